// HRTEM transfer-function tables (Microscope_Effects, src/microscope_effects.cuh:32-200), built once
// per engine and applied in the column pass of the image formation.
#include <cuda_runtime.h>

#include "common.hpp"
#include "kernels.cuh"
#include "line_kernels.cuh"

namespace mtb {

__global__ void ctf_table_kernel(ProbeDev lens, GridDev g, float2* __restrict__ out) {
    const int iy = blockIdx.x * blockDim.x + threadIdx.x, ix = blockIdx.y;
    if (iy >= g.ny) return;
    out[(size_t)ix * g.ny + iy] = probe_value(lens, g, ix, iy, make_float2(0.0f, 0.0f));
}

// apply_PCTF's factor: polar(st_inc, chi) inside the aperture, chi = g2 (c_c_30 g2 + c_c_10),
// st_inc = exp(-(spatial + temporal) / u) / sqrt(u) (linear-image weak-phase envelopes).
__global__ void pctf_table_kernel(PctfArgs p, GridDev g, float2* __restrict__ out) {
    const int iy = blockIdx.x * blockDim.x + threadIdx.x, ix = blockIdx.y;
    if (iy >= g.ny) return;
    const float gx = __fmul_rn((float)ig_shift(ix, g.nxh, g.nx), g.dgx);
    const float gy = __fmul_rn((float)ig_shift(iy, g.nyh, g.ny), g.dgy);
    const float g2 = __fadd_rn(__fmul_rn(gx, gx), __fmul_rn(gy, gy));
    float2 v = make_float2(0.0f, 0.0f);
    if ((p.g2_min <= g2) && (g2 < p.g2_max)) {
        const float pi = 3.141592653589793238463f;
        const float chi = __fmul_rn(g2, __fadd_rn(__fmul_rn(p.c_c_30, g2), p.c_c_10));
        float c = __fmul_rn(__fmul_rn(pi, p.si_theta_c), p.ti_iehwgd);
        const float u = __fadd_rn(1.0f, __fmul_rn(__fmul_rn(c, c), g2));
        c = __fmul_rn(__fmul_rn(__fmul_rn(pi, p.ti_iehwgd), p.lambda), g2);
        const float temp_inc = __fmul_rn(0.25f, __fmul_rn(c, c));
        c = __fmul_rn(__fmul_rn(pi, p.si_theta_c), __fadd_rn(__fmul_rn(__fmul_rn(p.c_30, p.lambda2), g2), p.c_10));
        const float spa_inc = __fmul_rn(__fmul_rn(c, c), g2);
        const float st = expf(-__fdiv_rn(__fadd_rn(spa_inc, temp_inc), u)) / sqrtf(u);
        float sn, cs;
        sincosf(chi, &sn, &cs);
        v = make_float2(__fmul_rn(st, cs), __fmul_rn(st, sn));
    }
    out[(size_t)ix * g.ny + iy] = v;
}

void launch_ctf_table(const ProbeDev& lens, const GridDev& g, float2* out, cudaStream_t s) {
    ctf_table_kernel<<<dim3((unsigned)((g.ny + 127) / 128), (unsigned)g.nx), 128, 0, s>>>(lens, g, out);
    note_launch();
    MTB_CUDA(cudaGetLastError());
}

void launch_pctf_table(const PctfArgs& p, const GridDev& g, float2* out, cudaStream_t s) {
    pctf_table_kernel<<<dim3((unsigned)((g.ny + 127) / 128), (unsigned)g.nx), 128, 0, s>>>(p, g, out);
    note_launch();
    MTB_CUDA(cudaGetLastError());
}

}  // namespace mtb
