// Line-pass kernels (contiguous y-lines and strided x-lines), templated on the line length.
// Each supported length is instantiated in its own translation unit (lines_<N>.cu) so the build
// parallelises; kernels.cu dispatches on the runtime size.
#pragma once

#include <cuda_runtime.h>

#include <type_traits>

#include "common.hpp"
#include "fft_core.cuh"
#include "kernels.cuh"

namespace mtb {

void note_launch();

template <int N>
constexpr int min_radix() {
    int r = LinePlan<N>::R[0];
    for (int s = 1; s < LinePlan<N>::NS; s++) r = LinePlan<N>::R[s] < r ? LinePlan<N>::R[s] : r;
    return r;
}

template <int N>
struct LineGeom {
    static constexpr int E = LinePlan<N>::E;
    static constexpr int TPL = N / E;
    static constexpr int NSG = LinePlan<N>::NS;
    static constexpr int R1 = LinePlan<N>::R[0];
    static constexpr int RL = LinePlan<N>::R[NSG - 1];
    static constexpr int RMIN = min_radix<N>();
    static constexpr int LS = N + N / RMIN + 1;  // padded line buffer (float2); odd
    static constexpr int TW_I = TwTable<N, false, 0>::SIZE + TwTable<N, false, 1>::SIZE + (NSG > 2 ? TwTable<N, false, 2>::SIZE : 0);
    static constexpr int TW_F = TwTable<N, true, 0>::SIZE + TwTable<N, true, 1>::SIZE + (NSG > 2 ? TwTable<N, true, 2>::SIZE : 0);
};

template <int N>
__device__ __forceinline__ void setup_twiddles(float2* base, const float2** twI, const float2** twF) {
    constexpr int NSG = LinePlan<N>::NS;
    float2* p = base;
    static_for<0, NSG>([&](auto sc) {
        constexpr int s = decltype(sc)::value;
        twI[s] = p;
        fill_twiddles<N, false, s>(p, threadIdx.x, blockDim.x);
        p += TwTable<N, false, s>::SIZE;
    });
    static_for<0, NSG>([&](auto sc) {
        constexpr int s = decltype(sc)::value;
        twF[s] = p;
        fill_twiddles<N, true, s>(p, threadIdx.x, blockDim.x);
        p += TwTable<N, true, s>::SIZE;
    });
}

struct WarpSync {
    __device__ __forceinline__ void operator()() const { __syncwarp(); }
};
struct BlockSync {
    __device__ __forceinline__ void operator()() const { __syncthreads(); }
};

// ---------------------------------------------------------------------------------------------
// Contiguous-line pass. 256 threads; each line of NY points is owned by TPL = NY/E threads.
template <int NY, int MODE>
__global__ void __launch_bounds__(256) rows_kernel(RowArgs a) {
    using G = LineGeom<NY>;
    constexpr int E = G::E, TPL = G::TPL, LPC = 256 / TPL;
    extern __shared__ float2 smem2[];
    const float2* twI[3] = {nullptr, nullptr, nullptr};
    const float2* twF[3] = {nullptr, nullptr, nullptr};
    setup_twiddles<NY>(smem2, twI, twF);
    float2* lines = smem2 + G::TW_I + G::TW_F;
    __syncthreads();

    const int li = threadIdx.x / TPL, t = threadIdx.x % TPL;
    float2* buf = lines + li * G::LS;
    const int groups = a.nx / LPC;
    const int items = groups * a.nprobe;
    using Sync = typename std::conditional<(TPL <= 32), WarpSync, BlockSync>::type;

    for (int item = blockIdx.x; item < items; item += gridDim.x) {
        const int b = item / groups;
        const int ix = (item % groups) * LPC + li;
        const size_t off = ((size_t)b * a.nx + ix) * NY;
        float2 x[E];
        if constexpr (MODE == ROW_STEP || MODE == ROW_INVERSE) {
#pragma unroll
            for (int i = 0; i < E; i++) x[i] = a.in[off + reg_pos<NY, G::R1>(i, t)];
            line_fft<NY, false, +1>(x, buf, twI, t, Sync{});
        } else if constexpr (MODE == ROW_FIRST_REAL) {
#pragma unroll
            for (int i = 0; i < E; i++) x[i] = a.in[off + reg_pos<NY, G::RL>(i, t)];
        } else {
#pragma unroll
            for (int i = 0; i < E; i++) x[i] = make_float2(1.0f, 0.0f);
        }
        if constexpr (MODE == ROW_INVERSE) {
#pragma unroll
            for (int i = 0; i < E; i++) a.out[off + reg_pos<NY, G::RL>(i, t)] = cscale(x[i], a.scale);
        } else {
            const float2* Tr = a.trans + (size_t)ix * NY;
#pragma unroll
            for (int i = 0; i < E; i++) x[i] = cmul(x[i], __ldg(&Tr[reg_pos<NY, G::RL>(i, t)]));
            line_fft<NY, true, -1>(x, buf, twF, t, Sync{});
#pragma unroll
            for (int i = 0; i < E; i++) a.out[off + reg_pos<NY, G::R1>(i, t)] = x[i];
        }
    }
}

template <int NY>
static size_t rows_smem() {
    using G = LineGeom<NY>;
    return sizeof(float2) * (size_t)(G::TW_I + G::TW_F + (256 / G::TPL) * G::LS);
}

// ---------------------------------------------------------------------------------------------
// Strided-line pass. 256 threads; W = 256/TPL adjacent columns per CTA (coalesced rows of W
// complex values); column c is owned by threads c, c+W, c+2W, ...
__device__ __forceinline__ int ig_shift(int i, int nh, int n) { return (i < nh) ? i : (i - n); }

// exp_i_chi (src/cgpu_fcns.cuh:1951-1980) for one Fourier-space pixel, times the normalisation.
__device__ __forceinline__ float2 probe_value(const ProbeDev& pr, const GridDev& g, int ix, int iy, float2 beam) {
    const float gx = __fadd_rn(__fmul_rn((float)ig_shift(ix, g.nxh, g.nx), g.dgx), pr.gxu);
    const float gy = __fadd_rn(__fmul_rn((float)ig_shift(iy, g.nyh, g.ny), g.dgy), pr.gyu);
    const float g2 = __fadd_rn(__fmul_rn(gx, gx), __fmul_rn(gy, gy));
    if (!((pr.g2_min <= g2) && (g2 < pr.g2_max))) return make_float2(0.0f, 0.0f);
    const float g4 = __fmul_rn(g2, g2);
    const float g6 = __fmul_rn(g4, g2);
    float chi = __fadd_rn(__fmul_rn(beam.x, gx), __fmul_rn(beam.y, gy));
    chi = __fadd_rn(chi, pr.nz_c10 ? __fmul_rn(pr.c_c_10, g2) : 0.0f);
    chi = __fadd_rn(chi, pr.nz_c30 ? __fmul_rn(pr.c_c_30, g4) : 0.0f);
    chi = __fadd_rn(chi, pr.nz_c50 ? __fmul_rn(pr.c_c_50, g6) : 0.0f);
    if (pr.phi_required) {
        const float gg = sqrtf(g2);
        const float g3 = __fmul_rn(g2, gg), g5 = __fmul_rn(g4, gg);
        const float ph = atan2f(gy, gx);
        auto term = [](float cc, float gp, float k, float ph, float ph0) {
            return (cc != 0.0f) ? __fmul_rn(__fmul_rn(cc, gp), sinf(__fmul_rn(k, __fsub_rn(ph, ph0)))) : 0.0f;
        };
        float t1 = __fadd_rn((ph != 0.0f) ? __fmul_rn((float)pr.m, ph) : 0.0f, term(pr.c_c_12, g2, 2.0f, ph, pr.phi_12));
        chi = __fadd_rn(chi, t1);
        float t2 = __fadd_rn(__fadd_rn(term(pr.c_c_21, g3, 1.0f, ph, pr.phi_21), term(pr.c_c_23, g3, 3.0f, ph, pr.phi_23)),
                             __fadd_rn(term(pr.c_c_32, g4, 2.0f, ph, pr.phi_32), term(pr.c_c_34, g4, 4.0f, ph, pr.phi_34)));
        chi = __fadd_rn(chi, t2);
        float t3 = __fadd_rn(__fadd_rn(__fadd_rn(term(pr.c_c_41, g5, 1.0f, ph, pr.phi_41), term(pr.c_c_43, g5, 3.0f, ph, pr.phi_43)),
                                       term(pr.c_c_45, g5, 5.0f, ph, pr.phi_45)),
                             __fadd_rn(__fadd_rn(term(pr.c_c_52, g6, 2.0f, ph, pr.phi_52), term(pr.c_c_54, g6, 4.0f, ph, pr.phi_54)),
                                       term(pr.c_c_56, g6, 6.0f, ph, pr.phi_56)));
        chi = __fadd_rn(chi, t3);
    }
    float sn, cs;
    sincosf(chi, &sn, &cs);
    return make_float2(__fmul_rn(cs, pr.norm), __fmul_rn(sn, pr.norm));
}

// LDY is the line stride (= ny) when known at compile time (square grids), 0 for a runtime stride.
template <int NX, int FLAGS, int LDY>
__global__ void __launch_bounds__(256) cols_kernel(ColArgs a) {
    using G = LineGeom<NX>;
    constexpr int E = G::E, TPL = G::TPL, W = 256 / TPL;
    constexpr bool LOAD = FLAGS & COL_LOAD, PROP = FLAGS & COL_PROP, DET = FLAGS & COL_DETECT;
    constexpr bool INV = FLAGS & COL_INVERSE, STORE = FLAGS & COL_STORE;
    extern __shared__ float2 smem2[];
    const float2* twF[3] = {nullptr, nullptr, nullptr};  // forward (plan order)
    const float2* twI[3] = {nullptr, nullptr, nullptr};  // inverse (reversed order)
    // forward transform uses plan order (REV=false), inverse uses reversed order (REV=true)
    {
        float2* p = smem2;
        static_for<0, G::NSG>([&](auto sc) {
            constexpr int s = decltype(sc)::value;
            twF[s] = p;
            fill_twiddles<NX, false, s>(p, threadIdx.x, blockDim.x);
            p += TwTable<NX, false, s>::SIZE;
        });
        static_for<0, G::NSG>([&](auto sc) {
            constexpr int s = decltype(sc)::value;
            twI[s] = p;
            fill_twiddles<NX, true, s>(p, threadIdx.x, blockDim.x);
            p += TwTable<NX, true, s>::SIZE;
        });
    }
    float2* s_px = smem2 + G::TW_I + G::TW_F;
    float2* lines = s_px + (PROP ? NX : 0);
    __shared__ double s_red[8][kMaxDet];
    if constexpr (PROP) {
        for (int i = threadIdx.x; i < NX; i += blockDim.x) s_px[i] = a.Px[i];
    }
    __syncthreads();

    const int c = threadIdx.x % W, t = threadIdx.x / W;
    float2* buf = lines + c * G::LS;
    const int ldy = LDY ? LDY : a.ny;
    const int tiles = ldy / W;
    const int items = tiles * a.nprobe;
    const size_t pstride = (size_t)NX * ldy;

    for (int item = blockIdx.x; item < items; item += gridDim.x) {
        const int b = item / tiles;
        const int ct = item % tiles;
        const int iy = ct * W + c;
        const size_t off = (size_t)b * pstride + iy + (size_t)t * ldy;
        const float2* src = a.in + off;
        float2* dst = a.out + off;
        float2 x[E];
        if constexpr (LOAD) {
#pragma unroll
            for (int i = 0; i < E; i++) x[i] = src[(reg_pos<NX, G::R1>(i, t) - t) * ldy];
            line_fft<NX, false, -1>(x, buf, twF, t, BlockSync{});
        } else {
            const float2 beam = a.beam[b];
#pragma unroll
            for (int i = 0; i < E; i++) x[i] = probe_value(a.probe, a.g, reg_pos<NX, G::RL>(i, t), iy, beam);
        }
        if constexpr (PROP) {
            const float2 py = a.Py[iy];
#pragma unroll
            for (int i = 0; i < E; i++) x[i] = cmul(x[i], cmul(s_px[reg_pos<NX, G::RL>(i, t)], py));
        }
        if constexpr (DET) {
            double acc[kMaxDet];
#pragma unroll
            for (int d = 0; d < kMaxDet; d++) acc[d] = 0.0;
            const float gy = __fsub_rn(__fmul_rn((float)ig_shift(iy, a.g.nyh, a.g.ny), a.g.dgy), 0.0f);
            const float gy2 = __fmul_rn(gy, gy);
#pragma unroll
            for (int i = 0; i < E; i++) {
                const int ix = reg_pos<NX, G::RL>(i, t);
                const float gx = __fmul_rn((float)ig_shift(ix, a.g.nxh, a.g.nx), a.g.dgx);
                const float g2 = __fadd_rn(__fmul_rn(gx, gx), gy2);
                const float v2 = __fadd_rn(__fmul_rn(x[i].x, x[i].x), __fmul_rn(x[i].y, x[i].y));
#pragma unroll
                for (int d = 0; d < kMaxDet; d++)
                    if (d < a.n_det && a.det_g2_min[d] <= g2 && g2 < a.det_g2_max[d]) acc[d] += (double)v2;
            }
            // deterministic block reduction: warp shuffles, then warps in order
#pragma unroll
            for (int d = 0; d < kMaxDet; d++) {
                double v = acc[d];
                for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
                if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5][d] = v;
            }
            __syncthreads();
            if (threadIdx.x < a.n_det) {
                double s = 0.0;
                for (int w = 0; w < 8; w++) s += s_red[w][threadIdx.x];
                a.det_partial[((size_t)b * tiles + ct) * a.n_det + threadIdx.x] = s;
            }
            __syncthreads();
        }
        if constexpr (INV) {
            line_fft<NX, true, +1>(x, buf, twI, t, BlockSync{});
#pragma unroll
            for (int i = 0; i < E; i++) dst[(reg_pos<NX, G::R1>(i, t) - t) * ldy] = x[i];
        } else if constexpr (STORE) {
#pragma unroll
            for (int i = 0; i < E; i++) dst[(reg_pos<NX, G::RL>(i, t) - t) * ldy] = x[i];
        }
    }
}

template <int NX, int FLAGS>
static size_t cols_smem() {
    using G = LineGeom<NX>;
    constexpr bool PROP = FLAGS & COL_PROP;
    return sizeof(float2) * (size_t)(G::TW_I + G::TW_F + (PROP ? NX : 0) + (256 / G::TPL) * G::LS);
}

// ---------------------------------------------------------------------------------------------
// launch helpers
template <class K>
static int max_ctas(K kernel, size_t smem) {
    static int nsm = 0;
    if (nsm == 0) {
        int dev = 0;
        MTB_CUDA(cudaGetDevice(&dev));
        MTB_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    }
    MTB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int occ = 0;
    MTB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, 256, smem));
    if (occ < 1) fail(MT_ERR_UNSUPPORTED, "line-pass kernel does not fit on an SM");
    return nsm * occ;
}

template <int NY, int MODE>
static void rows_launch(const RowArgs& a, int grid_ctas, cudaStream_t s) {
    using G = LineGeom<NY>;
    const size_t sm = rows_smem<NY>();
    static int cap = 0;
    if (cap == 0) cap = max_ctas(rows_kernel<NY, MODE>, sm);
    const int items = (a.nx / (256 / G::TPL)) * a.nprobe;
    int grid = grid_ctas > 0 ? grid_ctas : cap;
    if (grid > items) grid = items;
    rows_kernel<NY, MODE><<<grid, 256, sm, s>>>(a);
    note_launch();
    MTB_CUDA(cudaGetLastError());
}

template <int NY>
void rows_dispatch_mode(RowMode mode, const RowArgs& a, int grid_ctas, cudaStream_t s) {
    switch (mode) {
        case ROW_STEP: rows_launch<NY, ROW_STEP>(a, grid_ctas, s); break;
        case ROW_FIRST_ONE: rows_launch<NY, ROW_FIRST_ONE>(a, grid_ctas, s); break;
        case ROW_FIRST_REAL: rows_launch<NY, ROW_FIRST_REAL>(a, grid_ctas, s); break;
        case ROW_INVERSE: rows_launch<NY, ROW_INVERSE>(a, grid_ctas, s); break;
    }
}

template <int NX, int FLAGS, int LDY>
static void cols_launch_ld(const ColArgs& a, int grid_ctas, cudaStream_t s) {
    using G = LineGeom<NX>;
    const size_t sm = cols_smem<NX, FLAGS>();
    static int cap = 0;
    if (cap == 0) cap = max_ctas(cols_kernel<NX, FLAGS, LDY>, sm);
    const int items = (a.ny / (256 / G::TPL)) * a.nprobe;
    int grid = grid_ctas > 0 ? grid_ctas : cap;
    if (grid > items) grid = items;
    cols_kernel<NX, FLAGS, LDY><<<grid, 256, sm, s>>>(a);
    note_launch();
    MTB_CUDA(cudaGetLastError());
}

template <int NX, int FLAGS>
static void cols_launch(const ColArgs& a, int grid_ctas, cudaStream_t s) {
    if (a.ny == NX) cols_launch_ld<NX, FLAGS, NX>(a, grid_ctas, s);
    else cols_launch_ld<NX, FLAGS, 0>(a, grid_ctas, s);
}

constexpr int COL_F_PROBE = COL_INVERSE | COL_STORE;
constexpr int COL_F_STEP = COL_LOAD | COL_PROP | COL_INVERSE | COL_STORE;
constexpr int COL_F_STEP_DET = COL_LOAD | COL_PROP | COL_DETECT | COL_INVERSE | COL_STORE;
constexpr int COL_F_LAST_DET = COL_LOAD | COL_PROP | COL_DETECT;
constexpr int COL_F_FOURIER = COL_LOAD | COL_PROP | COL_STORE;
constexpr int COL_F_PROBE_FS = COL_STORE;

template <int NX>
void cols_dispatch_flags(int flags, const ColArgs& a, int grid_ctas, cudaStream_t s) {
    switch (flags) {
        case COL_F_PROBE: cols_launch<NX, COL_F_PROBE>(a, grid_ctas, s); break;
        case COL_F_STEP: cols_launch<NX, COL_F_STEP>(a, grid_ctas, s); break;
        case COL_F_STEP_DET: cols_launch<NX, COL_F_STEP_DET>(a, grid_ctas, s); break;
        case COL_F_LAST_DET: cols_launch<NX, COL_F_LAST_DET>(a, grid_ctas, s); break;
        case COL_F_FOURIER: cols_launch<NX, COL_F_FOURIER>(a, grid_ctas, s); break;
        case COL_F_PROBE_FS: cols_launch<NX, COL_F_PROBE_FS>(a, grid_ctas, s); break;
        default: fail(MT_ERR_INTERNAL, "unsupported column-pass flag combination");
    }
}

}  // namespace mtb
