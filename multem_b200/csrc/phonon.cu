// Frozen-phonon displacements generated on the GPU from a counter-based random number generator.
//
// The reference draws the displacements on the host, atom after atom, from three mt19937_64
// streams through std::normal_distribution (Spec::move_atoms, src/spec.hpp:85-127; Randn_3d,
// src/cgpu_rand.cuh:308-395). That sequence is inherently serial; the engine reproduces it on the
// host by default (pn_rng 0). With pn_rng 1 every displacement is instead a pure function of
// (pn_seed, configuration, atom index):
//   Philox4x32-10 (Salmon, Moraes, Dror and Shaw, "Parallel random numbers: as easy as 1, 2, 3",
//   SC'11): key (pn_seed, 0), counter (atom index, configuration, 0, 0), ten rounds of
//   (c0, c1, c2, c3) -> (hi(M1*c2) ^ c1 ^ k0, lo(M1*c2), hi(M0*c0) ^ c3 ^ k1, lo(M0*c0)) with the
//   key advanced by the Weyl increments (W0, W1) between rounds;
//   two of the four 32-bit words become uniforms u = (r + 1/2) 2^-32 in (0, 1), and the Box-Muller
//   transform (Box and Muller, Ann. Math. Statist. 29 (1958) 610) gives two independent standard
//   normals n_x = sqrt(-2 ln u0) cos(2 pi u1), n_y = sqrt(-2 ln u0) sin(2 pi u1), in double;
//   x += sigma * (float)n_x and y += sigma * (float)n_y as the host path does (float).
// One thread per atom, no state, no ordering: any configuration of any specimen is generated
// directly on the device, in the slot buffer the configuration's splat reads. The reference's plain
// path never displaces z (no subslicing: pn_dim.z is switched off, src/input_multislice.cuh:705-708),
// so the slicing does not depend on the configuration and is computed once.
#include <cuda_runtime.h>

#include "common.hpp"
#include "kernels.cuh"

namespace mtb {

namespace {

constexpr uint32_t kPhiloxM0 = 0xD2511F53u, kPhiloxM1 = 0xCD9E8D57u;
constexpr uint32_t kPhiloxW0 = 0x9E3779B9u, kPhiloxW1 = 0xBB67AE85u;

__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k) {
#pragma unroll
    for (int r = 0; r < 10; r++) {
        const uint32_t hi0 = __umulhi(kPhiloxM0, c.x), lo0 = kPhiloxM0 * c.x;
        const uint32_t hi1 = __umulhi(kPhiloxM1, c.z), lo1 = kPhiloxM1 * c.z;
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
        k.x += kPhiloxW0;
        k.y += kPhiloxW1;
    }
    return c;
}

__global__ void phonon_displace_kernel(const float4* __restrict__ base, const float* __restrict__ sigma, int n,
                                       uint32_t seed, uint32_t iconf, int pn_x, int pn_y, float4* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 a = base[i];
    const uint4 r = philox4x32_10(make_uint4((uint32_t)i, iconf, 0u, 0u), make_uint2(seed, 0u));
    const double u0 = ((double)r.x + 0.5) * 2.3283064365386963e-10;  // 2^-32
    const double u1 = ((double)r.y + 0.5) * 2.3283064365386963e-10;
    const double rad = sqrt(-2.0 * log(u0));
    double s, c;
    sincos(6.283185307179586 * u1, &s, &c);
    const float sg = sigma[i];
    // product and sum rounded separately (no fused multiply-add), as the host path rounds them
    if (pn_x) a.x = __fadd_rn(a.x, __fmul_rn(sg, (float)(rad * c)));
    if (pn_y) a.y = __fadd_rn(a.y, __fmul_rn(sg, (float)(rad * s)));
    out[i] = a;
}

// Standalone self-test of the generator (mt_philox4x32_10): one thread per counter.
__global__ void philox_kernel(const uint4* __restrict__ ctr, const uint2* __restrict__ key, int n, uint4* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = philox4x32_10(ctr[i], key[i]);
}

}  // namespace

void launch_phonon_displace(const float4* base, const float* sigma, int n, uint32_t seed, int iconf, bool pn_x,
                            bool pn_y, float4* out, cudaStream_t s) {
    if (n <= 0) return;
    phonon_displace_kernel<<<(n + 255) / 256, 256, 0, s>>>(base, sigma, n, seed, (uint32_t)iconf, pn_x, pn_y, out);
    MTB_CUDA(cudaGetLastError());
    add_launches(1);
}

void launch_philox(const uint4* ctr, const uint2* key, int n, uint4* out, cudaStream_t s) {
    if (n <= 0) return;
    philox_kernel<<<(n + 255) / 256, 256, 0, s>>>(ctr, key, n, out);
    MTB_CUDA(cudaGetLastError());
    add_launches(1);
}

}  // namespace mtb
