// BF16 GEMM on the fifth-generation tensor cores (tcgen05, sm_100a), FP32 accumulation in tensor
// memory, for the learned surrogate's convolutions (as implicit-GEMM operands built by
// surrogate.cu).
//
//   part[split][m][n] = sum_{k in split} A[m][k] * B[n][k]      (m < M, n < N)
//
// A [M][K] and B [N][K] are bf16, K-major (k contiguous), row pitch a multiple of 8 elements;
// the K range is cut into blocks of 64 (one 128-byte row of the 128-byte swizzle) and the blocks
// into `splits` contiguous ranges, one per grid.y, whose FP32 partial sums the caller reduces in a
// fixed order (deterministic results); with a single split the kernel applies bias and ReLU and
// stores the result itself (GemmOut). Tiles are 128 rows (the tensor-memory lanes) x BN columns;
// rows and columns past M, N and k past K arrive as zeros (tensor-copy out-of-bounds fill).
//
// One CTA of 4 warps per tile. Warp 0 allocates BN (at least 32) tensor-memory columns. Thread 0
// feeds a STAGES-deep ring of shared-memory stages with 2-D tensor copies (no multicast) and issues
// the MMAs: for block i it waits for stage i % STAGES to land, issues four 128 x BN x 16 MMAs
// (tcgen05.mma.cta_group::1.kind::f16, operands from shared-memory descriptors), commits them to the
// stage's "empty" barrier and refills the stage of block i-1 once its MMAs have completed, so the
// tensor pipe always has the next block queued. A final commit signals "done"; each warp then reads
// its 32 lanes of the accumulator (tcgen05.ld 32x32b) and stores its rows' partial sums.
//
// Bounded waits (mbarrier.cuh): a wait that runs out sets *err, thread 0 stops issuing, waits out
// the copies it issued and the MMAs it committed, and every thread still reaches the tensor-memory
// release.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cuda_bf16.h>

#include <cstdint>

#include "mbarrier.cuh"

namespace mtb {
namespace umma {

constexpr int BM = 128;            // tile rows: one per tensor-memory lane
constexpr int BK = 64;             // bf16 per K block: one 128-byte swizzled row
constexpr int STAGES = 4;          // shared-memory ring depth
constexpr unsigned A_BYTES = BM * BK * 2;

template <int BN>
struct Tile {
    static constexpr unsigned B_BYTES = BN * BK * 2;
    static constexpr int TCOLS = BN < 32 ? 32 : BN;  // tensor-memory columns (a power of 2, >= 32)
    // 1 KB of slack for aligning the ring to the 1024-byte swizzle atom
    static constexpr size_t SMEM = 1024 + (size_t)STAGES * (A_BYTES + B_BYTES);
    static_assert(BN % 16 == 0 && BN >= 16 && BN <= 256, "MMA N for M = 128 is a multiple of 16 in [16, 256]");
    static_assert(B_BYTES % 1024 == 0, "stages must stay on swizzle-atom boundaries");
};

// Instruction descriptor of kind::f16: FP32 accumulator (bits 4-5 = 1), A and B BF16 (bits 7-9,
// 10-12 = 1), both K-major (bits 15, 16 = 0), N >> 3 at bits 17-22, M >> 4 at bits 24-28.
constexpr uint32_t idesc_bf16(int m, int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

// Shared-memory matrix descriptor of a K-major operand in the canonical 128-byte swizzled layout
// that a SWIZZLE_128B tensor copy writes: rows of 128 bytes, 8-row atoms of 1024 bytes (stride
// byte offset 1024), leading byte offset unused for this layout (1), version 1 (bits 46-47),
// layout type 2 = SWIZZLE_128B (bits 61-63). Start address in 16-byte units at bits 0-13; the
// k-th 16-element step inside the 64-element row starts 32*k bytes further.
__device__ __forceinline__ uint64_t smem_desc_sw128(unsigned saddr) {
    return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
           ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_alloc(unsigned* slot, unsigned ncols) {  // whole warp
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(unsigned taddr, unsigned ncols) {  // whole warp
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void mma_bf16(unsigned tmem_d, uint64_t da, uint64_t db, uint32_t idesc, unsigned acc) {
    const unsigned z0 = 0, z1 = 0, z2 = 0, z3 = 0;  // no output lanes disabled
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n}\n" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(z0), "r"(z1), "r"(z2), "r"(z3)
        : "memory");
}
// arrive on `bar` once every MMA this thread issued before has completed
__device__ __forceinline__ void mma_commit(unsigned long long* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_ld16(unsigned taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tensor_load_2d(void* dst, const CUtensorMap* map, int x, int y, unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            smem_u32(dst)),
        "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

// Where the accumulator goes. With `part` set, the FP32 partial sums of each K split,
// part[split][m][n]; otherwise (one split) the finished result: v = acc + bias[n], ReLU when
// `relu`, stored as bf16 and/or float at (m / mdiv) * s_mq + (m % mdiv) * s_mr + n * s_n (an NCHW
// image when mdiv is H*W, s_mq the image stride, s_mr 1 and s_n H*W).
struct GemmOut {
    float* part;
    const float* bias;
    int relu;
    __nv_bfloat16* out_bf;
    float* out_f;
    long long mdiv, s_mq, s_mr, s_n;
};

template <int BN>
__global__ void __launch_bounds__(128, 1) gemm_kernel(const __grid_constant__ CUtensorMap mapA,
                                                      const __grid_constant__ CUtensorMap mapB, GemmOut o,
                                                      int M, int N, int nkb, int kb_per_split, int* err,
                                                      long long wait_ns) {
    using T = Tile<BN>;
    extern __shared__ unsigned char gemm_smem_raw[];
    unsigned char* ring = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(gemm_smem_raw) + 1023) &
                                                           ~static_cast<uintptr_t>(1023));
    unsigned char* sA = ring;
    unsigned char* sB = ring + STAGES * A_BYTES;
    __shared__ unsigned long long full[STAGES], empty[STAGES], done;
    __shared__ unsigned s_tmem;
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const int m0 = blockIdx.x * BM, n0 = blockIdx.z * BN, split = blockIdx.y;
    const int kb0 = split * kb_per_split;
    const int nk = nkb - kb0 < kb_per_split ? (nkb - kb0 > 0 ? nkb - kb0 : 0) : kb_per_split;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(&done, 1);
        mbar_fence_init();
    }
    if (warp == 0) tmem_alloc(&s_tmem, T::TCOLS);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const unsigned tmem = s_tmem;

    if (threadIdx.x == 0) {
        constexpr uint32_t idesc = idesc_bf16(BM, BN);
        const unsigned a0 = smem_u32(sA), b0 = smem_u32(sB);
        int loaded = 0;     // blocks whose copies were issued
        int consumed = 0;   // blocks whose copies were seen to land
        bool ok = !err_set(err);
        auto load = [&](int i) {
            const int s = i % STAGES;
            fence_proxy_async();
            mbar_expect_tx(&full[s], A_BYTES + T::B_BYTES);
            tensor_load_2d(sA + s * A_BYTES, &mapA, (kb0 + i) * BK, m0, &full[s]);
            tensor_load_2d(sB + s * T::B_BYTES, &mapB, (kb0 + i) * BK, n0, &full[s]);
        };
        for (; ok && loaded < nk && loaded < STAGES; loaded++) load(loaded);
        for (int i = 0; ok && i < nk; i++) {
            const int s = i % STAGES;
            if (!mbar_wait(&full[s], (unsigned)(i / STAGES) & 1u, err, wait_ns)) {
                ok = false;
                break;
            }
            consumed = i + 1;
            tc_fence_after();
#pragma unroll
            for (int kk = 0; kk < BK / 16; kk++)
                mma_bf16(tmem, smem_desc_sw128(a0 + s * A_BYTES + 32 * kk), smem_desc_sw128(b0 + s * T::B_BYTES + 32 * kk),
                         idesc, (i > 0 || kk > 0) ? 1u : 0u);
            mma_commit(&empty[s]);
            if (i >= 1 && loaded < nk) {
                // the stage of block i-1 takes block i-1+STAGES once block i-1's MMAs are done
                if (!mbar_wait(&empty[(i - 1) % STAGES], (unsigned)((i - 1) / STAGES) & 1u, err, wait_ns)) {
                    ok = false;
                    break;
                }
                load(loaded++);
            }
        }
        mma_commit(&done);  // every MMA issued above
        if (!ok) {
            // copies issued that nobody saw land: wait them out before the CTA can exit
            for (int i = consumed; i < loaded; i++) mbar_drain(&full[i % STAGES], (unsigned)(i / STAGES) & 1u);
        }
    }
    mbar_drain(&done, 0);  // the accumulator is final (bounded whatever the flag says)
    tc_fence_after();

    const int row = m0 + warp * 32 + lane;
    const bool have = nk > 0 && !err_set(err);
    long long obase = 0;
    if (!o.part) obase = (row / o.mdiv) * o.s_mq + (row % o.mdiv) * o.s_mr;
#pragma unroll 1
    for (int c0 = 0; c0 < BN; c0 += 16) {
        uint32_t r[16];
        tmem_ld16(tmem + ((unsigned)(warp * 32) << 16) + (unsigned)c0, r);
        if (row < M) {
            if (o.part) {
                float* dst = o.part + ((size_t)split * M + row) * N + n0 + c0;
#pragma unroll
                for (int j = 0; j < 16; j++)
                    if (n0 + c0 + j < N) dst[j] = have ? __uint_as_float(r[j]) : 0.0f;
            } else {
                // lanes hold consecutive rows: for each column the warp's stores are contiguous
#pragma unroll
                for (int j = 0; j < 16; j++) {
                    const int n = n0 + c0 + j;
                    if (n < N) {
                        float v = (have ? __uint_as_float(r[j]) : 0.0f) + (o.bias ? o.bias[n] : 0.0f);
                        if (o.relu) v = fmaxf(v, 0.0f);
                        const long long idx = obase + n * o.s_n;
                        if (o.out_bf) o.out_bf[idx] = __float2bfloat16_rn(v);
                        if (o.out_f) o.out_f[idx] = v;
                    }
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, T::TCOLS);
    }
}

}  // namespace umma
}  // namespace mtb
