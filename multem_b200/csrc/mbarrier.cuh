// Shared-memory barriers (mbarrier) with bounded waits, for kernels fed by the copy engine
// (bulk copies, tensor copies) or waiting on the tensor cores.
//
// Every wait gives up after a limit in nanoseconds (from the first failed check), sets the
// caller's error flag and returns false; once the flag is set, waits return at once. The drain
// wait, for copies or tensor-core work a thread issued itself, ignores the flag and is bounded by
// kDrainLimitNs, so a CTA never exits (or frees tensor memory) with work in flight it could still
// wait out.
#pragma once

#include <cuda_runtime.h>

namespace mtb {

constexpr long long kDrainLimitNs = 1000000000ll;  // bound of the wait for copies in flight at exit

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// non-blocking check of the phase with the given parity
__device__ __forceinline__ bool mbar_test_wait(unsigned long long* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ bool err_set(const int* err) { return *reinterpret_cast<const volatile int*>(err) != 0; }

// Wait for the phase with the given parity. Returns false without waiting when the error flag is
// already set; gives up after limit_ns (0: at the first failed check), sets the flag and returns
// false. The spin is also capped in iterations.
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity, int* err, long long limit_ns) {
    if (mbar_test_wait(bar, parity)) return true;
    if (err_set(err)) return false;
    if (limit_ns > 0) {
        const unsigned long long t0 = global_ns();
        for (unsigned it = 1; it < (1u << 30); it++) {
            if (mbar_try_wait(bar, parity)) return true;
            if ((it & 15u) == 0) {
                if (err_set(err)) return false;
                if ((long long)(global_ns() - t0) > limit_ns) break;
            }
        }
    }
    atomicOr(err, 1);
    return false;
}
// Exit path after an error: wait for the phase of a copy this thread issued, bounded by
// kDrainLimitNs whatever the flag says.
__device__ __forceinline__ void mbar_drain(unsigned long long* bar, unsigned parity) {
    if (mbar_test_wait(bar, parity)) return;
    const unsigned long long t0 = global_ns();
    for (unsigned it = 1; it < (1u << 30); it++) {
        if (mbar_try_wait(bar, parity)) return;
        if ((it & 15u) == 0 && (long long)(global_ns() - t0) > kDrainLimitNs) return;
    }
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

}  // namespace mtb
