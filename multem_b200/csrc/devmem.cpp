// Device memory for the engine's buffers: one CUDA memory pool per device, created by the
// library, with its release threshold at the maximum so that memory freed by one engine stays
// with the pool and the next engine in the process (for instance the next mt_multislice_run call)
// reuses it instead of obtaining fresh memory from the driver. The pool is trimmed and the
// allocation retried once when the device runs out of memory.
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <map>
#include <mutex>

#include "common.hpp"
#include "devmem.hpp"

namespace mtb {
namespace {

struct DevicePool {
    cudaMemPool_t pool = nullptr;
    cudaStream_t stream = nullptr;  // orders the pool's allocations and frees; never runs kernels
};

std::mutex g_mu;
std::atomic<long long> g_alloc_count{0};
std::map<int, DevicePool> g_pools;

DevicePool& pool_of(int dev) {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_pools.find(dev);
    if (it != g_pools.end()) return it->second;
    DevicePool P;
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    MTB_CUDA(cudaMemPoolCreate(&P.pool, &props));
    uint64_t keep = UINT64_MAX;
    MTB_CUDA(cudaMemPoolSetAttribute(P.pool, cudaMemPoolAttrReleaseThreshold, &keep));
    int cur = 0;
    MTB_CUDA(cudaGetDevice(&cur));
    if (cur != dev) MTB_CUDA(cudaSetDevice(dev));
    MTB_CUDA(cudaStreamCreateWithFlags(&P.stream, cudaStreamNonBlocking));
    if (cur != dev) MTB_CUDA(cudaSetDevice(cur));
    return g_pools.emplace(dev, P).first->second;
}

}  // namespace

void* dev_alloc(size_t bytes, int* dev_out) {
    int dev = 0;
    MTB_CUDA(cudaGetDevice(&dev));
    DevicePool& P = pool_of(dev);
    void* p = nullptr;
    cudaError_t e = cudaMallocFromPoolAsync(&p, bytes, P.pool, P.stream);
    if (e == cudaErrorMemoryAllocation) {
        (void)cudaGetLastError();
        MTB_CUDA(cudaStreamSynchronize(P.stream));
        MTB_CUDA(cudaMemPoolTrimTo(P.pool, 0));
        e = cudaMallocFromPoolAsync(&p, bytes, P.pool, P.stream);
    }
    cuda_check(e, "cudaMallocFromPoolAsync");
    g_alloc_count.fetch_add(1, std::memory_order_relaxed);
    // the allocation is complete once the pool's stream is, so any stream may use it afterwards
    MTB_CUDA(cudaStreamSynchronize(P.stream));
    *dev_out = dev;
    return p;
}

long long dev_alloc_count() { return g_alloc_count.load(std::memory_order_relaxed); }

void dev_free(void* p, int dev) {
    if (!p) return;
    // like cudaFree: wait for all work on the device, which may still read or write p
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != dev) cudaSetDevice(dev);
    cudaDeviceSynchronize();
    cudaFreeAsync(p, pool_of(dev).stream);
    cudaStreamSynchronize(pool_of(dev).stream);
    if (cur != dev) cudaSetDevice(cur);
}

void dev_free_idle(void* p, int dev) {
    if (!p) return;
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != dev) cudaSetDevice(dev);
    cudaFreeAsync(p, pool_of(dev).stream);
    cudaStreamSynchronize(pool_of(dev).stream);
    if (cur != dev) cudaSetDevice(cur);
}

}  // namespace mtb
