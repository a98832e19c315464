// Device memory for the engine's buffers (see devmem.cpp).
#pragma once

#include <cstddef>

namespace mtb {

// Allocate `bytes` on the current device from the library's pool; *dev receives the device.
void* dev_alloc(size_t bytes, int* dev);
// Number of dev_alloc calls that succeeded in this process.
long long dev_alloc_count();
// Return p (from dev_alloc on device dev) to the pool after all work on the device has finished.
void dev_free(void* p, int dev);
// Return p to the pool at once: the caller has already waited for every stream that used it (so
// engines on other host threads are not made to wait for each other).
void dev_free_idle(void* p, int dev);

}  // namespace mtb
