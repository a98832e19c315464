// Device memory for the engine's buffers (see devmem.cpp).
#pragma once

#include <cstddef>

namespace mtb {

// Allocate `bytes` on the current device from the library's pool; *dev receives the device.
void* dev_alloc(size_t bytes, int* dev);
// Return p (from dev_alloc on device dev) to the pool after all work on the device has finished.
void dev_free(void* p, int dev);

}  // namespace mtb
