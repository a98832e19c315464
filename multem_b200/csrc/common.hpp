// Shared error handling for the engine's host code.
#pragma once

#include <cuda_runtime.h>

#include <stdexcept>
#include <string>

#include "multem_b200.h"

namespace mtb {

struct Error : std::runtime_error {
    mt_status status;
    Error(mt_status s, const std::string& msg) : std::runtime_error(msg), status(s) {}
};

[[noreturn]] inline void fail(mt_status s, const std::string& msg) { throw Error(s, msg); }

inline void cuda_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        mt_status s = (e == cudaErrorMemoryAllocation) ? MT_ERR_OOM : MT_ERR_CUDA;
        throw Error(s, std::string(what) + ": " + cudaGetErrorString(e));
    }
}

#define MTB_CUDA(call) ::mtb::cuda_check((call), #call)

}  // namespace mtb
