// Errors inside the library: a status and a message, thrown as Failure and turned into a
// pg_status at the C boundary.
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "pine_gpu.h"

namespace pg {

struct Failure {
    pg_status status;
    std::string msg;
};

#define PG_CUDA(call)                                                                       \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess)                                                              \
            throw Failure{e_ == cudaErrorMemoryAllocation ? PG_ERR_OOM : PG_ERR_CUDA,       \
                          std::string(#call) + ": " + cudaGetErrorString(e_)};              \
    } while (0)

}  // namespace pg
