// CUDA status bookkeeping shared by the launchers: every CUDA status the library checks goes through
// cuda_status(), which records a failing one (the most recent wins, process-wide) so that
// dg_last_cuda_error() can name it, and maps it to DG_E_CUDA.
#pragma once
#include <cuda_runtime.h>

#include <atomic>

#include "dg_gpu.h"

namespace fvedg {

inline std::atomic<int>& last_cuda_error_slot() {
    static std::atomic<int> e{0};
    return e;
}

inline int cuda_status(cudaError_t e) {
    if (e == cudaSuccess) return DG_OK;
    last_cuda_error_slot().store((int)e);
    return DG_E_CUDA;
}

}  // namespace fvedg
