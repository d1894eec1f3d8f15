// Shared helpers of the vtem_b200 CUDA library (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/vtem_b200.h"

#define VTB_API extern "C" __attribute__((visibility("default")))

namespace vtb {

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// Records the CUDA error (if any) of the launch just issued and maps it to a
// status code.  Kernel launch errors are synchronous; execution faults are
// reported by the next synchronising call on the caller's side.
int launch_status();

void set_last_cuda_error(cudaError_t e);

// Polls after which a bounded device wait gives up: the process-wide value
// set by vtb_set_wait_limit, else the kernel's default.
uint32_t wait_limit(uint32_t default_polls);

constexpr int kNumSMs = 148;

inline int ceil_div(int64_t a, int64_t b) { return (int)((a + b - 1) / b); }

}  // namespace vtb

#define VTB_CHECK_ARG(cond)            \
    do {                               \
        if (!(cond)) return VTB_BAD_ARG; \
    } while (0)

#define VTB_CUDA_TRY(expr)                     \
    do {                                       \
        cudaError_t _e = (expr);               \
        if (_e != cudaSuccess) {               \
            vtb::set_last_cuda_error(_e);      \
            return VTB_CUDA_ERR;               \
        }                                      \
    } while (0)
