// Status codes, error bookkeeping, the bounded-wait limit and the version of
// the C ABI.
#include <atomic>

#include "common.cuh"

namespace vtb {

static thread_local int g_last_cuda_error = 0;

// 0: every kernel uses its own default limit; > 0: the number of polls after
// which every bounded device wait gives up (read at each launch).
static std::atomic<int64_t> g_wait_limit{0};

uint32_t wait_limit(uint32_t default_polls) {
    const int64_t v = g_wait_limit.load(std::memory_order_relaxed);
    return v > 0 ? (uint32_t)(v < 0xFFFFFFFFll ? v : 0xFFFFFFFFll) : default_polls;
}

void set_last_cuda_error(cudaError_t e) { g_last_cuda_error = (int)e; }

int launch_status() {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        g_last_cuda_error = (int)e;
        return VTB_CUDA_ERR;
    }
    return VTB_OK;
}

}  // namespace vtb

VTB_API int vtb_version(void) { return VTB_ABI_VERSION; }

VTB_API int vtb_set_wait_limit(int64_t polls, int64_t* previous) {
    VTB_CHECK_ARG(polls >= 0);
    const int64_t old = vtb::g_wait_limit.exchange(polls);
    if (previous) *previous = old;
    return VTB_OK;
}

VTB_API int vtb_last_cuda_error(void) { return vtb::g_last_cuda_error; }

VTB_API const char* vtb_status_string(int status) {
    switch (status) {
        case VTB_OK: return "ok";
        case VTB_BAD_ARG: return "bad argument";
        case VTB_OVERFLOW: return "spike buffer overflow";
        case VTB_OOM: return "out of device memory";
        case VTB_TIMEOUT: return "timed out";
        case VTB_CUDA_ERR: return "CUDA error";
        case VTB_NOT_CONVERGED: return "solver did not converge";
        case VTB_NO_DATA: return "no spikes to decode";
        case VTB_BLOCK_LIMIT: return "spikes in a frame block reached the buffer limit";
        default: return "unknown status";
    }
}
