// RNN (gradient-flow) decoder in the coefficient space.
//
// The reference's rnn3 (vtem/neural_network.py:15-99) runs, from c = 0,
// steps+1 updates c <- c + dt*alpha*(q - G c) on the n x n spike Gram
// G = Phi Phi^H.  The reconstruction only uses a = Phi^H c, and
//     Phi^H c_{i+1} = Phi^H c_i + dt*alpha*(Phi^H q - Phi^H Phi Phi^H c_i),
// so a_{i+1} = a_i + dt*alpha*(b - M a_i) with M = Phi^H Phi, b = Phi^H q:
// the same iterates, on the K x K system instead of n x n (1921 instead of
// ~25k at the GPU configuration).  In the real form (realsys.cu) this is
// x <- x + dt*alpha*(br - Mr x), float64 like the reference.
//
// One cooperative launch runs every step: each CTA owns a block of rows of
// Mr, kept in shared memory for the whole run when it fits (Mr is read from
// HBM/L2 once, not once per step), stages the previous iterate in shared
// memory, writes its rows of the next one, and meets the other CTAs at a
// grid barrier.  The barrier's wait is bounded: a CTA that waits longer than
// the limit sets *err and returns (the host reports VTB_TIMEOUT).
#include <algorithm>
#include <mutex>

#include "common.cuh"

namespace vtb {

constexpr unsigned kRnnSpinLimit = 1u << 24;   // x ~64 ns sleep: about a second
constexpr int kRnnThreads = 256;

// Generation barrier over all CTAs of the launch (cooperative launch: all
// co-resident).  count/gen live in global memory, zeroed before the launch.
__device__ bool rnn_grid_barrier(unsigned* count, unsigned* gen, unsigned nblocks, int* err, unsigned limit) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        ok = 1;
        volatile unsigned* vgen = gen;
        const unsigned g = *vgen;
        __threadfence();
        if (atomicAdd(count, 1u) == nblocks - 1) {
            atomicExch(count, 0u);
            __threadfence();
            atomicAdd(gen, 1u);
        } else {
            unsigned it = 0;
            while (*vgen == g) {
                if (++it > limit || *(volatile int*)err) {
                    atomicExch(err, 1);
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return ok != 0;
}

__global__ void __launch_bounds__(kRnnThreads) rnn_coeff_kernel(const double* __restrict__ Mr, int64_t ld,
                                                                const double* __restrict__ br, double* xa,
                                                                double* xb, int K, double dta, int updates,
                                                                int rows_per_block, int cache_rows,
                                                                unsigned* bar, int* err, unsigned limit) {
    extern __shared__ double rnn_sm[];
    double* sx = rnn_sm;                 // K: previous iterate
    double* sM = rnn_sm + K;             // rows_per_block x K (when cache_rows)
    const int r0 = blockIdx.x * rows_per_block;
    const int r1 = min(K, r0 + rows_per_block);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    if (cache_rows)
        for (int64_t e = threadIdx.x; e < (int64_t)(r1 - r0) * K; e += blockDim.x) {
            const int r = (int)(e / K), j = (int)(e % K);
            sM[e] = Mr[(int64_t)(r0 + r) * ld + j];
        }
    for (int it = 0; it < updates; ++it) {
        const double* cur = (it & 1) ? xb : xa;
        double* nxt = (it & 1) ? xa : xb;
        for (int j = threadIdx.x; j < K; j += blockDim.x) sx[j] = __ldcg(cur + j);
        __syncthreads();
        for (int r = r0 + warp; r < r1; r += nw) {
            const double* row = cache_rows ? sM + (int64_t)(r - r0) * K : Mr + (int64_t)r * ld;
            double s = 0.0;
            for (int j = lane; j < K; j += 32) s = fma(row[j], sx[j], s);
            for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            if (lane == 0) __stcg(nxt + r, sx[r] + dta * (br[r] - s));
        }
        if (!rnn_grid_barrier(bar, bar + 1, gridDim.x, err, limit)) return;
    }
}

}  // namespace vtb

using namespace vtb;

// x (K doubles, device) receives the iterate after steps+1 updates from x = 0;
// x_tmp (K doubles) and bar (2 unsigned + 1 int of scratch, 16 bytes) are
// caller-owned scratch.  Replaces rnn3 + rnn3_update (vtem/neural_network.py:
// 15-128) on the real coefficient system.  Synchronises nothing; an
// exceeded barrier wait is reported by vtb_rnn_coeff_status.
VTB_API int vtb_rnn_coeff(const double* Mr, int64_t ld, const double* br, double* x, double* x_tmp, int K,
                          double dt_alpha, int steps, void* bar, void* stream) {
    VTB_CHECK_ARG(K > 0 && ld >= K && steps >= 0 && Mr && br && x && x_tmp && bar);
    int dev = 0;
    VTB_CUDA_TRY(cudaGetDevice(&dev));
    cudaDeviceProp prop;
    VTB_CUDA_TRY(cudaGetDeviceProperties(&prop, dev));
    int coop = 0;
    VTB_CUDA_TRY(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
    if (!coop) return VTB_CUDA_ERR;
    const int nsm = prop.multiProcessorCount;
    const size_t smem_max = prop.sharedMemPerBlockOptin;
    int rows = (K + nsm - 1) / nsm;
    int blocks = (K + rows - 1) / rows;
    size_t sm = (size_t)K * 8 + (size_t)rows * K * 8;
    int cache = 1;
    if (sm > smem_max) {
        cache = 0;
        sm = (size_t)K * 8;
        VTB_CHECK_ARG(sm <= smem_max);
    }
    VTB_CUDA_TRY(cudaFuncSetAttribute(rnn_coeff_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    int per_sm = 0;
    VTB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, rnn_coeff_kernel, kRnnThreads, sm));
    if (per_sm * nsm < blocks) return VTB_CUDA_ERR;
    cudaStream_t s = as_stream(stream);
    VTB_CUDA_TRY(cudaMemsetAsync(x, 0, (size_t)K * 8, s));
    VTB_CUDA_TRY(cudaMemsetAsync(bar, 0, 16, s));
    const int updates = steps + 1;
    unsigned* b = reinterpret_cast<unsigned*>(bar);
    int* err = reinterpret_cast<int*>(b + 2);
    double* xa = x;
    double* xb = x_tmp;
    unsigned limit = wait_limit(kRnnSpinLimit);
    void* args[] = {(void*)&Mr, (void*)&ld, (void*)&br, (void*)&xa, (void*)&xb, (void*)&K, (void*)&dt_alpha,
                    (void*)&updates, (void*)&rows, (void*)&cache, (void*)&b, (void*)&err, (void*)&limit};
    VTB_CUDA_TRY(cudaLaunchCooperativeKernel((void*)rnn_coeff_kernel, dim3(blocks), dim3(kRnnThreads), args, sm, s));
    // the result is in xa after an even number of updates, else in xb
    if (updates & 1) VTB_CUDA_TRY(cudaMemcpyAsync(x, x_tmp, (size_t)K * 8, cudaMemcpyDeviceToDevice, s));
    return launch_status();
}
