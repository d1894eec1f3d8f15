// Pseudoinverse solve of G c = q (plain float64 path) and the RNN decoder.
//
//  vtb_solve_eq_sym: solve_eq_sym (vtem/utils/linalg.py:591-631) computes
//      c = U diag(1/s_i if s_i > rcond*s_0 else 0) U^H q from an SVD of the
//      symmetric Gram (CULA gesvd).  For a symmetric matrix the singular
//      values are |eigenvalues|, so the same c comes from the symmetric
//      eigendecomposition G = V diag(w) V^T (cuSOLVER dsyevd, the vendor
//      library in CULA's place) and the reference's truncation rule applied
//      to |w| (sq_Kernel, linalg.py:791-833).  The two GEMVs around the
//      truncation are hand-written, one warp per row.
//  vtb_rnn: rnn3 (vtem/neural_network.py:15-99): steps+1 updates
//      c <- c + dt*alpha*(q - G c) from c = 0, each one fused kernel (row
//      dot products of G with the previous iterate, then the update), double
//      buffered so that every row reads the same previous c.
#include <cusolverDn.h>

#include "common.cuh"

namespace vtb {

static cusolverDnHandle_t solver_handle(int dev) {
    static thread_local cusolverDnHandle_t h[64] = {nullptr};
    if (dev < 0 || dev >= 64) return nullptr;
    if (!h[dev]) {
        if (cusolverDnCreate(&h[dev]) != CUSOLVER_STATUS_SUCCESS) h[dev] = nullptr;
    }
    return h[dev];
}

// y[i] = sum_j A[i*lda + j] x[j] (trans = 0)   or   y[j] = sum_i A[i*lda+j] x[i] (trans = 1)
__global__ void gemv_rows_kernel(const double* __restrict__ A, int64_t lda, const double* __restrict__ x, int n,
                                 double* __restrict__ y) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= n) return;
    const double* row = A + (int64_t)warp * lda;
    double s = 0.0;
    for (int j = lane; j < n; j += 32) s = fma(row[j], x[j], s);
#pragma unroll
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) y[warp] = s;
}

// y = A^T x for row-major A: block of 32 columns x 8 row-groups, reduced in smem
__global__ void gemv_cols_kernel(const double* __restrict__ A, int64_t lda, const double* __restrict__ x, int n,
                                 double* __restrict__ y) {
    __shared__ double part[8][33];
    const int col = blockIdx.x * 32 + (threadIdx.x & 31);
    const int g = threadIdx.x >> 5;
    double s = 0.0;
    if (col < n)
        for (int i = g; i < n; i += 8) s = fma(A[(int64_t)i * lda + col], x[i], s);
    part[g][threadIdx.x & 31] = s;
    __syncthreads();
    if (g == 0 && col < n) {
        double t = 0.0;
        for (int k = 0; k < 8; ++k) t += part[k][threadIdx.x & 31];
        y[col] = t;
    }
}

// qq[i] = |w_i| > rcond*max|w| ? qq[i]/|w_i| : 0, counting the kept values
__global__ void truncate_kernel(const double* __restrict__ w, double* __restrict__ qq, int n, double rcond,
                                int32_t* __restrict__ kept) {
    __shared__ double s0;
    __shared__ int cnt;
    if (threadIdx.x == 0) {
        s0 = fmax(fabs(w[0]), fabs(w[n - 1])) * rcond;  // eigenvalues come sorted ascending
        cnt = 0;
    }
    __syncthreads();
    int local = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double s = fabs(w[i]);
        if (s > s0) {
            qq[i] = qq[i] / s;
            ++local;
        } else {
            qq[i] = 0.0;
        }
    }
    atomicAdd(&cnt, local);
    __syncthreads();
    if (threadIdx.x == 0 && kept) *kept = cnt;
}

__global__ void rnn_step_kernel(const double* __restrict__ G, int64_t ld, const double* __restrict__ q,
                                const double* __restrict__ c_old, double* __restrict__ c_new, double* __restrict__ y,
                                int n, double dt_alpha) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= n) return;
    const double* row = G + (int64_t)warp * ld;
    double s = 0.0;
    for (int j = lane; j < n; j += 32) s = fma(row[j], c_old[j], s);
#pragma unroll
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) {
        const double dy = q[warp] - s;
        c_new[warp] = c_old[warp] + dt_alpha * dy;
        if (y) y[warp] = dy;
    }
}

__global__ void sumsq_kernel(const double* __restrict__ v, int n, double* __restrict__ out) {
    __shared__ double part[32];
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s = fma(v[i], v[i], s);
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        s = threadIdx.x < (blockDim.x >> 5) ? part[threadIdx.x] : 0.0;
        for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (threadIdx.x == 0) *out = s;
    }
}

}  // namespace vtb

using namespace vtb;

// Workspace layout: [w: n doubles][qq: n doubles][info: 8 bytes][syevd work]
VTB_API int vtb_solve_eq_sym_workspace(int n, int64_t* bytes) {
    VTB_CHECK_ARG(n > 0 && bytes);
    int dev = 0;
    VTB_CUDA_TRY(cudaGetDevice(&dev));
    cusolverDnHandle_t h = solver_handle(dev);
    if (!h) return VTB_CUDA_ERR;
    int lwork = 0;
    if (cusolverDnDsyevd_bufferSize(h, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, n, nullptr, n, nullptr,
                                    &lwork) != CUSOLVER_STATUS_SUCCESS)
        return VTB_CUDA_ERR;
    *bytes = (int64_t)(2 * (int64_t)n + 1) * 8 + (int64_t)lwork * 8 + 256;
    return VTB_OK;
}

VTB_API int vtb_solve_eq_sym(double* G, int64_t ld, const double* q, double* c, int n, double rcond, void* work,
                             int64_t work_bytes, int32_t* kept, void* stream) {
    VTB_CHECK_ARG(n > 0 && ld >= n && G && q && c && work);
    int64_t need = 0;
    int st = vtb_solve_eq_sym_workspace(n, &need);
    if (st) return st;
    VTB_CHECK_ARG(work_bytes >= need);
    int dev = 0;
    VTB_CUDA_TRY(cudaGetDevice(&dev));
    cusolverDnHandle_t h = solver_handle(dev);
    cudaStream_t s = as_stream(stream);
    if (cusolverDnSetStream(h, s) != CUSOLVER_STATUS_SUCCESS) return VTB_CUDA_ERR;
    double* w = reinterpret_cast<double*>(work);
    double* qq = w + n;
    int* info = reinterpret_cast<int*>(qq + n);
    double* wk = reinterpret_cast<double*>(reinterpret_cast<char*>(info) + 8);
    const int lwork = (int)((need - (int64_t)(2 * (int64_t)n + 1) * 8 - 256) / 8);
    // Row-major symmetric G is its own column-major transpose.  The row-major
    // lower triangle is the column-major upper one.  On exit the column-major
    // eigenvectors (columns) are the rows of the row-major buffer.
    if (cusolverDnDsyevd(h, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, n, G, (int)ld, w, wk, lwork, info) !=
        CUSOLVER_STATUS_SUCCESS)
        return VTB_CUDA_ERR;
    int hinfo = 0;
    VTB_CUDA_TRY(cudaMemcpyAsync(&hinfo, info, sizeof(int), cudaMemcpyDeviceToHost, s));
    VTB_CUDA_TRY(cudaStreamSynchronize(s));
    if (hinfo != 0) return VTB_NOT_CONVERGED;
    const int blocks = ceil_div((int64_t)n * 32, 256);
    gemv_rows_kernel<<<blocks, 256, 0, s>>>(G, ld, q, n, qq);  // qq = V^T q
    truncate_kernel<<<1, 1024, 0, s>>>(w, qq, n, rcond, kept);
    gemv_cols_kernel<<<ceil_div(n, 32), 256, 0, s>>>(G, ld, qq, n, c);  // c = V qq
    return launch_status();
}

VTB_API int vtb_rnn(const double* G, int64_t ld, const double* q, double* c, double* y, double* c_tmp, int n,
                    double dt_alpha, int steps, double* ynorm_trace, int trace_every, void* stream) {
    VTB_CHECK_ARG(n > 0 && ld >= n && steps >= 0 && G && q && c && c_tmp);
    cudaStream_t s = as_stream(stream);
    VTB_CUDA_TRY(cudaMemsetAsync(c, 0, sizeof(double) * n, s));
    double* cur = c;
    double* nxt = c_tmp;
    const int blocks = ceil_div((int64_t)n * 32, 256);
    int traced = 0;
    for (int i = 0; i <= steps; ++i) {
        rnn_step_kernel<<<blocks, 256, 0, s>>>(G, ld, q, cur, nxt, y, n, dt_alpha);
        if (ynorm_trace && y && trace_every > 0 && i % trace_every == 0)
            sumsq_kernel<<<1, 1024, 0, s>>>(y, n, ynorm_trace + traced++);
        double* t = cur;
        cur = nxt;
        nxt = t;
    }
    if (cur != c) VTB_CUDA_TRY(cudaMemcpyAsync(c, cur, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    return launch_status();
}
