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

#include <cstdlib>

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

// Workspace layout (each piece 256-byte aligned): [w: n doubles][qq: n doubles][info][syevd work].
// The 64-bit cuSOLVER API sizes the eigensolver's workspace (2n^2 doubles at
// n = 25k is beyond the 32-bit interface); its small host workspace is
// allocated on the host per call.
static inline int64_t al256(int64_t x) { return (x + 255) & ~(int64_t)255; }

static cusolverDnParams_t solver_params() {
    static thread_local cusolverDnParams_t p = nullptr;
    if (!p && cusolverDnCreateParams(&p) != CUSOLVER_STATUS_SUCCESS) p = nullptr;
    return p;
}

static int syevd_sizes(cusolverDnHandle_t h, int n, size_t* dev_bytes, size_t* host_bytes) {
    cusolverDnParams_t prm = solver_params();
    if (!prm) return VTB_CUDA_ERR;
    if (cusolverDnXsyevd_bufferSize(h, prm, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, n, CUDA_R_64F, nullptr,
                                    n, CUDA_R_64F, nullptr, CUDA_R_64F, dev_bytes, host_bytes) !=
        CUSOLVER_STATUS_SUCCESS)
        return VTB_CUDA_ERR;
    return VTB_OK;
}

VTB_API int vtb_solve_eq_sym_workspace(int n, int64_t* bytes) {
    VTB_CHECK_ARG(n > 0 && bytes);
    int dev = 0;
    VTB_CUDA_TRY(cudaGetDevice(&dev));
    cusolverDnHandle_t h = solver_handle(dev);
    if (!h) return VTB_CUDA_ERR;
    size_t db = 0, hb = 0;
    int st = syevd_sizes(h, n, &db, &hb);
    if (st) return st;
    *bytes = 2 * al256((int64_t)n * 8) + 256 + al256((int64_t)db);
    return VTB_OK;
}

VTB_API int vtb_solve_eq_sym(double* G, int64_t ld, const double* q, double* c, int n, double rcond, void* work,
                             int64_t work_bytes, int32_t* kept, void* stream) {
    VTB_CHECK_ARG(n > 0 && ld >= n && G && q && c && work);
    VTB_CHECK_ARG(((uintptr_t)work & 255) == 0);
    int dev = 0;
    VTB_CUDA_TRY(cudaGetDevice(&dev));
    cusolverDnHandle_t h = solver_handle(dev);
    if (!h) return VTB_CUDA_ERR;
    size_t db = 0, hb = 0;
    int st = syevd_sizes(h, n, &db, &hb);
    if (st) return st;
    VTB_CHECK_ARG(work_bytes >= 2 * al256((int64_t)n * 8) + 256 + al256((int64_t)db));
    cudaStream_t s = as_stream(stream);
    if (cusolverDnSetStream(h, s) != CUSOLVER_STATUS_SUCCESS) return VTB_CUDA_ERR;
    char* base = reinterpret_cast<char*>(work);
    double* w = reinterpret_cast<double*>(base);
    double* qq = reinterpret_cast<double*>(base + al256((int64_t)n * 8));
    int* info = reinterpret_cast<int*>(base + 2 * al256((int64_t)n * 8));
    void* wk = base + 2 * al256((int64_t)n * 8) + 256;
    void* hwk = hb ? malloc(hb) : nullptr;
    if (hb && !hwk) return VTB_OOM;
    // Row-major symmetric G is its own column-major transpose.  The row-major
    // lower triangle is the column-major upper one.  On exit the column-major
    // eigenvectors (columns) are the rows of the row-major buffer.
    const cusolverStatus_t cs = cusolverDnXsyevd(h, solver_params(), CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER,
                                                 n, CUDA_R_64F, G, ld, CUDA_R_64F, w, CUDA_R_64F, wk, db, hwk, hb, info);
    int hinfo = 0;
    cudaError_t e1 = cudaMemcpyAsync(&hinfo, info, sizeof(int), cudaMemcpyDeviceToHost, s);
    cudaError_t e2 = cudaStreamSynchronize(s);
    free(hwk);
    if (cs != CUSOLVER_STATUS_SUCCESS) return VTB_CUDA_ERR;
    VTB_CUDA_TRY(e1);
    VTB_CUDA_TRY(e2);
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

// ---------------------------------------------------------------------------
// Hermitian K x K solve of the coefficient-space decoder (M a = b).
//   mode 0: pseudoinverse by eigendecomposition (cuSOLVER zheevd), the
//           reference's truncation |w| > rcond * max|w| (same rule as
//           vtb_solve_eq_sym, the eigenvalues being those of the spike Gram);
//   mode 1: Cholesky (zpotrf/zpotrs) with `refine` float64 refinement sweeps
//           against a saved copy of M.  Returns VTB_NOT_CONVERGED when the
//           factorisation fails or its pivots show a condition number beyond
//           1/rcond, in which case the caller falls back to mode 0.
// M is column-major (element (r, c) at c*ld + r), complex interleaved, and is
// overwritten.
namespace vtb {

// The GEMV and truncation kernels take a batch index from blockIdx.y (the
// truncation from blockIdx.x): matrix z at V + z*mstride, vectors at
// x/y + z*vstride (strides 0 for a single system).
__global__ void zgemv_conj_rows_kernel(const double2* __restrict__ V, int64_t ld, const double2* __restrict__ x,
                                       int n, double2* __restrict__ y, int64_t mstride = 0, int64_t vstride = 0) {
    // y[i] = sum_j conj(V[i*ld + j]) x[j]   (V row i = column i of the column-major eigenvector matrix)
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= n) return;
    V += blockIdx.y * mstride;
    x += blockIdx.y * vstride;
    y += blockIdx.y * vstride;
    const double2* row = V + (int64_t)warp * ld;
    double sr = 0.0, si = 0.0;
    for (int j = lane; j < n; j += 32) {
        const double2 v = row[j], b = x[j];
        sr += v.x * b.x + v.y * b.y;
        si += v.x * b.y - v.y * b.x;
    }
    for (int o = 16; o; o >>= 1) {
        sr += __shfl_xor_sync(0xffffffffu, sr, o);
        si += __shfl_xor_sync(0xffffffffu, si, o);
    }
    if (lane == 0) y[warp] = make_double2(sr, si);
}

__global__ void zgemv_cols_kernel(const double2* __restrict__ V, int64_t ld, const double2* __restrict__ x, int n,
                                  double2* __restrict__ y, const double2* __restrict__ b, int subtract,
                                  int64_t mstride = 0, int64_t vstride = 0) {
    // y[j] = sum_i V[i*ld + j] x[i]   (or b[j] - that when subtract)
    __shared__ double2 part[8][33];
    V += blockIdx.y * mstride;
    x += blockIdx.y * vstride;
    y += blockIdx.y * vstride;
    if (b) b += blockIdx.y * vstride;
    const int col = blockIdx.x * 32 + (threadIdx.x & 31);
    const int g = threadIdx.x >> 5;
    double sr = 0.0, si = 0.0;
    if (col < n)
        for (int i = g; i < n; i += 8) {
            const double2 v = V[(int64_t)i * ld + col], w = x[i];
            sr += v.x * w.x - v.y * w.y;
            si += v.x * w.y + v.y * w.x;
        }
    part[g][threadIdx.x & 31] = make_double2(sr, si);
    __syncthreads();
    if (g == 0 && col < n) {
        double tr = 0.0, ti = 0.0;
        for (int k = 0; k < 8; ++k) {
            tr += part[k][threadIdx.x & 31].x;
            ti += part[k][threadIdx.x & 31].y;
        }
        y[col] = subtract ? make_double2(b[col].x - tr, b[col].y - ti) : make_double2(tr, ti);
    }
}

__global__ void ztruncate_kernel(const double* __restrict__ w, double2* __restrict__ qq, int n, double rcond,
                                 int32_t* __restrict__ kept) {
    __shared__ double s0;
    __shared__ int cnt;
    w += (int64_t)blockIdx.x * n;
    qq += (int64_t)blockIdx.x * n;
    if (kept) kept += blockIdx.x;
    if (threadIdx.x == 0) {
        s0 = fmax(fabs(w[0]), fabs(w[n - 1])) * rcond;
        cnt = 0;
    }
    __syncthreads();
    int local = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double s = fabs(w[i]);
        if (s > s0) {
            qq[i] = make_double2(qq[i].x / s, qq[i].y / s);
            ++local;
        } else {
            qq[i] = make_double2(0.0, 0.0);
        }
    }
    atomicAdd(&cnt, local);
    __syncthreads();
    if (threadIdx.x == 0 && kept) *kept = cnt;
}

// pivots of the Cholesky factor: out[0] = min L_ii^2, out[1] = max L_ii^2
__global__ void chol_pivots_kernel(const double2* __restrict__ L, int64_t ld, int n, double* __restrict__ out) {
    __shared__ double smin[32], smax[32];
    double mn = 1e308, mx = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double d = L[(int64_t)i * ld + i].x;
        mn = fmin(mn, d * d);
        mx = fmax(mx, d * d);
    }
    for (int o = 16; o; o >>= 1) {
        mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
        mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    }
    if ((threadIdx.x & 31) == 0) {
        smin[threadIdx.x >> 5] = mn;
        smax[threadIdx.x >> 5] = mx;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < (int)(blockDim.x >> 5); ++k) {
            mn = fmin(mn, smin[k]);
            mx = fmax(mx, smax[k]);
        }
        mn = fmin(mn, smin[0]);
        mx = fmax(mx, smax[0]);
        out[0] = mn;
        out[1] = mx;
    }
}

__global__ void zaxpy_kernel(double2* __restrict__ a, const double2* __restrict__ d, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = make_double2(a[i].x + d[i].x, a[i].y + d[i].y);
}

}  // namespace vtb

// Workspace carve-up of vtb_herm_solve; every piece starts on a 256-byte
// boundary (the complex vectors are read as 16-byte double2).
namespace vtb {
struct HermWork {
    double* w;        // K eigenvalues / pivots
    double2* v1;      // K
    double2* v2;      // K
    int* info;
    double2* Mc;      // K*K copy of M (mode 1)
    cuDoubleComplex* wk;
    int lwork;
};
static inline int64_t align256(int64_t x) { return (x + 255) & ~(int64_t)255; }
static int64_t herm_layout(int K, int mode, int lwork, char* base, HermWork* hw) {
    int64_t off = 0;
    auto take = [&](int64_t bytes) {
        int64_t o = off;
        off = align256(off + bytes);
        return o;
    };
    const int64_t ow = take((int64_t)K * 8);
    const int64_t o1 = take((int64_t)K * 16);
    const int64_t o2 = take((int64_t)K * 16);
    const int64_t oi = take(64);
    const int64_t om = mode == 1 ? take((int64_t)K * K * 16) : 0;
    const int64_t ok = take((int64_t)lwork * 16);
    if (hw && base) {
        hw->w = reinterpret_cast<double*>(base + ow);
        hw->v1 = reinterpret_cast<double2*>(base + o1);
        hw->v2 = reinterpret_cast<double2*>(base + o2);
        hw->info = reinterpret_cast<int*>(base + oi);
        hw->Mc = mode == 1 ? reinterpret_cast<double2*>(base + om) : nullptr;
        hw->wk = reinterpret_cast<cuDoubleComplex*>(base + ok);
        hw->lwork = lwork;
    }
    return off;
}
static int herm_lwork(cusolverDnHandle_t h, int K, int mode, int* lwork) {
    if (mode == 0)
        return cusolverDnZheevd_bufferSize(h, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, K, nullptr, K, nullptr,
                                           lwork) == CUSOLVER_STATUS_SUCCESS ? VTB_OK : VTB_CUDA_ERR;
    return cusolverDnZpotrf_bufferSize(h, CUBLAS_FILL_MODE_LOWER, K, nullptr, K, lwork) == CUSOLVER_STATUS_SUCCESS
               ? VTB_OK : VTB_CUDA_ERR;
}
}  // namespace vtb

VTB_API int vtb_herm_solve_workspace(int K, int mode, int64_t* bytes) {
    VTB_CHECK_ARG(K > 0 && bytes && (mode == 0 || mode == 1));
    int dev = 0;
    VTB_CUDA_TRY(cudaGetDevice(&dev));
    cusolverDnHandle_t h = solver_handle(dev);
    if (!h) return VTB_CUDA_ERR;
    int lwork = 0;
    int st = herm_lwork(h, K, mode, &lwork);
    if (st) return st;
    *bytes = herm_layout(K, mode, lwork, nullptr, nullptr);
    return VTB_OK;
}

VTB_API int vtb_herm_solve(double* M, int64_t ld, const double* b, double* a, int K, double rcond, int mode,
                           int refine, void* work, int64_t work_bytes, int32_t* kept, double* pivots, void* stream) {
    VTB_CHECK_ARG(K > 0 && ld >= K && M && b && a && work && (mode == 0 || mode == 1));
    int64_t need = 0;
    int st = vtb_herm_solve_workspace(K, mode, &need);
    if (st) return st;
    VTB_CHECK_ARG(work_bytes >= need);
    VTB_CHECK_ARG(((uintptr_t)work & 255) == 0 && ((uintptr_t)M & 15) == 0 && ((uintptr_t)b & 15) == 0 &&
                  ((uintptr_t)a & 15) == 0);
    int dev = 0;
    VTB_CUDA_TRY(cudaGetDevice(&dev));
    cusolverDnHandle_t h = solver_handle(dev);
    cudaStream_t s = as_stream(stream);
    if (cusolverDnSetStream(h, s) != CUSOLVER_STATUS_SUCCESS) return VTB_CUDA_ERR;
    int lwork0 = 0;
    st = herm_lwork(h, K, mode, &lwork0);
    if (st) return st;
    HermWork hw;
    herm_layout(K, mode, lwork0, reinterpret_cast<char*>(work), &hw);
    double* w = hw.w;
    double2* v1 = hw.v1;
    double2* v2 = hw.v2;
    int* info = hw.info;
    double2* Mc = hw.Mc;
    cuDoubleComplex* wk = hw.wk;
    const int lwork = hw.lwork;
    cuDoubleComplex* Mz = reinterpret_cast<cuDoubleComplex*>(M);
    const double2* bz = reinterpret_cast<const double2*>(b);
    double2* az = reinterpret_cast<double2*>(a);
    int hinfo = 0;
    if (mode == 0) {
        if (cusolverDnZheevd(h, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, K, Mz, (int)ld, w, wk, lwork, info) !=
            CUSOLVER_STATUS_SUCCESS)
            return VTB_CUDA_ERR;
        double ev[2] = {0, 0};
        VTB_CUDA_TRY(cudaMemcpyAsync(&hinfo, info, sizeof(int), cudaMemcpyDeviceToHost, s));
        VTB_CUDA_TRY(cudaMemcpyAsync(&ev[0], w, 8, cudaMemcpyDeviceToHost, s));
        VTB_CUDA_TRY(cudaMemcpyAsync(&ev[1], w + K - 1, 8, cudaMemcpyDeviceToHost, s));
        VTB_CUDA_TRY(cudaStreamSynchronize(s));
        if (hinfo != 0) return VTB_NOT_CONVERGED;
        if (pivots) {
            pivots[0] = ev[0];
            pivots[1] = ev[1];
        }
        const double2* V = reinterpret_cast<const double2*>(M);  // column c (eigenvector c) at V + c*ld
        zgemv_conj_rows_kernel<<<ceil_div((int64_t)K * 32, 256), 256, 0, s>>>(V, ld, bz, K, v1);  // V^H b
        ztruncate_kernel<<<1, 1024, 0, s>>>(w, v1, K, rcond, kept);
        zgemv_cols_kernel<<<ceil_div(K, 32), 256, 0, s>>>(V, ld, v1, K, az, nullptr, 0);          // V qq
        return launch_status();
    }
    // mode 1: Cholesky + refinement
    VTB_CUDA_TRY(cudaMemcpy2DAsync(Mc, (size_t)K * 16, M, (size_t)ld * 16, (size_t)K * 16, K, cudaMemcpyDeviceToDevice, s));
    if (cusolverDnZpotrf(h, CUBLAS_FILL_MODE_LOWER, K, Mz, (int)ld, wk, lwork, info) != CUSOLVER_STATUS_SUCCESS)
        return VTB_CUDA_ERR;
    chol_pivots_kernel<<<1, 1024, 0, s>>>(reinterpret_cast<const double2*>(M), ld, K, w);
    double hp[2] = {0, 0};
    VTB_CUDA_TRY(cudaMemcpyAsync(&hinfo, info, sizeof(int), cudaMemcpyDeviceToHost, s));
    VTB_CUDA_TRY(cudaMemcpyAsync(hp, w, 16, cudaMemcpyDeviceToHost, s));
    VTB_CUDA_TRY(cudaStreamSynchronize(s));
    if (pivots) {
        pivots[0] = hp[0];
        pivots[1] = hp[1];
    }
    // (max/min pivot) is a lower bound of cond(M): beyond 1/rcond the pseudoinverse would truncate
    if (hinfo != 0 || !(hp[0] > 0.0) || hp[1] / hp[0] * rcond >= 1.0) return VTB_NOT_CONVERGED;
    VTB_CUDA_TRY(cudaMemcpyAsync(az, bz, (size_t)K * 16, cudaMemcpyDeviceToDevice, s));
    if (cusolverDnZpotrs(h, CUBLAS_FILL_MODE_LOWER, K, 1, Mz, (int)ld, reinterpret_cast<cuDoubleComplex*>(az), K,
                         info) != CUSOLVER_STATUS_SUCCESS)
        return VTB_CUDA_ERR;
    for (int it = 0; it < refine; ++it) {
        // r = b - M a with the saved M (column-major: row j of the buffer is column j)
        zgemv_cols_kernel<<<ceil_div(K, 32), 256, 0, s>>>(Mc, K, az, K, v2, bz, 1);
        if (cusolverDnZpotrs(h, CUBLAS_FILL_MODE_LOWER, K, 1, Mz, (int)ld, reinterpret_cast<cuDoubleComplex*>(v2), K,
                             info) != CUSOLVER_STATUS_SUCCESS)
            return VTB_CUDA_ERR;
        zaxpy_kernel<<<ceil_div(K, 256), 256, 0, s>>>(az, v2, K);
    }
    if (kept) VTB_CUDA_TRY(cudaMemsetAsync(kept, 0xff, sizeof(int32_t), s));
    return launch_status();
}

// Solve with a matrix already factorised by vtb_herm_solve(mode 1): x = M^-1 x
// in place (two triangular solves).  Used by the refinement sweeps.
VTB_API int vtb_herm_potrs(const double* Mfac, int64_t ld, double* x, int K, void* work, int64_t work_bytes,
                           void* stream) {
    VTB_CHECK_ARG(K > 0 && ld >= K && Mfac && x && work && ((uintptr_t)work & 255) == 0 && work_bytes >= 256);
    int dev = 0;
    VTB_CUDA_TRY(cudaGetDevice(&dev));
    cusolverDnHandle_t h = solver_handle(dev);
    if (!h) return VTB_CUDA_ERR;
    cudaStream_t s = as_stream(stream);
    if (cusolverDnSetStream(h, s) != CUSOLVER_STATUS_SUCCESS) return VTB_CUDA_ERR;
    int* info = reinterpret_cast<int*>(work);
    if (cusolverDnZpotrs(h, CUBLAS_FILL_MODE_LOWER, K, 1, reinterpret_cast<const cuDoubleComplex*>(Mfac), (int)ld,
                         reinterpret_cast<cuDoubleComplex*>(x), K, info) != CUSOLVER_STATUS_SUCCESS)
        return VTB_CUDA_ERR;
    return launch_status();
}

// Batched Cholesky solve of `batch` Hermitian K x K systems (one group of
// equally sized clips): cusolverDnZpotrfBatched then ZpotrsBatched.  Mptrs
// and bptrs are DEVICE arrays of device pointers (column-major M, lower
// factor in place; b overwritten by the solution).  infos (device, batch
// ints) receives each clip's status: the factorisation's own, or -1 when the
// pivot spread shows a condition number beyond 1/rcond (the same test as
// vtb_herm_solve mode 1); a nonzero entry means that clip needs the
// eigen-pseudoinverse instead (its b is then meaningless).
namespace vtb {
__global__ void batched_pivot_check_kernel(double2* const* __restrict__ Mptrs, int64_t ld, int K, double rcond,
                                           int32_t* __restrict__ infos) {
    __shared__ double smin[32], smax[32];
    const double2* L = Mptrs[blockIdx.x];
    double mn = 1e308, mx = 0.0;
    for (int i = threadIdx.x; i < K; i += blockDim.x) {
        const double d = L[(int64_t)i * ld + i].x;
        mn = fmin(mn, d * d);
        mx = fmax(mx, d * d);
    }
    for (int o = 16; o; o >>= 1) {
        mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
        mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    }
    if ((threadIdx.x & 31) == 0) {
        smin[threadIdx.x >> 5] = mn;
        smax[threadIdx.x >> 5] = mx;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < (int)(blockDim.x >> 5); ++k) {
            mn = fmin(mn, smin[k]);
            mx = fmax(mx, smax[k]);
        }
        if (infos[blockIdx.x] == 0 && (!(mn > 0.0) || mx / mn * rcond >= 1.0)) infos[blockIdx.x] = -1;
    }
}
}  // namespace vtb

VTB_API int vtb_herm_chol_batched(double** Mptrs, int64_t ld, double** bptrs, int K, int batch, double rcond,
                                  int32_t* infos, int32_t* solve_info, void* stream) {
    VTB_CHECK_ARG(K > 0 && ld >= K && batch > 0 && Mptrs && bptrs && infos && solve_info);
    int dev = 0;
    VTB_CUDA_TRY(cudaGetDevice(&dev));
    cusolverDnHandle_t h = solver_handle(dev);
    if (!h) return VTB_CUDA_ERR;
    cudaStream_t s = as_stream(stream);
    if (cusolverDnSetStream(h, s) != CUSOLVER_STATUS_SUCCESS) return VTB_CUDA_ERR;
    if (cusolverDnZpotrfBatched(h, CUBLAS_FILL_MODE_LOWER, K, reinterpret_cast<cuDoubleComplex**>(Mptrs), (int)ld,
                                infos, batch) != CUSOLVER_STATUS_SUCCESS)
        return VTB_CUDA_ERR;
    batched_pivot_check_kernel<<<batch, 256, 0, s>>>(reinterpret_cast<double2* const*>(Mptrs), ld, K, rcond, infos);
    int st = launch_status();
    if (st) return st;
    if (cusolverDnZpotrsBatched(h, CUBLAS_FILL_MODE_LOWER, K, 1, reinterpret_cast<cuDoubleComplex**>(Mptrs), (int)ld,
                                reinterpret_cast<cuDoubleComplex**>(bptrs), K, solve_info, batch) !=
        CUSOLVER_STATUS_SUCCESS)
        return VTB_CUDA_ERR;
    return launch_status();
}

// Batched pseudoinverse of Hermitian systems of one size K by
// eigendecomposition (cuSOLVER XsyevBatched): for every matrix z,
// a_z = V diag(1/w_i if |w_i| > rcond max|w| else 0) V^H b_z, the truncation
// of vtb_herm_solve mode 0.  The matrices are contiguous, column-major, at
// stride ld*K; b and a at stride K.  M is overwritten by the eigenvectors.
namespace vtb {
struct PinvBatchedWork {
    double* w;        // batch*K eigenvalues
    double2* v1;      // batch*K
    int* info;        // batch
    void* wk;
    size_t wk_bytes;
};
static int pinv_batched_sizes(cusolverDnHandle_t h, int K, int64_t ld, int batch, size_t* db, size_t* hb) {
    cusolverDnParams_t prm = solver_params();
    if (!prm) return VTB_CUDA_ERR;
    if (cusolverDnXsyevBatched_bufferSize(h, prm, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, K, CUDA_C_64F,
                                          nullptr, ld, CUDA_R_64F, nullptr, CUDA_C_64F, db, hb, batch) !=
        CUSOLVER_STATUS_SUCCESS)
        return VTB_CUDA_ERR;
    return VTB_OK;
}
static int64_t pinv_batched_layout(int K, int batch, size_t db, char* base, PinvBatchedWork* pw) {
    int64_t off = 0;
    auto take = [&](int64_t bytes) {
        int64_t o = off;
        off = al256(off + bytes);
        return o;
    };
    const int64_t ow = take((int64_t)batch * K * 8);
    const int64_t o1 = take((int64_t)batch * K * 16);
    const int64_t oi = take((int64_t)batch * 4);
    const int64_t ok = take((int64_t)db);
    if (pw && base) {
        pw->w = reinterpret_cast<double*>(base + ow);
        pw->v1 = reinterpret_cast<double2*>(base + o1);
        pw->info = reinterpret_cast<int*>(base + oi);
        pw->wk = base + ok;
        pw->wk_bytes = db;
    }
    return off;
}
}  // namespace vtb

VTB_API int vtb_herm_pinv_batched_workspace(int K, int batch, int64_t* bytes) {
    VTB_CHECK_ARG(K > 0 && batch > 0 && bytes);
    int dev = 0;
    VTB_CUDA_TRY(cudaGetDevice(&dev));
    cusolverDnHandle_t h = solver_handle(dev);
    if (!h) return VTB_CUDA_ERR;
    size_t db = 0, hb = 0;
    int st = pinv_batched_sizes(h, K, K, batch, &db, &hb);
    if (st) return st;
    *bytes = pinv_batched_layout(K, batch, db, nullptr, nullptr);
    return VTB_OK;
}

VTB_API int vtb_herm_pinv_batched(double* M, const double* b, double* a, int K, int batch, double rcond, void* work,
                                  int64_t work_bytes, int32_t* kept, int32_t* infos, void* stream) {
    VTB_CHECK_ARG(K > 0 && batch > 0 && M && b && a && work && infos);
    VTB_CHECK_ARG(((uintptr_t)work & 255) == 0 && ((uintptr_t)M & 15) == 0 && ((uintptr_t)b & 15) == 0 &&
                  ((uintptr_t)a & 15) == 0);
    int dev = 0;
    VTB_CUDA_TRY(cudaGetDevice(&dev));
    cusolverDnHandle_t h = solver_handle(dev);
    if (!h) return VTB_CUDA_ERR;
    size_t db = 0, hb = 0;
    int st = pinv_batched_sizes(h, K, K, batch, &db, &hb);
    if (st) return st;
    VTB_CHECK_ARG(work_bytes >= pinv_batched_layout(K, batch, db, nullptr, nullptr));
    PinvBatchedWork pw;
    pinv_batched_layout(K, batch, db, reinterpret_cast<char*>(work), &pw);
    cudaStream_t s = as_stream(stream);
    if (cusolverDnSetStream(h, s) != CUSOLVER_STATUS_SUCCESS) return VTB_CUDA_ERR;
    void* hwk = hb ? malloc(hb) : nullptr;
    if (hb && !hwk) return VTB_OOM;
    const cusolverStatus_t cs = cusolverDnXsyevBatched(h, solver_params(), CUSOLVER_EIG_MODE_VECTOR,
                                                       CUBLAS_FILL_MODE_LOWER, K, CUDA_C_64F, M, K, CUDA_R_64F, pw.w,
                                                       CUDA_C_64F, pw.wk, pw.wk_bytes, hwk, hb, pw.info, batch);
    // the host workspace must outlive the call's use of it
    cudaError_t e1 = cudaStreamSynchronize(s);
    free(hwk);
    if (cs != CUSOLVER_STATUS_SUCCESS) return VTB_CUDA_ERR;
    VTB_CUDA_TRY(e1);
    VTB_CUDA_TRY(cudaMemcpyAsync(infos, pw.info, (size_t)batch * 4, cudaMemcpyDeviceToDevice, s));
    const double2* V = reinterpret_cast<const double2*>(M);
    const int64_t ms = (int64_t)K * K;
    zgemv_conj_rows_kernel<<<dim3(ceil_div((int64_t)K * 32, 256), batch), 256, 0, s>>>(
        V, K, reinterpret_cast<const double2*>(b), K, pw.v1, ms, K);
    ztruncate_kernel<<<batch, 1024, 0, s>>>(pw.w, pw.v1, K, rcond, kept);
    zgemv_cols_kernel<<<dim3(ceil_div(K, 32), batch), 256, 0, s>>>(V, K, pw.v1, K, reinterpret_cast<double2*>(a),
                                                                 nullptr, 0, ms, K);
    return launch_status();
}
