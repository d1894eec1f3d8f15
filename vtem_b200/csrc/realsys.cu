// Real form of the coefficient-space system.
//
// The video is real, so its Dirichlet coefficients are Hermitian-symmetric:
// with the complex index j = s*Kt + (m + Mt) (s over the ascending storage
// indices of the spatial ellipse, which is symmetric about its centre), the
// mirrored index (-mx, -my, -m) is jb = K-1-j and a[jb] = conj(a[j]).  The
// system M a = b keeps that symmetry (M[jb][kb] = conj(M[j][k]) because
// Ds[n][-s] = conj(Ds[n][s]) for a real RF and T_k(-m) = conj(T_k(m))).  On
// the Hermitian-symmetric vectors the unitary change of variables
//     x_j = sqrt2 Re a_j,  x_{h+1+j} = sqrt2 Im a_j   (j < h = (K-1)/2),
//     x_h = a_h                                       (the centre, real)
// turns M a = b into a REAL symmetric K x K system Mr x = br with the same
// eigenvalues (the reference's truncation rule picks the same subspace), at a
// quarter of the arithmetic of the complex factorisation or eigensolver and
// half the storage.  With A = M[j][k], B = M[j][kb] (parts p, q of the real
// row/column indices; 0 = real part or centre, 1 = imaginary part):
//     Mr = s_r s_c * { A.re + B.re,  -A.im + B.im,  A.im + B.im,  A.re - B.re }
// for (p, q) = (0,0), (0,1), (1,0), (1,1), with s = 1/sqrt2 on the centre
// row/column and 1 elsewhere.
//
// Factorisations (cuSOLVER, the vendor library for dense LAPACK; the decoder
// keeps everything else in these kernels):
//   mode 1: float64 Cholesky (dpotrf) of a float64 Mr;
//   mode 2: float32 Cholesky (spotrf) of a float32 Mr (the mixed-precision
//           path: the tensor-core Gram and a float32 factor, with float64
//           refinement sweeps against the exact residual).
// Neither synchronises: a device flag receives 1 when the factorisation fails
// and 2 when the spread of the squared pivots, a lower bound of cond(Mr),
// reaches 1/rcond (the pseudoinverse might then truncate), so that a
// sequence of launches can be captured and checked once at its end.
#include <cusolverDn.h>

#include <algorithm>
#include <cstdlib>

#include "common.cuh"

namespace vtb {

constexpr double kInvSqrt2 = 0.70710678118654752440;
constexpr double kSqrt2 = 1.41421356237309504880;

// complex index and part of real index R (h = (K-1)/2)
__device__ __forceinline__ void real_split(int R, int h, int& j, int& part) {
    if (R <= h) {
        j = R;
        part = 0;
    } else {
        j = R - h - 1;
        part = 1;
    }
}

__device__ __forceinline__ double real_entry(double2 A, double2 B, int p, int q) {
    if (p == 0) return q == 0 ? A.x + B.x : -A.y + B.y;
    return q == 0 ? A.y + B.y : A.x - B.x;
}

// Element M[j][k] of the Hermitian M from the tensor-core Gram output
// C[(2p + pa) * ldc + 2u + pw] = sum_n {a.re, a.im}[pa] {W.re, W.im}[pw] for
// the pairs p of spatial indices s <= s' and the upper-triangular temporal
// entries u = (m, m'), m <= m' (both in row-major upper-triangular order):
// sum a W for m <= m', sum a conj(W[m'][m]) for m > m' (W_n is Hermitian).
// KT > 0: the temporal order is a compile-time constant (the divisions by
// Kt become multiply-shifts); KT == 0: Kt at run time
template <int KT>
__device__ __forceinline__ double2 gram_from_pairs(const float* __restrict__ C, int64_t ldc, int Ks, int Kt_rt, int j,
                                                   int k) {
    const int Kt = KT > 0 ? KT : Kt_rt;
    int s = j / Kt, m = j - s * Kt, s2 = k / Kt, m2 = k - s2 * Kt;
    bool conj = false;
    if (s > s2) {
        int t = s; s = s2; s2 = t;
        t = m; m = m2; m2 = t;
        conj = true;
    }
    const int64_t p = (int64_t)s * Ks - (int64_t)s * (s - 1) / 2 + (s2 - s);
    const bool lower = m > m2;
    const int ma = lower ? m2 : m, mb = lower ? m : m2;
    const int u = ma * Kt - ma * (ma - 1) / 2 + (mb - ma);
    const float* c = C + (2 * p) * ldc + 2 * u;
    const double rr = __ldg(c), ri = __ldg(c + 1), ir = __ldg(c + ldc), ii = __ldg(c + ldc + 1);
    const double re = lower ? rr + ii : rr - ii;
    const double im = lower ? ir - ri : ri + ir;
    return make_double2(re, conj ? -im : im);
}

// Mr from the tensor-core Gram: one block row of threads per real row R,
// one thread per complex column k <= h, which reads M[j][k] and M[j][K-1-k]
// once and writes both real columns they feed (k and h+1+k).
template <typename OutT, int KT>
__global__ void __launch_bounds__(256) real_scatter_kernel(const float* __restrict__ C, int64_t ldc, int Ks, int Kt,
                                                           OutT* __restrict__ Mr, int64_t ldr) {
    const int K = Ks * Kt, h = (K - 1) / 2;
    const int R = blockIdx.y;
    int j, p;
    real_split(R, h, j, p);
    OutT* row = Mr + (int64_t)R * ldr;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k <= h; k += gridDim.x * blockDim.x) {
        const double2 A = gram_from_pairs<KT>(C, ldc, Ks, Kt, j, k);
        const double2 B = gram_from_pairs<KT>(C, ldc, Ks, Kt, j, K - 1 - k);
        double v0 = real_entry(A, B, p, 0);
        if (R == h) v0 *= kInvSqrt2;
        if (k == h) v0 *= kInvSqrt2;
        row[k] = (OutT)v0;
        if (k < h) {
            double v1 = real_entry(A, B, p, 1);
            if (R == h) v1 *= kInvSqrt2;
            row[h + 1 + k] = (OutT)v1;
        }
    }
}

template <typename OutT>
static void launch_real_scatter(const float* C, int64_t ldc, int Ks, int Kt, OutT* Mr, int64_t ldr, dim3 grid,
                                cudaStream_t s) {
    switch (Kt) {
        case 7: real_scatter_kernel<OutT, 7><<<grid, 256, 0, s>>>(C, ldc, Ks, Kt, Mr, ldr); break;
        case 9: real_scatter_kernel<OutT, 9><<<grid, 256, 0, s>>>(C, ldc, Ks, Kt, Mr, ldr); break;
        case 11: real_scatter_kernel<OutT, 11><<<grid, 256, 0, s>>>(C, ldc, Ks, Kt, Mr, ldr); break;
        case 13: real_scatter_kernel<OutT, 13><<<grid, 256, 0, s>>>(C, ldc, Ks, Kt, Mr, ldr); break;
        case 15: real_scatter_kernel<OutT, 15><<<grid, 256, 0, s>>>(C, ldc, Ks, Kt, Mr, ldr); break;
        case 17: real_scatter_kernel<OutT, 17><<<grid, 256, 0, s>>>(C, ldc, Ks, Kt, Mr, ldr); break;
        default: real_scatter_kernel<OutT, 0><<<grid, 256, 0, s>>>(C, ldc, Ks, Kt, Mr, ldr); break;
    }
}

// From the complex column-major M (element (j, k) at k*ldm + j).
template <typename OutT>
__global__ void __launch_bounds__(256) realify_kernel(const double2* __restrict__ M, int64_t ldm, int K,
                                                      OutT* __restrict__ Mr, int64_t ldr) {
    const int h = (K - 1) / 2;
    const int64_t total = (int64_t)K * K;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int R = (int)(i / K), Q = (int)(i - (int64_t)R * K);
        int j, p, k, q;
        real_split(R, h, j, p);
        real_split(Q, h, k, q);
        const double2 A = M[(int64_t)k * ldm + j];
        const double2 B = M[(int64_t)(K - 1 - k) * ldm + j];
        double v = real_entry(A, B, p, q);
        if (R == h) v *= kInvSqrt2;
        if (Q == h) v *= kInvSqrt2;
        Mr[(int64_t)R * ldr + Q] = (OutT)v;
    }
}

// br from the Hermitian-symmetric complex b (batch index from blockIdx.y)
__global__ void realify_vec_kernel(const double2* __restrict__ b, int K, double* __restrict__ br) {
    const int h = (K - 1) / 2;
    b += (int64_t)blockIdx.y * K;
    br += (int64_t)blockIdx.y * K;
    for (int R = blockIdx.x * blockDim.x + threadIdx.x; R < K; R += gridDim.x * blockDim.x) {
        if (R < h) br[R] = kSqrt2 * b[R].x;
        else if (R == h) br[R] = b[h].x;
        else br[R] = kSqrt2 * b[R - h - 1].y;
    }
}

// a (=, or += when accumulate) the Hermitian-symmetric complex vector of x
__global__ void unrealify_vec_kernel(const double* __restrict__ x, int K, double2* __restrict__ a, int accumulate) {
    const int h = (K - 1) / 2;
    x += (int64_t)blockIdx.y * K;
    a += (int64_t)blockIdx.y * K;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j <= h; j += gridDim.x * blockDim.x) {
        if (j == h) {
            const double2 v = make_double2(x[h], 0.0);
            a[h] = accumulate ? make_double2(a[h].x + v.x, a[h].y) : v;
        } else {
            const double2 v = make_double2(x[j] * kInvSqrt2, x[h + 1 + j] * kInvSqrt2);
            const int jb = K - 1 - j;
            if (accumulate) {
                a[j] = make_double2(a[j].x + v.x, a[j].y + v.y);
                a[jb] = make_double2(a[jb].x + v.x, a[jb].y - v.y);
            } else {
                a[j] = v;
                a[jb] = make_double2(v.x, -v.y);
            }
        }
    }
}

__global__ void f64_to_f32_kernel(const double* __restrict__ x, float* __restrict__ y, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] = (float)x[i];
}
__global__ void f32_to_f64_kernel(const float* __restrict__ x, double* __restrict__ y, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] = (double)x[i];
}
__global__ void daxpy1_kernel(double* __restrict__ y, const double* __restrict__ x, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] += x[i];
}

// Squared pivots of a Cholesky factor (diagonal of L, row-major or
// column-major alike) -> piv[0] = min, piv[1] = max; flag = 1 if the
// factorisation reported a failure, 2 if max/min * rcond >= 1.
template <typename T>
__device__ void pivot_flag_body(const T* __restrict__ L, int64_t ld, int K, const int* __restrict__ info,
                                double rcond, double* __restrict__ piv, int32_t* __restrict__ flag) {
    __shared__ double smin[32], smax[32];
    double mn = 1e308, mx = 0.0;
    for (int i = threadIdx.x; i < K; i += blockDim.x) {
        const double d = (double)L[(int64_t)i * ld + i];
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
        if (piv) {
            piv[0] = mn;
            piv[1] = mx;
        }
        int f = 0;
        if (*info != 0 || !(mn > 0.0)) f = 1;
        else if (mx / mn * rcond >= 1.0) f = 2;
        *flag = f;
    }
}

template <typename T>
__global__ void pivot_flag_kernel(const T* __restrict__ L, int64_t ld, int K, const int* __restrict__ info,
                                  double rcond, double* __restrict__ piv, int32_t* __restrict__ flag) {
    pivot_flag_body<T>(L, ld, K, info, rcond, piv, flag);
}

// out = ||dx|| / ||x|| (the relative size of a refinement correction)
__global__ void norm_ratio_kernel(const double* __restrict__ dx, const double* __restrict__ x, int n,
                                  double* __restrict__ out) {
    __shared__ double sd[32], sx[32];
    double a = 0.0, b = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        a = fma(dx[i], dx[i], a);
        b = fma(x[i], x[i], b);
    }
    for (int o = 16; o; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
    }
    if ((threadIdx.x & 31) == 0) {
        sd[threadIdx.x >> 5] = a;
        sx[threadIdx.x >> 5] = b;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < (int)(blockDim.x >> 5); ++k) {
            a += sd[k];
            b += sx[k];
        }
        *out = sqrt(a) / fmax(sqrt(b), 1e-300);
    }
}

static cusolverDnHandle_t real_solver_handle(int dev) {
    static thread_local cusolverDnHandle_t h[64] = {nullptr};
    if (dev < 0 || dev >= 64) return nullptr;
    if (!h[dev]) {
        if (cusolverDnCreate(&h[dev]) != CUSOLVER_STATUS_SUCCESS) h[dev] = nullptr;
    }
    return h[dev];
}

static int64_t al256r(int64_t x) { return (x + 255) & ~(int64_t)255; }

// ------------------------------------------------------------------ float32 triangular solves
// x = L^-T L^-1 x for the lower float32 Cholesky factor L (column-major,
// element (i, j) at j*ld + i, as spotrf leaves it), for BATCHES of systems:
// one CTA of 1024 threads solves one system with the right-hand side in
// shared memory (many systems keep every SM busy; a single system goes to
// the multi-CTA trsv_flags_kernel below, since one CTA is bound by one SM's
// share of L2 bandwidth), in 32-wide block steps:
//   forward  (L y = b):  y_J = Dinv_J r_J (one warp), then every row below
//            the block subtracts L(i, J) y_J (the thread's rows of column
//            block J are loaded before the block barrier, hiding L2 latency);
//   backward (L^T x = y): warp w forms the dot product of column J*32+w below
//            the block with the solved tail, then x_J = Dinv_J^T (y_J - s).
// Dinv_J = L_JJ^-1 (32 x 32, row-major) is formed once per factorisation by
// diag_inv_batched_kernel.  Every read of L is a coalesced column segment.
constexpr int kTrsvThreads = 1024;
constexpr int kTrsvPrefetchRows = 1;

// One warp per diagonal block: lane c solves L_JJ X[:, c] = e_c; padding
// beyond K is the identity.
__device__ void diag_inv_body(const float* __restrict__ L, int64_t ld, int K, float* __restrict__ Dinv) {
    __shared__ float sL[4][32][33];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int J = blockIdx.x * 4 + w;
    const int nt = (K + 31) >> 5;
    if (J >= nt) return;
    const int base = J * 32;
    for (int r = 0; r < 32; ++r) {
        const int gr = base + r, gc = base + lane;
        float v = 0.f;
        if (gr < K && gc < K) {
            if (lane <= r) v = L[(int64_t)gc * ld + gr];
        } else if (r == lane) {
            v = 1.f;
        }
        sL[w][r][lane] = v;
    }
    __syncwarp();
    float X[32];
#pragma unroll
    for (int r = 0; r < 32; ++r) {
        float s = (r == lane) ? 1.f : 0.f;
#pragma unroll
        for (int k = 0; k < r; ++k) s = fmaf(-sL[w][r][k], X[k], s);
        X[r] = s / sL[w][r][r];
    }
#pragma unroll
    for (int r = 0; r < 32; ++r) Dinv[(int64_t)J * 1024 + r * 32 + lane] = X[r];
}


// Solves in place on the float32 vector r (shared memory, K entries); part
// is 32 floats of shared scratch.  Requires blockDim.x == kTrsvThreads.
__device__ void trsv_pair(const float* __restrict__ L, int64_t ld, const float* __restrict__ Dinv, int K,
                          float* __restrict__ r, float* __restrict__ part) {
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    const int nt = (K + 31) >> 5;
    // forward: L y = b
    for (int J = 0; J < nt; ++J) {
        const int c0 = J * 32, rs = c0 + 32;
        float Lr[kTrsvPrefetchRows][32];
#pragma unroll
        for (int m = 0; m < kTrsvPrefetchRows; ++m) {
            const int i = rs + t + m * kTrsvThreads;
            if (i < K) {
#pragma unroll
                for (int k = 0; k < 32; ++k) Lr[m][k] = L[(int64_t)(c0 + k) * ld + i];
            }
        }
        if (w == 0) {
            const float* D = Dinv + (int64_t)J * 1024 + lane * 32;
            float acc = 0.f;
#pragma unroll
            for (int k = 0; k < 32; ++k) {
                const float rk = (c0 + k < K) ? r[c0 + k] : 0.f;
                acc = fmaf(D[k], rk, acc);
            }
            __syncwarp();
            if (c0 + lane < K) r[c0 + lane] = acc;
        }
        __syncthreads();
        // rows below the block exist only when c0 + 32 <= K - 1, so every
        // column of the block is in range here
#pragma unroll
        for (int m = 0; m < kTrsvPrefetchRows; ++m) {
            const int i = rs + t + m * kTrsvThreads;
            if (i < K) {
                float s = 0.f;
#pragma unroll
                for (int k = 0; k < 32; ++k) s = fmaf(Lr[m][k], r[c0 + k], s);
                r[i] -= s;
            }
        }
        for (int i = rs + t + kTrsvPrefetchRows * kTrsvThreads; i < K; i += kTrsvThreads) {
            float s = 0.f;
            for (int k = 0; k < 32; ++k) s = fmaf(L[(int64_t)(c0 + k) * ld + i], r[c0 + k], s);
            r[i] -= s;
        }
        __syncthreads();
    }
    // backward: L^T x = y
    for (int J = nt - 1; J >= 0; --J) {
        const int c0 = J * 32, rs = c0 + 32;
        const int c = c0 + w;
        float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f;
        if (c < K) {
            const float* col = L + (int64_t)c * ld;
            int i = rs + lane;
            for (; i + 96 < K; i += 128) {
                s0 = fmaf(col[i], r[i], s0);
                s1 = fmaf(col[i + 32], r[i + 32], s1);
                s2 = fmaf(col[i + 64], r[i + 64], s2);
                s3 = fmaf(col[i + 96], r[i + 96], s3);
            }
            for (; i < K; i += 32) s0 = fmaf(col[i], r[i], s0);
        }
        float s = (s0 + s1) + (s2 + s3);
#pragma unroll
        for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) part[w] = s;
        __syncthreads();
        if (w == 0) {
            const float* D = Dinv + (int64_t)J * 1024;
            float acc = 0.f;
#pragma unroll
            for (int k = 0; k < 32; ++k) {
                const float yk = (c0 + k < K) ? r[c0 + k] - part[k] : 0.f;
                acc = fmaf(D[k * 32 + lane], yk, acc);
            }
            __syncwarp();
            if (c0 + lane < K) r[c0 + lane] = acc;
        }
        __syncthreads();
    }
}

using TrsvDesc = vtb_trsv_desc;
static_assert(sizeof(TrsvDesc) == 40, "vtb_trsv_desc layout");

// one CTA per system of a batch (descriptors in device memory)
__global__ void __launch_bounds__(kTrsvThreads) trsv_pair_batched_kernel(const TrsvDesc* __restrict__ descs) {
    extern __shared__ float trsv_sm[];
    const TrsvDesc d = descs[blockIdx.x];
    float* part = trsv_sm;
    float* r = trsv_sm + 32;
    for (int i = threadIdx.x; i < d.K; i += blockDim.x) r[i] = (float)d.x[i];
    __syncthreads();
    trsv_pair(d.L, d.ld, d.Dinv, d.K, r, part);
    for (int i = threadIdx.x; i < d.K; i += blockDim.x) d.x[i] = (double)r[i];
}

// Per-system pivot test of a batch of float32 factors (blockIdx.x = system).
__global__ void pivot_flag_batched_kernel(float* const* __restrict__ Mptrs, int64_t ld, int K,
                                          const int* __restrict__ infos, double rcond, double* __restrict__ piv,
                                          int32_t* __restrict__ flags) {
    const int z = blockIdx.x;
    pivot_flag_body<float>(Mptrs[z], ld, K, infos + z, rcond, piv ? piv + 2 * z : nullptr, flags + z);
}

__global__ void __launch_bounds__(128) diag_inv_batched_kernel(float* const* __restrict__ Mptrs, int64_t ld, int K,
                                                               float* __restrict__ Dinv, int64_t dinv_stride) {
    diag_inv_body(Mptrs[blockIdx.y], ld, K, Dinv + blockIdx.y * dinv_stride);
}

static int64_t dinv_floats(int K) { return (int64_t)((K + 31) / 32) * 1024; }

// ---------------------------------------------------------------------------
// Multi-CTA triangular solves for ONE system: x = L^-T L^-1 x.
//
// cuSOLVER's spotrs at K = 1921 is two chains of ~60 dependent 32-wide block
// steps (0.12-0.14 ms per triangle), each step a kernel-internal barrier.
// Here CTA j owns rows 64j..64j+63 (two 32-row sub-blocks A, B) and works
// left-looking: in the forward solve it accumulates L(rows, i) y_i for every
// earlier sub-block i as soon as that sub-block's owner has published y_i
// (a per-CTA flag), then solves its own two sub-blocks with the inverses of
// the 32 x 32 diagonal blocks (Dinv, from diag_inv_body) and publishes; the
// backward solve mirrors it from the last CTA down, reading column panels.
// The chain is 2 x ceil(K/64) flag hand-offs instead of 4 x ceil(K/32) block
// steps, and every CTA streams only its own panels of L.  The loads of a
// panel do not depend on the flag, so they are issued before the wait.
// All CTAs are co-resident (cooperative launch, one CTA per 64 rows, at
// most one per SM); each wait is bounded: after kTrsvSpinLimit polls the CTA
// sets *err = 3 and carries on (it still publishes, so no other CTA waits
// on it forever), and the caller treats the solve as failed.
constexpr int kTrsvFlagThreads = 256;
constexpr unsigned kTrsvSpinLimit = 1u << 21;   // x ~40 ns: well under a second

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// lane 0 polls, the warp learns the outcome; false after the limit
__device__ bool warp_wait_flag(const unsigned* f, int* err, unsigned limit) {
    int ok = 1;
    if ((threadIdx.x & 31) == 0) {
        unsigned it = 0;
        while (ld_acquire_u32(f) == 0u) {
            if (++it > limit || *(volatile int*)err == 3) {
                atomicExch(err, 3);
                ok = 0;
                break;
            }
        }
    }
    ok = __shfl_sync(0xffffffffu, ok, 0);
    __syncwarp();
    return ok != 0;
}

// publish: the warp's stores precede lane 0's release store of the flag
__device__ __forceinline__ void warp_publish(unsigned* f) {
    __syncwarp();
    if ((threadIdx.x & 31) == 0) asm volatile("st.release.gpu.global.u32 [%0], %1;\n" ::"l"(f), "r"(1u) : "memory");
}

// v[r] summed over the 32 lanes; lane r receives the total of v[r]
__device__ __forceinline__ float warp_transpose_reduce(float (&v)[32]) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) {
        const bool up = (lane & o) != 0;
#pragma unroll
        for (int k = 0; k < o; ++k) {
            const float send = up ? v[k] : v[k + o];
            const float keep = up ? v[k + o] : v[k];
            v[k] = keep + __shfl_xor_sync(0xffffffffu, send, o);
        }
    }
    return v[0];
}

// sum_k a[k] v[k], v in shared memory (broadcast reads), four chains
__device__ __forceinline__ float dot32(const float (&a)[32], const float* v) {
    float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f;
#pragma unroll
    for (int k = 0; k < 32; k += 4) {
        const float4 q = *reinterpret_cast<const float4*>(v + k);
        s0 = fmaf(a[k], q.x, s0);
        s1 = fmaf(a[k + 1], q.y, s1);
        s2 = fmaf(a[k + 2], q.z, s2);
        s3 = fmaf(a[k + 3], q.w, s3);
    }
    return (s0 + s1) + (s2 + s3);
}

__global__ void __launch_bounds__(kTrsvFlagThreads) trsv_flags_kernel(const float* __restrict__ L, int64_t ld,
                                                                      const float* __restrict__ Dinv, int K,
                                                                      double* x, float* ybuf, float* zbuf,
                                                                      unsigned* flags, int* err, unsigned limit) {
    __shared__ float part[2][8][32];
    __shared__ __align__(16) float sv[2][32];
    const int j = blockIdx.x, nc = gridDim.x;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int rA = 64 * j, rB = rA + 32;                 // first rows of sub-blocks A, B
    const int sA = 2 * j, sB = 2 * j + 1;                // their sub-block indices
    const bool hasB = rB < K;
    unsigned* ff = flags;                                // forward flags, one per CTA
    unsigned* fb = flags + nc;                           // backward flags
    const int ra = rA + lane, rb = rB + lane;
    // ---- forward: contributions of the sub-blocks i < 2j
    float accA = 0.f, accB = 0.f;
    for (int i = w; i < sA; i += 8) {
        float la[32], lb[32];
#pragma unroll
        for (int c = 0; c < 32; ++c) {
            const float* col = L + (int64_t)(32 * i + c) * ld;
            la[c] = ra < K ? col[ra] : 0.f;
            lb[c] = rb < K ? col[rb] : 0.f;
        }
        warp_wait_flag(ff + (i >> 1), err, limit);
        const float yv = __ldcg(ybuf + 32 * i + lane);   // sub-block i < 2j is full
#pragma unroll
        for (int c = 0; c < 32; ++c) {
            const float yc = __shfl_sync(0xffffffffu, yv, c);
            accA = fmaf(la[c], yc, accA);
            accB = fmaf(lb[c], yc, accB);
        }
    }
    part[0][w][lane] = accA;
    part[1][w][lane] = accB;
    // warp 0's operands, loaded before the barrier: rows of Dinv_A, Dinv_B and of L(B, A)
    float dA[32], dB[32], lba[32];
    if (w == 0) {
#pragma unroll
        for (int k = 0; k < 32; ++k) {
            dA[k] = Dinv[(int64_t)sA * 1024 + lane * 32 + k];
            dB[k] = hasB ? Dinv[(int64_t)sB * 1024 + lane * 32 + k] : 0.f;
            lba[k] = (hasB && rb < K && rA + k < K) ? L[(int64_t)(rA + k) * ld + rb] : 0.f;
        }
    }
    __syncthreads();
    float yA = 0.f, yB = 0.f;
    if (w == 0) {
        float s = ra < K ? (float)x[ra] : 0.f;
#pragma unroll
        for (int q = 0; q < 8; ++q) s -= part[0][q][lane];
        sv[0][lane] = s;
        __syncwarp();
        yA = dot32(dA, sv[0]);
        sv[1][lane] = yA;
        __syncwarp();
        if (hasB) {
            float t = rb < K ? (float)x[rb] : 0.f;
#pragma unroll
            for (int q = 0; q < 8; ++q) t -= part[1][q][lane];
            t -= dot32(lba, sv[1]);
            sv[0][lane] = t;
            __syncwarp();
            yB = dot32(dB, sv[0]);
        }
        if (ra < K) __stcg(ybuf + ra, yA);
        if (hasB && rb < K) __stcg(ybuf + rb, yB);
        warp_publish(ff + j);
    }
    __syncthreads();
    // ---- backward: contributions of the sub-blocks i > 2j+1, last first
    float cA[32], cB[32];
#pragma unroll
    for (int r = 0; r < 32; ++r) cA[r] = cB[r] = 0.f;
    const int nsub = (K + 31) >> 5;
    const int first = sB + 1;
    // warp w takes i = first + w + 8m, visited from the largest m down
    const int cnt = nsub > first + w ? (nsub - 1 - first - w) / 8 + 1 : 0;
    for (int m = cnt - 1; m >= 0; --m) {
        const int i = first + w + 8 * m;
        const int ri = 32 * i + lane;                    // row of L this lane reads
        float va[32], vb[32];
#pragma unroll
        for (int r = 0; r < 32; ++r) {
            va[r] = (ri < K && rA + r < K) ? L[(int64_t)(rA + r) * ld + ri] : 0.f;
            vb[r] = (ri < K && rB + r < K) ? L[(int64_t)(rB + r) * ld + ri] : 0.f;
        }
        warp_wait_flag(fb + (i >> 1), err, limit);
        const float xv = ri < K ? __ldcg(zbuf + ri) : 0.f;
#pragma unroll
        for (int r = 0; r < 32; ++r) {
            cA[r] = fmaf(va[r], xv, cA[r]);
            cB[r] = fmaf(vb[r], xv, cB[r]);
        }
    }
    part[0][w][lane] = warp_transpose_reduce(cA);
    part[1][w][lane] = warp_transpose_reduce(cB);
    // warp 0: columns of Dinv_A, Dinv_B (rows of their transposes)
    if (w == 0) {
#pragma unroll
        for (int k = 0; k < 32; ++k) {
            dA[k] = Dinv[(int64_t)sA * 1024 + k * 32 + lane];
            dB[k] = hasB ? Dinv[(int64_t)sB * 1024 + k * 32 + lane] : 0.f;
        }
    }
    __syncthreads();
    if (w == 0) {
        float xB = 0.f;
        if (hasB) {
            float t = yB;
#pragma unroll
            for (int q = 0; q < 8; ++q) t -= part[1][q][lane];
            sv[0][lane] = t;
            __syncwarp();
            xB = dot32(dB, sv[0]);
        }
        // L(B, A)^T x_B: lane c holds row c of L(B, A) in lba
        float pr[32];
#pragma unroll
        for (int r = 0; r < 32; ++r) pr[r] = lba[r] * xB;
        const float lt = warp_transpose_reduce(pr);
        float t = yA - lt;
#pragma unroll
        for (int q = 0; q < 8; ++q) t -= part[0][q][lane];
        sv[1][lane] = t;
        __syncwarp();
        const float xA = dot32(dA, sv[1]);
        if (ra < K) __stcg(zbuf + ra, xA);
        if (hasB && rb < K) __stcg(zbuf + rb, xB);
        warp_publish(fb + j);
        if (ra < K) x[ra] = (double)xA;
        if (hasB && rb < K) x[rb] = (double)xB;
    }
}

__global__ void __launch_bounds__(128) diag_inv_kernel(const float* __restrict__ L, int64_t ld, int K,
                                                       float* __restrict__ Dinv) {
    diag_inv_body(L, ld, K, Dinv);
}

static int flag_ctas(int K) { return (K + 63) / 64; }

// Workspace: [info 256][vec f32: K floats][w: K doubles][v1: K doubles][lapack work]

struct RealWork {
    int* info;
    float* vf;
    double* w;
    double* v1;
    void* wk;
    int lwork;   // elements of the factorisation's / eigensolver's work type
};

static int real_lwork(cusolverDnHandle_t h, int K, int mode, int* lwork) {
    cusolverStatus_t cs;
    if (mode == 0)
        cs = cusolverDnDsyevd_bufferSize(h, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, K, nullptr, K, nullptr,
                                         lwork);
    else if (mode == 1)
        cs = cusolverDnDpotrf_bufferSize(h, CUBLAS_FILL_MODE_LOWER, K, nullptr, K, lwork);
    else
        cs = cusolverDnSpotrf_bufferSize(h, CUBLAS_FILL_MODE_LOWER, K, nullptr, K, lwork);
    return cs == CUSOLVER_STATUS_SUCCESS ? VTB_OK : VTB_CUDA_ERR;
}

static int64_t real_layout(int K, int mode, int lwork, char* base, RealWork* rw) {
    int64_t off = 0;
    auto take = [&](int64_t bytes) {
        const int64_t o = off;
        off = al256r(off + bytes);
        return o;
    };
    const int64_t oi = take(256);
    const int64_t of = take((int64_t)K * 4);
    const int64_t ow = take((int64_t)K * 8);
    const int64_t o1 = take((int64_t)K * 8);
    const int64_t ok = take((int64_t)lwork * (mode == 2 ? 4 : 8));
    if (base && rw) {
        rw->info = reinterpret_cast<int*>(base + oi);
        rw->vf = reinterpret_cast<float*>(base + of);
        rw->w = reinterpret_cast<double*>(base + ow);
        rw->v1 = reinterpret_cast<double*>(base + o1);
        rw->wk = base + ok;
        rw->lwork = lwork;
    }
    return off;
}

static int real_setup(int K, int mode, void* work, int64_t work_bytes, void* stream, cusolverDnHandle_t* ph,
                      RealWork* rw) {
    int dev = 0;
    VTB_CUDA_TRY(cudaGetDevice(&dev));
    cusolverDnHandle_t h = real_solver_handle(dev);
    if (!h) return VTB_CUDA_ERR;
    int lwork = 0;
    int st = real_lwork(h, K, mode, &lwork);
    if (st) return st;
    const int64_t need = real_layout(K, mode, lwork, nullptr, nullptr);
    VTB_CHECK_ARG(work_bytes >= need && ((uintptr_t)work & 255) == 0);
    real_layout(K, mode, lwork, reinterpret_cast<char*>(work), rw);
    if (cusolverDnSetStream(h, as_stream(stream)) != CUSOLVER_STATUS_SUCCESS) return VTB_CUDA_ERR;
    *ph = h;
    return VTB_OK;
}

// x = V diag(1/w if |w| > rcond*max|w| else 0) V^T b for the column-major
// eigenvector matrix V (columns = eigenvectors): v1 = V^T b (one warp per
// column), truncation, x = V v1 (column blocks).
__global__ void dgemv_t_kernel(const double* __restrict__ V, int64_t ld, const double* __restrict__ x, int n,
                               double* __restrict__ y) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= n) return;
    const double* col = V + (int64_t)warp * ld;
    double s = 0.0;
    for (int i = lane; i < n; i += 32) s = fma(col[i], x[i], s);
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) y[warp] = s;
}

__global__ void dgemv_n_kernel(const double* __restrict__ V, int64_t ld, const double* __restrict__ x, int n,
                               double* __restrict__ y) {
    __shared__ double part[8][33];
    const int row = blockIdx.x * 32 + (threadIdx.x & 31);
    const int g = threadIdx.x >> 5;
    double s = 0.0;
    if (row < n)
        for (int c = g; c < n; c += 8) s = fma(V[(int64_t)c * ld + row], x[c], s);
    part[g][threadIdx.x & 31] = s;
    __syncthreads();
    if (g == 0 && row < n) {
        double t = 0.0;
        for (int k = 0; k < 8; ++k) t += part[k][threadIdx.x & 31];
        y[row] = t;
    }
}

__device__ void dtruncate_body(const double* __restrict__ w, double* __restrict__ v, int n, double rcond,
                               int32_t* __restrict__ kept) {
    __shared__ double s0;
    __shared__ int cnt;
    if (threadIdx.x == 0) {
        s0 = fmax(fabs(w[0]), fabs(w[n - 1])) * rcond;
        cnt = 0;
    }
    __syncthreads();
    int local = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double s = fabs(w[i]);
        if (s > s0) {
            v[i] = v[i] / s;
            ++local;
        } else {
            v[i] = 0.0;
        }
    }
    atomicAdd(&cnt, local);
    __syncthreads();
    if (threadIdx.x == 0 && kept) *kept = cnt;
}

__global__ void dtruncate_kernel(const double* __restrict__ w, double* __restrict__ v, int n, double rcond,
                                 int32_t* __restrict__ kept) {
    dtruncate_body(w, v, n, rcond, kept);
}

}  // namespace vtb

using namespace vtb;

VTB_API int vtb_coeff_real_scatter(const float* C, int64_t ldc, int Ks, int Kt, void* Mr, int64_t ldr, int out_f64,
                                   void* stream) {
    VTB_CHECK_ARG(Ks > 0 && (Ks & 1) && Kt > 0 && (Kt & 1) && C && Mr && ldr >= (int64_t)Ks * Kt &&
                  ldc >= (int64_t)Kt * (Kt + 1));
    const int K = Ks * Kt, h = (K - 1) / 2;
    VTB_CHECK_ARG(K <= 65535);
    const dim3 grid(ceil_div(h + 1, 256), K);
    if (out_f64)
        launch_real_scatter<double>(C, ldc, Ks, Kt, reinterpret_cast<double*>(Mr), ldr, grid, as_stream(stream));
    else
        launch_real_scatter<float>(C, ldc, Ks, Kt, reinterpret_cast<float*>(Mr), ldr, grid, as_stream(stream));
    return launch_status();
}

VTB_API int vtb_coeff_realify(const double* M, int64_t ldm, int K, void* Mr, int64_t ldr, int out_f64, void* stream) {
    VTB_CHECK_ARG(K > 0 && (K & 1) && M && Mr && ldm >= K && ldr >= K);
    const int64_t total = (int64_t)K * K;
    const int blocks = (int)std::min<int64_t>(ceil_div(total, 256), 16 * kNumSMs);
    if (out_f64)
        realify_kernel<double><<<blocks, 256, 0, as_stream(stream)>>>(reinterpret_cast<const double2*>(M), ldm, K,
                                                                      reinterpret_cast<double*>(Mr), ldr);
    else
        realify_kernel<float><<<blocks, 256, 0, as_stream(stream)>>>(reinterpret_cast<const double2*>(M), ldm, K,
                                                                     reinterpret_cast<float*>(Mr), ldr);
    return launch_status();
}

VTB_API int vtb_coeff_realify_vec(const double* b, int K, int batch, double* br, void* stream) {
    VTB_CHECK_ARG(K > 0 && (K & 1) && batch > 0 && b && br);
    realify_vec_kernel<<<dim3(ceil_div(K, 256), batch), 256, 0, as_stream(stream)>>>(
        reinterpret_cast<const double2*>(b), K, br);
    return launch_status();
}

VTB_API int vtb_coeff_unrealify_vec(const double* x, int K, int batch, double* a, int accumulate, void* stream) {
    VTB_CHECK_ARG(K > 0 && (K & 1) && batch > 0 && x && a);
    unrealify_vec_kernel<<<dim3(ceil_div((K + 1) / 2, 256), batch), 256, 0, as_stream(stream)>>>(
        x, K, reinterpret_cast<double2*>(a), accumulate);
    return launch_status();
}

VTB_API int vtb_sym_workspace(int K, int mode, int64_t* bytes) {
    VTB_CHECK_ARG(K > 0 && bytes && mode >= 0 && mode <= 2);
    int dev = 0;
    VTB_CUDA_TRY(cudaGetDevice(&dev));
    cusolverDnHandle_t h = real_solver_handle(dev);
    if (!h) return VTB_CUDA_ERR;
    int lwork = 0;
    int st = real_lwork(h, K, mode, &lwork);
    if (st) return st;
    *bytes = real_layout(K, mode, lwork, nullptr, nullptr);
    return VTB_OK;
}

VTB_API int vtb_sym_factor(void* M, int64_t ld, int K, int mode, double rcond, void* work, int64_t work_bytes,
                           int32_t* flag, double* pivots, void* stream) {
    VTB_CHECK_ARG(K > 0 && ld >= K && M && work && flag && (mode == 1 || mode == 2));
    cusolverDnHandle_t h;
    RealWork rw;
    int st = real_setup(K, mode, work, work_bytes, stream, &h, &rw);
    if (st) return st;
    cudaStream_t s = as_stream(stream);
    cusolverStatus_t cs;
    if (mode == 1)
        cs = cusolverDnDpotrf(h, CUBLAS_FILL_MODE_LOWER, K, reinterpret_cast<double*>(M), (int)ld,
                              reinterpret_cast<double*>(rw.wk), rw.lwork, rw.info);
    else
        cs = cusolverDnSpotrf(h, CUBLAS_FILL_MODE_LOWER, K, reinterpret_cast<float*>(M), (int)ld,
                              reinterpret_cast<float*>(rw.wk), rw.lwork, rw.info);
    if (cs != CUSOLVER_STATUS_SUCCESS) return VTB_CUDA_ERR;
    if (mode == 1)
        pivot_flag_kernel<double><<<1, 1024, 0, s>>>(reinterpret_cast<const double*>(M), ld, K, rw.info, rcond, pivots,
                                                     flag);
    else {
        pivot_flag_kernel<float><<<1, 1024, 0, s>>>(reinterpret_cast<const float*>(M), ld, K, rw.info, rcond, pivots,
                                                    flag);
    }
    return launch_status();
}

VTB_API int vtb_sym_potrs(const void* Mfac, int64_t ld, double* x, int K, int mode, void* work, int64_t work_bytes,
                          void* stream) {
    VTB_CHECK_ARG(K > 0 && ld >= K && Mfac && x && work && (mode == 1 || mode == 2));
    cusolverDnHandle_t h;
    RealWork rw;
    int st = real_setup(K, mode, work, work_bytes, stream, &h, &rw);
    if (st) return st;
    cudaStream_t s = as_stream(stream);
    if (mode == 1) {
        if (cusolverDnDpotrs(h, CUBLAS_FILL_MODE_LOWER, K, 1, reinterpret_cast<const double*>(Mfac), (int)ld, x, K,
                             rw.info) != CUSOLVER_STATUS_SUCCESS)
            return VTB_CUDA_ERR;
        return launch_status();
    }
    // one system: cuSOLVER's multi-CTA solves (the mixed decoder uses
    // vtb_sym_potrs_flags instead); batches use trsv_pair_batched_kernel
    f64_to_f32_kernel<<<ceil_div(K, 256), 256, 0, s>>>(x, rw.vf, K);
    if (cusolverDnSpotrs(h, CUBLAS_FILL_MODE_LOWER, K, 1, reinterpret_cast<const float*>(Mfac), (int)ld, rw.vf, K,
                         rw.info) != CUSOLVER_STATUS_SUCCESS)
        return VTB_CUDA_ERR;
    f32_to_f64_kernel<<<ceil_div(K, 256), 256, 0, s>>>(rw.vf, x, K);
    return launch_status();
}

// Inverses of the 32 x 32 diagonal blocks of one float32 factor (lower,
// column-major) for vtb_sym_potrs_flags: Dinv receives vtb_sym_dinv_floats(K)
// floats.
VTB_API int vtb_sym_dinv(const float* L, int64_t ld, int K, float* Dinv, void* stream) {
    VTB_CHECK_ARG(K > 0 && ld >= K && L && Dinv);
    const int nt = (K + 31) / 32;
    diag_inv_kernel<<<ceil_div(nt, 4), 128, 0, as_stream(stream)>>>(L, ld, K, Dinv);
    return launch_status();
}

VTB_API int64_t vtb_sym_potrs_flags_bytes(int K) {
    if (K <= 0) return 0;
    const int64_t nsub = (K + 31) / 32;
    return al256r(2 * (int64_t)flag_ctas(K) * 4) + 2 * al256r(nsub * 32 * 4);
}

// x = L^-T L^-1 x (float64 x, float32 arithmetic) for one system with the
// multi-CTA flag hand-off solve (trsv_flags_kernel); Dinv from vtb_sym_dinv.
// work: vtb_sym_potrs_flags_bytes(K).  err (device int32): set to 3 if a
// wait exceeded its limit (the result is then invalid).  VTB_BAD_ARG when
// the ceil(K/64) CTAs cannot all be resident (K above ~9400 on a B200).
VTB_API int vtb_sym_potrs_flags(const float* L, int64_t ld, const float* Dinv, int K, double* x, void* work,
                                int64_t work_bytes, int32_t* err, void* stream) {
    VTB_CHECK_ARG(K > 0 && ld >= K && L && Dinv && x && work && err);
    VTB_CHECK_ARG(work_bytes >= vtb_sym_potrs_flags_bytes(K));
    int dev = 0;
    VTB_CUDA_TRY(cudaGetDevice(&dev));
    int coop = 0, nsm = 0, per_sm = 0;
    VTB_CUDA_TRY(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
    VTB_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    VTB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, trsv_flags_kernel, kTrsvFlagThreads, 0));
    int nc = flag_ctas(K);
    VTB_CHECK_ARG(coop && nc <= nsm * per_sm);
    const int64_t nsub = (K + 31) / 32;
    char* wb = reinterpret_cast<char*>(work);
    unsigned* flags = reinterpret_cast<unsigned*>(wb);
    float* ybuf = reinterpret_cast<float*>(wb + al256r(2 * (int64_t)nc * 4));
    float* zbuf = reinterpret_cast<float*>(reinterpret_cast<char*>(ybuf) + al256r(nsub * 32 * 4));
    cudaStream_t s = as_stream(stream);
    VTB_CUDA_TRY(cudaMemsetAsync(flags, 0, 2 * (size_t)nc * 4, s));
    int* errp = reinterpret_cast<int*>(err);
    unsigned limit = wait_limit(kTrsvSpinLimit);
    void* args[] = {(void*)&L, (void*)&ld, (void*)&Dinv, (void*)&K, (void*)&x, (void*)&ybuf, (void*)&zbuf,
                    (void*)&flags, (void*)&errp, (void*)&limit};
    VTB_CUDA_TRY(cudaLaunchCooperativeKernel((void*)trsv_flags_kernel, dim3(nc), dim3(kTrsvFlagThreads), args, 0, s));
    return launch_status();
}

// Batched float32 Cholesky of `batch` systems of one size K (a group of clips
// with equal K): cusolverDnSpotrfBatched, then per system the pivot test of
// vtb_sym_factor (flags[z]) and the diagonal-block inverses used by
// vtb_sym_potrs_batched (Dinv + z * vtb_sym_dinv_floats(K)).  infos (device,
// batch ints) receives cuSOLVER's per-system status.  Does not synchronise.
VTB_API int vtb_sym_factor_batched(float** Mptrs, int64_t ld, int K, int batch, double rcond, float* Dinv,
                                   int32_t* infos, int32_t* flags, double* pivots, void* stream) {
    VTB_CHECK_ARG(K > 0 && ld >= K && batch >= 0);
    if (batch == 0) return VTB_OK;
    VTB_CHECK_ARG(Mptrs && Dinv && infos && flags);
    int dev = 0;
    VTB_CUDA_TRY(cudaGetDevice(&dev));
    cusolverDnHandle_t h = real_solver_handle(dev);
    if (!h) return VTB_CUDA_ERR;
    cudaStream_t s = as_stream(stream);
    if (cusolverDnSetStream(h, s) != CUSOLVER_STATUS_SUCCESS) return VTB_CUDA_ERR;
    if (cusolverDnSpotrfBatched(h, CUBLAS_FILL_MODE_LOWER, K, Mptrs, (int)ld, infos, batch) != CUSOLVER_STATUS_SUCCESS)
        return VTB_CUDA_ERR;
    pivot_flag_batched_kernel<<<batch, 1024, 0, s>>>(Mptrs, ld, K, infos, rcond, pivots, flags);
    int st = launch_status();
    if (st) return st;
    diag_inv_batched_kernel<<<dim3(ceil_div((K + 31) / 32, 4), batch), 128, 0, s>>>(Mptrs, ld, K, Dinv,
                                                                                   dinv_floats(K));
    return launch_status();
}

VTB_API int64_t vtb_sym_dinv_floats(int K) { return K > 0 ? dinv_floats(K) : 0; }

// Batched float32 solves x_z = L_z^-T L_z^-1 x_z, one CTA per system.  descs
// (device) holds per system {L (column-major float32 factor of
// vtb_sym_factor mode 2 or vtb_sym_factor_batched), Dinv (the inverses of its
// 32 x 32 diagonal blocks), x (float64, in place), ld, K}; Kmax bounds K.
VTB_API int vtb_sym_potrs_batched(const void* descs, int batch, int Kmax, void* stream) {
    VTB_CHECK_ARG(batch >= 0 && Kmax > 0);
    if (batch == 0) return VTB_OK;
    VTB_CHECK_ARG(descs);
    const size_t sm = (size_t)(Kmax + 32) * sizeof(float);
    VTB_CHECK_ARG(sm <= 200 * 1024);
    if (sm > 48 * 1024)
        VTB_CUDA_TRY(
            cudaFuncSetAttribute(trsv_pair_batched_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    trsv_pair_batched_kernel<<<batch, kTrsvThreads, sm, as_stream(stream)>>>(reinterpret_cast<const TrsvDesc*>(descs));
    return launch_status();
}

VTB_API int vtb_norm_ratio(const double* dx, const double* x, int n, double* out, void* stream) {
    VTB_CHECK_ARG(n > 0 && dx && x && out);
    norm_ratio_kernel<<<1, 1024, 0, as_stream(stream)>>>(dx, x, n, out);
    return launch_status();
}

VTB_API int vtb_daxpy1(double* y, const double* x, int n, void* stream) {
    VTB_CHECK_ARG(n >= 0 && y && x);
    if (n == 0) return VTB_OK;
    daxpy1_kernel<<<ceil_div(n, 256), 256, 0, as_stream(stream)>>>(y, x, n);
    return launch_status();
}

VTB_API int vtb_sym_pinv(double* M, int64_t ld, const double* b, double* x, int K, double rcond, void* work,
                         int64_t work_bytes, int32_t* kept, double* eig_range, void* stream) {
    VTB_CHECK_ARG(K > 0 && ld >= K && M && b && x && work);
    cusolverDnHandle_t h;
    RealWork rw;
    int st = real_setup(K, 0, work, work_bytes, stream, &h, &rw);
    if (st) return st;
    cudaStream_t s = as_stream(stream);
    if (cusolverDnDsyevd(h, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, K, M, (int)ld, rw.w,
                         reinterpret_cast<double*>(rw.wk), rw.lwork, rw.info) != CUSOLVER_STATUS_SUCCESS)
        return VTB_CUDA_ERR;
    int hinfo = 0;
    double ev[2] = {0, 0};
    VTB_CUDA_TRY(cudaMemcpyAsync(&hinfo, rw.info, sizeof(int), cudaMemcpyDeviceToHost, s));
    VTB_CUDA_TRY(cudaMemcpyAsync(&ev[0], rw.w, 8, cudaMemcpyDeviceToHost, s));
    VTB_CUDA_TRY(cudaMemcpyAsync(&ev[1], rw.w + K - 1, 8, cudaMemcpyDeviceToHost, s));
    VTB_CUDA_TRY(cudaStreamSynchronize(s));
    if (hinfo != 0) return VTB_NOT_CONVERGED;
    if (eig_range) {
        eig_range[0] = ev[0];
        eig_range[1] = ev[1];
    }
    dgemv_t_kernel<<<ceil_div((int64_t)K * 32, 256), 256, 0, s>>>(M, ld, b, K, rw.v1);
    dtruncate_kernel<<<1, 1024, 0, s>>>(rw.w, rw.v1, K, rcond, kept);
    dgemv_n_kernel<<<ceil_div(K, 32), 256, 0, s>>>(M, ld, rw.v1, K, x);
    return launch_status();
}

// Batched eigen-pseudoinverse of `batch` real symmetric systems of one size K
// (cuSOLVER XsyevBatched): x_z = V diag(1/w if |w| > rcond*max|w| else 0)
// V^T b_z, the rule of vtb_sym_pinv per system.  M holds the matrices
// contiguously (stride K*K, overwritten by the eigenvectors), b and x at
// stride K; kept[z] (device, may be NULL) the kept counts, infos[z] (device)
// the eigensolver's status.  Synchronises the stream (the host workspace of
// the eigensolver must outlive the call).
namespace vtb {
static cusolverDnParams_t real_params() {
    static thread_local cusolverDnParams_t p = nullptr;
    if (!p && cusolverDnCreateParams(&p) != CUSOLVER_STATUS_SUCCESS) p = nullptr;
    return p;
}
static int pinv_batched_real_sizes(cusolverDnHandle_t h, int K, int batch, size_t* db, size_t* hb) {
    cusolverDnParams_t prm = real_params();
    if (!prm) return VTB_CUDA_ERR;
    if (cusolverDnXsyevBatched_bufferSize(h, prm, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, K, CUDA_R_64F,
                                          nullptr, K, CUDA_R_64F, nullptr, CUDA_R_64F, db, hb, batch) !=
        CUSOLVER_STATUS_SUCCESS)
        return VTB_CUDA_ERR;
    return VTB_OK;
}
// [w: batch*K][v: batch*K][info: batch][eigensolver work]
static int64_t pinv_batched_real_layout(int K, int batch, size_t db) {
    return al256r((int64_t)batch * K * 8) * 2 + al256r((int64_t)batch * 4) + al256r((int64_t)db);
}

__global__ void dgemv_t_batched_kernel(const double* __restrict__ V, int K, const double* __restrict__ x,
                                       double* __restrict__ y) {
    const int z = blockIdx.y;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= K) return;
    const double* col = V + (int64_t)z * K * K + (int64_t)warp * K;
    const double* xz = x + (int64_t)z * K;
    double s = 0.0;
    for (int i = lane; i < K; i += 32) s = fma(col[i], xz[i], s);
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) y[(int64_t)z * K + warp] = s;
}

__global__ void dgemv_n_batched_kernel(const double* __restrict__ V, int K, const double* __restrict__ x,
                                       double* __restrict__ y) {
    __shared__ double part[8][33];
    const int z = blockIdx.y;
    const double* Vz = V + (int64_t)z * K * K;
    const double* xz = x + (int64_t)z * K;
    const int row = blockIdx.x * 32 + (threadIdx.x & 31);
    const int g = threadIdx.x >> 5;
    double s = 0.0;
    if (row < K)
        for (int c = g; c < K; c += 8) s = fma(Vz[(int64_t)c * K + row], xz[c], s);
    part[g][threadIdx.x & 31] = s;
    __syncthreads();
    if (g == 0 && row < K) {
        double t = 0.0;
        for (int k = 0; k < 8; ++k) t += part[k][threadIdx.x & 31];
        y[(int64_t)z * K + row] = t;
    }
}

__global__ void dtruncate_batched_kernel(const double* __restrict__ w, double* __restrict__ v, int K, double rcond,
                                         int32_t* __restrict__ kept) {
    const int z = blockIdx.x;
    dtruncate_body(w + (int64_t)z * K, v + (int64_t)z * K, K, rcond, kept ? kept + z : nullptr);
}
}  // namespace vtb

VTB_API int vtb_sym_pinv_batched_workspace(int K, int batch, int64_t* bytes) {
    VTB_CHECK_ARG(K > 0 && batch > 0 && bytes);
    int dev = 0;
    VTB_CUDA_TRY(cudaGetDevice(&dev));
    cusolverDnHandle_t h = real_solver_handle(dev);
    if (!h) return VTB_CUDA_ERR;
    size_t db = 0, hb = 0;
    int st = pinv_batched_real_sizes(h, K, batch, &db, &hb);
    if (st) return st;
    *bytes = pinv_batched_real_layout(K, batch, db);
    return VTB_OK;
}

VTB_API int vtb_sym_pinv_batched(double* M, const double* b, double* x, int K, int batch, double rcond, void* work,
                                 int64_t work_bytes, int32_t* kept, int32_t* infos, void* stream) {
    VTB_CHECK_ARG(K > 0 && batch > 0 && M && b && x && work && infos && ((uintptr_t)work & 255) == 0);
    int dev = 0;
    VTB_CUDA_TRY(cudaGetDevice(&dev));
    cusolverDnHandle_t h = real_solver_handle(dev);
    if (!h) return VTB_CUDA_ERR;
    size_t db = 0, hb = 0;
    int st = pinv_batched_real_sizes(h, K, batch, &db, &hb);
    if (st) return st;
    VTB_CHECK_ARG(work_bytes >= pinv_batched_real_layout(K, batch, db));
    char* base = reinterpret_cast<char*>(work);
    double* w = reinterpret_cast<double*>(base);
    double* v = reinterpret_cast<double*>(base + al256r((int64_t)batch * K * 8));
    int* info = reinterpret_cast<int*>(base + 2 * al256r((int64_t)batch * K * 8));
    void* wk = base + 2 * al256r((int64_t)batch * K * 8) + al256r((int64_t)batch * 4);
    cudaStream_t s = as_stream(stream);
    if (cusolverDnSetStream(h, s) != CUSOLVER_STATUS_SUCCESS) return VTB_CUDA_ERR;
    void* hwk = hb ? malloc(hb) : nullptr;
    if (hb && !hwk) return VTB_OOM;
    const cusolverStatus_t cs = cusolverDnXsyevBatched(h, real_params(), CUSOLVER_EIG_MODE_VECTOR,
                                                       CUBLAS_FILL_MODE_LOWER, K, CUDA_R_64F, M, K, CUDA_R_64F, w,
                                                       CUDA_R_64F, wk, db, hwk, hb, info, batch);
    cudaError_t e1 = cudaStreamSynchronize(s);
    free(hwk);
    if (cs != CUSOLVER_STATUS_SUCCESS) return VTB_CUDA_ERR;
    VTB_CUDA_TRY(e1);
    VTB_CUDA_TRY(cudaMemcpyAsync(infos, info, (size_t)batch * 4, cudaMemcpyDeviceToDevice, s));
    dgemv_t_batched_kernel<<<dim3(ceil_div((int64_t)K * 32, 256), batch), 256, 0, s>>>(M, K, b, v);
    dtruncate_batched_kernel<<<batch, 1024, 0, s>>>(w, v, K, rcond, kept);
    dgemv_n_batched_kernel<<<dim3(ceil_div(K, 32), batch), 256, 0, s>>>(M, K, v, x);
    return launch_status();
}
