// Coefficient-space decoder.
//
// The plain decoder solves G c = q with G = Phi Phi^H (n x n, n = spike
// intervals) and synthesises u = sum_k c_k psi_k phi_{n_k}.  With
//   Phi[k, (s, m)] = norm_n conj(Ds_n[s]) T_k(m),   T_k(m) = int_{tk1}^{tk2} e^{jmWt} dt,
// the reconstruction only ever needs a = Phi^H c, and
//   Phi^H G^+ q = Phi^+ q = M^+ b,   M = Phi^H Phi (K x K),  b = Phi^H q,
// with the same truncation (the nonzero eigenvalues of Phi Phi^H and
// Phi^H Phi coincide, so rcond * s_0 selects the same subspace).  K =
// (ellipse size) * (2 Mt + 1) is independent of the spike count.
//
// M has Kronecker structure: with d_n = norm_n Ds_n and the per-neuron
// temporal Gram W_n[m, m'] = sum_{k in n} conj(T_k(m)) T_k(m'),
//   M[(s,m),(s',m')] = sum_n d_n[s] conj(d_n[s']) W_n[m, m'],
//   b[(s,m)]         = sum_n d_n[s] g_n[m],  g_n[m] = sum_{k in n} conj(T_k(m)) q_k,
// so Phi (n x K) is never formed: one pass over the spikes builds W_n, g_n
// (temporal_gram_kernel), one tiled pass over the neurons builds M
// (kron_gram_kernel).  The synthesis expands a on the separable
// space-time basis: A[t, s] = sum_m a[s, m] e^{jmWt}, then per frame
// u = Re(ey^T A_t ex) on the decode grid (synth_kernel), whose output write is
// the one HBM-sized stream of the whole decode.
#include <cooperative_groups.h>
#include <cuda_bf16.h>

#include <algorithm>

#include "common.cuh"

namespace vtb {

// lower_bound of v in the sorted a[0..n) by one full warp: 32-way probes
// (three dependent rounds for 25k entries instead of fifteen), the same
// result on every lane.
__device__ int warp_lower_bound(const int32_t* __restrict__ a, int n, int v) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    int lo = 0, hi = n;
    while (hi - lo > 32) {
        const int step = (hi - lo + 31) / 32;
        const int pos = lo + lane * step;
        const int c = __popc(__ballot_sync(full, pos < hi && a[pos] < v));
        if (c == 0) {
            hi = lo;
        } else {
            const int nlo = lo + (c - 1) * step + 1;
            hi = min(hi, lo + c * step);
            lo = nlo;
        }
    }
    const int pos = lo + lane;
    return lo + __popc(__ballot_sync(full, pos < hi && a[pos] < v));
}

// [lo, hi) of neuron nr in the neuron-sorted index array, found by warp 0 and
// shared with the block (all threads must call it).
__device__ __forceinline__ void neuron_range(const int32_t* __restrict__ ind, int nspk, int nr, int& lo, int& hi) {
    __shared__ int s_range[2];
    if (threadIdx.x < 32) {
        const int a = warp_lower_bound(ind, nspk, nr);
        const int b = warp_lower_bound(ind, nspk, nr + 1);
        if (threadIdx.x == 0) {
            s_range[0] = a;
            s_range[1] = b;
        }
    }
    __syncthreads();
    lo = s_range[0];
    hi = s_range[1];
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cmulc(double2 a, double2 b) {  // a * conj(b)
    return make_double2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}

// ------------------------------------------------------------------ W_n, g_n
// One block per neuron.  Spikes must be sorted by neuron.  T_k(m) for m in
// [-Mt, Mt] uses the product form (2/(mW)) sin(mW dt/2) e^{jmW tbar}, exact
// for the integral and free of the cancellation of e^{a} - e^{b}; its
// harmonics come from powers of e^{jW tbar} and e^{jW dt/2} (two sincos per
// interval; a few ulp per power).
constexpr int kTChunk = 32;

__device__ __forceinline__ void spike_T(double a, double b, int Mt, double W, double2* __restrict__ T) {
    const double d = b - a;
    double s1, c1, sh, ch;
    sincos(W * (0.5 * (a + b)), &s1, &c1);
    sincos(0.5 * W * d, &sh, &ch);
    T[Mt] = make_double2(d, 0.0);
    const double2 e1 = make_double2(c1, s1), h1 = make_double2(ch, sh);
    double2 pe = make_double2(1.0, 0.0), ph = make_double2(1.0, 0.0);
    for (int m = 1; m <= Mt; ++m) {
        pe = cmul(pe, e1);
        ph = cmul(ph, h1);
        const double amp = (2.0 / (m * W)) * ph.y;   // (2/(mW)) sin(mW d/2), even in m
        T[Mt + m] = make_double2(amp * pe.x, amp * pe.y);
        T[Mt - m] = make_double2(amp * pe.x, -amp * pe.y);
    }
}

// Thread t owns the entries e = t, t+256, ... (at most kTgEntries) of the
// upper triangle (m <= m') of the Hermitian W_n (the mirror is written from
// the same sum); threads m < Kt also g_n[m].
constexpr int kTgEntries = 4;   // Kt(Kt+1)/2 <= 1024: Mt <= 21

__global__ void __launch_bounds__(256) temporal_gram_kernel(
    const double* __restrict__ tk1, const double* __restrict__ tk2, const int32_t* __restrict__ ind, int nspk,
    const double* __restrict__ kappa, const double* __restrict__ delta, const double* __restrict__ bias,
    const double* __restrict__ norm, int Mt, double W, double2* __restrict__ Wn, double2* __restrict__ gn) {
    extern __shared__ double2 sT[];  // kTChunk x Kt, then kTChunk q values (as double2.x)
    const int Kt = 2 * Mt + 1;
    double2* sq = sT + kTChunk * Kt;
    const int nr = blockIdx.x;
    int lo, hi;
    neuron_range(ind, nspk, nr, lo, hi);
    const int KK = Kt * Kt, nup = Kt * (Kt + 1) / 2;
    const double kd = kappa[nr] * delta[nr], bb = bias[nr], nn = norm[nr];
    int em[kTgEntries], emp[kTgEntries];
    double2 acc[kTgEntries];
#pragma unroll
    for (int u = 0; u < kTgEntries; ++u) {
        int e = threadIdx.x + u * blockDim.x, m = 0;
        em[u] = -1;
        emp[u] = 0;
        acc[u] = make_double2(0, 0);
        if (e < nup) {
            while (e >= Kt - m) {
                e -= Kt - m;
                ++m;
            }
            em[u] = m;
            emp[u] = m + e;
        }
    }
    const bool own_g = threadIdx.x < Kt;
    double2 gacc = make_double2(0, 0);
    for (int k0 = lo; k0 < hi; k0 += kTChunk) {
        const int nk = min(kTChunk, hi - k0);
        __syncthreads();
        if (threadIdx.x < nk) {
            const double a = tk1[k0 + threadIdx.x], b = tk2[k0 + threadIdx.x];
            spike_T(a, b, Mt, W, sT + threadIdx.x * Kt);
            sq[threadIdx.x].x = (kd - bb * (b - a)) * nn;  // q_k, compute_q_Kernel's formula
        }
        __syncthreads();
#pragma unroll
        for (int u = 0; u < kTgEntries; ++u) {
            if (em[u] < 0) continue;
            for (int kk = 0; kk < nk; ++kk) {
                const double2 a = sT[kk * Kt + em[u]], b = sT[kk * Kt + emp[u]];
                // conj(a) * b
                acc[u].x += a.x * b.x + a.y * b.y;
                acc[u].y += a.x * b.y - a.y * b.x;
            }
        }
        if (own_g) {
            for (int kk = 0; kk < nk; ++kk) {
                const double2 a = sT[kk * Kt + threadIdx.x];
                const double q = sq[kk].x;
                gacc.x += a.x * q;
                gacc.y -= a.y * q;
            }
        }
    }
#pragma unroll
    for (int u = 0; u < kTgEntries; ++u) {
        if (em[u] < 0) continue;
        const int m = em[u], mp = emp[u];
        Wn[(int64_t)nr * KK + m * Kt + mp] = acc[u];
        if (m != mp) Wn[(int64_t)nr * KK + mp * Kt + m] = make_double2(acc[u].x, -acc[u].y);
    }
    if (own_g) gn[(int64_t)nr * Kt + threadIdx.x] = gacc;
}

// ---- one warp per neuron (Kt(Kt+1)/2 <= 32 * kWarpEntries): no block-wide
// barrier between the phases of a neuron, four neurons per block, so the
// short per-neuron chains of many neurons overlap on each SM.
constexpr int kNrWarps = 4;        // neurons (warps) per block
constexpr int kWarpEntries = 8;    // upper W_n entries per lane: Kt(Kt+1)/2 <= 256, Mt <= 10

static inline bool warp_per_neuron(int Kt) { return Kt * (Kt + 1) / 2 <= 32 * kWarpEntries; }

// The temporal Gram W_n and g_n of one neuron per warp: lane l computes the
// spike T_k(m) of the chunk's l-th spike into the warp's shared memory, then
// owns the upper entries e = l, l + 32, ... and (l < Kt) g_n[l].  Chunks of
// kTChunk spikes in order, the same sums in the same order as
// temporal_gram_kernel.
__global__ void __launch_bounds__(kNrWarps * 32) temporal_gram_warp_kernel(
    const double* __restrict__ tk1, const double* __restrict__ tk2, const int32_t* __restrict__ ind, int nspk, int N,
    const double* __restrict__ kappa, const double* __restrict__ delta, const double* __restrict__ bias,
    const double* __restrict__ norm, int Mt, double W, double2* __restrict__ Wn, double2* __restrict__ gn) {
    extern __shared__ double2 shw[];
    const int Kt = 2 * Mt + 1, KK = Kt * Kt, nup = Kt * (Kt + 1) / 2;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nr = blockIdx.x * kNrWarps + w;
    if (nr >= N) return;   // whole warps only; no block-wide barrier below
    double2* T = shw + (size_t)w * kTChunk * (Kt + 1);
    double* q = reinterpret_cast<double*>(T + kTChunk * Kt);
    const int lo = warp_lower_bound(ind, nspk, nr), hi = warp_lower_bound(ind, nspk, nr + 1);
    const double kd = kappa[nr] * delta[nr], bb = bias[nr], nn = norm[nr];
    int em[kWarpEntries], emp[kWarpEntries];
    double2 acc[kWarpEntries];
#pragma unroll
    for (int u = 0; u < kWarpEntries; ++u) {
        int e = lane + 32 * u, m = 0;
        em[u] = -1;
        emp[u] = 0;
        acc[u] = make_double2(0, 0);
        if (e < nup) {
            while (e >= Kt - m) {
                e -= Kt - m;
                ++m;
            }
            em[u] = m;
            emp[u] = m + e;
        }
    }
    double2 gacc = make_double2(0, 0);
    for (int k0 = lo; k0 < hi; k0 += kTChunk) {
        const int nk = min(kTChunk, hi - k0);
        __syncwarp();
        if (lane < nk) {
            const double a = tk1[k0 + lane], b = tk2[k0 + lane];
            spike_T(a, b, Mt, W, T + lane * Kt);
            q[lane] = (kd - bb * (b - a)) * nn;   // q_k, compute_q_Kernel's formula
        }
        __syncwarp();
#pragma unroll
        for (int u = 0; u < kWarpEntries; ++u) {
            if (em[u] < 0) continue;
            for (int kk = 0; kk < nk; ++kk) {
                const double2 a = T[kk * Kt + em[u]], b = T[kk * Kt + emp[u]];
                // conj(a) * b
                acc[u].x += a.x * b.x + a.y * b.y;
                acc[u].y += a.x * b.y - a.y * b.x;
            }
        }
        if (lane < Kt) {
            for (int kk = 0; kk < nk; ++kk) {
                const double2 a = T[kk * Kt + lane];
                const double qk = q[kk];
                gacc.x += a.x * qk;
                gacc.y -= a.y * qk;
            }
        }
    }
#pragma unroll
    for (int u = 0; u < kWarpEntries; ++u) {
        if (em[u] < 0) continue;
        const int m = em[u], mp = emp[u];
        Wn[(int64_t)nr * KK + m * Kt + mp] = acc[u];
        if (m != mp) Wn[(int64_t)nr * KK + mp * Kt + m] = make_double2(acc[u].x, -acc[u].y);
    }
    if (lane < Kt) gn[(int64_t)nr * Kt + lane] = gacc;
}

// The residual's per-neuron part, one neuron per warp: v(m) = sum_s
// conj(d_n[s]) a(s, m) (lane m, two partial sums over s), then per chunk of
// spikes y_k = q_k - Re sum_m T_k(m) v(m) (lane k) and g(m) += sum_k
// conj(T_k(m)) y_k (lane m).
__global__ void __launch_bounds__(kNrWarps * 32) coeff_residual_warp_kernel(
    const double* __restrict__ tk1, const double* __restrict__ tk2, const int32_t* __restrict__ ind, int nspk, int N,
    const double* __restrict__ kappa, const double* __restrict__ delta, const double* __restrict__ bias,
    const double* __restrict__ norm, int Mt, double W, const double2* __restrict__ d, int Ks,
    const double2* __restrict__ a, double2* __restrict__ gres) {
    extern __shared__ double2 shw[];
    const int Kt = 2 * Mt + 1;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nr = blockIdx.x * kNrWarps + w;
    if (nr >= N) return;   // whole warps only; no block-wide barrier below
    double2* T = shw + (size_t)w * (kTChunk * Kt + Kt + kTChunk);
    double2* v = T + kTChunk * Kt;
    double* y = reinterpret_cast<double*>(v + Kt);
    const int lo = warp_lower_bound(ind, nspk, nr), hi = warp_lower_bound(ind, nspk, nr + 1);
    const double kd = kappa[nr] * delta[nr], bb = bias[nr], nn = norm[nr];
    if (lane < Kt) {
        // loads of 8 spatial indices are issued together (one L2 latency per 8)
        constexpr int kU = 8;
        double sr0 = 0.0, si0 = 0.0, sr1 = 0.0, si1 = 0.0;
        const double2* dn = d + (int64_t)nr * Ks;
        int s = 0;
        for (; s + kU <= Ks; s += kU) {
            double2 dd[kU], aa[kU];
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                dd[u] = dn[s + u];
                aa[u] = a[(int64_t)(s + u) * Kt + lane];
            }
#pragma unroll
            for (int u = 0; u < kU; u += 2) {
                sr0 += dd[u].x * aa[u].x + dd[u].y * aa[u].y;   // conj(d) * a
                si0 += dd[u].x * aa[u].y - dd[u].y * aa[u].x;
                sr1 += dd[u + 1].x * aa[u + 1].x + dd[u + 1].y * aa[u + 1].y;
                si1 += dd[u + 1].x * aa[u + 1].y - dd[u + 1].y * aa[u + 1].x;
            }
        }
        for (; s < Ks; ++s) {
            const double2 d0 = dn[s], a0 = a[(int64_t)s * Kt + lane];
            sr0 += d0.x * a0.x + d0.y * a0.y;
            si0 += d0.x * a0.y - d0.y * a0.x;
        }
        v[lane] = make_double2(sr0 + sr1, si0 + si1);
    }
    double2 gacc = make_double2(0, 0);
    for (int k0 = lo; k0 < hi; k0 += kTChunk) {
        const int nk = min(kTChunk, hi - k0);
        __syncwarp();
        if (lane < nk) spike_T(tk1[k0 + lane], tk2[k0 + lane], Mt, W, T + lane * Kt);
        __syncwarp();
        if (lane < nk) {
            double acc = 0.0;
            for (int m = 0; m < Kt; ++m) {
                const double2 t = T[lane * Kt + m], vv = v[m];
                acc += t.x * vv.x - t.y * vv.y;
            }
            const double qk = (kd - bb * (tk2[k0 + lane] - tk1[k0 + lane])) * nn;
            y[lane] = qk - acc;
        }
        __syncwarp();
        if (lane < Kt) {
            for (int kk = 0; kk < nk; ++kk) {
                const double2 t = T[kk * Kt + lane];
                gacc.x += t.x * y[kk];
                gacc.y -= t.y * y[kk];
            }
        }
    }
    if (lane < Kt) gres[(int64_t)nr * Kt + lane] = gacc;
}

// ------------------------------------------------------------------ M
// Block = 4 x 4 tile of (s, s') pairs (s-tile <= s'-tile: M is Hermitian and
// the mirror half is written from the same accumulators); threads own (m, m')
// entries of the Kt x Kt sub-blocks.  d products for a chunk of neurons are
// staged in shared memory; W_n entries stream from L2, coalesced.
constexpr int kKT = 4;
constexpr int kKN = 32;

__global__ void __launch_bounds__(256) kron_gram_kernel(const double2* __restrict__ d, int N, int Ks,
                                                        const double2* __restrict__ Wn, int Kt,
                                                        double2* __restrict__ M, int64_t ldm) {
    __shared__ double2 sa[kKN][kKT * kKT];
    // map blockIdx.x to an upper-triangular tile pair (ti <= tj)
    const int T = (Ks + kKT - 1) / kKT;
    int b = blockIdx.x, ti = 0;
    while (b >= T - ti) { b -= T - ti; ++ti; }
    const int tj = ti + b;
    const int s0 = ti * kKT, s1 = tj * kKT;
    const int KK = Kt * Kt;
    for (int e0 = 0; e0 < KK; e0 += blockDim.x) {
        const int e = e0 + threadIdx.x;
        double2 acc[kKT][kKT];
#pragma unroll
        for (int i = 0; i < kKT; ++i)
#pragma unroll
            for (int j = 0; j < kKT; ++j) acc[i][j] = make_double2(0, 0);
        for (int n0 = 0; n0 < N; n0 += kKN) {
            const int nn = min(kKN, N - n0);
            __syncthreads();
            for (int x = threadIdx.x; x < nn * kKT * kKT; x += blockDim.x) {
                const int r = x / (kKT * kKT), ij = x % (kKT * kKT), i = ij / kKT, j = ij % kKT;
                const int si = s0 + i, sj = s1 + j;
                double2 v = make_double2(0, 0);
                if (si < Ks && sj < Ks) v = cmulc(d[(int64_t)(n0 + r) * Ks + si], d[(int64_t)(n0 + r) * Ks + sj]);
                sa[r][ij] = v;
            }
            __syncthreads();
            if (e < KK) {
                double2 wnext = Wn[(int64_t)n0 * KK + e];
                for (int r = 0; r < nn; ++r) {
                    const double2 w = wnext;
                    if (r + 1 < nn) wnext = Wn[(int64_t)(n0 + r + 1) * KK + e];
#pragma unroll
                    for (int i = 0; i < kKT; ++i)
#pragma unroll
                        for (int j = 0; j < kKT; ++j) {
                            const double2 a = sa[r][i * kKT + j];
                            acc[i][j].x = fma(a.x, w.x, fma(-a.y, w.y, acc[i][j].x));
                            acc[i][j].y = fma(a.x, w.y, fma(a.y, w.x, acc[i][j].y));
                        }
                }
            }
        }
        if (e < KK) {
            const int m = e / Kt, mp = e % Kt;
#pragma unroll
            for (int i = 0; i < kKT; ++i)
#pragma unroll
                for (int j = 0; j < kKT; ++j) {
                    const int si = s0 + i, sj = s1 + j;
                    if (si >= Ks || sj >= Ks) continue;
                    const int64_t row = (int64_t)si * Kt + m, col = (int64_t)sj * Kt + mp;
                    M[col * ldm + row] = acc[i][j];  // column-major
                    if (ti != tj) M[row * ldm + col] = make_double2(acc[i][j].x, -acc[i][j].y);
                }
        }
    }
}

// b[(s, m)] = sum_n d[n][s] g[n][m]: a cluster of kRhsSplit CTAs per group
// of kRhsS spatial indices, each CTA summing a contiguous eighth of the
// neurons.  The CTA stages up to `chunk` neurons' d[n][s0..s0+3] and
// g[n][0..Kt) in shared memory (coalesced row reads; one chunk covers the
// CTA's neurons at the usual sizes), and two threads per output (s, m) sum
// the even and the odd neurons, added in that order; the cluster's first CTA
// adds the others' partial sums through distributed shared memory in rank
// order (deterministic).
constexpr int kRhsS = 4;       // spatial indices per cluster
constexpr int kRhsM = 32;      // temporal indices per pass
constexpr int kRhsSplit = 8;   // CTAs per cluster (neuron eighths)

static inline int rhs_grid(int Ks) { return ceil_div(Ks, kRhsS) * kRhsSplit; }

// neurons staged per pass, so that the staging and the partial sums fit the
// 48 KB a kernel gets without an opt-in
static inline int rhs_chunk(int Kt) {
    int c = 128;
    while (c > 8 && (size_t)c * (kRhsS + Kt) * sizeof(double2) > 46 * 1024) c /= 2;
    return c;
}

static inline size_t rhs_smem(int Kt) { return (size_t)rhs_chunk(Kt) * (kRhsS + Kt) * sizeof(double2); }

__global__ void __cluster_dims__(kRhsSplit, 1, 1) __launch_bounds__(256)
    kron_rhs_kernel(const double2* __restrict__ d, int N, int Ks, const double2* __restrict__ gn, int Kt,
                    double2* __restrict__ b, int chunk) {
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    extern __shared__ double2 shr[];
    double2* sd = shr;                  // chunk x kRhsS
    double2* sg = shr + chunk * kRhsS;  // chunk x Kt
    __shared__ double2 part[kRhsS * kRhsM];
    const int rank = (int)cluster.block_rank();
    const int s0 = (blockIdx.x / kRhsSplit) * kRhsS;
    const int nq = (N + kRhsSplit - 1) / kRhsSplit;
    const int n_lo = rank * nq, n_hi = min(N, n_lo + nq);
    const int t = threadIdx.x, h = t & 1, o = t >> 1, si = o / kRhsM, mm = o % kRhsM;
    for (int mb = 0; mb < Kt; mb += kRhsM) {
        const int m = mb + mm;
        double2 acc = make_double2(0, 0);
        for (int c = n_lo; c < n_hi; c += chunk) {
            const int nc = min(chunk, n_hi - c);
            __syncthreads();
            for (int e = t; e < nc * kRhsS; e += blockDim.x) {
                const int n = e / kRhsS, j = e % kRhsS;
                sd[e] = s0 + j < Ks ? d[(int64_t)(c + n) * Ks + s0 + j] : make_double2(0, 0);
            }
            for (int e = t; e < nc * Kt; e += blockDim.x) sg[e] = gn[(int64_t)c * Kt + e];
            __syncthreads();
            if (m < Kt) {
                for (int n = h; n < nc; n += 2) {
                    const double2 p = cmul(sd[n * kRhsS + si], sg[n * Kt + m]);
                    acc.x += p.x;
                    acc.y += p.y;
                }
            }
        }
        // even + odd neurons (lanes 2o and 2o + 1 of the same warp)
        const double ox = __shfl_xor_sync(0xffffffffu, acc.x, 1), oy = __shfl_xor_sync(0xffffffffu, acc.y, 1);
        if (h == 0) part[o] = make_double2(acc.x + ox, acc.y + oy);
        cluster.sync();
        if (rank == 0 && h == 0 && s0 + si < Ks && m < Kt) {
            double2 v = part[o];
#pragma unroll
            for (int r = 1; r < kRhsSplit; ++r) {
                const double2 w = cluster.map_shared_rank(part, r)[o];
                v.x += w.x;
                v.y += w.y;
            }
            b[(int64_t)(s0 + si) * Kt + m] = v;
        }
        cluster.sync();   // the partial sums stay valid until rank 0 has read them
    }
}

// d[n][s] = norm_n * Ds[n][smap[s]]
__global__ void pack_d_kernel(const double2* __restrict__ Ds, int N, int Kfull, const int32_t* __restrict__ smap,
                              int Ks, const double* __restrict__ norm, double2* __restrict__ d) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= N * Ks) return;
    const int n = e / Ks, s = e % Ks;
    const double2 v = Ds[(int64_t)n * Kfull + smap[s]];
    d[e] = make_double2(v.x * norm[n], v.y * norm[n]);
}

// ------------------------------------------------------------------ synthesis
// A[t][s] = sum_m a[s][m] e^{jmW t_i}, t_i = t0 + i dt
__global__ void temporal_expand_kernel(const double2* __restrict__ a, int Ks, int Mt, double W, double t0,
                                       double dt, int Nt, double2* __restrict__ A) {
    extern __shared__ double2 se[];
    const int Kt = 2 * Mt + 1;
    const int it = blockIdx.x;
    const double tt = t0 + it * dt;
    for (int mi = threadIdx.x; mi < Kt; mi += blockDim.x) {
        double s, c;
        sincos((mi - Mt) * W * tt, &s, &c);
        se[mi] = make_double2(c, s);
    }
    __syncthreads();
    for (int s = threadIdx.x; s < Ks; s += blockDim.x) {
        double2 acc = make_double2(0, 0);
        for (int mi = 0; mi < Kt; ++mi) {
            const double2 p = cmul(a[(int64_t)s * Kt + mi], se[mi]);
            acc.x += p.x;
            acc.y += p.y;
        }
        A[(int64_t)it * Ks + s] = acc;
    }
}

// u[t][py][px] = Re sum_{r,c} A_t[(r,c)] ey[r][py] ex[c][px]; one block per
// group of frames; ex/ey (with the (-1)^{mx+my} signs and the crop offsets of
// the period grid) are built in shared memory by the block.  Per frame the
// block forms B[r][px] = sum_c A_t[(r,c)] ex[c][px], then each of the 256
// threads accumulates a 4 x 4 set of pixels (py = ty + 16i, px = tx + 16j,
// over 64 x 64 pixel tiles): 32 FMAs per 8 complex shared-memory reads, the
// strided pixel map keeping those reads free of bank conflicts and the
// stores in 128-byte rows.
constexpr int kSynthFrames = 8;

template <typename OutT>
__global__ void __launch_bounds__(256) synth_kernel(const double2* __restrict__ A, const int32_t* __restrict__ smap,
                                                    int Ks, int Mx, int My, int Px, int Py, int Px1, int Py1, int Nt,
                                                    OutT* __restrict__ u) {
    extern __shared__ double2 sm2[];
    const int Kx = 2 * Mx + 1, Ky = 2 * My + 1;
    double2* ex = sm2;                 // Kx x Px
    double2* ey = ex + Kx * Px;        // Ky x Py
    double2* G = ey + Ky * Py;         // Ky x Kx (frame's coefficients on the grid)
    double2* B = G + Ky * Kx;          // Ky x Px
    const int xd = (Px1 - Px) / 2, yd = (Py1 - Py) / 2;
    for (int e = threadIdx.x; e < Kx * Px; e += blockDim.x) {
        const int c = e / Px, px = e % Px, mx = c - Mx;
        const int64_t r = ((((int64_t)mx * (px + xd)) % Px1) + Px1) % Px1;
        double s, co;
        sincospi(2.0 * r / Px1, &s, &co);
        const double sg = (mx & 1) ? -1.0 : 1.0;
        ex[e] = make_double2(sg * co, sg * s);
    }
    for (int e = threadIdx.x; e < Ky * Py; e += blockDim.x) {
        const int rr = e / Py, py = e % Py, my = My - rr;   // storage row rr holds my = My - rr
        const int64_t r = ((((int64_t)my * (py + yd)) % Py1) + Py1) % Py1;
        double s, co;
        sincospi(2.0 * r / Py1, &s, &co);
        const double sg = (my & 1) ? -1.0 : 1.0;
        ey[e] = make_double2(sg * co, sg * s);
    }
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int f0 = blockIdx.x * kSynthFrames;
    for (int f = f0; f < min(f0 + kSynthFrames, Nt); ++f) {
        __syncthreads();
        for (int e = threadIdx.x; e < Ky * Kx; e += blockDim.x) G[e] = make_double2(0, 0);
        __syncthreads();
        for (int s = threadIdx.x; s < Ks; s += blockDim.x) G[smap[s]] = A[(int64_t)f * Ks + s];
        __syncthreads();
        for (int e = threadIdx.x; e < Ky * Px; e += blockDim.x) {
            const int rr = e / Px, px = e % Px;
            double2 acc = make_double2(0, 0);
            for (int c = 0; c < Kx; ++c) {
                const double2 g = G[rr * Kx + c], x = ex[c * Px + px];
                acc.x = fma(g.x, x.x, fma(-g.y, x.y, acc.x));
                acc.y = fma(g.x, x.y, fma(g.y, x.x, acc.y));
            }
            B[e] = acc;
        }
        __syncthreads();
        OutT* uf = u + (int64_t)f * Px * Py;
        for (int y0 = 0; y0 < Py; y0 += 64) {
            for (int x0 = 0; x0 < Px; x0 += 64) {
                double acc[4][4];
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                    for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
                for (int rr = 0; rr < Ky; ++rr) {
                    double2 bv[4], ev[4];
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const int px = x0 + tx + 16 * j;
                        bv[j] = px < Px ? B[rr * Px + px] : make_double2(0, 0);
                    }
#pragma unroll
                    for (int i = 0; i < 4; ++i) {
                        const int py = y0 + ty + 16 * i;
                        ev[i] = py < Py ? ey[rr * Py + py] : make_double2(0, 0);
                    }
#pragma unroll
                    for (int i = 0; i < 4; ++i)
#pragma unroll
                        for (int j = 0; j < 4; ++j) acc[i][j] = fma(bv[j].x, ev[i].x, fma(-bv[j].y, ev[i].y, acc[i][j]));
                }
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const int py = y0 + ty + 16 * i;
                    if (py >= Py) continue;
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const int px = x0 + tx + 16 * j;
                        if (px < Px) uf[(int64_t)py * Px + px] = (OutT)acc[i][j];
                    }
                }
            }
        }
    }
}

// Fused synthesis over half the spectrum.  The spatial factors are
// Hermitian (ey[-my] = conj ey[my], ex[-mx] = conj ex[mx]), so the real part
// of the full sum pairs every (my, mx) with (-my, -mx):
//     u[py][px] = Re B[0][px] + sum_{my >= 1} Re(ey[my][py] B'[my][px]),
//     B'[my][px] = sum_mx (A_t[my][mx] + conj A_t[-my][-mx]) ex[mx][px]
//               = sum_k Y[k][py] X[k][px],  k < 2My+1 real rows
// (Y[0] = 1, Y[2my-1] = Re ey, Y[2my] = -Im ey; X[0] = Re B[0],
// X[2my-1] = Re B'[my], X[2my] = Im B'[my]); for the Hermitian-symmetric
// coefficients every decoder produces, B' = 2 B.  Per frame: the temporal
// expansion of the ellipse (a[s][m] staged in shared memory once per block),
// B for my >= 0, then the rank-(2My+1) real product, each thread a 4 x 4
// pixel block (8 shared-memory reads per 16 FMAs, two blocks per SM): 13 FMAs
// per voxel at Mx = My = 6, no intermediate buffer in HBM, streaming stores.
constexpr int kHalfMaxRows = 13;   // 2My+1 served by the fused kernel (My <= 6)

constexpr int kHalfFrames = 2;     // frames per iteration: more threads busy in the per-frame setup

template <typename OutT>
__global__ void __launch_bounds__(256, 2) synth_half_kernel(const double2* __restrict__ a,
                                                            const int32_t* __restrict__ smap, int Ks, int Mx, int My,
                                                            int Mt, double W, double t0, double dt, int Nt, int Px,
                                                            int Py, int Px1, int Py1, OutT* __restrict__ u) {
    extern __shared__ double2 hs[];
    const int Kx = 2 * Mx + 1, Ky = 2 * My + 1, Kt = 2 * Mt + 1, R = Ky, H = My + 1, KG = Ky * Kx;
    double2* ex = hs;                               // Kx x Px
    double2* as = ex + Kx * Px;                     // Ks x Kt
    double2* E = as + Ks * Kt;                      // kHalfFrames x Kt
    double2* G = E + kHalfFrames * Kt;              // kHalfFrames x Ky x Kx (zero outside the ellipse)
    double* X = reinterpret_cast<double*>(G + kHalfFrames * KG);   // kHalfFrames x R x Px
    double* Ys = X + kHalfFrames * R * Px;          // R x Py
    const int xd = (Px1 - Px) / 2, yd = (Py1 - Py) / 2;
    // spatial factors from one sincospi per pixel column / row and powers of
    // it (a few ulp per power; a per-entry sincospi here would cost more than
    // the frames a block renders)
    for (int px = threadIdx.x; px < Px; px += blockDim.x) {
        double sn, co;
        sincospi(2.0 * ((px + xd) % Px1) / Px1, &sn, &co);
        const double2 base = make_double2(co, sn);
        double2 pw = make_double2(1.0, 0.0);
        ex[Mx * Px + px] = pw;
        for (int mx = 1; mx <= Mx; ++mx) {
            pw = cmul(pw, base);
            const double sg = (mx & 1) ? -1.0 : 1.0;
            ex[(Mx + mx) * Px + px] = make_double2(sg * pw.x, sg * pw.y);
            ex[(Mx - mx) * Px + px] = make_double2(sg * pw.x, -sg * pw.y);
        }
    }
    for (int py = threadIdx.x; py < Py; py += blockDim.x) {
        double sn, co;
        sincospi(2.0 * ((py + yd) % Py1) / Py1, &sn, &co);
        const double2 base = make_double2(co, sn);
        double2 pw = make_double2(1.0, 0.0);
        Ys[py] = 1.0;
        for (int my = 1; my <= My; ++my) {
            pw = cmul(pw, base);
            const double sg = (my & 1) ? -1.0 : 1.0;
            Ys[(2 * my - 1) * Py + py] = sg * pw.x;
            Ys[(2 * my) * Py + py] = -sg * pw.y;
        }
    }
    // transposed, as[m][s]: the expansion's threads (consecutive s) read consecutive entries
    for (int e = threadIdx.x; e < Ks * Kt; e += blockDim.x) as[(e % Kt) * Ks + e / Kt] = a[e];
    for (int e = threadIdx.x; e < kHalfFrames * KG; e += blockDim.x) G[e] = make_double2(0, 0);
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    for (int f0 = blockIdx.x * kHalfFrames; f0 < Nt; f0 += gridDim.x * kHalfFrames) {
        const int nf = min(kHalfFrames, Nt - f0);
        __syncthreads();
        for (int q = threadIdx.x; q < nf; q += blockDim.x) {
            double sn, co;
            sincos(W * (t0 + (f0 + q) * dt), &sn, &co);
            const double2 base = make_double2(co, sn);
            double2 pw = make_double2(1.0, 0.0);
            E[q * Kt + Mt] = pw;
            for (int m = 1; m <= Mt; ++m) {
                pw = cmul(pw, base);
                E[q * Kt + Mt + m] = pw;
                E[q * Kt + Mt - m] = make_double2(pw.x, -pw.y);
            }
        }
        __syncthreads();
        for (int e = threadIdx.x; e < nf * Ks; e += blockDim.x) {
            const int q = e / Ks, sidx = e % Ks;
            double2 acc = make_double2(0, 0);
            for (int mi = 0; mi < Kt; ++mi) {
                const double2 p = cmul(as[mi * Ks + sidx], E[q * Kt + mi]);
                acc.x += p.x;
                acc.y += p.y;
            }
            G[q * KG + smap[sidx]] = acc;
        }
        __syncthreads();
        // storage row rr holds my = My - rr: rows rr <= My are my >= 0
        for (int e = threadIdx.x; e < nf * H * Px; e += blockDim.x) {
            const int q = e / (H * Px), r2 = e % (H * Px);
            const int my = r2 / Px, px = r2 % Px, rr = My - my;
            const double2* Gq = G + q * KG;
            double2 acc = make_double2(0, 0);
            for (int c = 0; c < Kx; ++c) {
                double2 g = Gq[rr * Kx + c];
                if (my > 0) {
                    const double2 gm = Gq[KG - 1 - (rr * Kx + c)];   // (-my, -mx)
                    g = make_double2(g.x + gm.x, g.y - gm.y);
                }
                const double2 x = ex[c * Px + px];
                acc.x = fma(g.x, x.x, fma(-g.y, x.y, acc.x));
                acc.y = fma(g.x, x.y, fma(g.y, x.x, acc.y));
            }
            double* Xq = X + q * R * Px;
            if (my == 0) {
                Xq[px] = acc.x;
            } else {
                Xq[(2 * my - 1) * Px + px] = acc.x;
                Xq[(2 * my) * Px + px] = acc.y;
            }
        }
        __syncthreads();
        // each thread: pixels (y0 + ty + 16i, x0 + tx + 16j), i, j < 4: the X
        // reads of a warp are 16 consecutive doubles, the Y reads two, both
        // free of bank conflicts, and the stores 128-byte rows
        for (int y0 = 0; y0 < Py; y0 += 64) {
            for (int q = 0; q < nf; ++q) {
                const double* Xq = X + q * R * Px;
                OutT* uf = u + (int64_t)(f0 + q) * Px * Py;
                for (int x0 = 0; x0 < Px; x0 += 64) {
                    double acc[4][4];
#pragma unroll
                    for (int i = 0; i < 4; ++i)
#pragma unroll
                        for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
#pragma unroll 1
                    for (int k = 0; k < R; ++k) {
                        double xv[4], yv[4];
#pragma unroll
                        for (int j = 0; j < 4; ++j) {
                            const int px = x0 + tx + 16 * j;
                            xv[j] = px < Px ? Xq[k * Px + px] : 0.0;
                        }
#pragma unroll
                        for (int i = 0; i < 4; ++i) {
                            const int py = y0 + ty + 16 * i;
                            yv[i] = py < Py ? Ys[k * Py + py] : 0.0;
                        }
#pragma unroll
                        for (int i = 0; i < 4; ++i)
#pragma unroll
                            for (int j = 0; j < 4; ++j) acc[i][j] = fma(yv[i], xv[j], acc[i][j]);
                    }
#pragma unroll
                    for (int i = 0; i < 4; ++i) {
                        const int py = y0 + ty + 16 * i;
                        if (py >= Py) continue;
#pragma unroll
                        for (int j = 0; j < 4; ++j) {
                            const int px = x0 + tx + 16 * j;
                            if (px < Px) __stcs(uf + (int64_t)py * Px + px, (OutT)acc[i][j]);
                        }
                    }
                }
            }
        }
    }
}

// Warp-specialised synthesis for frames up to 64 pixels wide with Mx, My <= 6
// (the decoder's usual orders).  Same sum as synth_half_kernel:
//     u[py][px] = sum_k Y[k][py] X_f[k][px],  k < 2My+1 real rows,
// with the per-frame rows X_f built from the expanded, Hermitian-folded
// coefficients.  Each 384-thread block renders a contiguous range of frames
// (balanced to one frame) with two roles that run concurrently:
//  * producer warps (4): per chunk of kFoldFrames frames, E = e^{j m W t} by
//    powers, A_t[s] = sum_m a[s][m] E[m] (consecutive threads on consecutive
//    s: contiguous coefficient reads, E broadcast) scattered into a zeroed
//    (2My+1) x (2Mx+1) grid, the fold
//        g[c] = A_t[my][c] + conj A_t[-my][-c]   (g = A_t[0] for my = 0),
//        Re = g0.x + sum_m (S.x exr - D.y exi),  Im = g0.y + sum_m (S.y exr + D.x exi),
//    S = g[m] + g[-m], D = g[m] - g[-m] (4 FMAs per |m|; exr/exi of the
//    thread's pixel column in registers), and per frame the X rows into one
//    of kWsSlots shared-memory slots;
//  * consumer warps (8): per frame, u = Y^T X on the float64 tensor cores
//    (mma.sync m8n8k4, k padded to a multiple of 4 with zero rows), warp w
//    rows 8w..8w+7 of a 64-row tile, all 64 columns; column pairs written
//    with streaming stores.
// The slots are handed over with named barriers (bar.arrive by the side that
// fills or frees a slot, bar.sync by the side that waits): both sides walk
// the same frame list, so every arrive has its matching sync and no wait is
// open-ended.  Row strides 68 (X) and 64k + 4 (Y) put the four k rows of an
// mma fragment on distinct banks.
constexpr int kFoldMaxM = 6;
constexpr int kFoldFrames = 8;
constexpr int kFoldXS = 68;
constexpr int kWsSlots = 3;
constexpr int kWsConsumers = 256;   // 8 warps
constexpr int kWsProducers = 128;   // 4 warps
constexpr int kWsThreads = kWsConsumers + kWsProducers;
// named barrier ids: 0 = __syncthreads, 1 = producers only, then FULL and EMPTY per slot
constexpr int kBarProd = 1, kBarFull = 2, kBarEmpty = 2 + kWsSlots;

// Barrier ids as immediates (so that only the ids used are reserved).
template <int ID>
__device__ __forceinline__ void named_sync(int n) {
    asm volatile("bar.sync %0, %1;\n" ::"n"(ID), "r"(n) : "memory");
}
template <int ID>
__device__ __forceinline__ void named_arrive(int n) {
    asm volatile("bar.arrive %0, %1;\n" ::"n"(ID), "r"(n) : "memory");
}
template <int BASE>
__device__ __forceinline__ void slot_sync(int slot, int n) {
    static_assert(kWsSlots == 3, "one case per slot");
    if (slot == 0) named_sync<BASE>(n);
    else if (slot == 1) named_sync<BASE + 1>(n);
    else named_sync<BASE + 2>(n);
}
template <int BASE>
__device__ __forceinline__ void slot_arrive(int slot, int n) {
    if (slot == 0) named_arrive<BASE>(n);
    else if (slot == 1) named_arrive<BASE + 1>(n);
    else named_arrive<BASE + 2>(n);
}

// D (8x8) += A (8x4) B (4x8) on the float64 tensor cores: lane l holds
// A[l/4][l%4], B[l%4][l/4] and D[l/4][2(l%4) + {0,1}].
__device__ __forceinline__ void dmma_8x8x4(double (&d)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}

__device__ __forceinline__ void store_pair(double* p, double x, double y) {
    __stcs(reinterpret_cast<double2*>(p), make_double2(x, y));
}
__device__ __forceinline__ void store_pair(float* p, double x, double y) {
    __stcs(reinterpret_cast<float2*>(p), make_float2((float)x, (float)y));
}

template <typename OutT, int MY>
__global__ void __launch_bounds__(kWsThreads, 2) synth_ws_kernel(const double2* __restrict__ a,
                                                                 const int32_t* __restrict__ smap, int Ks, int Mx,
                                                                 int Mt, double W, double t0, double dt, int Nt,
                                                                 int Px, int Py, int Px1, int Py1, int YS,
                                                                 OutT* __restrict__ u) {
    constexpr int R = 2 * MY + 1, H = MY + 1, KS = (R + 3) / 4;
    extern __shared__ double2 fs[];
    const int Kx = 2 * Mx + 1, Kt = 2 * Mt + 1, KG = R * Kx;
    const int RS = 2 + 4 * Mx;                              // doubles per folded row
    double2* as = fs;                                       // Kt x Ks (transposed)
    double2* E = as + Ks * Kt;                              // kFoldFrames x Kt
    double2* Ag = E + kFoldFrames * Kt;                     // kFoldFrames x KG (zero outside the ellipse)
    double* Fold = reinterpret_cast<double*>(Ag + kFoldFrames * KG);   // kFoldFrames x H x RS
    double* X = Fold + kFoldFrames * H * RS;                // kWsSlots x 16 x kFoldXS (rows >= R zero)
    double* Ys = X + kWsSlots * 16 * kFoldXS;               // 16 x YS (zero beyond Py and R)
    const int tid = threadIdx.x;
    for (int e = tid; e < 16 * YS; e += blockDim.x) Ys[e] = 0.0;
    for (int e = tid; e < kFoldFrames * KG; e += blockDim.x) Ag[e] = make_double2(0.0, 0.0);
    for (int e = tid; e < kWsSlots * 16 * kFoldXS; e += blockDim.x) X[e] = 0.0;
    __syncthreads();
    {
        const int yd = (Py1 - Py) / 2;
        for (int py = tid; py < Py; py += blockDim.x) {
            double sn, co;
            sincospi(2.0 * ((py + yd) % Py1) / Py1, &sn, &co);
            const double2 base = make_double2(co, sn);
            double2 pw = make_double2(1.0, 0.0);
            Ys[py] = 1.0;
            for (int my = 1; my <= MY; ++my) {
                pw = cmul(pw, base);
                const double sg = (my & 1) ? -1.0 : 1.0;
                Ys[(2 * my - 1) * YS + py] = sg * pw.x;
                Ys[(2 * my) * YS + py] = -sg * pw.y;
            }
        }
    }
    for (int e = tid; e < Ks * Kt; e += blockDim.x) as[(e % Kt) * Ks + e / Kt] = a[e];
    __syncthreads();
    const int fb = (int)((int64_t)blockIdx.x * Nt / gridDim.x);
    const int fe = (int)((int64_t)(blockIdx.x + 1) * Nt / gridDim.x);
    const int n = fe - fb;
    if (tid < kWsConsumers) {
        // ---- consumer: u = Y^T X per frame on the tensor cores
        const int warp = tid >> 5, lane = tid & 31;
        const bool vec2 = (Px % 2) == 0;                    // pair stores stay aligned
        for (int i = 0; i < n; ++i) {
            const int slot = i % kWsSlots;
            slot_sync<kBarFull>(slot, kWsThreads);
            const double* Xq = X + slot * 16 * kFoldXS;
            OutT* uf = u + (int64_t)(fb + i) * Px * Py;
            for (int y0 = 0; y0 < Py; y0 += 64) {
                const int r0 = y0 + 8 * warp;               // this warp's 8 rows
                if (r0 >= Py) continue;                     // warp-uniform
                double af[KS];                              // A = Y^T (8 rows x 4 k) fragments
#pragma unroll
                for (int ks = 0; ks < KS; ++ks) af[ks] = Ys[(4 * ks + (lane & 3)) * YS + r0 + (lane >> 2)];
                double acc[8][2];
#pragma unroll
                for (int t = 0; t < 8; ++t) acc[t][0] = acc[t][1] = 0.0;
#pragma unroll
                for (int ks = 0; ks < KS; ++ks) {
                    const double* Xk = Xq + (4 * ks + (lane & 3)) * kFoldXS + (lane >> 2);
#pragma unroll
                    for (int t = 0; t < 8; ++t) dmma_8x8x4(acc[t], af[ks], Xk[8 * t]);
                }
                const int py = r0 + (lane >> 2);
                if (py < Py) {
                    OutT* ur = uf + (int64_t)py * Px;
#pragma unroll
                    for (int t = 0; t < 8; ++t) {
                        const int px = 8 * t + 2 * (lane & 3);
                        if (px + 1 < Px && vec2) {
                            store_pair(ur + px, acc[t][0], acc[t][1]);
                        } else {
                            if (px < Px) __stcs(ur + px, (OutT)acc[t][0]);
                            if (px + 1 < Px) __stcs(ur + px + 1, (OutT)acc[t][1]);
                        }
                    }
                }
            }
            if (i + kWsSlots < n) slot_arrive<kBarEmpty>(slot, kWsThreads);
        }
        return;
    }
    // ---- producer: expansion, fold and X rows, kWsSlots frames ahead at most
    const int ptid = tid - kWsConsumers;
    const int cpx = ptid & 63;
    double exr[kFoldMaxM], exi[kFoldMaxM];
    {
        const int xd = (Px1 - Px) / 2;
        double sn = 0.0, co = 1.0;
        if (cpx < Px) sincospi(2.0 * ((cpx + xd) % Px1) / Px1, &sn, &co);
        const double2 base = make_double2(co, sn);
        double2 pw = make_double2(1.0, 0.0);
#pragma unroll
        for (int m = 0; m < kFoldMaxM; ++m) {
            pw = cmul(pw, base);
            const double sg = (m & 1) ? 1.0 : -1.0;         // (-1)^(m+1)
            exr[m] = sg * pw.x;
            exi[m] = sg * pw.y;
        }
    }
    int i = 0;
    for (int c0 = fb; c0 < fe; c0 += kFoldFrames) {
        const int nf = min(kFoldFrames, fe - c0);
        if (ptid < nf) {
            double sn, co;
            sincos(W * (t0 + (c0 + ptid) * dt), &sn, &co);
            const double2 base = make_double2(co, sn);
            double2 pw = make_double2(1.0, 0.0);
            double2* Eq = E + ptid * Kt;
            Eq[Mt] = pw;
            for (int m = 1; m <= Mt; ++m) {
                pw = cmul(pw, base);
                Eq[Mt + m] = pw;
                Eq[Mt - m] = make_double2(pw.x, -pw.y);
            }
        }
        named_sync<kBarProd>(kWsProducers);
        // temporal expansion: thread per (frame, ellipse entry)
        // two entries per thread at a time: four independent FMA chains
        for (int e0 = ptid; e0 < nf * Ks; e0 += 2 * kWsProducers) {
            const int e1 = min(e0 + kWsProducers, nf * Ks - 1);   // a duplicate of e0's work when past the end
            const int q0 = e0 / Ks, s0 = e0 - q0 * Ks, q1 = e1 / Ks, s1 = e1 - q1 * Ks;
            const double2 *E0 = E + q0 * Kt, *E1 = E + q1 * Kt;
            double ax0 = 0.0, ay0 = 0.0, ax1 = 0.0, ay1 = 0.0;
            for (int mi = 0; mi < Kt; ++mi) {
                const double2 c0 = as[mi * Ks + s0], v0 = E0[mi];
                const double2 c1 = as[mi * Ks + s1], v1 = E1[mi];
                ax0 = fma(c0.x, v0.x, fma(-c0.y, v0.y, ax0));
                ay0 = fma(c0.x, v0.y, fma(c0.y, v0.x, ay0));
                ax1 = fma(c1.x, v1.x, fma(-c1.y, v1.y, ax1));
                ay1 = fma(c1.x, v1.y, fma(c1.y, v1.x, ay1));
            }
            Ag[q0 * KG + __ldg(smap + s0)] = make_double2(ax0, ay0);
            if (e0 + kWsProducers < nf * Ks) Ag[q1 * KG + __ldg(smap + s1)] = make_double2(ax1, ay1);
        }
        named_sync<kBarProd>(kWsProducers);
        // fold: task (q, my, m), my in [0, My], m in [0, Mx]; grid row My - my'
        for (int e = ptid; e < nf * H * (Mx + 1); e += kWsProducers) {
            const int q = e / (H * (Mx + 1)), r = e % (H * (Mx + 1));
            const int my = r / (Mx + 1), m = r % (Mx + 1);
            const double2* Aq = Ag + q * KG;
            const double2* up = Aq + (MY - my) * Kx + Mx;   // row my, column 0
            const double2* dn = Aq + (MY + my) * Kx + Mx;   // row -my, column 0
            double* row = Fold + (q * H + my) * RS;
            if (m == 0) {
                double2 g = up[0];
                if (my > 0) g = make_double2(g.x + dn[0].x, g.y - dn[0].y);
                row[0] = g.x;
                row[1] = g.y;
            } else {
                double2 gp = up[m], gm = up[-m];
                if (my > 0) {
                    const double2 hp = dn[-m], hm = dn[m];
                    gp = make_double2(gp.x + hp.x, gp.y - hp.y);
                    gm = make_double2(gm.x + hm.x, gm.y - hm.y);
                }
                double* v = row + 2 + 4 * (m - 1);
                v[0] = gp.x + gm.x;
                v[1] = -(gp.y - gm.y);
                v[2] = gp.y + gm.y;
                v[3] = gp.x - gm.x;
            }
        }
        named_sync<kBarProd>(kWsProducers);
        for (int q = 0; q < nf; ++q, ++i) {
            const int slot = i % kWsSlots;
            if (i >= kWsSlots) slot_sync<kBarEmpty>(slot, kWsThreads);
            double* Xq = X + slot * 16 * kFoldXS;
            if (cpx < Px) {
                // this thread's rows my = g, g + 2, ... together: independent FMA chains
                constexpr int NR = (MY + 2) / 2;
                const int g = ptid >> 6;
                double re[NR], im[NR];
#pragma unroll
                for (int j = 0; j < NR; ++j) {
                    const int my = min(g + 2 * j, MY);
                    const double* row = Fold + (q * H + my) * RS;
                    re[j] = row[0];
                    im[j] = row[1];
                }
#pragma unroll
                for (int m = 0; m < kFoldMaxM; ++m) {
                    if (m < Mx) {
#pragma unroll
                        for (int j = 0; j < NR; ++j) {
                            const double* row = Fold + (q * H + min(g + 2 * j, MY)) * RS;
                            const double2 v01 = *reinterpret_cast<const double2*>(row + 2 + 4 * m);
                            const double2 v23 = *reinterpret_cast<const double2*>(row + 4 + 4 * m);
                            re[j] = fma(v01.x, exr[m], fma(v01.y, exi[m], re[j]));
                            im[j] = fma(v23.x, exr[m], fma(v23.y, exi[m], im[j]));
                        }
                    }
                }
#pragma unroll
                for (int j = 0; j < NR; ++j) {
                    const int my = g + 2 * j;
                    if (my > MY) continue;
                    if (my == 0) {
                        Xq[cpx] = re[j];
                    } else {
                        Xq[(2 * my - 1) * kFoldXS + cpx] = re[j];
                        Xq[(2 * my) * kFoldXS + cpx] = im[j];
                    }
                }
            }
            slot_arrive<kBarFull>(slot, kWsThreads);
        }
    }
}

template <typename OutT>
static void launch_ws(int My, int blocks, size_t smf, cudaStream_t s, const double2* a, const int32_t* smap, int Ks,
                      int Mx, int Mt, double W, double t0, double dt, int Nt, int Px, int Py, int Px1, int Py1, int YS,
                      OutT* u, cudaError_t* err) {
    auto go = [&](auto kern) {
        *err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smf);
        if (*err == cudaSuccess)
            kern<<<blocks, kWsThreads, smf, s>>>(a, smap, Ks, Mx, Mt, W, t0, dt, Nt, Px, Py, Px1, Py1, YS, u);
    };
    switch (My) {
        case 0: go(synth_ws_kernel<OutT, 0>); break;
        case 1: go(synth_ws_kernel<OutT, 1>); break;
        case 2: go(synth_ws_kernel<OutT, 2>); break;
        case 3: go(synth_ws_kernel<OutT, 3>); break;
        case 4: go(synth_ws_kernel<OutT, 4>); break;
        case 5: go(synth_ws_kernel<OutT, 5>); break;
        default: go(synth_ws_kernel<OutT, 6>); break;
    }
}

}  // namespace vtb

using namespace vtb;

VTB_API int vtb_coeff_temporal_gram(const double* tk1, const double* tk2, const int32_t* ind, int nspk, int N,
                                    const double* kappa, const double* delta, const double* bias, const double* norm,
                                    int Mt, double W, double* Wn, double* gn, void* stream) {
    VTB_CHECK_ARG(nspk >= 0 && N > 0 && Mt >= 1 && Mt <= 128 && Wn && gn && kappa && delta && bias && norm);
    VTB_CHECK_ARG(nspk == 0 || (tk1 && tk2 && ind));
    const int Kt = 2 * Mt + 1;
    const size_t sm = (size_t)kTChunk * (Kt + 1) * sizeof(double2);
    VTB_CHECK_ARG(Kt * (Kt + 1) / 2 <= 256 * kTgEntries);
    if (warp_per_neuron(Kt)) {
        temporal_gram_warp_kernel<<<ceil_div(N, kNrWarps), kNrWarps * 32, kNrWarps * sm, as_stream(stream)>>>(
            tk1, tk2, ind, nspk, N, kappa, delta, bias, norm, Mt, W, reinterpret_cast<double2*>(Wn),
            reinterpret_cast<double2*>(gn));
        return launch_status();
    }
    temporal_gram_kernel<<<N, 256, sm, as_stream(stream)>>>(tk1, tk2, ind, nspk, kappa, delta, bias, norm, Mt, W,
                                                           reinterpret_cast<double2*>(Wn),
                                                           reinterpret_cast<double2*>(gn));
    return launch_status();
}

VTB_API int vtb_coeff_pack(const double* Ds, int N, int Kfull, const int32_t* smap, int Ks, const double* norm,
                           double* d, void* stream) {
    VTB_CHECK_ARG(N > 0 && Ks > 0 && Ks <= Kfull && Ds && smap && norm && d);
    pack_d_kernel<<<ceil_div((int64_t)N * Ks, 256), 256, 0, as_stream(stream)>>>(
        reinterpret_cast<const double2*>(Ds), N, Kfull, smap, Ks, norm, reinterpret_cast<double2*>(d));
    return launch_status();
}

VTB_API int vtb_coeff_gram(const double* d, int N, int Ks, const double* Wn, const double* gn, int Kt, double* M,
                           int64_t ldm, double* b, void* stream) {
    VTB_CHECK_ARG(N > 0 && Ks > 0 && Kt > 0 && d && Wn && gn && M && b && ldm >= (int64_t)Ks * Kt);
    const int T = (Ks + kKT - 1) / kKT;
    const int tiles = T * (T + 1) / 2;
    kron_gram_kernel<<<tiles, 256, 0, as_stream(stream)>>>(reinterpret_cast<const double2*>(d), N, Ks,
                                                           reinterpret_cast<const double2*>(Wn), Kt,
                                                           reinterpret_cast<double2*>(M), ldm);
    int st = launch_status();
    if (st) return st;
    kron_rhs_kernel<<<rhs_grid(Ks), 256, rhs_smem(Kt), as_stream(stream)>>>(
        reinterpret_cast<const double2*>(d), N, Ks, reinterpret_cast<const double2*>(gn), Kt,
        reinterpret_cast<double2*>(b), rhs_chunk(Kt));
    return launch_status();
}

VTB_API int vtb_coeff_synthesize(const double* a, const int32_t* smap, int Ks, int Mx, int My, int Mt, double W,
                                 double t0, double dt, int Nt, int Px, int Py, int Px1, int Py1, double* A_work,
                                 void* u, int out_f32, void* stream) {
    VTB_CHECK_ARG(Ks > 0 && Mx >= 0 && My >= 0 && Mt >= 0 && Nt >= 0 && Px > 0 && Py > 0 && Px1 >= Px && Py1 >= Py);
    VTB_CHECK_ARG(2 * Mx + 1 <= Px1 && 2 * My + 1 <= Py1);
    if (Nt == 0) return VTB_OK;
    VTB_CHECK_ARG(a && smap && u);
    cudaStream_t s = as_stream(stream);
    const int Kt = 2 * Mt + 1;
    const int Kx = 2 * Mx + 1, Ky = 2 * My + 1;
    if (Px <= 64 && Mx <= kFoldMaxM && My <= kFoldMaxM && Py <= 256) {
        // warp-specialised kernel (A_work unused)
        const int H = My + 1, YS = ceil_div(Py, 64) * 64 + 4;   // padded: A fragments hit distinct banks
        const size_t smf = (size_t)(Ks * Kt + kFoldFrames * (Kt + Ky * Kx)) * sizeof(double2) +
                           (size_t)(kFoldFrames * H * (2 + 4 * Mx) + kWsSlots * 16 * kFoldXS + 16 * YS) *
                               sizeof(double);
        VTB_CHECK_ARG(smf <= 200 * 1024);
        const int blocks = (int)std::min<int64_t>(Nt, 2 * kNumSMs);
        cudaError_t err = cudaSuccess;
        if (out_f32)
            launch_ws<float>(My, blocks, smf, s, reinterpret_cast<const double2*>(a), smap, Ks, Mx, Mt, W, t0, dt, Nt,
                             Px, Py, Px1, Py1, YS, reinterpret_cast<float*>(u), &err);
        else
            launch_ws<double>(My, blocks, smf, s, reinterpret_cast<const double2*>(a), smap, Ks, Mx, Mt, W, t0, dt, Nt,
                              Px, Py, Px1, Py1, YS, reinterpret_cast<double*>(u), &err);
        VTB_CUDA_TRY(err);
        return launch_status();
    }
    if (Ky <= kHalfMaxRows) {
        // fused half-spectrum kernel (A_work unused)
        const size_t smh = (size_t)(Kx * Px + Ks * Kt + kHalfFrames * (Kt + Ky * Kx)) * sizeof(double2) +
                           (size_t)(kHalfFrames * Ky * Px + Ky * Py) * sizeof(double);
        VTB_CHECK_ARG(smh <= 200 * 1024);
        const int blocks = (int)std::min<int64_t>(ceil_div(Nt, kHalfFrames), 2 * kNumSMs);
        if (out_f32) {
            if (smh > 48 * 1024)
                VTB_CUDA_TRY(cudaFuncSetAttribute(synth_half_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                  (int)smh));
            synth_half_kernel<float><<<blocks, 256, smh, s>>>(reinterpret_cast<const double2*>(a), smap, Ks, Mx, My, Mt,
                                                              W, t0, dt, Nt, Px, Py, Px1, Py1,
                                                              reinterpret_cast<float*>(u));
        } else {
            if (smh > 48 * 1024)
                VTB_CUDA_TRY(cudaFuncSetAttribute(synth_half_kernel<double>,
                                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smh));
            synth_half_kernel<double><<<blocks, 256, smh, s>>>(reinterpret_cast<const double2*>(a), smap, Ks, Mx, My,
                                                               Mt, W, t0, dt, Nt, Px, Py, Px1, Py1,
                                                               reinterpret_cast<double*>(u));
        }
        return launch_status();
    }
    VTB_CHECK_ARG(A_work);
    temporal_expand_kernel<<<Nt, 128, Kt * sizeof(double2), s>>>(reinterpret_cast<const double2*>(a), Ks, Mt, W, t0,
                                                                 dt, Nt, reinterpret_cast<double2*>(A_work));
    int st = launch_status();
    if (st) return st;
    const size_t sm = (size_t)(Kx * Px + Ky * Py + Ky * Kx + Ky * Px) * sizeof(double2);
    VTB_CHECK_ARG(sm <= 200 * 1024);
    const int blocks = ceil_div(Nt, kSynthFrames);
    if (out_f32) {
        if (sm > 48 * 1024)
            VTB_CUDA_TRY(cudaFuncSetAttribute(synth_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        synth_kernel<float><<<blocks, 256, sm, s>>>(reinterpret_cast<const double2*>(A_work), smap, Ks, Mx, My, Px,
                                                   Py, Px1, Py1, Nt, reinterpret_cast<float*>(u));
    } else {
        if (sm > 48 * 1024)
            VTB_CUDA_TRY(cudaFuncSetAttribute(synth_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        synth_kernel<double><<<blocks, 256, sm, s>>>(reinterpret_cast<const double2*>(A_work), smap, Ks, Mx, My, Px,
                                                    Py, Px1, Py1, Nt, reinterpret_cast<double*>(u));
    }
    return launch_status();
}

// ---------------------------------------------------------------------------
// Synthesis for callers that cannot allocate device memory.
//
// Some hosts of this library cannot call cudaMalloc: a plugin running inside
// another runtime's fixed memory pool, a process whose allocations all go
// through a framework allocator it may not bypass, or code replayed inside
// an already-instantiated execution graph.  For them this variant keeps its
// temporal-expansion scratch in a fixed file-scope device array instead of a
// caller-provided buffer.  The array (kNoAllocScratchBytes = 4 MiB) exists on
// every GPU that loads the library, until the process exits.  Frames are
// processed in chunks that fit in it, so any clip length works as long as
// one frame's coefficients (Ks * 16 bytes) fit.
#include <mutex>

namespace vtb {

constexpr int64_t kNoAllocScratchBytes = 4ll << 20;
constexpr int64_t kNoAllocScratchElems = kNoAllocScratchBytes / (int64_t)sizeof(double2);

static __device__ __align__(256) double2 g_noalloc_synth_scratch[kNoAllocScratchElems];

// A[i][s] = sum_m a[s][m] e^{jmW t}, t = t0 + (f0 + i) dt, for i < gridDim.x
__global__ void temporal_expand_chunk_kernel(const double2* __restrict__ a, int Ks, int Mt, double W, double t0,
                                             double dt, int f0, double2* __restrict__ A) {
    extern __shared__ double2 se[];
    const int Kt = 2 * Mt + 1;
    const int it = f0 + blockIdx.x;
    const double tt = t0 + it * dt;
    for (int mi = threadIdx.x; mi < Kt; mi += blockDim.x) {
        double s, c;
        sincos((mi - Mt) * W * tt, &s, &c);
        se[mi] = make_double2(c, s);
    }
    __syncthreads();
    for (int s = threadIdx.x; s < Ks; s += blockDim.x) {
        double2 acc = make_double2(0, 0);
        for (int mi = 0; mi < Kt; ++mi) {
            const double2 p = cmul(a[(int64_t)s * Kt + mi], se[mi]);
            acc.x += p.x;
            acc.y += p.y;
        }
        A[(int64_t)blockIdx.x * Ks + s] = acc;
    }
}

// Device address of the scratch array on the current device (in host code
// the array's name is only a host-side stand-in).  Looked up on every call,
// not cached: after a device reset the module is loaded again and an older
// address would point at freed memory.  Only the first lookup on a device
// loads the module; later ones are a table lookup.
static double2* noalloc_scratch(int* status) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_synth_scratch);
    if (e != cudaSuccess || !p) {
        set_last_cuda_error(e);
        *status = VTB_CUDA_ERR;
        return nullptr;
    }
    return reinterpret_cast<double2*>(p);
}

}  // namespace vtb

VTB_API int vtb_coeff_synthesize_noalloc(const double* a, const int32_t* smap, int Ks, int Mx, int My, int Mt,
                                         double W, double t0, double dt, int Nt, int Px, int Py, int Px1, int Py1,
                                         void* u, int out_f32, void* stream) {
    VTB_CHECK_ARG(Ks > 0 && Mx >= 0 && My >= 0 && Mt >= 0 && Nt >= 0 && Px > 0 && Py > 0 && Px1 >= Px && Py1 >= Py);
    VTB_CHECK_ARG(2 * Mx + 1 <= Px1 && 2 * My + 1 <= Py1);
    // one frame of expanded coefficients must fit in the fixed scratch
    VTB_CHECK_ARG((int64_t)Ks <= kNoAllocScratchElems);
    if (Nt == 0) return VTB_OK;
    VTB_CHECK_ARG(a && smap && u);
    int st = VTB_OK;
    double2* scratch = noalloc_scratch(&st);
    if (!scratch) return st;
    cudaStream_t s = as_stream(stream);
    const int Kt = 2 * Mt + 1;
    const int Kx = 2 * Mx + 1, Ky = 2 * My + 1;
    const size_t sm = (size_t)(Kx * Px + Ky * Py + Ky * Kx + Ky * Px) * sizeof(double2);
    VTB_CHECK_ARG(sm <= 200 * 1024);
    if (sm > 48 * 1024) {
        if (out_f32)
            VTB_CUDA_TRY(cudaFuncSetAttribute(synth_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        else
            VTB_CUDA_TRY(cudaFuncSetAttribute(synth_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    }
    const int chunk = (int)std::min<int64_t>(kNoAllocScratchElems / Ks, (int64_t)Nt);
    const int64_t frame = (int64_t)Px * Py;
    for (int f0 = 0; f0 < Nt; f0 += chunk) {
        const int nf = std::min(chunk, Nt - f0);
        temporal_expand_chunk_kernel<<<nf, 128, Kt * sizeof(double2), s>>>(reinterpret_cast<const double2*>(a), Ks,
                                                                            Mt, W, t0, dt, f0, scratch);
        st = launch_status();
        if (st) return st;
        const int blocks = ceil_div(nf, kSynthFrames);
        if (out_f32)
            synth_kernel<float><<<blocks, 256, sm, s>>>(scratch, smap, Ks, Mx, My, Px, Py, Px1, Py1, nf,
                                                       reinterpret_cast<float*>(u) + f0 * frame);
        else
            synth_kernel<double><<<blocks, 256, sm, s>>>(scratch, smap, Ks, Mx, My, Px, Py, Px1, Py1, nf,
                                                        reinterpret_cast<double*>(u) + f0 * frame);
        st = launch_status();
        if (st) return st;
    }
    return VTB_OK;
}

// ---------------------------------------------------------------------------
// Mixed-precision pieces of the coefficient-space decoder.
//
// (1) The Kronecker Gram as one tensor-core GEMM.  For s <= s' (M is
//     Hermitian) and a_n = d_n[s] conj(d_n[s']),
//        M((s,m),(s',m')) = sum_n a_n W_n[m][m'],
//     and W_n is Hermitian, so the four real sums over n of
//     {a.re, a.im} x {W.re, W.im}[m][m'] for m <= m' give both
//     (m, m') (= sum a W) and (m', m) (= sum a conj W).  C = L R^T with
//     L[(pair, part), n] built from the RF bank only (split once per decoder)
//     and R[(u, part), n] for the Kt(Kt+1)/2 upper-triangular entries u of
//     W_n (split per decode): half the products of the real form of the
//     complex GEMM.  Split-bf16 products, fp32 accumulation.
// (2) The exact float64 residual r = Phi^H (q - Phi a) through the same
//     Kronecker factors (never forming M in float64), for refinement sweeps
//     on top of a factorisation of the tensor-core M.
namespace vtb {

// x -> bf16 hi at dst[0] and the bf16 of the remainder x - hi at dst[seg]
__device__ __forceinline__ void split_bf16_store(double x, __nv_bfloat16* dst, int seg) {
    const __nv_bfloat16 hi = __float2bfloat16_rn((float)x);
    dst[0] = hi;
    dst[seg] = __float2bfloat16_rn((float)(x - (double)__bfloat162float(hi)));
}

// L[row][seg * Kh + n], row = 2 * pair + part, Kh = N rounded up to 64,
// segments [hi | lo]: part 0 the real, part 1 the imaginary part of
// a_n[p] = d_n[s_p] conj(d_n[s'_p]) (zero for the padding n >= N).
__global__ void kron_lhs_sym_kernel(const double2* __restrict__ d, int N, int Ks, const int32_t* __restrict__ ps,
                                    const int32_t* __restrict__ ps2, int npairs, int Kh,
                                    __nv_bfloat16* __restrict__ L) {
    const int64_t total = (int64_t)npairs * Kh;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        const int p = (int)(e / Kh), n = (int)(e % Kh);
        double2 a = make_double2(0.0, 0.0);
        if (n < N) a = cmulc(d[(int64_t)n * Ks + ps[p]], d[(int64_t)n * Ks + ps2[p]]);
        __nv_bfloat16* row = L + (int64_t)(2 * p) * 2 * Kh + n;
        split_bf16_store(a.x, row, Kh);
        split_bf16_store(a.y, row + 2 * Kh, Kh);
    }
}

constexpr int kWnChunk = 32;  // neurons per block of kron_rhs_sym_kernel

// R[row][seg * Kh + n], row = 2u + part for the upper-triangular entries
// u = (m, m'), m <= m' (row-major order) of the Hermitian W_n, segments
// [hi | lo]: part 0 the real, part 1 the imaginary part of W_n[m][m'].
// Block (neuron chunk, m): row m of 32 neurons' W_n read contiguously into
// shared memory, then written as 32-neuron runs of each output row.
__global__ void __launch_bounds__(256) kron_rhs_sym_kernel(const double2* __restrict__ Wn, int N, int Kt, int Kh,
                                                           __nv_bfloat16* __restrict__ R) {
    __shared__ double2 sw[kWnChunk * 32];
    const int n0 = blockIdx.x * kWnChunk, m = blockIdx.y, nm = Kt - m, KK = Kt * Kt;
    for (int e = threadIdx.x; e < kWnChunk * nm; e += blockDim.x) {
        const int i = e / nm, j = e - i * nm;
        sw[i * nm + j] = n0 + i < N ? Wn[(int64_t)(n0 + i) * KK + m * Kt + m + j] : make_double2(0.0, 0.0);
    }
    __syncthreads();
    const int u0 = m * Kt - m * (m - 1) / 2;
    for (int e = threadIdx.x; e < nm * 2 * kWnChunk; e += blockDim.x) {
        const int i = e & (kWnChunk - 1), part = (e / kWnChunk) & 1, j = e / (2 * kWnChunk);
        const double2 w = sw[i * nm + j];
        split_bf16_store(part ? w.y : w.x, R + (int64_t)(2 * (u0 + j) + part) * 2 * Kh + n0 + i, Kh);
    }
}

// One block per neuron: v(m) = sum_s conj(d_n[s]) a(s, m); for each of the
// neuron's spikes y_k = q_k - Re sum_m T_k(m) v(m); g(m) = sum_k conj(T_k(m)) y_k.
__global__ void __launch_bounds__(256) coeff_residual_kernel(
    const double* __restrict__ tk1, const double* __restrict__ tk2, const int32_t* __restrict__ ind, int nspk,
    const double* __restrict__ kappa, const double* __restrict__ delta, const double* __restrict__ bias,
    const double* __restrict__ norm, int Mt, double W, const double2* __restrict__ d, int Ks,
    const double2* __restrict__ a, double2* __restrict__ gres) {
    extern __shared__ double2 sh[];
    const int Kt = 2 * Mt + 1;
    double2* v = sh;                 // Kt
    double2* T = v + Kt;             // kTChunk x Kt
    double* y = reinterpret_cast<double*>(T + kTChunk * Kt);  // kTChunk
    const int nr = blockIdx.x;
    int lo, hi;
    neuron_range(ind, nspk, nr, lo, hi);
    const double kd = kappa[nr] * delta[nr], bb = bias[nr], nn = norm[nr];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // v(m): warp w handles m = w, w+8, ...
    for (int m = w; m < Kt; m += 8) {
        double sr = 0.0, si = 0.0;
        for (int s = lane; s < Ks; s += 32) {
            const double2 dd = d[(int64_t)nr * Ks + s], aa = a[(int64_t)s * Kt + m];
            sr += dd.x * aa.x + dd.y * aa.y;   // conj(dd) * aa
            si += dd.x * aa.y - dd.y * aa.x;
        }
        for (int o = 16; o; o >>= 1) {
            sr += __shfl_xor_sync(0xffffffffu, sr, o);
            si += __shfl_xor_sync(0xffffffffu, si, o);
        }
        if (lane == 0) v[m] = make_double2(sr, si);
    }
    double2 gacc = make_double2(0, 0);
    for (int k0 = lo; k0 < hi; k0 += kTChunk) {
        const int nk = min(kTChunk, hi - k0);
        __syncthreads();
        if (threadIdx.x < nk) spike_T(tk1[k0 + threadIdx.x], tk2[k0 + threadIdx.x], Mt, W, T + threadIdx.x * Kt);
        __syncthreads();
        // y_k, one warp per spike
        for (int kk = w; kk < nk; kk += 8) {
            double acc = 0.0;
            for (int mi = lane; mi < Kt; mi += 32) {
                const double2 t = T[kk * Kt + mi], vv = v[mi];
                acc += t.x * vv.x - t.y * vv.y;
            }
            for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
            if (lane == 0) {
                const double qk = (kd - bb * (tk2[k0 + kk] - tk1[k0 + kk])) * nn;
                y[kk] = qk - acc;
            }
        }
        __syncthreads();
        if (threadIdx.x < Kt) {
            for (int kk = 0; kk < nk; ++kk) {
                const double2 t = T[kk * Kt + threadIdx.x];
                gacc.x += t.x * y[kk];
                gacc.y -= t.y * y[kk];
            }
        }
    }
    if (threadIdx.x < Kt) gres[(int64_t)nr * Kt + threadIdx.x] = gacc;
}

__global__ void zadd_kernel(double2* __restrict__ a, const double2* __restrict__ d, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = make_double2(a[i].x + d[i].x, a[i].y + d[i].y);
}

}  // namespace vtb

VTB_API int vtb_coeff_lhs_sym(const double* d, int N, int Ks, const int32_t* ps, const int32_t* ps2, int npairs,
                              void* L, void* stream) {
    VTB_CHECK_ARG(N > 0 && Ks > 0 && npairs > 0 && d && ps && ps2 && L && ((uintptr_t)L & 15) == 0);
    const int Kh = ceil_div(N, 64) * 64;
    const int64_t total = (int64_t)npairs * Kh;
    const int blocks = (int)std::min<int64_t>(ceil_div(total, 256), 32 * kNumSMs);
    kron_lhs_sym_kernel<<<blocks, 256, 0, as_stream(stream)>>>(reinterpret_cast<const double2*>(d), N, Ks, ps, ps2,
                                                               npairs, Kh, reinterpret_cast<__nv_bfloat16*>(L));
    return launch_status();
}

VTB_API int vtb_coeff_wn_sym(const double* Wn, int N, int Kt, void* R, void* stream) {
    VTB_CHECK_ARG(N > 0 && Kt > 0 && Kt <= 32 && Wn && R && ((uintptr_t)R & 15) == 0);
    const int Kh = ceil_div(N, 64) * 64;
    kron_rhs_sym_kernel<<<dim3(Kh / kWnChunk, Kt), 256, 0, as_stream(stream)>>>(
        reinterpret_cast<const double2*>(Wn), N, Kt, Kh, reinterpret_cast<__nv_bfloat16*>(R));
    return launch_status();
}

VTB_API int vtb_coeff_rhs(const double* d, int N, int Ks, const double* gn, int Kt, double* b, void* stream) {
    VTB_CHECK_ARG(N > 0 && Ks > 0 && Kt > 0 && d && gn && b);
    kron_rhs_kernel<<<rhs_grid(Ks), 256, rhs_smem(Kt), as_stream(stream)>>>(
        reinterpret_cast<const double2*>(d), N, Ks, reinterpret_cast<const double2*>(gn), Kt,
        reinterpret_cast<double2*>(b), rhs_chunk(Kt));
    return launch_status();
}

VTB_API int vtb_coeff_residual(const double* tk1, const double* tk2, const int32_t* ind, int nspk, int N,
                               const double* kappa, const double* delta, const double* bias, const double* norm,
                               int Mt, double W, const double* d, int Ks, const double* a, double* gres, double* r,
                               void* stream) {
    VTB_CHECK_ARG(nspk > 0 && N > 0 && Ks > 0 && Mt >= 1 && Mt <= 128 && tk1 && tk2 && ind && kappa && delta &&
                  bias && norm && d && a && gres && r);
    const int Kt = 2 * Mt + 1;
    const size_t sm = (size_t)Kt * sizeof(double2) + (size_t)kTChunk * Kt * sizeof(double2) + kTChunk * sizeof(double);
    cudaStream_t s = as_stream(stream);
    if (warp_per_neuron(Kt)) {
        const size_t smw = (size_t)(kTChunk * Kt + Kt + kTChunk) * sizeof(double2);
        coeff_residual_warp_kernel<<<ceil_div(N, kNrWarps), kNrWarps * 32, kNrWarps * smw, s>>>(
            tk1, tk2, ind, nspk, N, kappa, delta, bias, norm, Mt, W, reinterpret_cast<const double2*>(d), Ks,
            reinterpret_cast<const double2*>(a), reinterpret_cast<double2*>(gres));
    } else {
        coeff_residual_kernel<<<N, 256, sm, s>>>(tk1, tk2, ind, nspk, kappa, delta, bias, norm, Mt, W,
                                                 reinterpret_cast<const double2*>(d), Ks,
                                                 reinterpret_cast<const double2*>(a),
                                                 reinterpret_cast<double2*>(gres));
    }
    int st = launch_status();
    if (st) return st;
    kron_rhs_kernel<<<rhs_grid(Ks), 256, rhs_smem(Kt), s>>>(reinterpret_cast<const double2*>(d), N, Ks,
                                                            reinterpret_cast<const double2*>(gres), Kt,
                                                            reinterpret_cast<double2*>(r), rhs_chunk(Kt));
    return launch_status();
}

VTB_API int vtb_zadd(double* a, const double* d, int n, void* stream) {
    VTB_CHECK_ARG(n >= 0 && a && d);
    if (n == 0) return VTB_OK;
    zadd_kernel<<<ceil_div(n, 256), 256, 0, as_stream(stream)>>>(reinterpret_cast<double2*>(a),
                                                                 reinterpret_cast<const double2*>(d), n);
    return launch_status();
}

// g[n][m] = sum_{k in n} conj(T_k(m)) w_k for per-interval weights w (the
// coefficients c of the spike-space solve): with vtb_coeff_rhs this gives
// a = Phi^H c, the reconstruction coefficients of the reference's n x n
// pseudoinverse solution (used when a window has fewer intervals than
// coefficients, where the n x n system is the smaller one).
namespace vtb {
__global__ void __launch_bounds__(256) temporal_weighted_kernel(const double* __restrict__ tk1,
                                                                const double* __restrict__ tk2,
                                                                const int32_t* __restrict__ ind, int nspk,
                                                                const double* __restrict__ wk, int Mt, double W,
                                                                double2* __restrict__ g) {
    const int Kt = 2 * Mt + 1;
    const int nr = blockIdx.x;
    int lo, hi;
    neuron_range(ind, nspk, nr, lo, hi);
    for (int mi = threadIdx.x; mi < Kt; mi += blockDim.x) {
        const int m = mi - Mt;
        double gr = 0.0, gi = 0.0;
        for (int k = lo; k < hi; ++k) {
            const double a = tk1[k], b = tk2[k], d = b - a, w = wk[k];
            if (m == 0) {
                gr += d * w;
            } else {
                const double mw = m * W;
                const double amp = (2.0 / mw) * sin(0.5 * mw * d);
                double s, c;
                sincos(mw * (0.5 * (a + b)), &s, &c);
                gr += amp * c * w;   // conj(T) = amp e^{-j mW tbar}
                gi -= amp * s * w;
            }
        }
        g[(int64_t)nr * Kt + mi] = make_double2(gr, gi);
    }
}
}  // namespace vtb

VTB_API int vtb_coeff_from_spike_weights(const double* tk1, const double* tk2, const int32_t* ind, int nspk, int N,
                                         const double* w, int Mt, double W, const double* d, int Ks, double* g,
                                         double* a, void* stream) {
    VTB_CHECK_ARG(nspk > 0 && N > 0 && Ks > 0 && Mt >= 1 && tk1 && tk2 && ind && w && d && g && a);
    const int Kt = 2 * Mt + 1;
    cudaStream_t s = as_stream(stream);
    temporal_weighted_kernel<<<N, 64, 0, s>>>(tk1, tk2, ind, nspk, w, Mt, W, reinterpret_cast<double2*>(g));
    int st = launch_status();
    if (st) return st;
    kron_rhs_kernel<<<rhs_grid(Ks), 256, rhs_smem(Kt), s>>>(reinterpret_cast<const double2*>(d), N, Ks,
                                                            reinterpret_cast<const double2*>(g), Kt,
                                                            reinterpret_cast<double2*>(a), rhs_chunk(Kt));
    return launch_status();
}
