// Float32 Cholesky factorisation of ONE symmetric positive definite system
// (the mixed decoder's real-form coefficient system, K = 1921 at the GPU
// configuration), written for the B200 instead of cuSOLVER's spotrf, with the
// inverse of the factor formed in the same launch when asked for.
//
// spotrf at K = 1921 is latency-bound (a chain of dependent panel steps, 0.65
// ms for 2.4 GFLOP).  Here one cooperative launch factorises the matrix in
// 64 x 64 tiles (T = ceil(K/64) tile rows) as a data-flow graph:
//
//   CTA 0 ("diagonal") walks the critical path, step k = 0..T-1:
//     one panel factorisation [A_kk; I] -> [L_kk; L_kk^-T] with all its warps
//     (8-column blocks: warp 0 factorises and inverts each 8 x 8 diagonal
//     block while the others apply the previous block's update; the panel's
//     rows below a block are multiplied by its inverse); publishes L_kk^-1
//     (Dinv) first, then L_kk and the packed X_kk after the sub-diagonal;
//     the sub-diagonal tile L_{k+1,k} = A_{k+1,k} L_kk^-T as a product;
//     SYRK of the next diagonal tile A_{k+1,k+1} -= L_{k+1,k} L_{k+1,k}^T,
//     which it keeps in shared memory for step k+1.
//   CTAs 1.. ("workers") run every other piece: for tile (I,J) the updates
//     A_IJ -= sum_{k'} L_Ik' L_Jk'^T (the 4 x 4 register block of each thread
//     stays in registers across all of them), then for I >= J+2 the TRSM as
//     the product with the published L_JJ^-T.  Diagonal and sub-diagonal
//     tiles receive from the workers all updates but the last (the diagonal
//     CTA applies that one), so the diagonal CTA never waits on a round trip
//     through a worker for data its own previous step produced.  With the
//     inverse asked for, the workers also form X = L^-1 tile by tile,
//     X_ij = -X_ii sum_{k=j}^{i-1} L_ik X_kj, as soon as its operands are
//     published; the solves are then two matrix-vector products.
//
// Worker tasks are ordered by the step whose outputs they need ("group" g:
// the TRSM tiles (I, g) for I >= g+2, then the sub-diagonal (g+2, g+1), then
// the diagonal (g+2, g+2), pre-updated through g; the inverse tiles of row s
// before group s) and dealt round-robin; each worker runs its tasks in that
// order.  Every dependency of a task lies in an earlier position or in a
// diagonal step that depends only on earlier groups, so with all CTAs
// co-resident (cooperative launch) the graph cannot deadlock.
//
// Hand-offs: a tile's producer stores it, then (after a CTA barrier) thread
// 0 release-stores the tile's flag (release is cumulative: the barrier
// orders the other threads' stores before it); a consumer's thread 0 acquire-polls the flag, the CTA barrier
// follows, and the tile is read through L2 (ld.global.cg / cp.async.cg).
// Every wait is bounded: after the limit the CTA marks the call aborted
// (status 3) and all CTAs stop waiting and return.
//
// Rows and columns beyond K behave as the identity (0 off the diagonal, 1
// on it), so K needs no padding.  The factor L is written over the lower
// triangle of A (column-major, element (i, j) at j*ld + i, as spotrf leaves
// it); Dinv receives T tiles of 64 x 64 holding L_kk^-1 ROW-major (tile k at
// k*4096, element (r, c) at r*64 + c).  A failed pivot (<= 0 or not a
// number) or a spread of the squared pivots max/min >= 1/rcond sets the
// status word to 1 or 2, as vtb_sym_factor's pivot test does.
#include <cooperative_groups.h>

#include <algorithm>

#include "common.cuh"

namespace vtb {

constexpr int kCT = 64;               // tile
constexpr int kCTE = kCT * kCT;       // tile elements
constexpr int kCThreads = 256;
constexpr int kSMaxT = 160;           // solves: K <= 10240
constexpr unsigned kCholSpin = 1u << 20;

__device__ __forceinline__ unsigned c_ld_acquire(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void c_st_release(unsigned* p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;\n" ::"l"(p), "r"(v) : "memory");
}

struct CholCtx {
    float* A;
    int64_t ld;
    int K, T;
    float* Dinv;
    unsigned* tflag;     // T*T tile flags: 1 = worker part done, 2 = final L tile published
    int* abort_word;     // nonzero: some CTA gave up
    int32_t* status;     // caller's status word
    double* piv;         // caller's [min, max] squared pivots (may be null)
    double rcond;
    unsigned limit;
    float* Xinv;         // packed L^-1 tiles, row-major (null: no inverse)
    unsigned* xflag;     // T*T flags: 1 = X tile (i, j) published
    unsigned* pflag;     // T*T counts of the partial chunks of X tile (i, j) done
};

// thread 0 waits until *f >= v; every thread learns the outcome
__device__ bool cta_wait(const CholCtx& c, const unsigned* f, unsigned v, int* s_ok) {
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        unsigned it = 0;
        while (c_ld_acquire(f) < v) {
            if (++it > c.limit || *(volatile int*)c.abort_word != 0) {
                atomicExch(c.abort_word, 1);
                atomicMax(c.status, 3);
                ok = 0;
                break;
            }
        }
        *s_ok = ok;
    }
    __syncthreads();
    return *s_ok != 0;
}

// cta_wait on two flags at once (f2 may be null): thread 0 issues both loads
// per poll, so two flags that are already set cost one round trip
__device__ bool cta_wait2(const CholCtx& c, const unsigned* f1, unsigned v1, const unsigned* f2, unsigned v2,
                          int* s_ok) {
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        unsigned it = 0;
        for (;;) {
            const unsigned a = c_ld_acquire(f1);
            const unsigned b = f2 ? c_ld_acquire(f2) : v2;
            if (a >= v1 && b >= v2) break;
            if (++it > c.limit || *(volatile int*)c.abort_word != 0) {
                atomicExch(c.abort_word, 1);
                atomicMax(c.status, 3);
                ok = 0;
                break;
            }
        }
        *s_ok = ok;
    }
    __syncthreads();
    return *s_ok != 0;
}

// the CTA barrier orders every thread's stores before thread 0's release
// store, whose release semantics are cumulative at GPU scope
__device__ __forceinline__ void cta_publish(unsigned* f, unsigned v) {
    __syncthreads();
    if (threadIdx.x == 0) c_st_release(f, v);
}

// tile (I, J) of A into shared memory s (column-major, 64 x 64); entries
// beyond K are the identity's.  A tile inside K whose columns start on 16
// bytes (ld % 4 == 0, A aligned) is copied asynchronously (cp.async, 16-byte
// chunks, L2 only): the caller waits with cp.async.wait_group and a CTA
// barrier before reading it.  Other tiles are loaded synchronously.  Every
// call commits exactly one cp.async group (empty for a synchronous load), so
// callers can count groups.
__device__ __forceinline__ void cp_async16(float* dst, const float* src) {
    const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

__device__ void load_tile(const CholCtx& c, float* s, int I, int J) {
    const int r0 = I * kCT, c0 = J * kCT;
    const bool full = r0 + kCT <= c.K && c0 + kCT <= c.K;
    if (full && (c.ld & 3) == 0 && ((uintptr_t)c.A & 15) == 0) {
        for (int e = threadIdx.x; e < kCTE / 4; e += kCThreads) {
            const int cc = e >> 4, r = (e & 15) * 4;
            cp_async16(s + cc * kCT + r, c.A + (int64_t)(c0 + cc) * c.ld + r0 + r);
        }
        cp_async_commit();
        return;
    }
    for (int e = threadIdx.x; e < kCTE; e += kCThreads) {
        const int cc = e >> 6, r = e & 63;
        const int gr = r0 + r, gc = c0 + cc;
        float v;
        if (full || (gr < c.K && gc < c.K)) v = __ldcg(c.A + (int64_t)gc * c.ld + gr);
        else v = gr == gc ? 1.f : 0.f;
        s[e] = v;
    }
    cp_async_commit();   // an empty group: every call commits exactly one
}

__device__ __forceinline__ unsigned c_ld_relaxed(const unsigned* p) {
    unsigned v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// The diagonal CTA's look-ahead copies: during the panel factorisation of
// step k, warp 7 leaves the panel (whose barriers then count warps 0-6 only)
// and polls the flags of the next sub-diagonal and diagonal tiles with
// relaxed loads (each read one poll later); a tile whose flag it saw set is
// ordered after the flag (one fence for all such tiles) and copied by warp
// 7's own cp.async groups.  The fences and copies never hold up a panel
// barrier.  Only full, 16-byte-aligned tiles are copied this way; the others
// take the CTA-wide path.
struct LookAhead {
    const unsigned* f[2];
    float* dst[2];
    int I[2], J[2];
    unsigned seen[2];  // the flag values the last poll read
    bool on[2];
    int issued;        // tiles whose copies were issued (bits)
};

// one poll of warp 7: fence and copy the tiles whose flags the previous poll
// saw set, then new relaxed looks at the other flags
__device__ __forceinline__ void look_ahead_poll(const CholCtx& c, LookAhead& la) {
    const int lane = threadIdx.x & 31;
    int nb = 0;
#pragma unroll
    for (int t = 0; t < 2; ++t)
        if (la.on[t] && !((la.issued >> t) & 1) && la.seen[t] >= 1u) nb |= 1 << t;
    if (nb) {
        asm volatile("fence.acq_rel.gpu;\n" ::: "memory");
        __syncwarp();
#pragma unroll
        for (int t = 0; t < 2; ++t) {
            if (!((nb >> t) & 1)) continue;
            const int r0 = la.I[t] * kCT, c0 = la.J[t] * kCT;
            for (int e = lane; e < kCTE / 4; e += 32) {
                const int cc = e >> 4, r = (e & 15) * 4;
                cp_async16(la.dst[t] + cc * kCT + r, c.A + (int64_t)(c0 + cc) * c.ld + r0 + r);
            }
        }
        cp_async_commit();
        la.issued |= nb;
    }
#pragma unroll
    for (int t = 0; t < 2; ++t)
        if (la.on[t] && !((la.issued >> t) & 1)) la.seen[t] = c_ld_relaxed(la.f[t]);
}

__device__ __forceinline__ bool look_ahead_open(const LookAhead& la) {
    return (la.on[0] && !(la.issued & 1)) || (la.on[1] && !(la.issued & 2));
}

// barrier of the panel's warps 0-6 (warp 7 runs the look-ahead meanwhile)
__device__ __forceinline__ void panel_sync() { asm volatile("bar.sync 1, 224;" ::: "memory"); }

constexpr int kLookAheadPolls = 1 << 12;   // bound of warp 7's poll loop (a panel takes ~30 polls)

// thread 0 checks *f >= v once (no wait); every thread learns the answer
__device__ bool cta_ready(const unsigned* f, unsigned v, int* s_ok) {
    __syncthreads();
    if (threadIdx.x == 0) *s_ok = c_ld_acquire(f) >= v;
    __syncthreads();
    return *s_ok != 0;
}

// two such checks in one round trip (thread 0 issues both loads before
// using either); bit 0 of the result for f1, bit 1 for f2
__device__ int cta_ready2(const unsigned* f1, unsigned v1, const unsigned* f2, unsigned v2, int* s_ok) {
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned a = c_ld_acquire(f1), b = c_ld_acquire(f2);
        *s_ok = (a >= v1 ? 1 : 0) | (b >= v2 ? 2 : 0);
    }
    __syncthreads();
    return *s_ok;
}

// shared tile s into tile (I, J) of A (rows and columns below K; for a
// diagonal tile the lower triangle only)
__device__ void store_tile(const CholCtx& c, const float* s, int I, int J) {
    const int r0 = I * kCT, c0 = J * kCT;
    if (r0 + kCT <= c.K && c0 + kCT <= c.K && (c.ld & 3) == 0 && ((uintptr_t)c.A & 15) == 0) {
        // full tile: 16-byte stores (4 rows of a column); a diagonal tile keeps
        // the matrix's upper triangle (chunks across the diagonal entry by entry)
        for (int e = threadIdx.x; e < kCTE / 4; e += kCThreads) {
            const int cc = e >> 4, r = (e & 15) * 4;
            float* g = c.A + (int64_t)(c0 + cc) * c.ld + r0 + r;
            const float4 v = reinterpret_cast<const float4*>(s)[e];
            if (I != J || r >= cc) {
                __stcg(reinterpret_cast<float4*>(g), v);
            } else if (r + 3 >= cc) {
                if (r + 1 >= cc) __stcg(g + 1, v.y);
                if (r + 2 >= cc) __stcg(g + 2, v.z);
                __stcg(g + 3, v.w);
            }
        }
        return;
    }
    for (int e = threadIdx.x; e < kCTE; e += kCThreads) {
        const int cc = e >> 6, r = e & 63;
        const int gr = r0 + r, gc = c0 + cc;
        if (gr < c.K && gc < c.K && (I != J || r >= cc)) __stcg(c.A + (int64_t)gc * c.ld + gr, s[e]);
    }
}

// acc[i][j] -= p_i q_j over a 4 x 4 patch with the packed FP32 FMA (rows in
// pairs, two fma.rn per instruction: the same roundings as fmaf)
__device__ __forceinline__ void rank1_sub(float (&acc)[4][4], float4 p, const float (&q)[4]) {
    const float2 p01 = make_float2(p.x, p.y), p23 = make_float2(p.z, p.w);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const float2 nq = make_float2(-q[j], -q[j]);
        const float2 a01 = __ffma2_rn(p01, nq, make_float2(acc[0][j], acc[1][j]));
        const float2 a23 = __ffma2_rn(p23, nq, make_float2(acc[2][j], acc[3][j]));
        acc[0][j] = a01.x;
        acc[1][j] = a01.y;
        acc[2][j] = a23.x;
        acc[3][j] = a23.y;
    }
}

// acc[i][j] -= sum_{t0 <= t < t1} P[t][4tr+i] Q[t][4tc+j]  (P, Q column-major 64 x 64)
__device__ __forceinline__ void sub_ptq(float (&acc)[4][4], const float* P, const float* Q, int tr, int tc, int t0,
                                        int t1) {
#pragma unroll 4
    for (int t = t0; t < t1; ++t) {
        const float4 p = *reinterpret_cast<const float4*>(P + t * kCT + 4 * tr);
        const float4 q = *reinterpret_cast<const float4*>(Q + t * kCT + 4 * tc);
        const float qv[4] = {q.x, q.y, q.z, q.w};
        rank1_sub(acc, p, qv);
    }
}

// acc[i][j] -= sum_t P[t][4tr+i] Q[4tc+j][t]  (P column-major 64 x 64; Q with the t index contiguous: Q[c][t]
// at Q + c*64 + t).  The Q reads of a quarter-warp are one address (same tc): broadcasts.
__device__ __forceinline__ void sub_pq_rowq(float (&acc)[4][4], const float* P, const float* Q, int tr, int tc) {
#pragma unroll 2
    for (int t = 0; t < kCT; t += 4) {
        float4 q[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) q[j] = *reinterpret_cast<const float4*>(Q + (4 * tc + j) * kCT + t);
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const float4 p = *reinterpret_cast<const float4*>(P + (t + u) * kCT + 4 * tr);
            float qv[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) qv[j] = u == 0 ? q[j].x : u == 1 ? q[j].y : u == 2 ? q[j].z : q[j].w;
            rank1_sub(acc, p, qv);
        }
    }
}

__device__ __forceinline__ void acc_from(float (&acc)[4][4], const float* s, int tr, int tc) {
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = s[(4 * tc + j) * kCT + 4 * tr + i];
}

__device__ __forceinline__ void acc_to(const float (&acc)[4][4], float* s, int tr, int tc) {
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) s[(4 * tc + j) * kCT + 4 * tr + i] = acc[i][j];
}

// ---------------------------------------------------------------- 64 x 64 POTRF
// The 8 x 8 diagonal block at (8bb, 8bb) of the column-major 64 x 64 tile S,
// in one warp: every lane loads the whole block (broadcast reads) and
// factorises it in its registers, so no step waits on another lane; the
// warp then writes L (zeros above the diagonal) and rinv[8bb + j] = 1/L_jj.
// Pivots of rows beyond K (nvalid: rows of the tile below K) do not enter
// pmin/pmax; a pivot <= 0 or NaN sets bad.
__device__ __forceinline__ void potrf8_warp(float* S, float* rinv, int bb, float& pmin, float& pmax, int& bad,
                                            int nvalid) {
    const int o = 8 * bb;
    float a[8][8];     // a[i][j]: row i, column j (lower part used)
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const float4 lo = *reinterpret_cast<const float4*>(S + (o + j) * kCT + o);
        const float4 hi = *reinterpret_cast<const float4*>(S + (o + j) * kCT + o + 4);
        a[0][j] = lo.x; a[1][j] = lo.y; a[2][j] = lo.z; a[3][j] = lo.w;
        a[4][j] = hi.x; a[5][j] = hi.y; a[6][j] = hi.z; a[7][j] = hi.w;
    }
    float rs[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        float p = a[j][j];
        if (!(p > 0.f)) {
            bad = 1;
            p = 1.f;
        }
        if (o + j < nvalid) {
            pmin = fminf(pmin, p);
            pmax = fmaxf(pmax, p);
        }
        rs[j] = rsqrtf(p);
#pragma unroll
        for (int i = j; i < 8; ++i) a[i][j] *= rs[j];
#pragma unroll
        for (int c = j + 1; c < 8; ++c)
#pragma unroll
            for (int i = c; i < 8; ++i) a[i][c] = fmaf(-a[i][j], a[c][j], a[i][c]);
    }
    // every lane holds the same values: warp-wide stores to one address each
    // (no divergent branch, one shared-memory wavefront per store)
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        float col[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) col[i] = i >= c ? a[i][c] : 0.f;
        *reinterpret_cast<float4*>(S + (o + c) * kCT + o) = make_float4(col[0], col[1], col[2], col[3]);
        *reinterpret_cast<float4*>(S + (o + c) * kCT + o + 4) = make_float4(col[4], col[5], col[6], col[7]);
    }
    *reinterpret_cast<float4*>(rinv + o) = make_float4(rs[0], rs[1], rs[2], rs[3]);
    *reinterpret_cast<float4*>(rinv + o + 4) = make_float4(rs[4], rs[5], rs[6], rs[7]);
}

// row r of column block bb: x <- x L_bb^-T by substitution (x the row's 8
// entries in that block, already updated by every earlier block)
__device__ __forceinline__ void subst_row8(float* X, const float* L, const float* rinv, int bb, int r) {
    const int o = 8 * bb;
    float x[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) x[c] = X[(o + c) * kCT + r];
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        float v = x[c];
#pragma unroll
        for (int t = 0; t < c; ++t) v = fmaf(-x[t], L[(o + t) * kCT + o + c], v);
        x[c] = v * rinv[o + c];
    }
#pragma unroll
    for (int c = 0; c < 8; ++c) X[(o + c) * kCT + r] = x[c];
}

// X[r0..r0+3][c0..c0+3] -= sum_{t<8} X[r0..][o+t] L[c0..][o+t]: one 4 x 4 patch of
// a rank-8 update (X, L column-major 64 x 64 in shared memory)
__device__ __forceinline__ void patch_update(float* X, const float* L, int r0, int c0, int o) {
    float acc[4][4];
#pragma unroll
    for (int jj = 0; jj < 4; ++jj) {
        const float4 v = *reinterpret_cast<const float4*>(X + (c0 + jj) * kCT + r0);
        acc[0][jj] = v.x;
        acc[1][jj] = v.y;
        acc[2][jj] = v.z;
        acc[3][jj] = v.w;
    }
#pragma unroll
    for (int t = 0; t < 8; ++t) {
        const float4 pv = *reinterpret_cast<const float4*>(X + (o + t) * kCT + r0);
        const float4 qv = *reinterpret_cast<const float4*>(L + (o + t) * kCT + c0);
        const float qa[4] = {qv.x, qv.y, qv.z, qv.w};
        rank1_sub(acc, pv, qa);
    }
#pragma unroll
    for (int jj = 0; jj < 4; ++jj)
        *reinterpret_cast<float4*>(X + (c0 + jj) * kCT + r0) = make_float4(acc[0][jj], acc[1][jj], acc[2][jj], acc[3][jj]);
}

// Cholesky and inverse of the symmetric positive definite 64 x 64 tile S
// (column-major, lower triangle read), as ONE panel [S; E] with E = I:
// S <- L (zeros above the diagonal), E <- I L^-T = L^-T (column-major, i.e.
// L^-1 row-major), rinv <- 1/diag(L).  Blocks of 8 columns, all 8 warps:
// after the column block bb is solved (one thread per panel row that is not
// zero in it: the rows of S below the block and rows 0..8bb+7 of E, 64 in
// all), warp 0 updates and factorises the next diagonal block while warps 1-7
// apply the rank-8 update to the rest of the panel in 4 x 4 register patches
// (consecutive threads on consecutive row patches of one column patch:
// conflict-free rows, broadcast column operand).  Rows 8bb+8.. of E are
// still the identity's in the columns of block bb and need no work.
__device__ void potrf_inv64(const CholCtx& c, float* S, float* E, float* rinv, float& pmin, float& pmax, int& bad,
                            int nvalid, LookAhead& la, volatile int* done) {
    const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
    if (w == 0) {
        potrf8_warp(S, rinv, 0, pmin, pmax, bad, nvalid);
    } else {
        for (int e = tid - 32; e < kCTE / 4; e += kCThreads - 32) {
            const int col = e >> 4, r = (e & 15) * 4;
            *reinterpret_cast<float4*>(E + 4 * e) =
                make_float4(r == col ? 1.f : 0.f, r + 1 == col ? 1.f : 0.f, r + 2 == col ? 1.f : 0.f,
                            r + 3 == col ? 1.f : 0.f);
        }
    }
    __syncthreads();
    if (w == kCThreads / 32 - 1) {
        // warp 7: the look-ahead, until both tiles are on their way or the panel is done
        for (int it = 0; it < kLookAheadPolls && look_ahead_open(la) && !*done; ++it) look_ahead_poll(c, la);
        __syncthreads();
        return;
    }
    // blocks past the last row inside K (the last tile of a K that is not a
    // multiple of 64) hold the identity and stay as they are
    const int nb = nvalid >= kCT ? 8 : max(1, (nvalid + 7) / 8);
    for (int bb = 0; bb < 8; ++bb) {
        const int o = 8 * bb, c0 = o + 8, nd = kCT - c0;
        if (tid < kCT) {
            // one code path for both kinds of row (no divergence inside a warp)
            const bool srow = tid < nd;
            subst_row8(srow ? S : E, S, rinv, bb, srow ? c0 + tid : tid - nd);
        }
        panel_sync();
        if (bb == nb - 1) break;
        if (w == 0) {
            // next diagonal block: S[c0+i][c0+j] -= sum_t L[c0+i][o+t] L[c0+j][o+t], two entries per lane
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int e = lane + 32 * h, i = e & 7, j = e >> 3;
                float v = S[(c0 + j) * kCT + c0 + i];
#pragma unroll
                for (int t = 0; t < 8; ++t) v = fmaf(-S[(o + t) * kCT + c0 + i], S[(o + t) * kCT + c0 + j], v);
                S[(c0 + j) * kCT + c0 + i] = v;
            }
            __syncwarp();
            potrf8_warp(S, rinv, bb + 1, pmin, pmax, bad, nvalid);
        } else {
            // warps 1-6: E rows 0..c0-1 (2bb+2 row patches) x columns [c0, 64); then the lower
            // triangle of S's rows and columns [c0, 64) without the next diagonal block
            const int m = nd / 4, me = 2 * bb + 2, ne = me * m;
            for (int q = tid - 32; q < ne + m * m; q += kCThreads - 64) {
                // one code path for E and S patches (no divergence inside a warp)
                const bool ep = q < ne;
                const int q2 = q - ne, pc = q2 / m, pr = q2 % m;
                if (!ep && (pr < pc || (pr < 2 && pc < 2))) continue;
                patch_update(ep ? E : S, S, ep ? 4 * (q % me) : c0 + 4 * pr, c0 + 4 * (ep ? q / me : pc), o);
            }
        }
        panel_sync();
    }
    // the panel is done: warp 7 stops polling and joins
    if (tid == 0) *done = 1;
    __syncthreads();
}

// ---------------------------------------------------------------- worker tasks
// Factorisation tasks, group g (0 <= g <= T-3), T-g of them: the TRSM tiles
// (I, g) for I = g+2..T-1 (type 0), then the sub-diagonal (g+2, g+1) (type 1)
// and the diagonal (g+2, g+2) (type 2), pre-updated through g.
//
// Inverse tasks (when L^-1 is asked for), X_ij = -X_ii S_ij with
// S_ij = sum_{k=j}^{i-1} L_ik X_kj (the diagonal CTA forms X_ii = L_ii^-1):
// the terms k = j..i-2 are summed in chunks of kXChunk consecutive k
// (type 4, the chunk ending at k1 runs as soon as L_{i,k1} and X_{k1,j}
// exist), each chunk adding to the running partial -S_ij kept in X_ij's own
// storage; the last term k = i-1 and the product with X_ii are the final
// task (type 5), so after the last diagonal step only one product per tile
// of the last row remains.
//
// The workers form two pools (half each when the inverse is asked for): one
// runs the factorisation tasks in group order, the other the inverse tasks
// in slot order, s = 0..T-1: the chunks ending at k1 = s-1 (rows i >= s+1),
// then the final tasks of row s.  A factorisation group s needs the
// diagonal steps <= s and earlier groups; the diagonal step s needs groups
// <= s-1; a chunk ending at s-1 needs L_{i,s-1} (group s-1 or step s-1),
// rows <= s-1 of X and the row's earlier chunks; a final task of row s needs
// step s and row s-1 of X.  The factorisation never waits on the inverse,
// and within each pool every dependency lies earlier in its order (or in the
// other pool, or on the diagonal), so with every CTA resident no task waits
// on one behind it.
constexpr int kXChunk = 4;

// factorisation task t in group order
__device__ __forceinline__ void factor_task(int T, int t, int& I, int& J, int& type) {
    for (int g = 0; g <= T - 3; ++g) {
        const int n = T - g, n0 = T - g - 2;
        if (t < n) {
            if (t < n0) { I = g + 2 + t; J = g; type = 0; }
            else if (t == n0) { I = g + 2; J = g + 1; type = 1; }
            else { I = g + 2; J = g + 2; type = 2; }
            return;
        }
        t -= n;
    }
    I = J = type = -1;
}

__host__ __device__ __forceinline__ int factor_count(int T) { return T >= 3 ? T * (T + 1) / 2 - 3 : 0; }

// inverse task t in slot order
__device__ __forceinline__ void inverse_task(int T, int t, int& I, int& J, int& type, int& k0, int& k1) {
    for (int sl = 0; sl < T; ++sl) {
        // chunks of row sl+1 ending at its last non-final term k = sl-1 (possibly short)
        if (sl >= 1 && sl + 1 <= T - 1) {
            if (t < sl) {
                I = sl + 1;
                J = t;
                k1 = sl - 1;
                k0 = J + ((k1 - J) / kXChunk) * kXChunk;
                type = 4;
                return;
            }
            t -= sl;
        }
        // full chunks [sl-kXChunk, sl-1] of rows sl+2..T-1
        const int nb = sl / kXChunk;
        if (nb > 0 && T - 1 >= sl + 2) {
            const int cnt = (T - 2 - sl) * nb;
            if (t < cnt) {
                I = sl + 2 + t / nb;
                J = sl - kXChunk - kXChunk * (t % nb);
                k0 = sl - kXChunk;
                k1 = sl - 1;
                type = 4;
                return;
            }
            t -= cnt;
        }
        // final tasks of row sl
        if (t < sl) {
            I = sl;
            J = t;
            k0 = k1 = sl - 1;
            type = 5;
            return;
        }
        t -= sl;
    }
    I = J = type = k0 = k1 = -1;
}

__host__ __device__ __forceinline__ int inverse_count(int T) {
    int n = 0;
    for (int sl = 0; sl < T; ++sl) {
        if (sl >= 1 && sl + 1 <= T - 1) n += sl;
        if (T - 1 >= sl + 2) n += (T - 2 - sl) * (sl / kXChunk);
        n += sl;
    }
    return n;
}

// Inverse tasks of the last kTailSlots slots go round-robin over ALL workers
// (the factorisation pool runs out of work there while these chunks pile
// up); the index of the first of them in slot order.
constexpr int kTailSlots = 4;

__host__ __device__ __forceinline__ int inverse_tail_start(int T) {
    int n = 0;
    for (int sl = 0; sl < T - kTailSlots; ++sl) {
        if (sl >= 1 && sl + 1 <= T - 1) n += sl;
        if (T - 1 >= sl + 2) n += (T - 2 - sl) * (sl / kXChunk);
        n += sl;
    }
    return n;
}

__host__ __device__ __forceinline__ int task_count(int T, bool inv) {
    return factor_count(T) + (inv ? inverse_count(T) : 0);
}

// workers of the factorisation when the inverse is formed too (the rest form
// the inverse); all of them without it
__host__ __device__ __forceinline__ int factor_workers(int W, int T, bool inv) {
    if (!inv || inverse_count(T) == 0) return W;
    if (factor_count(T) == 0) return 0;
    const int wf = W / 2;
    return wf < 1 ? 1 : wf;
}

// packed lower-triangular tile index of (i, j), i >= j
__device__ __forceinline__ int64_t packed_tile(int i, int j) { return (int64_t)i * (i + 1) / 2 + j; }

struct CholSmem {
    float a[2][kCTE];     // worker: operand L_Ik' (double buffer); diagonal CTA: current and next diagonal tile
    float b[2][kCTE];     // worker: operand L_Jk' (double buffer), then L_JJ^-1; diagonal CTA: sub-diagonal tile
    float x[kCTE];        // worker: the task's tile (staging); diagonal CTA: L_kk^-T
    float rinv[kCT];
    int ok;
    int la;               // diagonal CTA: look-ahead tiles copied in (bit 0 sub-diagonal, bit 1 diagonal)
    int panel_done;       // diagonal CTA: set when the panel factorisation ends (warp 7 stops polling)
};

// 64 x 64 floats at src (16-byte aligned) into shared memory, one cp.async group
__device__ __forceinline__ void load_flat(float* s, const float* src) {
    for (int e = threadIdx.x; e < kCTE / 4; e += kCThreads) cp_async16(s + 4 * e, src + 4 * e);
    cp_async_commit();
}

// shared 64 x 64 floats to global dst (16-byte aligned)
__device__ __forceinline__ void store_flat(float* dst, const float* s) {
    for (int e = threadIdx.x; e < kCTE / 4; e += kCThreads)
        __stcg(reinterpret_cast<float4*>(dst) + e, reinterpret_cast<const float4*>(s)[e]);
}

__device__ __forceinline__ void acc_zero(float (&acc)[4][4]) {
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[p][q] = 0.f;
}

__device__ __forceinline__ void acc_neg(float (&acc)[4][4]) {
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[p][q] = -acc[p][q];
}

// the running partial -S_ij of an inverse tile (row-major in X_ij's storage)
__device__ __forceinline__ void partial_load(const float* X, float (&acc)[4][4], int tr, int tc) {
#pragma unroll
    for (int p = 0; p < 4; ++p) {
        const float4 v = __ldcg(reinterpret_cast<const float4*>(X + (4 * tr + p) * kCT + 4 * tc));
        acc[p][0] = v.x;
        acc[p][1] = v.y;
        acc[p][2] = v.z;
        acc[p][3] = v.w;
    }
}

__device__ __forceinline__ void partial_store(float* X, const float (&acc)[4][4], int tr, int tc) {
#pragma unroll
    for (int p = 0; p < 4; ++p)
        __stcg(reinterpret_cast<float4*>(X + (4 * tr + p) * kCT + 4 * tc),
               make_float4(acc[p][0], acc[p][1], acc[p][2], acc[p][3]));
}

// acc -= sum_{k=k0}^{k1} L_ik X_kj, operands double-buffered as in the
// factorisation updates (P = L_ik column-major, Q = X_kj row-major)
__device__ bool inv_accumulate(const CholCtx& c, CholSmem& sm, int i, int j, int k0, int k1, float (&acc)[4][4]) {
    const int T = c.T;
    const int tr = threadIdx.x & 15, tc = threadIdx.x >> 4;
    const int n = k1 - k0 + 1;
    if (!cta_wait2(c, c.tflag + i * T + k0, 2u, c.xflag + k0 * T + j, 1u, &sm.ok)) return false;
    load_tile(c, sm.a[0], i, k0);
    load_flat(sm.b[0], c.Xinv + packed_tile(k0, j) * kCTE);
    for (int q = 0; q < n; ++q) {
        const int k = k0 + q, nb = (q + 1) & 1;
        bool next = false;
        if (q + 1 < n) {
            next = cta_ready2(c.tflag + i * T + k + 1, 2u, c.xflag + (k + 1) * T + j, 1u, &sm.ok) == 3;
            if (next) {
                load_tile(c, sm.a[nb], i, k + 1);
                load_flat(sm.b[nb], c.Xinv + packed_tile(k + 1, j) * kCTE);
            }
        }
        if (next) asm volatile("cp.async.wait_group 2;\n" ::: "memory");
        else cp_async_wait_all();
        __syncthreads();
        sub_ptq(acc, sm.a[q & 1], sm.b[q & 1], tr, tc, 0, kCT);
        if (q + 1 < n && !next) {
            if (!cta_wait2(c, c.tflag + i * T + k + 1, 2u, c.xflag + (k + 1) * T + j, 1u, &sm.ok)) return false;
            load_tile(c, sm.a[nb], i, k + 1);
            load_flat(sm.b[nb], c.Xinv + packed_tile(k + 1, j) * kCTE);
        }
    }
    return true;
}

// Type 4: one chunk k0..k1 of the partial of X_ij
__device__ bool task_inverse_chunk(const CholCtx& c, CholSmem& sm, int i, int j, int k0, int k1) {
    const int T = c.T;
    const int tr = threadIdx.x & 15, tc = threadIdx.x >> 4;
    const int ch = (k0 - j) / kXChunk;
    float* X = c.Xinv + packed_tile(i, j) * kCTE;
    float acc[4][4];
    if (ch > 0) {
        if (!cta_wait(c, c.pflag + i * T + j, (unsigned)ch, &sm.ok)) return false;
        partial_load(X, acc, tr, tc);
    } else {
        acc_zero(acc);
    }
    if (!inv_accumulate(c, sm, i, j, k0, k1, acc)) return false;
    partial_store(X, acc, tr, tc);
    cta_publish(c.pflag + i * T + j, (unsigned)ch + 1u);
    return true;
}

// Type 5: the last term k = i-1, then X_ij = -X_ii S_ij
__device__ bool task_inverse_final(const CholCtx& c, CholSmem& sm, int i, int j) {
    const int T = c.T;
    const int tr = threadIdx.x & 15, tc = threadIdx.x >> 4;
    const int nch = (i - 1 - j + kXChunk - 1) / kXChunk;     // chunks of k = j..i-2
    float* X = c.Xinv + packed_tile(i, j) * kCTE;
    float acc[4][4];
    if (nch > 0) {
        if (!cta_wait(c, c.pflag + i * T + j, (unsigned)nch, &sm.ok)) return false;
        partial_load(X, acc, tr, tc);
    } else {
        acc_zero(acc);
    }
    if (!inv_accumulate(c, sm, i, j, i - 1, i - 1, acc)) return false;
    // acc = -S.  With P = -S row-major and Q = X_ii row-major, sub_pq_rowq
    // gives out[a][b] = sum_t S[t][a] X_ii[b][t] = (X_ii S)[b][a]; X_ij = -(X_ii S)
    if (!cta_wait(c, c.xflag + i * T + i, 1u, &sm.ok)) return false;
    load_flat(sm.b[0], c.Xinv + packed_tile(i, i) * kCTE);
#pragma unroll
    for (int p = 0; p < 4; ++p)
        *reinterpret_cast<float4*>(sm.x + (4 * tr + p) * kCT + 4 * tc) =
            make_float4(acc[p][0], acc[p][1], acc[p][2], acc[p][3]);
    cp_async_wait_all();
    __syncthreads();
    float out[4][4];
    acc_zero(out);
    sub_pq_rowq(out, sm.x, sm.b[0], tr, tc);
    __syncthreads();
    acc_neg(out);
    acc_to(out, sm.x, tr, tc);     // X_ij[4tc+q][4tr+p] at (4tc+q)*64 + 4tr+p: row-major
    __syncthreads();
    store_flat(X, sm.x);
    cta_publish(c.xflag + i * T + j, 1u);
    return true;
}

__device__ bool worker_task(const CholCtx& c, CholSmem& sm, int t);

// Each pool deals its tasks round-robin (pool worker w runs tasks w, w + Wp,
// ...) in its order.
__device__ void worker(const CholCtx& c, CholSmem& sm) {
    const int W = gridDim.x - 1, wid = blockIdx.x - 1;
    const int T = c.T;
    const bool inv = c.Xinv != nullptr;
    const int wf = factor_workers(W, T, inv);
    const int n_inv = inv ? inverse_count(T) : 0;
    const int tail = (inv && wf > 0 && wf < W) ? min(inverse_tail_start(T), n_inv) : n_inv;
    auto inverse = [&](int t) -> bool {
        int I, J, type, k0, k1;
        inverse_task(T, t, I, J, type, k0, k1);
        if (type == 4) return task_inverse_chunk(c, sm, I, J, k0, k1);
        if (type == 5) return task_inverse_final(c, sm, I, J);
        return true;
    };
    if (wid < wf) {
        const int n = factor_count(T);
        for (int t = wid; t < n; t += wf)
            if (!worker_task(c, sm, t)) return;
    } else {
        const int wi = W - wf;
        for (int t = wid - wf; t < tail; t += wi)
            if (!inverse(t)) return;
    }
    // the inverse's tail, every worker in slot order (each CTA's tasks stay
    // in increasing global order: no task waits on one behind it)
    for (int t = tail + wid; t < n_inv; t += W)
        if (!inverse(t)) return;
}

// factorisation task t
__device__ bool worker_task(const CholCtx& c, CholSmem& sm, int t) {
    const int T = c.T;
    const int tr = threadIdx.x & 15, tc = threadIdx.x >> 4;
    int I, J, type;
    factor_task(T, t, I, J, type);
    // updates k' < kend, kend = J for type 0, I-1 for types 1 and 2
    const int kend = type == 0 ? J : I - 1;
    __syncthreads();
    load_tile(c, sm.x, I, J);
    cp_async_wait_all();
    __syncthreads();
    float acc[4][4];
    acc_from(acc, sm.x, tr, tc);
    // operands of update k in buffer k & 1; the next update's operands are
    // requested before this one's product when their flags are already set
    if (kend > 0) {
        if (!cta_wait2(c, c.tflag + I * T + 0, 2u, I != J ? c.tflag + J * T + 0 : nullptr, 2u, &sm.ok))
            return false;
        load_tile(c, sm.a[0], I, 0);
        if (I != J) load_tile(c, sm.b[0], J, 0);
    }
    for (int k = 0; k < kend; ++k) {
        const int nb = (k + 1) & 1;
        bool next = false;
        if (k + 1 < kend) {
            next = I == J ? cta_ready(c.tflag + I * T + k + 1, 2u, &sm.ok)
                          : cta_ready2(c.tflag + I * T + k + 1, 2u, c.tflag + J * T + k + 1, 2u, &sm.ok) == 3;
            if (next) {
                // the buffers of update k-1 are free: every thread passed the barriers above
                load_tile(c, sm.a[nb], I, k + 1);
                if (I != J) load_tile(c, sm.b[nb], J, k + 1);
            }
        }
        // this update's groups complete; the next update's (one per operand) may stay in flight
        if (next && I != J) asm volatile("cp.async.wait_group 2;\n" ::: "memory");
        else if (next) asm volatile("cp.async.wait_group 1;\n" ::: "memory");
        else cp_async_wait_all();
        __syncthreads();
        const float* pa = sm.a[k & 1];
        sub_ptq(acc, pa, I != J ? sm.b[k & 1] : pa, tr, tc, 0, kCT);
        if (k + 1 < kend && !next) {
            if (!cta_wait2(c, c.tflag + I * T + k + 1, 2u, I != J ? c.tflag + J * T + k + 1 : nullptr, 2u, &sm.ok))
                return false;
            load_tile(c, sm.a[nb], I, k + 1);
            if (I != J) load_tile(c, sm.b[nb], J, k + 1);
        }
    }
    __syncthreads();
    acc_to(acc, sm.x, tr, tc);
    if (type == 0) {
        // TRSM as a product with the published L_JJ^-T: L_IJ = A_IJ L_JJ^-T
        if (!cta_wait(c, c.tflag + J * T + J, 2u, &sm.ok)) return false;
        load_flat(sm.b[0], c.Dinv + (int64_t)J * kCTE);
        cp_async_wait_all();
        __syncthreads();
        float out[4][4];
        acc_zero(out);
        sub_pq_rowq(out, sm.x, sm.b[0], tr, tc);
        __syncthreads();
        acc_neg(out);
        acc_to(out, sm.x, tr, tc);
    }
    __syncthreads();
    store_tile(c, sm.x, I, J);
    cta_publish(c.tflag + I * T + J, type == 0 ? 2u : 1u);
    return true;
}

// Step k: the panel factorisation of the diagonal tile (L_kk and its
// inverse, published together), the sub-diagonal tile as a product with
// L_kk^-T, and the next diagonal tile's last update.
__device__ void diagonal(const CholCtx& c, CholSmem& sm) {
    const int T = c.T;
    const int tr = threadIdx.x & 15, tc = threadIdx.x >> 4;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const bool inv = c.Xinv != nullptr;
    float pmin = 3.4e38f, pmax = 0.f;
    int bad = 0;
    int cur = 0;                         // sm.a[cur]: the diagonal tile of this step
    float* X = sm.b[1];
    float* E = sm.x;
    load_tile(c, sm.a[0], 0, 0);
    cp_async_wait_all();
    __syncthreads();
    for (int k = 0; k < T; ++k) {
        float* D = sm.a[cur];
        float* Y = sm.a[cur ^ 1];
        // the next two tiles, requested now when the workers have published
        // them, arrive during the factorisation of this one
        // step 0's neighbours need no worker update: copied now; later ones are
        // polled for and copied by warp 7 during the panel (look-ahead)
        LookAhead la;
        la.on[0] = la.on[1] = false;
        la.issued = 0;
        la.seen[0] = la.seen[1] = 0u;
        if (threadIdx.x == 0) {
            sm.la = 0;
            sm.panel_done = 0;
        }
        if (k + 1 < T) {
            if (k < 1) {
                load_tile(c, X, k + 1, k);
                load_tile(c, Y, k + 1, k + 1);
            } else if ((k + 2) * kCT <= c.K && (c.ld & 3) == 0 && ((uintptr_t)c.A & 15) == 0) {
                la.f[0] = c.tflag + (k + 1) * T + k;
                la.f[1] = c.tflag + (k + 1) * T + k + 1;
                la.dst[0] = X;
                la.dst[1] = Y;
                la.I[0] = la.I[1] = k + 1;
                la.J[0] = k;
                la.J[1] = k + 1;
                la.on[0] = la.on[1] = true;
            }
        }
        const bool hx = k < 1, hy = k < 1;
        potrf_inv64(c, D, E, sm.rinv, pmin, pmax, bad, c.K - k * kCT, la, &sm.panel_done);
        // the workers need L_kk^-T first (their TRSMs); L_kk itself and the
        // packed X_kk are written after the sub-diagonal tile is out, so the
        // release stores on this CTA's path wait for as few stores as possible
        store_flat(c.Dinv + (int64_t)k * kCTE, E);
        cta_publish(c.tflag + k * T + k, 2u);
        // X_{k-1,k-1} was stored during the previous step: this release covers it
        if (inv && k > 0 && threadIdx.x == 0) c_st_release(c.xflag + (k - 1) * T + k - 1, 1u);
        if (k + 1 >= T) {
            store_tile(c, D, k, k);
            if (inv) {
                store_flat(c.Xinv + packed_tile(k, k) * kCTE, E);
                cta_publish(c.xflag + k * T + k, 1u);
            }
            break;
        }
        // warp 7's last poll (tiles its previous poll saw set), then its
        // copies are complete for everyone after this barrier
        if (threadIdx.x >= kCThreads - 32) {
            look_ahead_poll(c, la);
            cp_async_wait_all();
            if (threadIdx.x == kCThreads - 32) sm.la = la.issued;
        }
        __syncthreads();
        const int pre = sm.la;
        // sub-diagonal tile: the workers applied updates k' < k (none when k = 0);
        // L_{k+1,k} = X L_kk^-T
        if (!hx && !(pre & 1)) {
            if (!cta_wait(c, c.tflag + (k + 1) * T + k, 1u, &sm.ok)) return;
            load_tile(c, X, k + 1, k);
        }
        cp_async_wait_all();
        __syncthreads();
        {
            float out[4][4];
            acc_zero(out);
            sub_pq_rowq(out, X, E, tr, tc);
            __syncthreads();
            acc_neg(out);
            acc_to(out, X, tr, tc);
        }
        __syncthreads();
        // L_{k+1,k}, L_kk and the packed X_kk go out now and drain during the
        // SYRK; L_{k+1,k}'s flag is released after it (the workers need that
        // tile several microseconds later), by a thread outside warp 0 so
        // that the next block factorisation does not wait on the release
        store_tile(c, X, k + 1, k);
        store_tile(c, D, k, k);
        if (inv) store_flat(c.Xinv + packed_tile(k, k) * kCTE, E);     // flag set with the next step's release
        // next diagonal tile: the workers applied updates k' < k; this CTA applies k
        if (!hy && !(pre & 2)) {
            if (!cta_wait(c, c.tflag + (k + 1) * T + k + 1, 1u, &sm.ok)) return;
            load_tile(c, Y, k + 1, k + 1);
        }
        cp_async_wait_all();
        __syncthreads();
        // lower 4 x 4 patches only (the factorisation reads the lower triangle)
        float acc[4][4];
        if (tc <= tr) {
            acc_from(acc, Y, tr, tc);
            sub_ptq(acc, X, X, tr, tc, 0, kCT);
        }
        __syncthreads();
        if (tc <= tr) acc_to(acc, Y, tr, tc);
        __syncthreads();
        if (threadIdx.x == kCThreads - 32) c_st_release(c.tflag + (k + 1) * T + k, 2u);
        cur ^= 1;
    }
    // pivot test (pivots of warp 0, which ran every 8 x 8 factorisation)
    if (w == 0 && lane == 0) {
        int f = 0;
        if (bad) f = 1;
        else if ((double)pmax / (double)pmin * c.rcond >= 1.0) f = 2;
        if (f) atomicMax(c.status, f);
        if (c.piv) {
            c.piv[0] = (double)pmin;
            c.piv[1] = (double)pmax;
        }
    }
}

__global__ void __launch_bounds__(kCThreads, 1) chol_tiles_kernel(CholCtx c) {
    extern __shared__ __align__(16) uint8_t chol_smem[];
    CholSmem& sm = *reinterpret_cast<CholSmem*>(chol_smem);
    if (blockIdx.x == 0) diagonal(c, sm);
    else worker(c, sm);
}

static int chol_tiles(int K) { return (K + kCT - 1) / kCT; }

}  // namespace vtb

using namespace vtb;

VTB_API int64_t vtb_chol_dinv_floats(int K) { return K > 0 ? (int64_t)chol_tiles(K) * kCTE : 0; }

VTB_API int64_t vtb_chol_work_bytes(int K) {
    if (K <= 0) return 0;
    const int64_t T = chol_tiles(K);
    return 3 * ((T * T * 4 + 255) & ~(int64_t)255) + 256;
}

VTB_API int64_t vtb_chol_inverse_floats(int K) {
    if (K <= 0) return 0;
    const int64_t T = chol_tiles(K);
    return T * (T + 1) / 2 * kCTE;
}

static int chol_launch(float* A, int64_t ld, int K, float* Dinv, float* Linv, void* work, int64_t work_bytes,
                       int32_t* status, double* pivots, double rcond, void* stream) {
    VTB_CHECK_ARG(K > 0 && ld >= K && A && Dinv && work && status);
    VTB_CHECK_ARG(work_bytes >= vtb_chol_work_bytes(K) && ((uintptr_t)work & 255) == 0);
    VTB_CHECK_ARG(((uintptr_t)Linv & 15) == 0 && ((uintptr_t)Dinv & 15) == 0);
    int dev = 0;
    VTB_CUDA_TRY(cudaGetDevice(&dev));
    int coop = 0, nsm = 0;
    VTB_CUDA_TRY(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
    VTB_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    if (!coop) return VTB_CUDA_ERR;
    const size_t sm = sizeof(CholSmem);
    VTB_CUDA_TRY(cudaFuncSetAttribute(chol_tiles_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    int per_sm = 0;
    VTB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, chol_tiles_kernel, kCThreads, sm));
    if (per_sm < 1) return VTB_CUDA_ERR;
    const int T = chol_tiles(K);
    const bool inv = Linv != nullptr;
    const int ntask = task_count(T, inv);
    const int need = (inv && factor_count(T) > 0 && inverse_count(T) > 0) ? 2 : 1;
    const int grid = 1 + std::max(need, std::min(nsm - 1, ntask));
    cudaStream_t s = as_stream(stream);
    const int64_t fbytes = ((int64_t)T * T * 4 + 255) & ~(int64_t)255;
    VTB_CUDA_TRY(cudaMemsetAsync(work, 0, (size_t)(3 * fbytes + 256), s));
    CholCtx c;
    c.A = A;
    c.ld = ld;
    c.K = K;
    c.T = T;
    c.Dinv = Dinv;
    c.tflag = reinterpret_cast<unsigned*>(work);
    c.xflag = reinterpret_cast<unsigned*>(reinterpret_cast<char*>(work) + fbytes);
    c.pflag = reinterpret_cast<unsigned*>(reinterpret_cast<char*>(work) + 2 * fbytes);
    c.abort_word = reinterpret_cast<int*>(reinterpret_cast<char*>(work) + 3 * fbytes);
    c.status = status;
    c.piv = pivots;
    c.rcond = rcond;
    c.limit = wait_limit(kCholSpin);
    c.Xinv = Linv;
    void* args[] = {(void*)&c};
    VTB_CUDA_TRY(cudaLaunchCooperativeKernel((void*)chol_tiles_kernel, dim3(grid), dim3(kCThreads), args, sm, s));
    return launch_status();
}

// Float32 Cholesky of the symmetric positive definite K x K matrix A
// (column-major, leading dimension ld; only the lower triangle is written:
// A = L L^T with L over the lower triangle).  Dinv (vtb_chol_dinv_floats(K)
// floats, 16-byte aligned) receives the inverses of the 64 x 64 diagonal
// tiles of L, row-major, for vtb_chol_solve.  work: vtb_chol_work_bytes(K) bytes of scratch (cleared
// here).  status (device int32, cleared by the caller) receives 1 when a
// pivot fails, 2 when max/min of the squared pivots reaches 1/rcond, 3 when
// a wait between CTAs ran out; pivots (device, may be NULL) receives [min,
// max] squared pivots.  Replaces spotrf (cuSOLVER) in the mixed decoder's
// solve of G c = q (vtem/utils/linalg.py:591-631 as called at
// vtem/vtdm.py:645-648).  Stream-ordered; does not synchronise.
VTB_API int vtb_chol_factor(float* A, int64_t ld, int K, float* Dinv, void* work, int64_t work_bytes, int32_t* status,
                            double* pivots, double rcond, void* stream) {
    return chol_launch(A, ld, K, Dinv, nullptr, work, work_bytes, status, pivots, rcond, stream);
}

// vtb_chol_factor that also forms L^-1 in the same launch: Linv
// (vtb_chol_inverse_floats(K) floats, 16-byte aligned) receives the tiles
// (i, j), i >= j, of L^-1, row-major, tile (i, j) at (i(i+1)/2 + j) * 4096.
VTB_API int vtb_chol_factor_inverse(float* A, int64_t ld, int K, float* Dinv, float* Linv, void* work,
                                    int64_t work_bytes, int32_t* status, double* pivots, double rcond, void* stream) {
    VTB_CHECK_ARG(Linv);
    return chol_launch(A, ld, K, Dinv, Linv, work, work_bytes, status, pivots, rcond, stream);
}

namespace vtb {

// y = L^-1 b and x = L^-T y with the packed inverse X, one block per tile:
// block (i, j) forms its tile's product with the vector (X_ij b_j forward,
// X_ij^T y_i backward) into a partial, and the last block of a block row
// (column) to finish -- counted by an atomic ticket -- adds the partials in
// a fixed order, so the result does not depend on the block schedule.
constexpr int kGThreads = 256;

__device__ __forceinline__ void unpack_tile(int t, int& i, int& j) {
    i = (int)((sqrtf(8.f * (float)t + 1.f) - 1.f) * 0.5f);
    while ((int64_t)i * (i + 1) / 2 > t) --i;
    while ((int64_t)(i + 1) * (i + 2) / 2 <= t) ++i;
    j = t - i * (i + 1) / 2;
}

__global__ void __launch_bounds__(kGThreads) inv_fwd_kernel(const float* __restrict__ X, int K,
                                                            const double* __restrict__ b, float* __restrict__ part,
                                                            float* __restrict__ y, unsigned* __restrict__ cnt) {
    __shared__ float bs[kCT];
    __shared__ float red[4][kCT];
    __shared__ int last;
    const int t = blockIdx.x, tid = threadIdx.x;
    int i, j;
    unpack_tile(t, i, j);
    if (tid < kCT) {
        const int g = j * kCT + tid;
        bs[tid] = g < K ? (float)b[g] : 0.f;
    }
    __syncthreads();
    const int r = tid >> 2, q = tid & 3;
    const float4* row = reinterpret_cast<const float4*>(X + (int64_t)t * kCTE + r * kCT + 16 * q);
    float4 v[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) v[e] = __ldg(row + e);
    float a0 = 0.f, a1 = 0.f;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        const float* bq = bs + 16 * q + 4 * e;
        a0 = fmaf(v[e].x, bq[0], a0);
        a1 = fmaf(v[e].y, bq[1], a1);
        a0 = fmaf(v[e].z, bq[2], a0);
        a1 = fmaf(v[e].w, bq[3], a1);
    }
    float acc = a0 + a1;
    acc += __shfl_xor_sync(0xffffffffu, acc, 1);
    acc += __shfl_xor_sync(0xffffffffu, acc, 2);
    if (q == 0) part[(int64_t)t * kCT + r] = acc;
    __threadfence();
    __syncthreads();
    if (tid == 0) last = atomicAdd(cnt + i, 1u) == (unsigned)i;      // row i has i + 1 tiles
    __syncthreads();
    if (!last) return;
    __threadfence();
    {
        // four threads per row, each over every fourth partial, then a fixed-order combine
        const int rr = tid & 63, qq = tid >> 6;
        float sum = 0.f;
#pragma unroll 4
        for (int jj = qq; jj <= i; jj += 4) sum += __ldcg(part + ((int64_t)i * (i + 1) / 2 + jj) * kCT + rr);
        red[qq][rr] = sum;
    }
    __syncthreads();
    if (tid < kCT) y[i * kCT + tid] = (red[0][tid] + red[1][tid]) + (red[2][tid] + red[3][tid]);
    if (tid == 0) cnt[i] = 0u;
}

__global__ void __launch_bounds__(kGThreads) inv_bwd_kernel(const float* __restrict__ X, int K, int T,
                                                            const float* __restrict__ y, float* __restrict__ part,
                                                            double* __restrict__ x, unsigned* __restrict__ cnt) {
    __shared__ float ys[kCT];
    __shared__ float red[4][kCT];
    __shared__ int last;
    const int t = blockIdx.x, tid = threadIdx.x;
    int i, j;
    unpack_tile(t, i, j);
    if (tid < kCT) ys[tid] = y[i * kCT + tid];
    __syncthreads();
    const int c = tid & 63, rq = tid >> 6;
    const float* col = X + (int64_t)t * kCTE + (16 * rq) * kCT + c;
    float v[16];
#pragma unroll
    for (int e = 0; e < 16; ++e) v[e] = __ldg(col + e * kCT);
    float a0 = 0.f, a1 = 0.f;
#pragma unroll
    for (int e = 0; e < 16; e += 2) {
        a0 = fmaf(v[e], ys[16 * rq + e], a0);
        a1 = fmaf(v[e + 1], ys[16 * rq + e + 1], a1);
    }
    red[rq][c] = a0 + a1;
    __syncthreads();
    if (tid < kCT) part[(int64_t)t * kCT + tid] = (red[0][tid] + red[1][tid]) + (red[2][tid] + red[3][tid]);
    __threadfence();
    __syncthreads();
    if (tid == 0) last = atomicAdd(cnt + T + j, 1u) == (unsigned)(T - 1 - j);   // column j has T - j tiles
    __syncthreads();
    if (!last) return;
    __threadfence();
    {
        const int cc2 = tid & 63, qq = tid >> 6;
        float sum = 0.f;
#pragma unroll 4
        for (int ii = j + qq; ii < T; ii += 4) sum += __ldcg(part + ((int64_t)ii * (ii + 1) / 2 + j) * kCT + cc2);
        __syncthreads();       // every thread has read red[][] above
        red[qq][cc2] = sum;
    }
    __syncthreads();
    if (tid < kCT) {
        const int g = j * kCT + tid;
        if (g < K) x[g] = (double)((red[0][tid] + red[1][tid]) + (red[2][tid] + red[3][tid]));
    }
    if (tid == 0) cnt[T + j] = 0u;
}

}  // namespace vtb

VTB_API int64_t vtb_chol_solve_inverse_bytes(int K) {
    if (K <= 0) return 0;
    const int64_t T = chol_tiles(K);
    return (T * (T + 1) / 2 * kCT + T * kCT) * 4 + 2 * T * 4;
}

// x = L^-T L^-1 x (x float64 in and out, float32 arithmetic) with the packed
// inverse of vtb_chol_factor_inverse: two triangular matrix-vector products,
// one block per tile of X, every tile read once.  work:
// vtb_chol_solve_inverse_bytes(K) bytes, 4-byte aligned, ZEROED before the
// first call (each call leaves its counters zeroed again); calls sharing a
// work buffer must be stream-ordered.  Replaces spotrs in the mixed
// decoder's solve (linalg.py:591-631).  Stream-ordered.
VTB_API int vtb_chol_solve_inverse(const float* Linv, int K, double* x, void* work, int64_t work_bytes,
                                   void* stream) {
    VTB_CHECK_ARG(K > 0 && Linv && x && work && ((uintptr_t)Linv & 15) == 0 && ((uintptr_t)work & 3) == 0);
    VTB_CHECK_ARG(work_bytes >= vtb_chol_solve_inverse_bytes(K));
    const int T = chol_tiles(K);
    const int nt = T * (T + 1) / 2;
    float* part = reinterpret_cast<float*>(work);
    float* y = part + (int64_t)nt * kCT;
    unsigned* cnt = reinterpret_cast<unsigned*>(y + T * kCT);
    cudaStream_t s = as_stream(stream);
    inv_fwd_kernel<<<nt, kGThreads, 0, s>>>(Linv, K, x, part, y, cnt);
    int st = launch_status();
    if (st) return st;
    inv_bwd_kernel<<<nt, kGThreads, 0, s>>>(Linv, K, T, y, part, x, cnt);
    return launch_status();
}

namespace vtb {

// ---------------------------------------------------------------------------
// x = L^-T L^-1 x for the factor of vtb_chol_factor, in ONE thread-block
// cluster (C CTAs on one GPC): block-row substitution over the 64-row tiles,
// the diagonal blocks applied through Dinv (L_kk^-1).  CTA q owns the tile
// rows k = q, q + C, ...; every CTA keeps the whole solved vector in its
// shared memory.  Forward step j (one cluster barrier each):
//   owner(j):  y_j = Dinv_j (b_j - s_j - L_{j,j-1} y_{j-1}), then stores y_j
//              into every CTA's shared memory (distributed shared memory);
//   every CTA: s_k += L_{k,j-1} y_{j-1} for its rows k > j
// (s_k: the running sum of the already solved blocks), so the chain between
// two barriers is one 64 x 64 product and one application of Dinv.  The
// backward pass is the mirror image with L^T.  Four threads share a row
// (forward) or a column (backward: columns of the column-major factor are
// contiguous) of a tile, 16 elements each, and combine with warp shuffles.
// Every tile a step needs is loaded into registers BEFORE the barrier that
// releases the previous block, so its L2 latency overlaps the wait.  No
// spin-wait: the cluster barrier is the hardware's, and every CTA takes every
// step.
constexpr int kSThreads = 256;
constexpr int kSPre = 4;          // own tiles per step loaded ahead in registers
constexpr int kSMaxOwn = 24;      // ceil(T / C) for C >= 8

struct SolveSmem {
    float v[kSMaxT * kCT];        // y (forward), then x (backward)
    float s[kSMaxOwn][kCT];       // running sums of own rows
    float t[kCT];                 // the owner's block before Dinv
};

__device__ __forceinline__ void dsm_store(float* local_addr, unsigned rank, float v) {
    uint32_t a = static_cast<uint32_t>(__cvta_generic_to_shared(local_addr)), r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(rank));
    asm volatile("st.shared::cluster.f32 [%0], %1;" ::"r"(r), "f"(v) : "memory");
}

__device__ __forceinline__ void cluster_sync_all() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory");
    asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}

// row mapping: thread (r = tid >> 2, part = tid & 3) holds M[r][16 part + i]
// of tile (I, J) of the column-major A; entries beyond K are the identity's
__device__ __forceinline__ void load_rows(const float* A, int64_t ld, int K, int I, int J, float (&v)[16]) {
    const int r = threadIdx.x >> 2, part = threadIdx.x & 3;
    const int gr = I * kCT + r;
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        const int gc = J * kCT + 16 * part + i;
        v[i] = (gr < K && gc < K) ? __ldcg(A + (int64_t)gc * ld + gr) : (gr == gc ? 1.f : 0.f);
    }
}

// column mapping: thread (c = tid >> 2, part = tid & 3) holds M[16 part + i][c]
__device__ __forceinline__ void load_cols(const float* A, int64_t ld, int K, int I, int J, float (&v)[16]) {
    const int c = threadIdx.x >> 2, part = threadIdx.x & 3;
    const int gc = J * kCT + c;
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        const int gr = I * kCT + 16 * part + i;
        v[i] = (gr < K && gc < K) ? __ldcg(A + (int64_t)gc * ld + gr) : (gr == gc ? 1.f : 0.f);
    }
}

// sum over the four threads of a row / column, every one of them gets it
__device__ __forceinline__ float quad_sum(float x) {
    x += __shfl_xor_sync(0xffffffffu, x, 1);
    x += __shfl_xor_sync(0xffffffffu, x, 2);
    return x;
}

__device__ __forceinline__ float dot16(const float (&w)[16], const float* v) {
    float a0 = 0.f, a1 = 0.f;
#pragma unroll
    for (int i = 0; i < 16; i += 2) {
        a0 = fmaf(w[i], v[i], a0);
        a1 = fmaf(w[i + 1], v[i + 1], a1);
    }
    return a0 + a1;
}

__global__ void __launch_bounds__(kSThreads, 1) chol_solve_kernel(const float* __restrict__ A, int64_t ld,
                                                                  const float* __restrict__ Dinv, int K, double* x) {
    extern __shared__ __align__(16) uint8_t solve_smem[];
    SolveSmem& sm = *reinterpret_cast<SolveSmem*>(solve_smem);
    const int T = (K + kCT - 1) / kCT;
    unsigned C, q;
    asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(C));
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(q));
    const int tid = threadIdx.x, rc = tid >> 2, part = tid & 3;
    const int nown = ((int)T - (int)q + (int)C - 1) / (int)C;   // own rows k = q + C m
    for (int e = tid; e < kSMaxOwn * kCT; e += kSThreads) (&sm.s[0][0])[e] = 0.f;
    cluster_sync_all();

    // ------------------------------------------------ forward: L y = b
    for (int j = 0; j < T; ++j) {
        const bool own = (j % (int)C) == (int)q;
        float crit[16], dv[16], pre[kSPre][16];
        if (own) {
            if (j >= 1) load_rows(A, ld, K, j, j - 1, crit);
#pragma unroll
            for (int i = 0; i < 16; ++i) dv[i] = __ldcg(Dinv + (int64_t)j * kCTE + rc * kCT + 16 * part + i);
        }
        const int mstart = (j + 1 - (int)q + (int)C - 1) / (int)C;  // first own row k = q + C m > j
        if (j >= 1) {
#pragma unroll
            for (int p = 0; p < kSPre; ++p)
                if (mstart + p < nown) load_rows(A, ld, K, (int)q + (int)C * (mstart + p), j - 1, pre[p]);
        }
        cluster_sync_all();                     // y_{j-1} is in every CTA's v
        const float* yp = sm.v + (j - 1) * kCT + 16 * part;
        if (own) {
            const int mj = (j - (int)q) / (int)C;
            float lv = j >= 1 ? quad_sum(dot16(crit, yp)) : 0.f;
            if (part == 0) {
                const int gr = j * kCT + rc;
                const float b = gr < K ? (float)x[gr] : 0.f;
                sm.t[rc] = b - sm.s[mj][rc] - lv;
            }
            __syncthreads();
            const float yj = quad_sum(dot16(dv, sm.t + 16 * part));
            if (part == 0)
                for (unsigned d = 0; d < C; ++d) dsm_store(sm.v + j * kCT + rc, d, yj);
        }
        // non-critical: s_k += L_{k,j-1} y_{j-1} for own k > j (row rc owned by its part-0 thread)
        if (j >= 1) {
#pragma unroll
            for (int p = 0; p < kSPre; ++p) {
                if (mstart + p < nown) {
                    const float lv = quad_sum(dot16(pre[p], yp));
                    if (part == 0) sm.s[mstart + p][rc] += lv;
                }
            }
            for (int m = mstart + kSPre; m < nown; ++m) {
                float w[16];
                load_rows(A, ld, K, (int)q + (int)C * m, j - 1, w);
                const float lv = quad_sum(dot16(w, yp));
                if (part == 0) sm.s[m][rc] += lv;
            }
        }
    }
    cluster_sync_all();                         // y complete everywhere
    for (int e = tid; e < kSMaxOwn * kCT; e += kSThreads) (&sm.s[0][0])[e] = 0.f;
    __syncthreads();

    // ------------------------------------------------ backward: L^T x = y
    // step j = T-1 .. 0: owner(j): x_j = Dinv_j^T (y_j - s_j - L_{j+1,j}^T x_{j+1});
    // every CTA: s_k += L_{j+1,k}^T x_{j+1} for own k < j (column rc owned by its part-0 thread)
    for (int j = T - 1; j >= 0; --j) {
        const bool own = (j % (int)C) == (int)q;
        const bool has = j + 1 < T;
        float crit[16], dv[16], pre[kSPre][16];
        if (own) {
            if (has) load_cols(A, ld, K, j + 1, j, crit);
#pragma unroll
            for (int i = 0; i < 16; ++i) dv[i] = __ldcg(Dinv + (int64_t)j * kCTE + (16 * part + i) * kCT + rc);
        }
        // own rows k < j, in increasing k: k = q + C m for m < mend
        const int mend = (j - (int)q + (int)C - 1) / (int)C;         // own k < j  <=>  m < mend
        const int mlim = mend < 0 ? 0 : (mend < nown ? mend : nown);
        if (has) {
#pragma unroll
            for (int p = 0; p < kSPre; ++p)
                if (p < mlim) load_cols(A, ld, K, j + 1, (int)q + (int)C * p, pre[p]);
        }
        cluster_sync_all();                     // x_{j+1} is in every CTA's v
        const float* xp = sm.v + (j + 1) * kCT + 16 * part;
        if (own) {
            const int mj = (j - (int)q) / (int)C;
            const float lv = has ? quad_sum(dot16(crit, xp)) : 0.f;
            if (part == 0) sm.t[rc] = sm.v[j * kCT + rc] - sm.s[mj][rc] - lv;
            __syncthreads();
            const float xj = quad_sum(dot16(dv, sm.t + 16 * part));
            if (part == 0)
                for (unsigned d = 0; d < C; ++d) dsm_store(sm.v + j * kCT + rc, d, xj);
        }
        if (has) {
#pragma unroll
            for (int p = 0; p < kSPre; ++p) {
                if (p < mlim) {
                    const float lv = quad_sum(dot16(pre[p], xp));
                    if (part == 0) sm.s[p][rc] += lv;
                }
            }
            for (int m = kSPre; m < mlim; ++m) {
                float w[16];
                load_cols(A, ld, K, j + 1, (int)q + (int)C * m, w);
                const float lv = quad_sum(dot16(w, xp));
                if (part == 0) sm.s[m][rc] += lv;
            }
        }
    }
    cluster_sync_all();
    if (q == 0)
        for (int i = tid; i < K; i += kSThreads) x[i] = (double)sm.v[i];
    cluster_sync_all();                         // no CTA leaves while its shared memory may be written
}

// cluster size: 16 CTAs where the non-portable size can be scheduled, else 8
static int g_solve_cs = 0;

static cudaError_t launch_solve(int cs, const float* L, int64_t ld, const float* Dinv, int K, double* x,
                                cudaStream_t s) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cs);
    cfg.blockDim = dim3(kSThreads);
    cfg.dynamicSmemBytes = sizeof(SolveSmem);
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = cs;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, chol_solve_kernel, L, ld, Dinv, K, x);
}

}  // namespace vtb

// x = L^-T L^-1 x (x float64 in and out, float32 arithmetic) with the factor
// and the diagonal-tile inverses of vtb_chol_factor, in one thread-block
// cluster.  K <= 10240.  Replaces spotrs (cuSOLVER) in the mixed decoder.
// Stream-ordered; does not synchronise.
VTB_API int vtb_chol_solve(const float* L, int64_t ld, const float* Dinv, int K, double* x, void* stream) {
    VTB_CHECK_ARG(K > 0 && K <= kSMaxT * kCT && ld >= K && L && Dinv && x);
    if (g_solve_cs == 0) {
        VTB_CUDA_TRY(cudaFuncSetAttribute(chol_solve_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)sizeof(SolveSmem)));
        int cs = 8;
        if (cudaFuncSetAttribute(chol_solve_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) ==
            cudaSuccess) {
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3(16);
            cfg.blockDim = dim3(kSThreads);
            cfg.dynamicSmemBytes = sizeof(SolveSmem);
            cudaLaunchAttribute at[1];
            at[0].id = cudaLaunchAttributeClusterDimension;
            at[0].val.clusterDim.x = 16;
            at[0].val.clusterDim.y = 1;
            at[0].val.clusterDim.z = 1;
            cfg.attrs = at;
            cfg.numAttrs = 1;
            int nclusters = 0;
            if (cudaOccupancyMaxActiveClusters(&nclusters, chol_solve_kernel, &cfg) == cudaSuccess && nclusters > 0)
                cs = 16;
        }
        cudaGetLastError();
        g_solve_cs = cs;
    }
    VTB_CUDA_TRY(launch_solve(g_solve_cs, L, ld, Dinv, K, x, as_stream(stream)));
    return launch_status();
}

// CTAs of the cluster vtb_chol_solve launches (0 before its first call).
VTB_API int vtb_chol_solve_cluster(void) { return vtb::g_solve_cs; }
