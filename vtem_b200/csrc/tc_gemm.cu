// Tensor-core GEMM for sm_100a: C = alpha * A B^T with A (M x K) and B (N x K)
// in bf16, K-major, accumulated in fp32 in tensor memory (tcgen05).
//
// Used with split-bf16 operands: a float64/float32 value x is written as
// hi = bf16(x), lo = bf16(x - hi), and the operands are laid out along K as
// A' = [A_hi | A_hi | A_lo], B' = [B_hi | B_lo | B_hi], so one accumulator
// sums hi*hi + hi*lo + lo*hi (relative error ~2^-16 per product, fp32
// accumulation), the "split BF16" products of the mixed-precision path.
//
// Structure (one 128 x BN output tile per CTA, 128 threads):
//   thread 0   : TMA producer, 2-D tiled loads with 128-byte swizzle into a
//                kStages-deep ring of shared-memory stages (no multicast);
//   thread 32  : MMA issuer, tcgen05.mma.cta_group::1.kind::f16 (M=128,
//                N=BN, K=16 per instruction), tcgen05.commit to free stages;
//   warps 0..3 : epilogue, tcgen05.ld 32x32b of their 32 TMEM lanes (rows),
//                scaled and stored as fp32 or fp64 with arbitrary strides.
// Every mbarrier wait is bounded; a timeout sets *err and the CTA still
// drains, releases its tensor memory and returns.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include <cstring>
#include <type_traits>
#include <mutex>

#include "common.cuh"

namespace vtb {

constexpr int kTcBM = 128;
constexpr int kTcBK = 64;   // 64 bf16 = 128 bytes = one swizzle row
constexpr int kTcStages = 4;
constexpr uint32_t kWaitLimit = 1u << 22;
// drain of a CTA that gave up: its own TMA loads and MMAs complete without
// depending on anything else, so this bound is only a backstop
constexpr uint32_t kDrainLimit = 1u << 24;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// bounded wait on the phase with the given parity; returns false on timeout
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t limit) {
    const uint32_t a = smem_u32(bar);
    for (uint32_t it = 0; it < limit; ++it) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(a), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::
            "r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y)
        : "memory");
}

// K-major operand tile, 128-byte swizzle: 8-row atoms of 1024 bytes.
template <int BK>
__device__ __forceinline__ uint64_t smem_desc_k(const void* base);

// K-major operand tile, 64-byte swizzle (BK = 32 bf16 per row): 8-row atoms of 512 bytes.
template <>
__device__ __forceinline__ uint64_t smem_desc_k<32>(const void* base) {
    const uint64_t addr = smem_u32(base);
    return ((addr >> 4) & 0x3FFFull) | (1ull << 16) | (32ull << 32) | (1ull << 46) | (4ull << 61);
}

__device__ __forceinline__ uint64_t smem_desc_sw128(const void* base) {
    const uint64_t addr = smem_u32(base);
    return ((addr >> 4) & 0x3FFFull) | (1ull << 16) | (64ull << 32) | (1ull << 46) | (2ull << 61);
}

template <>
__device__ __forceinline__ uint64_t smem_desc_k<64>(const void* base) {
    return smem_desc_sw128(base);
}

// 16 consecutive fp32 accumulator columns of this warp's 32 TMEM lanes (one
// row per thread); the registers are valid after tmem_ld_wait
__device__ __forceinline__ void tmem_ld16_async(uint32_t taddr, uint32_t (&v)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(taddr));
}

__device__ __forceinline__ void tmem_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
    tmem_ld16_async(taddr, v);
    tmem_ld_wait();
}

template <int BN>
struct TcIdesc {
    // c_format f32 (bit 4), a/b bf16 (bits 7, 10), K-major A and B, N>>3 at 17, M>>4 at 24
    static constexpr uint32_t value = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
                                      ((uint32_t)(kTcBM >> 4) << 24);
};

// X3 (three-product mode): the operands are [hi | lo] along K (2K columns)
// and every k-block issues hi*hi, hi*lo and lo*hi from the same
// shared-memory tiles, so no operand part is stored or loaded twice.
// NS sub-tiles of BN columns share each A tile: a CTA computes a
// 128 x (NS * BN) tile with NS accumulators side by side in tensor memory
// (BN <= 256 is the largest N of one MMA), loading its A rows once.
constexpr int kSmemRing = 225 * 1024;  // stage ring; barriers and 1 KB alignment slack fit in the rest of 227 KB

// BK: the k-block (64 bf16 = 128-byte rows with the 128-byte swizzle, or
// 32 = 64-byte rows with the 64-byte swizzle: half-size stages, twice as
// many in the same ring, for tiles whose stage would otherwise leave only
// two in flight)
template <int BN, bool X3, int NS = 1, int BK = kTcBK>
struct TcCfg {
    static_assert(BK == 64 || BK == 32, "k-block of 64 or 32");
    static constexpr int kParts = X3 ? 2 : 1;
    static constexpr int kCols = NS * BN;
    static constexpr int kStageBytes = kParts * (kTcBM + kCols) * BK * 2;
    static constexpr int kFit = kSmemRing / kStageBytes;
    static constexpr int kMaxStages = kTcStages * (kTcBK / BK);
    static constexpr int kStages = kFit < kMaxStages ? kFit : kMaxStages;
    static_assert(kStages >= 2, "at least two pipeline stages");
    static constexpr uint32_t kTmemCols = kCols <= 32 ? 32 : kCols <= 64 ? 64 : kCols <= 128 ? 128
                                                       : kCols <= 256 ? 256 : 512;
};

template <int BN, bool X3 = false, int NS = 1, int BK = kTcBK>
struct TcSmem {
    using Cfg = TcCfg<BN, X3, NS, BK>;
    __nv_bfloat16 a[Cfg::kStages][Cfg::kParts][kTcBM * BK];
    __nv_bfloat16 b[Cfg::kStages][Cfg::kParts][Cfg::kCols * BK];
    uint64_t full[Cfg::kStages];
    uint64_t empty[Cfg::kStages];
    uint64_t done;
    uint32_t tmem_base;
};

// 2-D tiled store of a shared-memory box to global memory (bulk async group)
__device__ __forceinline__ void tma_store_2d(const CUtensorMap* map, const void* src, int x, int y) {
    asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%2, %3}], [%1];" ::"l"(
                     reinterpret_cast<uint64_t>(map)),
                 "r"(smem_u32(src)), "r"(x), "r"(y)
                 : "memory");
}

// One 128 x (NS * BN) output tile (rows m0.., columns n0..) of C = alpha A B^T;
// the tensor maps may live in kernel parameters or in global memory.  With
// X3, K is the width of one operand part and C = A_hi B_hi^T + A_hi B_lo^T +
// A_lo B_hi^T.  tmC (nullable): a float32 map of C (box 32 x 128, 128-byte
// swizzle) for the tensor-store epilogue.
template <int BN, typename OutT, bool X3 = false, int NS = 1, int BK = kTcBK>
__device__ __forceinline__ void tc_tile(const CUtensorMap* tmA, const CUtensorMap* tmB, const CUtensorMap* tmC,
                                        int M, int N, int K, int m0, int n0, OutT* __restrict__ C, int64_t c_m,
                                        int64_t c_n, double alpha, int accumulate, int32_t* __restrict__ err,
                                        uint32_t limit, uint8_t* smem_raw) {
    using Sm = TcSmem<BN, X3, NS, BK>;
    using Cfg = typename Sm::Cfg;
    constexpr int S = Cfg::kStages;
    constexpr int kCols = Cfg::kCols;
    constexpr uint32_t kTmemCols = Cfg::kTmemCols;
    // 1024-byte alignment of the stage buffers (the swizzle atoms)
    Sm& sm = *reinterpret_cast<Sm*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
    const int tid = threadIdx.x;
    const int warp = tid >> 5;
    const int nk = K / BK;

    if (tid == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(&sm.full[s], 1);
            mbar_init(&sm.empty[s], 1);
        }
        mbar_init(&sm.done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&sm.tmem_base)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = sm.tmem_base;
    bool ok = true;

    int issued = 0;   // TMA stages the producer issued
    if (tid == 0) {
        // producer
        constexpr uint32_t bytes = Cfg::kStageBytes;
        for (int kb = 0; kb < nk && ok; ++kb) {
            const int s = kb % S;
            if (kb >= S) ok = mbar_wait(&sm.empty[s], ((kb / S) + 1) & 1, limit);
            if (!ok) break;
            mbar_expect_tx(&sm.full[s], bytes);
#pragma unroll
            for (int part = 0; part < Cfg::kParts; ++part) {
                tma_load_2d(sm.a[s][part], tmA, &sm.full[s], part * K + kb * BK, m0);
#pragma unroll
                for (int ns = 0; ns < NS; ++ns)
                    tma_load_2d(sm.b[s][part] + ns * BN * BK, tmB, &sm.full[s], part * K + kb * BK,
                                n0 + ns * BN);
            }
            issued = kb + 1;
        }
        if (!ok) atomicExch(err, VTB_TIMEOUT);
    } else if (tid == 32) {
        // MMA issuer
        constexpr uint32_t idesc = TcIdesc<BN>::value;
        for (int kb = 0; kb < nk && ok; ++kb) {
            const int s = kb % S;
            ok = mbar_wait(&sm.full[s], (kb / S) & 1, limit);
            if (!ok) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            // products of this k-block: (A part, B part) = (0,0); with X3 also (0,1) and (1,0)
#pragma unroll
            for (int pr = 0; pr < (X3 ? 3 : 1); ++pr) {
                const uint64_t da = smem_desc_k<BK>(sm.a[s][pr == 2 ? Cfg::kParts - 1 : 0]);
#pragma unroll
                for (int ns = 0; ns < NS; ++ns) {
                    const uint64_t db = smem_desc_k<BK>(sm.b[s][pr == 1 ? Cfg::kParts - 1 : 0] + ns * BN * BK);
#pragma unroll
                    for (int j = 0; j < BK / 16; ++j) {
                        // advance 16 bf16 (32 bytes) along K inside the swizzle row
                        const uint64_t adv = (uint64_t)(j * 2);
                        const uint32_t acc = (kb > 0 || pr > 0 || j > 0) ? 1u : 0u;
                        asm volatile(
                            "{\n\t.reg .pred p;\n\t"
                            "setp.ne.b32 p, %4, 0;\n\t"
                            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem + ns * BN),
                            "l"(da + adv), "l"(db + adv), "r"(idesc), "r"(acc)
                            : "memory");
                    }
                }
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_u32(&sm.empty[s]))
                         : "memory");
        }
        // committed also after a timeout: `done` then tracks the MMAs that
        // were issued, so the tensor memory is freed only after they finish
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         smem_u32(&sm.done))
                     : "memory");
        if (!ok) atomicExch(err, VTB_TIMEOUT);
    }
    __syncwarp();
    // epilogue: every warp waits for the accumulator (or gives up with the others)
    bool have = (nk > 0) && mbar_wait(&sm.done, 0, limit);
    if (!have && nk > 0) {
        if ((tid & 31) == 0) atomicExch(err, VTB_TIMEOUT);
        // the issued MMAs finish before the accumulator is touched or freed
        mbar_wait(&sm.done, 0, kDrainLimit);
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    // a CTA that gave up drains its producer's issued TMA loads before the
    // stage ring is reused or the CTA exits
    if (tid == 0)
        for (int kb = issued > S ? issued - S : 0; kb < issued; ++kb)
            mbar_wait(&sm.full[kb % S], (kb / S) & 1, kDrainLimit);
    const bool rowf = std::is_same<OutT, float>::value && c_n == 1 && !accumulate;
    const bool unit = alpha == 1.0;
    const int r = warp * 32 + (tid & 31);   // this thread's accumulator row (TMEM lane)
    static_assert(kCols % 32 == 0, "32-column accumulator chunks");
    if (rowf && tmC != nullptr) {
        // row-major float output by tensor stores: 32-column slabs of 128 rows
        // x 128 bytes in the C map's 128-byte swizzle, staged in the (now
        // idle) stage ring
        constexpr int kSlabBytes = kTcBM * 128;
        static_assert(sizeof(sm.a) + sizeof(sm.b) >= (size_t)(kCols / 32) * kSlabBytes, "slabs fit the ring");
        uint8_t* st = reinterpret_cast<uint8_t*>(&sm.a[0][0][0]);
        __syncthreads();
#pragma unroll 1
        for (int c0 = 0; c0 < kCols; c0 += 32) {
            uint32_t v[2][16];
            tmem_ld16_async(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v[0]);
            tmem_ld16_async(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(c0 + 16), v[1]);
            tmem_ld_wait();
            uint8_t* row = st + (c0 / 32) * kSlabBytes + r * 128;
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const uint32_t* w = &v[q >> 2][(q & 3) * 4];
                float4 f;
                if (unit) {
                    f = make_float4(__uint_as_float(w[0]), __uint_as_float(w[1]), __uint_as_float(w[2]),
                                    __uint_as_float(w[3]));
                } else {
                    f = make_float4((float)(alpha * (double)__uint_as_float(w[0])),
                                    (float)(alpha * (double)__uint_as_float(w[1])),
                                    (float)(alpha * (double)__uint_as_float(w[2])),
                                    (float)(alpha * (double)__uint_as_float(w[3])));
                }
                *reinterpret_cast<float4*>(row + ((q ^ (r & 7)) << 4)) = f;
            }
        }
        // the generic-proxy writes become visible to the tensor stores
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        // the map covers the first N4 = N rounded down to 4 columns (whole
        // 16-byte chunks: the tensor store clips at chunk granularity); the
        // last N - N4 columns are written from the slabs by plain stores
        const int N4 = N & ~3;
        if (tid == 0 && have) {
            for (int j = 0; j < kCols / 32; ++j)
                if (n0 + 32 * j < N4) tma_store_2d(tmC, st + j * kSlabBytes, n0 + 32 * j, m0);
            asm volatile("cp.async.bulk.commit_group;" ::: "memory");
        }
        if (have && N4 < N && m0 + r < M) {
            for (int col = max(N4, n0); col < min(N, n0 + kCols); ++col) {
                const int cc = col - n0, q = (cc & 31) >> 2;
                const float* src = reinterpret_cast<const float*>(st + (cc >> 5) * kSlabBytes + r * 128 +
                                                                  ((q ^ (r & 7)) << 4)) + (cc & 3);
                reinterpret_cast<float*>(C)[(int64_t)(m0 + r) * c_m + col] = *src;
            }
        }
        // the slabs are read before the CTA exits
        if (tid == 0 && have) asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
    } else if (rowf) {
        // row-major float output without a map: the tile goes through the
        // stage ring so that each warp's global stores run along a row (one
        // thread per row would scatter every store over 32 rows)
        constexpr int kLds = kCols + 4;  // rows 4 banks apart: conflict-free float4 stores
        static_assert(sizeof(sm.a) + sizeof(sm.b) >= sizeof(float) * kTcBM * kLds, "staging tile fits the ring");
        float* st = reinterpret_cast<float*>(&sm.a[0][0][0]);
        __syncthreads();
#pragma unroll 1
        for (int c0 = 0; c0 < kCols; c0 += 32) {
            uint32_t v[2][16];
            tmem_ld16_async(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v[0]);
            tmem_ld16_async(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(c0 + 16), v[1]);
            tmem_ld_wait();
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                float f[16];
#pragma unroll
                for (int j = 0; j < 16; ++j)
                    f[j] = unit ? __uint_as_float(v[h][j]) : (float)(alpha * (double)__uint_as_float(v[h][j]));
                float4* dst = reinterpret_cast<float4*>(st + r * kLds + c0 + 16 * h);
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    dst[q] = make_float4(f[4 * q], f[4 * q + 1], f[4 * q + 2], f[4 * q + 3]);
            }
        }
        __syncthreads();
        if (have) {
            // warp w writes rows w, w + 4, ...: 8-byte pairs along the row when
            // the row starts allow it, else single floats
            const int rows = min(kTcBM, M - m0), cols = min(kCols, N - n0), lane = tid & 31;
            float* Cf = reinterpret_cast<float*>(C) + (int64_t)m0 * c_m + n0;
            const bool pairs = (c_m & 1) == 0 && (reinterpret_cast<uintptr_t>(Cf) & 7) == 0;
            constexpr int kRowsPerIter = 4;
#pragma unroll 1
            for (int rr0 = warp; rr0 < rows; rr0 += 4 * kRowsPerIter) {
#pragma unroll
                for (int u = 0; u < kRowsPerIter; ++u) {
                    const int rr = rr0 + 4 * u;
                    if (rr >= rows) break;
                    const float* srow = st + rr * kLds;
                    float* grow = Cf + (int64_t)rr * c_m;
                    if (pairs) {
#pragma unroll
                        for (int cc = 2 * lane; cc < kCols; cc += 64) {
                            if (cc + 1 < cols) {
                                *reinterpret_cast<float2*>(grow + cc) = *reinterpret_cast<const float2*>(srow + cc);
                            } else if (cc < cols) {
                                grow[cc] = srow[cc];
                            }
                        }
                    } else {
#pragma unroll
                        for (int cc = lane; cc < kCols; cc += 32)
                            if (cc < cols) grow[cc] = srow[cc];
                    }
                }
            }
        }
    } else {
        const int row = m0 + r;
#pragma unroll 1
        for (int c0 = 0; c0 < kCols; c0 += 16) {
            uint32_t v[16];
            tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
            if (have && row < M) {
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const int col = n0 + c0 + j;
                    if (col < N) {
                        OutT* c = C + (int64_t)row * c_m + (int64_t)col * c_n;
                        const double x = alpha * (double)__uint_as_float(v[j]);
                        *c = accumulate ? (OutT)((double)*c + x) : (OutT)x;
                    }
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
    }
}

template <int BN, typename OutT, bool X3, int NS, int BK>
__global__ void __launch_bounds__(128, 1) tc_gemm_kernel(const __grid_constant__ CUtensorMap tmA,
                                                         const __grid_constant__ CUtensorMap tmB,
                                                         const __grid_constant__ CUtensorMap tmC, int use_c_map,
                                                         int M, int N, int K, OutT* __restrict__ C, int64_t c_m,
                                                         int64_t c_n, double alpha, int accumulate,
                                                         int32_t* __restrict__ err, uint32_t limit) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    tc_tile<BN, OutT, X3, NS, BK>(&tmA, &tmB, use_c_map ? &tmC : nullptr, M, N, K, blockIdx.y * kTcBM,
                                  blockIdx.x * (NS * BN), C, c_m, c_n, alpha, accumulate, err, limit, smem_raw);
}

// Grouped GEMM: many independent problems C_p = A_p B_p^T (float32 output,
// row-major, leading dimension ldc) in one launch.  Problem p owns the tiles
// [tile_start, tile_start + ceil(M/128) * ceil(N/BN)); a CTA finds its
// problem by binary search and runs the same tile pipeline, its tensor maps
// read from global memory (written by the host before the launch).
struct TcGroupProblem {
    CUtensorMap ma;
    CUtensorMap mb;
    float* C;
    int64_t ldc;
    int M, N, K, tile_start;
    int32_t* err;
    int pad[6];
};

template <int BN, bool X3>
__global__ void __launch_bounds__(128, 1) tc_gemm_grouped_kernel(const TcGroupProblem* __restrict__ probs, int nprob,
                                                                  uint32_t limit) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    const int tile = blockIdx.x;
    int lo = 0, hi = nprob - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (probs[mid].tile_start <= tile) lo = mid;
        else hi = mid - 1;
    }
    const TcGroupProblem* p = probs + lo;
    if (threadIdx.x == 0) {
        // the TMA unit reads the maps through the tensor-map proxy: order
        // it after the generic-proxy writes that placed them
        asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(&p->ma) : "memory");
        asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(&p->mb) : "memory");
    }
    const int ntn = (p->N + BN - 1) / BN;
    const int t = tile - p->tile_start;
    tc_tile<BN, float, X3>(&p->ma, &p->mb, nullptr, p->M, p->N, p->K, (t / ntn) * kTcBM, (t % ntn) * BN, p->C, p->ldc, 1, 1.0,
                           0, p->err, limit, smem_raw);
}

// ------------------------------------------------------------------ split-bf16 operands
// dst[r][seg*Kp + k] for seg in {0,1,2}: pattern 0 = [hi, hi, lo] (A side),
// pattern 1 = [hi, lo, hi] (B side); zero padding for k >= K.
template <typename InT>
__global__ void split_bf16x3_kernel(const InT* __restrict__ src, int rows, int K, int64_t ld, int64_t ks,
                                    double scale, int Kp, int pattern, __nv_bfloat16* __restrict__ dst) {
    const int64_t total = (int64_t)rows * Kp;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        const int r = (int)(e / Kp), k = (int)(e % Kp);
        const double x = k < K ? (double)src[(int64_t)r * ld + (int64_t)k * ks] * scale : 0.0;
        const float xf = (float)x;
        const __nv_bfloat16 hi = __float2bfloat16_rn(xf);
        const __nv_bfloat16 lo = __float2bfloat16_rn((float)(x - (double)__bfloat162float(hi)));
        __nv_bfloat16* d = dst + (int64_t)r * 3 * Kp + k;
        d[0] = hi;
        d[Kp] = pattern == 0 ? hi : lo;
        d[2 * Kp] = pattern == 0 ? lo : hi;
    }
}

// dst[r][seg*Kp + k]: seg 0 = hi, seg 1 = lo (the three-product mode's
// layout).  A thread converts 8 consecutive k and writes 16 bytes per part.
template <typename InT>
__global__ void split_bf16x2_kernel(const InT* __restrict__ src, int rows, int K, int64_t ld, int64_t ks,
                                    double scale, int Kp, __nv_bfloat16* __restrict__ dst) {
    const int gpr = Kp / 8;     // groups of 8 per row
    const int64_t total = (int64_t)rows * gpr;
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < total; g += (int64_t)gridDim.x * blockDim.x) {
        const int r = (int)(g / gpr), k0 = (int)(g % gpr) * 8;
        const InT* row = src + (int64_t)r * ld;
        __align__(16) __nv_bfloat16 hi[8], lo[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int k = k0 + i;
            const double x = k < K ? (double)__ldg(row + (int64_t)k * ks) * scale : 0.0;
            hi[i] = __float2bfloat16_rn((float)x);
            lo[i] = __float2bfloat16_rn((float)(x - (double)__bfloat162float(hi[i])));
        }
        __nv_bfloat16* d = dst + (int64_t)r * 2 * Kp + k0;
        *reinterpret_cast<uint4*>(d) = *reinterpret_cast<const uint4*>(hi);
        *reinterpret_cast<uint4*>(d + Kp) = *reinterpret_cast<const uint4*>(lo);
    }
}

// ------------------------------------------------------------------ host side
static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, []() {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

// rows x K bf16 row-major (row pitch ld elements), box = box_rows x box_k
// (64: 128-byte rows, 128-byte swizzle; 32: 64-byte rows, 64-byte swizzle)
static int make_map(CUtensorMap* map, const void* base, int rows, int K, int64_t ld, int box_rows,
                    int box_k = kTcBK) {
    auto fn = encode_fn();
    if (!fn) return VTB_CUDA_ERR;
    cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
    cuuint32_t box[2] = {(cuuint32_t)box_k, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, box_k == 32 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_128B,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? VTB_OK : VTB_BAD_ARG;
}

// float32 C (rows x cols, row pitch ldc elements) for the tensor-store
// epilogue: box 32 x 128, 128-byte swizzle, over the first cols rounded down
// to 4 columns (the kernel writes the rest); false when the layout does not
// allow a map (base not 16-byte aligned, pitch not a multiple of 16 bytes)
static bool make_c_map(CUtensorMap* map, const float* C, int rows, int cols, int64_t ldc) {
    auto fn = encode_fn();
    const int cols4 = cols & ~3;
    if (!fn || cols4 == 0 || ((uintptr_t)C & 15) != 0 || ((ldc * 4) & 15) != 0 || ldc < cols) return false;
    cuuint64_t dims[2] = {(cuuint64_t)cols4, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)ldc * 4};
    cuuint32_t box[2] = {32, (cuuint32_t)kTcBM};
    cuuint32_t estr[2] = {1, 1};
    return fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(C), dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_NONE,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int BN, typename OutT, bool X3, int NS, int BK>
static int launch_tc(const CUtensorMap& ma, const CUtensorMap& mb, int M, int N, int K, OutT* C, int64_t c_m,
                     int64_t c_n, double alpha, int accumulate, int32_t* err, cudaStream_t s) {
    const size_t sm = sizeof(TcSmem<BN, X3, NS, BK>) + 1024;
    static std::once_flag once;
    static cudaError_t attr = cudaSuccess;
    std::call_once(once, [&]() {
        attr = cudaFuncSetAttribute(tc_gemm_kernel<BN, OutT, X3, NS, BK>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    });
    if (attr != cudaSuccess) {
        set_last_cuda_error(attr);
        return VTB_CUDA_ERR;
    }
    CUtensorMap mc;
    std::memset(&mc, 0, sizeof(mc));
    int use_c = 0;
    if (std::is_same<OutT, float>::value && c_n == 1 && !accumulate)
        use_c = make_c_map(&mc, reinterpret_cast<const float*>(C), M, N, c_m) ? 1 : 0;
    dim3 grid(ceil_div(N, NS * BN), ceil_div(M, kTcBM));
    tc_gemm_kernel<BN, OutT, X3, NS, BK><<<grid, 128, sm, s>>>(ma, mb, mc, use_c, M, N, K, C, c_m, c_n, alpha,
                                                               accumulate, err, wait_limit(kWaitLimit));
    return launch_status();
}

}  // namespace vtb

using namespace vtb;

VTB_API int vtb_split_bf16x3(const void* src, int src_f32, int rows, int K, int64_t ld, int64_t k_stride,
                             double scale, int pattern, void* dst, void* stream) {
    VTB_CHECK_ARG(rows >= 0 && K >= 0 && (pattern == 0 || pattern == 1));
    if (rows == 0) return VTB_OK;
    VTB_CHECK_ARG(src && dst && ((uintptr_t)dst & 15) == 0);
    const int Kp = ceil_div(K, kTcBK) * kTcBK;
    const int64_t total = (int64_t)rows * Kp;
    const int blocks = (int)std::min<int64_t>(ceil_div(total, 256), 16 * kNumSMs);
    if (src_f32)
        split_bf16x3_kernel<float><<<blocks, 256, 0, as_stream(stream)>>>(
            reinterpret_cast<const float*>(src), rows, K, ld, k_stride, scale, Kp, pattern,
            reinterpret_cast<__nv_bfloat16*>(dst));
    else
        split_bf16x3_kernel<double><<<blocks, 256, 0, as_stream(stream)>>>(
            reinterpret_cast<const double*>(src), rows, K, ld, k_stride, scale, Kp, pattern,
            reinterpret_cast<__nv_bfloat16*>(dst));
    return launch_status();
}

VTB_API int vtb_split_bf16x2(const void* src, int src_f32, int rows, int K, int64_t ld, int64_t k_stride,
                             double scale, void* dst, void* stream) {
    VTB_CHECK_ARG(rows >= 0 && K >= 0);
    if (rows == 0) return VTB_OK;
    VTB_CHECK_ARG(src && dst && ((uintptr_t)dst & 15) == 0);
    const int Kp = ceil_div(K, kTcBK) * kTcBK;
    const int64_t total = (int64_t)rows * (Kp / 8);
    const int blocks = (int)std::min<int64_t>(ceil_div(total, 256), 16 * kNumSMs);
    if (src_f32)
        split_bf16x2_kernel<float><<<blocks, 256, 0, as_stream(stream)>>>(
            reinterpret_cast<const float*>(src), rows, K, ld, k_stride, scale, Kp,
            reinterpret_cast<__nv_bfloat16*>(dst));
    else
        split_bf16x2_kernel<double><<<blocks, 256, 0, as_stream(stream)>>>(
            reinterpret_cast<const double*>(src), rows, K, ld, k_stride, scale, Kp,
            reinterpret_cast<__nv_bfloat16*>(dst));
    return launch_status();
}

template <int BN, bool X3, int NS = 1, int BK = kTcBK>
static int tc_dispatch(const void* A, int M, const void* B, int N, int K, void* C, int64_t c_m, int64_t c_n,
                       int out_f64, double alpha, int accumulate, int32_t* err, cudaStream_t s) {
    CUtensorMap ma, mb;
    const int Kw = X3 ? 2 * K : K;     // columns of the operand arrays
    int st = make_map(&ma, A, M, Kw, Kw, kTcBM, BK);
    if (st) return st;
    st = make_map(&mb, B, N, Kw, Kw, BN, BK);
    if (st) return st;
    if (out_f64)
        return launch_tc<BN, double, X3, NS, BK>(ma, mb, M, N, K, reinterpret_cast<double*>(C), c_m, c_n, alpha,
                                                 accumulate, err, s);
    return launch_tc<BN, float, X3, NS, BK>(ma, mb, M, N, K, reinterpret_cast<float*>(C), c_m, c_n, alpha,
                                            accumulate, err, s);
}

template <bool X3>
static int tc_gemm_bn(const void* A, int M, const void* B, int N, int K, void* C, int64_t c_m, int64_t c_n,
                      int out_f64, double alpha, int accumulate, int32_t* err, int bn, void* stream) {
    VTB_CHECK_ARG(M >= 0 && N >= 0 && K > 0 && (K % kTcBK) == 0);
    if (M == 0 || N == 0) return VTB_OK;
    VTB_CHECK_ARG(A && B && C && err && ((uintptr_t)A & 15) == 0 && ((uintptr_t)B & 15) == 0);
    VTB_CHECK_ARG(ceil_div(M, kTcBM) <= 65535);
    cudaStream_t s = as_stream(stream);
    switch (bn) {
        case 64: return tc_dispatch<64, X3>(A, M, B, N, K, C, c_m, c_n, out_f64, alpha, accumulate, err, s);
        case 96: return tc_dispatch<96, X3>(A, M, B, N, K, C, c_m, c_n, out_f64, alpha, accumulate, err, s);
        case 128: return tc_dispatch<128, X3>(A, M, B, N, K, C, c_m, c_n, out_f64, alpha, accumulate, err, s);
        case 160: return tc_dispatch<160, X3>(A, M, B, N, K, C, c_m, c_n, out_f64, alpha, accumulate, err, s);
        case 192: return tc_dispatch<192, X3>(A, M, B, N, K, C, c_m, c_n, out_f64, alpha, accumulate, err, s);
        case 256: return tc_dispatch<256, X3>(A, M, B, N, K, C, c_m, c_n, out_f64, alpha, accumulate, err, s);
        // two 160-column accumulators sharing each A tile, 32-wide k-blocks
        case 320: return tc_dispatch<160, X3, 2, 32>(A, M, B, N, K, C, c_m, c_n, out_f64, alpha, accumulate, err, s);
        default: return VTB_BAD_ARG;
    }
}

// Output tile widths the kernel is built for (M tile = 128): the autotuner
// of vtem_b200.autotune picks one per problem shape.
VTB_API int vtb_tc_gemm_bf16_bn(const void* A, int M, const void* B, int N, int K, void* C, int64_t c_m, int64_t c_n,
                                int out_f64, double alpha, int accumulate, int32_t* err, int bn, void* stream) {
    return tc_gemm_bn<false>(A, M, B, N, K, C, c_m, c_n, out_f64, alpha, accumulate, err, bn, stream);
}

// Three-product split-bf16 GEMM: A (M x 2K) = [A_hi | A_lo] and B (N x 2K) =
// [B_hi | B_lo] (vtb_split_bf16x2), C = alpha (A_hi B_hi^T + A_hi B_lo^T +
// A_lo B_hi^T): the products of the three-part layout of vtb_split_bf16x3
// with two thirds of its operand bytes.
VTB_API int vtb_tc_gemm_bf16x3_bn(const void* A, int M, const void* B, int N, int K, void* C, int64_t c_m,
                                  int64_t c_n, int out_f64, double alpha, int accumulate, int32_t* err, int bn,
                                  void* stream) {
    return tc_gemm_bn<true>(A, M, B, N, K, C, c_m, c_n, out_f64, alpha, accumulate, err, bn, stream);
}

VTB_API int vtb_tc_gemm_bf16(const void* A, int M, const void* B, int N, int K, void* C, int64_t c_m, int64_t c_n,
                             int out_f64, double alpha, int accumulate, int32_t* err, void* stream) {
    return vtb_tc_gemm_bf16_bn(A, M, B, N, K, C, c_m, c_n, out_f64, alpha, accumulate, err, 128, stream);
}

VTB_API int64_t vtb_tc_group_bytes(int nprob) { return nprob > 0 ? (int64_t)nprob * (int64_t)sizeof(TcGroupProblem) : 0; }

// Fill the HOST descriptor array of a grouped GEMM (nprob problems C_p =
// A_p B_p^T, A_p M_p x K_p and B_p N_p x K_p bf16 K-major, C_p float32
// row-major with leading dimension ldc_p; all arrays are host arrays of the
// problems' device pointers and sizes); *total_tiles receives the grid size.
// The caller copies the array to device memory (vtb_tc_group_bytes bytes,
// 64-byte aligned) before vtb_tc_gemm_grouped.
static int group_build(void* host_desc, int nprob, const uint64_t* A, const int* M, const uint64_t* B, const int* N,
                       const int* K, const uint64_t* C, const int64_t* ldc, const uint64_t* err, int bn, int parts,
                       int* total_tiles) {
    VTB_CHECK_ARG(host_desc && nprob > 0 && A && M && B && N && K && C && ldc && err && total_tiles);
    VTB_CHECK_ARG(bn == 64 || bn == 128 || bn == 256);
    TcGroupProblem* d = reinterpret_cast<TcGroupProblem*>(host_desc);
    int tiles = 0;
    for (int p = 0; p < nprob; ++p) {
        VTB_CHECK_ARG(M[p] > 0 && N[p] > 0 && K[p] > 0 && (K[p] % kTcBK) == 0 && A[p] && B[p] && C[p] && err[p]);
        VTB_CHECK_ARG((A[p] & 15) == 0 && (B[p] & 15) == 0);
        memset(&d[p], 0, sizeof(TcGroupProblem));
        const int Kw = parts * K[p];
        int st = make_map(&d[p].ma, reinterpret_cast<const void*>(A[p]), M[p], Kw, Kw, kTcBM);
        if (st) return st;
        st = make_map(&d[p].mb, reinterpret_cast<const void*>(B[p]), N[p], Kw, Kw, bn);
        if (st) return st;
        d[p].C = reinterpret_cast<float*>(C[p]);
        d[p].ldc = ldc[p];
        d[p].M = M[p];
        d[p].N = N[p];
        d[p].K = K[p];
        d[p].tile_start = tiles;
        d[p].err = reinterpret_cast<int32_t*>(err[p]);
        tiles += ceil_div(M[p], kTcBM) * ceil_div(N[p], bn);
    }
    *total_tiles = tiles;
    return VTB_OK;
}

VTB_API int vtb_tc_group_build(void* host_desc, int nprob, const uint64_t* A, const int* M, const uint64_t* B,
                               const int* N, const int* K, const uint64_t* C, const int64_t* ldc, const uint64_t* err,
                               int bn, int* total_tiles) {
    return group_build(host_desc, nprob, A, M, B, N, K, C, ldc, err, bn, 1, total_tiles);
}

// The same for the three-product mode: A_p (M_p x 2K_p) = [hi | lo], B_p
// (N_p x 2K_p) = [hi | lo], K_p the width of one part.
VTB_API int vtb_tc_group_build_x3(void* host_desc, int nprob, const uint64_t* A, const int* M, const uint64_t* B,
                                  const int* N, const int* K, const uint64_t* C, const int64_t* ldc,
                                  const uint64_t* err, int bn, int* total_tiles) {
    return group_build(host_desc, nprob, A, M, B, N, K, C, ldc, err, bn, 2, total_tiles);
}

template <int BN, bool X3>
static int launch_grouped(const void* desc, int nprob, int tiles, cudaStream_t s) {
    const size_t sm = sizeof(TcSmem<BN, X3>) + 1024;
    static std::once_flag once;
    static cudaError_t attr = cudaSuccess;
    std::call_once(once, [&]() {
        attr = cudaFuncSetAttribute(tc_gemm_grouped_kernel<BN, X3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)sm);
    });
    if (attr != cudaSuccess) {
        set_last_cuda_error(attr);
        return VTB_CUDA_ERR;
    }
    tc_gemm_grouped_kernel<BN, X3><<<tiles, 128, sm, s>>>(reinterpret_cast<const TcGroupProblem*>(desc), nprob,
                                                           wait_limit(kWaitLimit));
    return launch_status();
}

template <bool X3>
static int grouped(const void* dev_desc, int nprob, int total_tiles, int bn, void* stream) {
    VTB_CHECK_ARG(dev_desc && nprob > 0 && total_tiles > 0 && ((uintptr_t)dev_desc & 63) == 0);
    cudaStream_t s = as_stream(stream);
    switch (bn) {
        case 64: return launch_grouped<64, X3>(dev_desc, nprob, total_tiles, s);
        case 128: return launch_grouped<128, X3>(dev_desc, nprob, total_tiles, s);
        case 256: return launch_grouped<256, X3>(dev_desc, nprob, total_tiles, s);
        default: return VTB_BAD_ARG;
    }
}

// One launch over all problems of a descriptor array built with the same bn.
VTB_API int vtb_tc_gemm_grouped(const void* dev_desc, int nprob, int total_tiles, int bn, void* stream) {
    return grouped<false>(dev_desc, nprob, total_tiles, bn, stream);
}

// One launch over a descriptor array of vtb_tc_group_build_x3.
VTB_API int vtb_tc_gemm_grouped_x3(const void* dev_desc, int nprob, int total_tiles, int bn, void* stream) {
    return grouped<true>(dev_desc, nprob, total_tiles, bn, stream);
}
