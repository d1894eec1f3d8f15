// Ideal IAF time encoder: warp-per-neuron FP64 scan.
//
// Semantics follow the reference kernels exactly (vtem/ensemble_encode.py:
// 438-552 deterministic thresholds, :555-674 random thresholds, including the
// draw of the next threshold before `area -= (delta - v0)` at :623-627) and
// VTEM_IAF's block loop (vtem/vtem.py:165-200): frames are grouped in blocks of
// `block_frames` sharing one boundary frame, time_count restarts at 0 at every
// block boundary and v0 carries over.  Spike times are block-relative, as the
// reference stores them.
//
// This file is compiled with --fmad=false: every product and sum rounds
// separately, in the reference's source order, so spike times and sample
// indices are bit-identical to a non-contracting host execution of the
// reference kernel.
//
// Work split: one warp per neuron.  For each chunk of 32 steps the lanes load
// 32 samples (coalesced when the input is neuron-major; the loads run
// kIafAhead chunks ahead of their use, in registers), form y = (x+b)/kappa
// and the trapezoid area of their own step in parallel, and stage them in
// shared memory; the warp then walks the 32 steps in order (the membrane
// recursion is a strict sequential FP64 chain that no reordering may touch).
// The common step is one add and one compare; steps with a threshold crossing
// or a negative slope take the reference's full loop.  Spikes are appended by
// lane 0 to the neuron's slice of the output.  Each neuron stops once its
// spike count reaches `cap`, which bounds every loop by the buffer size.
#include "common.cuh"

namespace vtb {

struct IafArgs {
    const double* in;
    int64_t ts, ns;          // strides of in(t, n)
    int N, F, block_frames;
    double dt;
    const double* kappa;
    const double* bias;
    const double* delta;     // threshold (mean threshold for random thresholds)
    double* v0;
    double* time_count;
    // random thresholds (randn == nullptr: deterministic)
    const double* randn;
    int64_t rb, rs, rn;      // strides of randn(block, slot, n)
    int block_cap;           // slots per block in randn
    const double* sigma;
    double* delta_value;
    // outputs, neuron-major [n * cap + j]
    double* spike_time;
    int32_t* spike_step;
    int32_t* spike_count;
    int cap;
    unsigned long long* near_count;
    double near_eps;
    int32_t* status;
    double block_rate;       // > 0: per-block spike limit ceil(block length / block_rate)
};

constexpr int kIafWarps = 4;
constexpr int kIafAhead = 8;   // chunks of 32 samples prefetched ahead

template <bool RT>
__global__ void __launch_bounds__(kIafWarps * 32, 1) iaf_scan_kernel(IafArgs p) {
    __shared__ __align__(16) double s_area[kIafWarps][32];
    __shared__ double s_y1[kIafWarps][32];
    __shared__ double s_y2[kIafWarps][32];
    __shared__ __align__(16) double s_v[kIafWarps][32];
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int w = threadIdx.x >> 5;
    const int n = blockIdx.x * kIafWarps + w;
    if (n >= p.N) return;  // uniform per warp

    const double kap = p.kappa[n];
    const double bia = p.bias[n];
    const double dt = p.dt;
    const double dmean = p.delta[n];
    const double sg = RT ? p.sigma[n] : 0.0;
    double delta = RT ? p.delta_value[n] : dmean;
    double v0 = p.v0[n];
    double tc = p.time_count[n];
    int count = 0;
    int cnt_block = 0;
    int block = 0;
    unsigned long long near = 0;
    bool stop = false;

    const int steps = p.F - 1;
    const int bstep = p.block_frames - 1;
    int next_reset = bstep > 0 ? bstep : 0x7fffffff;
    // spike limit of the current frame block (the reference's per-call buffer)
    auto block_limit = [&](int b) -> int {
        if (!(p.block_rate > 0.0)) return 0x7fffffff;
        const int len = min(p.block_frames, p.F - b * bstep);
        const double lim = ceil((double)len / p.block_rate);
        return lim < 2147483647.0 ? (int)lim : 0x7fffffff;
    };
    int lim_block = block_limit(0);
    bool limit_hit = false;
    const double* base = p.in + (int64_t)n * p.ns;
    auto ld = [&](int t) -> double { return t < p.F ? __ldg(base + (int64_t)t * p.ts) : 0.0; };

    double ycur = (ld(lane) + bia) / kap;
    double ynext = (ld(32 + lane) + bia) / kap;
    // input samples kIafAhead chunks beyond ynext, in flight while the chain
    // walks the current chunk (one chunk takes far less than an HBM round trip)
    double ahead[kIafAhead];
#pragma unroll
    for (int i = 0; i < kIafAhead; ++i) ahead[i] = ld(64 + 32 * i + lane);

    for (int t0 = 0; t0 < steps && !stop; t0 += 32) {
        const double xpre = ahead[0];
#pragma unroll
        for (int i = 0; i + 1 < kIafAhead; ++i) ahead[i] = ahead[i + 1];
        ahead[kIafAhead - 1] = ld(t0 + 64 + 32 * kIafAhead + lane);
        double y2l = __shfl_down_sync(full, ycur, 1);
        const double yn0 = __shfl_sync(full, ynext, 0);
        if (lane == 31) y2l = yn0;
        const double areal = (ycur + y2l) / 2 * dt;
        const bool posl = (y2l >= 0 || (y2l < 0 && ycur <= 0));
        const unsigned posmask = __ballot_sync(full, posl);
        s_area[w][lane] = areal;
        s_y1[w][lane] = ycur;
        s_y2[w][lane] = y2l;
        __syncwarp();
        const int nst = min(32, steps - t0);
        // The chunk is walked as register chains between slow steps.  A
        // chain covers the steps j0.. of the positive-slope form: the warp
        // runs the membrane and time recursions v += area_j, tc += dt in the
        // reference's order (uniform across lanes: the 32 areas are loaded
        // from shared memory into registers first, so the chain is nothing
        // but dependent adds) and stores the membrane value after each step;
        // lane j tests step j's value and ballots find the first step that is
        // a crossing or not of the positive-slope form.  Steps before it are
        // final as computed (the same float64 operations in the same order as
        // the reference's step loop); tc before it is recomputed by the same
        // additions.  That step runs the reference's full loop (slow_step)
        // from the exact state, and the next chain starts after it.  With
        // frame blocks shorter than 32 steps every step takes the full loop.
        auto slow_step = [&](int j) {
            const int g = t0 + j;
            if (g == next_reset) {  // start of the next frame block
                tc = 0.0;
                cnt_block = 0;
                ++block;
                next_reset += bstep;
                lim_block = block_limit(block);
            }
            const double area0 = s_area[w][j];
            const bool pos = (posmask >> j) & 1u;
            if (pos) {
                const double s = v0 + area0;
                near += (fabs(s - delta) < p.near_eps) ? 1ull : 0ull;
                if (!(s >= delta)) {  // the common step: no crossing
                    v0 = s;
                    tc += dt;
                    return;
                }
                // crossing(s) inside this step: the reference's loop
                double y1 = s_y1[w][j];
                const double y2 = s_y2[w][j];
                double area = area0;
                double ddt = dt;
                for (;;) {
                    const double a = ((y2 - y1) / ddt);
                    const double remain = (fabs(a) <= 1e-12) ? ((delta - v0) / y1)
                                                             : (sqrt(y1 * y1 + 2 * (delta - v0) * a) - y1) / (a);
                    tc += remain;
                    if (RT) {
                        const int slot = cnt_block < p.block_cap - 1 ? cnt_block : p.block_cap - 1;
                        delta = p.randn[(int64_t)block * p.rb + (int64_t)slot * p.rs + (int64_t)n * p.rn] * sg + dmean;
                    }
                    if (lane == 0) {
                        p.spike_time[(int64_t)n * p.cap + count] = tc;
                        p.spike_step[(int64_t)n * p.cap + count] = g;
                    }
                    ++count;
                    ++cnt_block;
                    limit_hit |= cnt_block >= lim_block;
                    area -= (delta - v0);
                    v0 = 0;
                    ddt -= remain;
                    y1 = y1 + remain * a;
                    if (count >= p.cap) { stop = true; break; }
                    const double s2 = v0 + area;
                    near += (fabs(s2 - delta) < p.near_eps) ? 1ull : 0ull;
                    if (!(s2 >= delta)) break;
                }
                if (stop) return;
                v0 += area;
                tc += ddt;
            } else {
                // negative slope through zero (ensemble_encode.py:515-535)
                double y1 = s_y1[w][j];
                const double y2 = s_y2[w][j];
                double ddt = dt;
                double a = ((y2 - y1) / ddt);
                double remain;
                for (;;) {
                    remain = y1 * y1 + 2 * (delta - v0) * a;
                    near += (fabs(remain) < p.near_eps) ? 1ull : 0ull;
                    if (!(remain >= 0)) break;
                    remain = (sqrt(remain) - y1) / a;
                    tc += remain;
                    if (RT) {
                        const int slot = cnt_block < p.block_cap - 1 ? cnt_block : p.block_cap - 1;
                        delta = p.randn[(int64_t)block * p.rb + (int64_t)slot * p.rs + (int64_t)n * p.rn] * sg + dmean;
                    }
                    if (lane == 0) {
                        p.spike_time[(int64_t)n * p.cap + count] = tc;
                        p.spike_step[(int64_t)n * p.cap + count] = g;
                    }
                    ++count;
                    ++cnt_block;
                    limit_hit |= cnt_block >= lim_block;
                    v0 = 0;
                    ddt -= remain;
                    y1 = y1 + remain * a;
                    a = ((y2 - y1) / ddt);
                    if (count >= p.cap) { stop = true; break; }
                }
                if (stop) return;
                v0 += (y1 + y2) / 2 * ddt;
                tc += ddt;
            }
        };
        // the next chunk's inputs, issued before the walk so the division overlaps it
        const double ynn = (xpre + bia) / kap;
        const bool fastok = bstep >= 32 || bstep <= 0;
        int j0 = 0;
        while (j0 < nst && !stop) {
            int f = j0;
            if (fastok) {
                const int rpos = (next_reset >= t0 + j0 && next_reset < t0 + nst) ? next_reset - t0 : -1;
                double ar[32];
#pragma unroll
                for (int j = 0; j < 32; j += 2) {
                    const double2 q = *reinterpret_cast<const double2*>(&s_area[w][j]);
                    ar[j] = q.x;
                    ar[j + 1] = q.y;
                }
                double v = v0, tt = tc;
                if (j0 == 0 && nst == 32 && rpos < 0) {
#pragma unroll
                    for (int j = 0; j < 32; j += 2) {
                        v = v + ar[j];
                        tt = tt + dt;
                        const double va = v;
                        v = v + ar[j + 1];
                        tt = tt + dt;
                        *reinterpret_cast<double2*>(&s_v[w][j]) = make_double2(va, v);
                    }
                } else {
#pragma unroll
                    for (int j = 0; j < 32; j += 2) {
                        if (j >= j0 && j < nst) {
                            if (j == rpos) tt = 0.0;
                            v = v + ar[j];
                            tt = tt + dt;
                        }
                        const double va = v;
                        if (j + 1 >= j0 && j + 1 < nst) {
                            if (j + 1 == rpos) tt = 0.0;
                            v = v + ar[j + 1];
                            tt = tt + dt;
                        }
                        *reinterpret_cast<double2*>(&s_v[w][j]) = make_double2(va, v);
                    }
                }
                __syncwarp();
                const double s_l = s_v[w][lane];
                const bool inseg = lane >= j0 && lane < nst;
                const unsigned npos = __ballot_sync(full, inseg && !((posmask >> lane) & 1u));
                const unsigned cross = __ballot_sync(full, inseg && s_l >= delta);
                const unsigned nearm = __ballot_sync(full, inseg && fabs(s_l - delta) < p.near_eps);
                const unsigned stopm = npos | cross;
                f = stopm ? __ffs(stopm) - 1 : nst;
                near += (unsigned long long)__popc(f < 32 ? (nearm & ((1u << f) - 1u)) : nearm);
                if (f == nst) {
                    v0 = v;
                    tc = tt;
                } else if (f > j0) {
                    v0 = s_v[w][f - 1];
                    double t2 = tc;
                    for (int j = j0; j < f; ++j) {
                        if (j == rpos) t2 = 0.0;
                        t2 = t2 + dt;
                    }
                    tc = t2;
                }
                if (rpos >= j0 && rpos < f) {
                    cnt_block = 0;
                    ++block;
                    next_reset += bstep;
                    lim_block = block_limit(block);
                }
                __syncwarp();
                if (f >= nst) break;
            }
            slow_step(f);
            j0 = f + 1;
        }
        __syncwarp();
        ycur = ynext;
        ynext = ynn;
    }
    if (lane == 0) {
        p.v0[n] = v0;
        p.time_count[n] = tc;
        p.spike_count[n] = count;
        if (RT) p.delta_value[n] = delta;
        if (p.near_count && near) atomicAdd(p.near_count, near);
        if (p.status) {
            if (limit_hit) atomicExch(p.status, VTB_BLOCK_LIMIT);
            else if (stop) atomicCAS(p.status, 0, VTB_OVERFLOW);
        }
    }
}

// Consecutive pairs of each neuron's spikes, one warp per neuron (this file
// is compiled without FMA contraction, so t rounds as the reference's
// expression time + block * refresh - t0 does).
__global__ void __launch_bounds__(256) spike_pairs_kernel(const double* __restrict__ time,
                                                          const int32_t* __restrict__ step,
                                                          const int32_t* __restrict__ count, int N, int cap,
                                                          int bstep, double R, double t0, double T,
                                                          const int64_t* __restrict__ offs, double* __restrict__ tk1,
                                                          double* __restrict__ tk2, int32_t* __restrict__ ind,
                                                          int32_t* __restrict__ outside) {
    const int n = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (n >= N) return;
    const int c = min(count[n], cap);
    const int64_t o = offs[n];
    bool bad = false;
    for (int j = lane; j < c; j += 32) {
        const int64_t k = (int64_t)n * cap + j;
        const double blk = (double)(step[k] / bstep);
        const double t = time[k] + blk * R - t0;
        bad |= !(t > 0.0 && t < T);
        if (j + 1 < c) {
            tk1[o + j] = t;
            ind[o + j] = n;
        }
        if (j > 0) tk2[o + j - 1] = t;
    }
    if (__any_sync(0xffffffffu, bad) && lane == 0) atomicExch(outside, 1);
}

}  // namespace vtb

using namespace vtb;

VTB_API int vtb_iaf_encode(const double* input, int64_t in_t_stride, int64_t in_n_stride, int N, int F,
                           int block_frames, double dt, const double* kappa, const double* bias,
                           const double* delta, double* v0, double* time_count, const double* randn,
                           int64_t randn_block_stride, int64_t randn_slot_stride, int64_t randn_n_stride,
                           int randn_block_cap, const double* sigma, double* delta_value, double* spike_time,
                           int32_t* spike_step, int32_t* spike_count, int cap,
                           unsigned long long* near_count, double near_eps, int32_t* status, double block_rate,
                           void* stream) {
    VTB_CHECK_ARG(N >= 0 && F >= 0 && block_frames >= 1 && cap >= 1);
    if (N == 0) return VTB_OK;
    VTB_CHECK_ARG(input && kappa && bias && delta && v0 && time_count && spike_time && spike_step &&
                  spike_count);
    if (randn) VTB_CHECK_ARG(sigma && delta_value && randn_block_cap >= 1);
    IafArgs a{input, in_t_stride, in_n_stride, N, F, block_frames, dt, kappa, bias, delta, v0, time_count,
              randn, randn_block_stride, randn_slot_stride, randn_n_stride, randn_block_cap, sigma,
              delta_value, spike_time, spike_step, spike_count, cap, near_count, near_eps, status, block_rate};
    const int blocks = ceil_div(N, kIafWarps);
    if (randn)
        iaf_scan_kernel<true><<<blocks, kIafWarps * 32, 0, as_stream(stream)>>>(a);
    else
        iaf_scan_kernel<false><<<blocks, kIafWarps * 32, 0, as_stream(stream)>>>(a);
    return launch_status();
}

VTB_API int vtb_spike_pairs(const double* spike_time, const int32_t* spike_step, const int32_t* spike_count, int N,
                            int cap, int block_frames, double refresh_interval, double t0, double T,
                            const int64_t* offsets, double* tk1, double* tk2, int32_t* ind, int32_t* outside,
                            void* stream) {
    VTB_CHECK_ARG(N >= 0 && cap >= 1 && block_frames >= 2);
    if (N == 0) return VTB_OK;
    VTB_CHECK_ARG(spike_time && spike_step && spike_count && offsets && outside);
    spike_pairs_kernel<<<ceil_div((int64_t)N * 32, 256), 256, 0, as_stream(stream)>>>(
        spike_time, spike_step, spike_count, N, cap, block_frames - 1, refresh_interval, t0, T, offsets, tk1, tk2,
        ind, outside);
    return launch_status();
}
