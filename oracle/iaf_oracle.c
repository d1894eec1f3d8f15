/*
 * Test infrastructure only: the CPU oracle of the ideal integrate-and-fire
 * (IAF) time encoder.  Nothing in the product links this file; the tests and
 * the CPU baseline of bench.py load it through ctypes as the checker.
 *
 * This is a scalar restatement of the reference's IAF kernels, one neuron at
 * a time, in the reference's exact floating-point operation order:
 *   - deterministic thresholds: vtem/ensemble_encode.py:438-552
 *     (get_IAF_kernel_linear, both the y2>=0 branch at :493-514 and the
 *     negative-slope branch at :515-535)
 *   - random thresholds:        vtem/ensemble_encode.py:555-674
 *     (get_IAF_kernel_linear_rt; the next threshold is drawn at :623/:645
 *     *before* `area -= (delta - v0)` at :627, which is kept as is)
 * It must be compiled without floating-point contraction
 * (-ffp-contract=off) so that every product and sum rounds separately, the
 * same as the CUDA kernel built with --fmad=false.
 *
 * One call is one launch of the reference kernel (one encode() call on one
 * block of frames).  The caller owns the block loop of VTEM_IAF
 * (vtem/vtem.py:165-200): time_count is reset between blocks, v0 carries over.
 *
 * Differences from the reference, all on paths the reference leaves
 * undefined: a neuron stops scanning once its spike count exceeds
 * max_spike (the reference keeps writing into the clamped last slot and the
 * caller then raises, ensemble_encode.py:163-164); nothing is written for
 * neurons >= N (the reference writes g_v0/g_time_count/g_spike_count for
 * every thread of the last block, ensemble_encode.py:541-545).
 */
#include <math.h>
#include <stdint.h>

typedef long long i64;

/* Returns the number of neurons whose spike count went past max_spike. */
int iaf_oracle_encode_block(
    const double* in, i64 t_stride, i64 n_stride, int N, int size, double dt,
    const double* kappa, const double* bias, const double* delta_mean,
    double* v0_io, double* time_count_io,
    /* random thresholds (NULL randn = deterministic thresholds) */
    const double* randn, i64 randn_slot_stride, i64 randn_n_stride,
    const double* sigma, double* delta_value_io,
    /* outputs: neuron-major [n * max_spike + slot] */
    double* spike_time, int32_t* spike_step, int max_spike,
    int32_t* spike_count, double near_eps, i64* near_count)
{
    int overflowed = 0;
    i64 near = 0;
    for (int n = 0; n < N; ++n) {
        const double k = kappa[n];
        const double b = bias[n];
        double delta = randn ? delta_value_io[n] : delta_mean[n];
        const double dmean = delta_mean[n];
        const double sg = randn ? sigma[n] : 0.0;
        double v0 = v0_io[n];
        double time_count = time_count_io[n];
        double ddt = dt;
        int count = 0;
        int stop = 0;
        for (int i = 0; i < size - 1 && !stop; ++i) {
            double y1 = (in[(i64)i * t_stride + (i64)n * n_stride] + b) / k;
            double y2 = (in[(i64)(i + 1) * t_stride + (i64)n * n_stride] + b) / k;
            if (y2 >= 0 || (y2 < 0 && y1 <= 0)) {
                double area = (y1 + y2) / 2 * ddt;
                for (;;) {
                    double s = v0 + area;
                    if (fabs(s - delta) < near_eps) ++near;
                    if (!(s >= delta)) break;
                    double a = ((y2 - y1) / ddt);
                    double remain = (fabs(a) <= 1e-12)
                        ? ((delta - v0) / y1)
                        : (sqrt(y1 * y1 + 2 * (delta - v0) * a) - y1) / (a);
                    time_count += remain;
                    int slot = count < max_spike - 1 ? count : max_spike - 1;
                    if (randn)
                        delta = randn[(i64)slot * randn_slot_stride + (i64)n * randn_n_stride] * sg + dmean;
                    spike_time[(i64)n * max_spike + slot] = time_count;
                    spike_step[(i64)n * max_spike + slot] = i;
                    count++;
                    area -= (delta - v0);
                    v0 = 0;
                    ddt -= remain;
                    y1 = y1 + remain * a;
                    if (count > max_spike) { stop = 1; break; }
                }
                if (stop) break;
                v0 += area;
                time_count += ddt;
                ddt = dt;
            } else {
                double a = ((y2 - y1) / ddt);
                double remain;
                for (;;) {
                    remain = y1 * y1 + 2 * (delta - v0) * a;
                    if (fabs(remain) < near_eps) ++near;
                    if (!(remain >= 0)) break;
                    remain = (sqrt(remain) - y1) / a;
                    time_count += remain;
                    int slot = count < max_spike - 1 ? count : max_spike - 1;
                    if (randn)
                        delta = randn[(i64)slot * randn_slot_stride + (i64)n * randn_n_stride] * sg + dmean;
                    spike_time[(i64)n * max_spike + slot] = time_count;
                    spike_step[(i64)n * max_spike + slot] = i;
                    count++;
                    v0 = 0;
                    ddt -= remain;
                    y1 = y1 + remain * a;
                    a = ((y2 - y1) / ddt);
                    if (count > max_spike) { stop = 1; break; }
                }
                if (stop) break;
                v0 += (y1 + y2) / 2 * ddt;
                time_count += ddt;
                ddt = dt;
            }
        }
        if (count >= max_spike) overflowed++;
        v0_io[n] = v0;
        time_count_io[n] = time_count;
        spike_count[n] = count;
        if (randn) delta_value_io[n] = delta;
    }
    if (near_count) *near_count += near;
    return overflowed;
}
