// FP64 register-tiled GEMM on the CUDA cores (DFMA), used by the plain
// float64 path: C[m, n] = alpha * sum_k A(m, k) B(n, k) + beta * C[m, n]
// with arbitrary element strides, so one kernel serves the RF projection
// (video x RFs), the synthesis (H x spatial functions) and the small
// cross-weight products.  64x64 output tile per 256-thread block, 4x4 per
// thread, k staged through shared memory in slabs of 16.
#pragma once
#include "common.cuh"

namespace vtb {

struct GemmF64Args {
    int M, N, K;
    const double* A;
    int64_t a_m, a_k;   // strides of A(m, k)
    const double* B;
    int64_t b_n, b_k;   // strides of B(n, k)
    double* C;
    int64_t c_m, c_n;   // strides of C(m, n)
    double alpha, beta;
};

// C(m, n) = alpha sum_k A(m, k) B(n, k) + beta C(m, n) on `s` (gemm_f64.cu).
int gemm_f64(const GemmF64Args& p, cudaStream_t s);

}  // namespace vtb
