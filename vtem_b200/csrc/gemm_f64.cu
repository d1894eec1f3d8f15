// FP64 register-tiled GEMM kernel (declared in gemm_f64.cuh).
#include "gemm_f64.cuh"

namespace vtb {

constexpr int kGemmBM = 64, kGemmBN = 64, kGemmBK = 16;

__global__ void __launch_bounds__(256) gemm_f64_kernel(GemmF64Args p) {
    __shared__ double As[kGemmBK][kGemmBM + 1];
    __shared__ double Bs[kGemmBK][kGemmBN + 1];
    const int tid = threadIdx.x;
    const int m0 = blockIdx.y * kGemmBM;
    const int n0 = blockIdx.x * kGemmBN;
    const int tm = (tid / 16) * 4;
    const int tn = (tid % 16) * 4;
    double acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;

    // loader mapping: 64 rows x 16 k = 1024 elements, 4 per thread
    const bool a_kfast = p.a_k == 1;
    const bool b_kfast = p.b_k == 1;
    for (int k0 = 0; k0 < p.K; k0 += kGemmBK) {
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            int e = tid + r * 256;
            int row, kk;
            if (a_kfast) { row = e / kGemmBK; kk = e % kGemmBK; }
            else { kk = e / kGemmBM; row = e % kGemmBM; }
            int gm = m0 + row, gk = k0 + kk;
            As[kk][row] = (gm < p.M && gk < p.K) ? p.A[(int64_t)gm * p.a_m + (int64_t)gk * p.a_k] : 0.0;
            if (b_kfast) { row = e / kGemmBK; kk = e % kGemmBK; }
            else { kk = e / kGemmBN; row = e % kGemmBN; }
            int gn = n0 + row;
            gk = k0 + kk;
            Bs[kk][row] = (gn < p.N && gk < p.K) ? p.B[(int64_t)gn * p.b_n + (int64_t)gk * p.b_k] : 0.0;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < kGemmBK; ++kk) {
            double a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = As[kk][tm + i];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tn + j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        int gm = m0 + tm + i;
        if (gm >= p.M) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            int gn = n0 + tn + j;
            if (gn >= p.N) continue;
            double* c = p.C + (int64_t)gm * p.c_m + (int64_t)gn * p.c_n;
            double v = p.alpha * acc[i][j];
            if (p.beta != 0.0) v += p.beta * *c;
            *c = v;
        }
    }
}

int gemm_f64(const GemmF64Args& p, cudaStream_t s) {
    if (p.M <= 0 || p.N <= 0) return VTB_OK;
    dim3 grid(ceil_div(p.N, kGemmBN), ceil_div(p.M, kGemmBM));
    if (grid.y > 65535) return VTB_BAD_ARG;
    gemm_f64_kernel<<<grid, 256, 0, s>>>(p);
    return launch_status();
}

}  // namespace vtb
