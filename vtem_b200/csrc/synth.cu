// Reconstruction (synthesis) of the plain float64 decoder.
//
// The reference evaluates, for every voxel, a sum over all spikes of
//   c_k norm_{n_k} phi_{n_k}(x, y) psi_k(t),
//   psi_k(t) = (t_k2 - t_k1) + (2/W) sum_{m=1..Mt} [sin(mW(t-t_k1)) - sin(mW(t-t_k2))]/m
// (reconstruct_Kernel, vtem/dirichlet.py:354-420), O(voxels * spikes * Mt)
// sine evaluations.  The same sum is regrouped here without approximation:
//   psi_k(t) = sum_{|m|<=Mt} conj(T_k(m)) e^{jmWt},
//   T_k(m) = int_{t_k1}^{t_k2} e^{jmWs} ds = (2/(mW)) sin(mW dt_k/2) e^{jmW tbar_k},
// so with beta_n(m) = sum_{k in n} c_k norm_n conj(T_k(m)) (one pass over the
// spikes) the temporal weights are H[t, n] = beta_n(0) + 2 Re sum_{m>=1}
// beta_n(m) e^{jmWt}, and the video is the FP64 GEMM u = H * phi.
#include "common.cuh"
#include "gemm_f64.cuh"

namespace vtb {

__device__ __forceinline__ int lower_bound_i32(const int32_t* a, int n, int v) {
    int lo = 0, hi = n;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (a[mid] < v) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// beta[n][m] (m = 0..Mt, complex interleaved), one warp per neuron.  The
// spike list must be sorted by neuron index (the reference's spike reader
// emits it neuron by neuron, spike_store.py:345-348).
template <int MAXM>
__global__ void beta_kernel(const double* __restrict__ tk1, const double* __restrict__ tk2,
                            const int32_t* __restrict__ ind, const double* __restrict__ c,
                            const double* __restrict__ norm, int nspk, int N, int Mt, double W,
                            double2* __restrict__ beta) {
    const int nr = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (nr >= N) return;
    const int lo = lower_bound_i32(ind, nspk, nr);
    const int hi = lower_bound_i32(ind, nspk, nr + 1);
    double br[MAXM + 1], bi[MAXM + 1];
#pragma unroll
    for (int m = 0; m <= MAXM; ++m) br[m] = bi[m] = 0.0;
    const double nn = norm[nr];
    for (int k = lo + lane; k < hi; k += 32) {
        const double a = tk1[k], b = tk2[k];
        const double w = c[k] * nn;
        const double d = b - a, tb = 0.5 * (a + b);
        br[0] += w * d;
#pragma unroll
        for (int m = 1; m <= MAXM; ++m) {
            if (m > Mt) break;
            const double mw = m * W;
            const double amp = w * (2.0 / mw) * sin(0.5 * mw * d);
            double s, co;
            sincos(mw * tb, &s, &co);
            br[m] += amp * co;   // conj(T) = amp e^{-j mW tbar}
            bi[m] -= amp * s;
        }
    }
#pragma unroll
    for (int m = 0; m <= MAXM; ++m) {
        if (m > Mt) break;
        double r = br[m], i = bi[m];
#pragma unroll
        for (int o = 16; o; o >>= 1) {
            r += __shfl_xor_sync(0xffffffffu, r, o);
            i += __shfl_xor_sync(0xffffffffu, i, o);
        }
        if (lane == 0) beta[(int64_t)nr * (Mt + 1) + m] = make_double2(r, i);
    }
}

// H[t][n] = beta_n(0) + 2 sum_m Re(beta_n(m) e^{jmW t}); one block per time sample
__global__ void h_kernel(const double2* __restrict__ beta, int N, int Mt, double W, const double* __restrict__ t,
                         double* __restrict__ H) {
    extern __shared__ double2 e[];
    const int it = blockIdx.x;
    const double tt = t[it];
    for (int m = threadIdx.x; m <= Mt; m += blockDim.x) {
        double s, c;
        sincos(m * W * tt, &s, &c);
        e[m] = make_double2(c, s);
    }
    __syncthreads();
    for (int nr = threadIdx.x; nr < N; nr += blockDim.x) {
        const double2* b = beta + (int64_t)nr * (Mt + 1);
        double acc = 0.0;
        for (int m = 1; m <= Mt; ++m) acc += b[m].x * e[m].x - b[m].y * e[m].y;
        H[(int64_t)it * N + nr] = b[0].x + 2.0 * acc;
    }
}

}  // namespace vtb

using namespace vtb;

VTB_API int vtb_reconstruct_workspace(int N, int Nt, int Mt, int64_t* bytes) {
    VTB_CHECK_ARG(N >= 0 && Nt >= 0 && Mt >= 0 && bytes);
    *bytes = (int64_t)N * (Mt + 1) * 16 + (int64_t)Nt * N * 8 + 256;
    return VTB_OK;
}

VTB_API int vtb_reconstruct(const double* dirich, int N, int P, const double* tk1, const double* tk2,
                            const double* c, const int32_t* ind, const double* norm, int nspk, const double* t,
                            int Nt, int Mt, double WM, double* u, void* work, int64_t work_bytes, void* stream) {
    VTB_CHECK_ARG(N > 0 && P > 0 && nspk >= 0 && Nt >= 0 && Mt >= 1 && Mt <= 64);
    if (Nt == 0) return VTB_OK;
    VTB_CHECK_ARG(dirich && norm && t && u && work);
    VTB_CHECK_ARG(nspk == 0 || (tk1 && tk2 && c && ind));
    int64_t need = 0;
    vtb_reconstruct_workspace(N, Nt, Mt, &need);
    VTB_CHECK_ARG(work_bytes >= need);
    cudaStream_t s = as_stream(stream);
    double2* beta = reinterpret_cast<double2*>(work);
    double* H = reinterpret_cast<double*>(reinterpret_cast<char*>(work) + (((int64_t)N * (Mt + 1) * 16 + 255) & ~255));
    const int blocks = ceil_div((int64_t)N * 32, 256);
    if (nspk == 0) {
        VTB_CUDA_TRY(cudaMemsetAsync(beta, 0, (size_t)N * (Mt + 1) * 16, s));
    } else if (Mt <= 8) {
        beta_kernel<8><<<blocks, 256, 0, s>>>(tk1, tk2, ind, c, norm, nspk, N, Mt, WM, beta);
    } else if (Mt <= 16) {
        beta_kernel<16><<<blocks, 256, 0, s>>>(tk1, tk2, ind, c, norm, nspk, N, Mt, WM, beta);
    } else {
        beta_kernel<64><<<blocks, 256, 0, s>>>(tk1, tk2, ind, c, norm, nspk, N, Mt, WM, beta);
    }
    int st = launch_status();
    if (st) return st;
    h_kernel<<<Nt, 256, (Mt + 1) * sizeof(double2), s>>>(beta, N, Mt, WM, t, H);
    st = launch_status();
    if (st) return st;
    GemmF64Args g{Nt, P, N, H, N, 1, dirich, 1, P, u, P, 1, 1.0, 0.0};
    return gemm_f64(g, s);
}
