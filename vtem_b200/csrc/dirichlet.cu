// Dirichlet-space kernels of the plain float64 decoder.
//
//  vtb_dirichlet_coeffs : Ds[n, My-my, mx+Mx] = dxdy (-1)^(mx+my) DFT2(RF_n)
//      restricted to the spatial ellipse (compute_Ds + fft2Ds_kernel,
//      vtem/vrf.py:333-377, :1293-1350).  Only (2Mx+1)(2My+1) of the
//      LPy*LPx frequencies are ever used, so instead of a full 2-D FFT the
//      kernel evaluates a separable DFT for just those bins: rows are staged
//      through shared memory 16 at a time and reduced against an exact
//      twiddle table (sincospi of integer ratios), one block per RF.
//  vtb_dirich_space : phi_n on the decode grid, equal to the reference's
//      unnormalised inverse FFT on the (Py1, Px1) period grid followed by the
//      centred crop (compute_dirich_space_fft, vrf.py:437-499, :585-677),
//      evaluated as a separable direct sum over the nonzero bins.
//  vtb_dsw : Dsw = Re(Ds Ds^H) scaled by norm_a norm_b (compute_Dsw + put_norm,
//      vrf.py:502-559), as one real GEMM over the interleaved (re, im) planes.
//  vtb_compute_q : compute_q_Kernel (vtem/dirichlet.py:204-222).
//  vtb_compute_G : compute_G_Kernel + diag_add_Kernel (dirichlet.py:272-350),
//      same per-element formula, 2-D tiled.
#include "common.cuh"
#include "gemm_f64.cuh"

namespace vtb {

// ---------------------------------------------------------------- Ds (DFT)

constexpr int kDsRows = 16;

__global__ void __launch_bounds__(256) ds_kernel(const double* __restrict__ rf, int64_t rf_ld, int LPy, int LPx,
                                                  int Mx, int My, double dxdy, double2* __restrict__ Ds) {
    extern __shared__ double smem[];
    const int Kx = 2 * Mx + 1, Ky = 2 * My + 1;
    double2* twx = reinterpret_cast<double2*>(smem);               // LPx entries: e^{-2 pi i r / LPx}
    double2* twy = twx + LPx;                                        // LPy entries
    double* rows = reinterpret_cast<double*>(twy + LPy);             // kDsRows x LPx
    double2* R = reinterpret_cast<double2*>(rows + kDsRows * LPx);   // kDsRows x Kx
    const int n = blockIdx.x;
    const int tid = threadIdx.x;
    for (int r = tid; r < LPx; r += blockDim.x) {
        double s, c;
        sincospi(2.0 * r / LPx, &s, &c);
        twx[r] = make_double2(c, -s);
    }
    for (int r = tid; r < LPy; r += blockDim.x) {
        double s, c;
        sincospi(2.0 * r / LPy, &s, &c);
        twy[r] = make_double2(c, -s);
    }
    // accumulator of F(my, mx) owned by thread tid < Kx*Ky
    double accr = 0.0, acci = 0.0;
    const int my_t = tid / Kx - My, mx_t = tid % Kx - Mx;
    const double* src = rf + (int64_t)n * rf_ld;
    for (int py0 = 0; py0 < LPy; py0 += kDsRows) {
        const int nr = min(kDsRows, LPy - py0);
        __syncthreads();
        for (int e = tid; e < nr * LPx; e += blockDim.x) rows[e] = src[(int64_t)py0 * LPx + e];
        __syncthreads();
        // row DFT at the Kx bins: R[row][mx] = sum_px rows[row][px] e^{-2 pi i mx px / LPx}
        for (int o = tid; o < nr * Kx; o += blockDim.x) {
            const int row = o / Kx, mx = o % Kx - Mx;
            const int mxm = ((mx % LPx) + LPx) % LPx;
            double sr = 0.0, si = 0.0;
            int r = 0;
            const double* rr = rows + row * LPx;
            for (int px = 0; px < LPx; ++px) {
                const double2 w = twx[r];
                sr = fma(rr[px], w.x, sr);
                si = fma(rr[px], w.y, si);
                r += mxm;
                if (r >= LPx) r -= LPx;
            }
            R[row * Kx + mx + Mx] = make_double2(sr, si);
        }
        __syncthreads();
        if (tid < Kx * Ky) {
            const int mym = ((my_t % LPy) + LPy) % LPy;
            for (int row = 0; row < nr; ++row) {
                const int py = py0 + row;
                const int r = (int)(((int64_t)mym * py) % LPy);
                const double2 w = twy[r];
                const double2 v = R[row * Kx + mx_t + Mx];
                accr = fma(v.x, w.x, fma(-v.y, w.y, accr));
                acci = fma(v.x, w.y, fma(v.y, w.x, acci));
            }
        }
    }
    if (tid < Kx * Ky) {
        const int mx = mx_t, my = my_t;
        double2 out = make_double2(0.0, 0.0);
        if ((int64_t)mx * mx * My * My + (int64_t)my * my * Mx * Mx <= (int64_t)Mx * Mx * My * My) {
            const double sgn = ((mx + my) % 2 == 0) ? dxdy : -dxdy;
            out = make_double2(sgn * accr, sgn * acci);
        }
        Ds[(int64_t)n * Kx * Ky + (My - my) * Kx + (mx + Mx)] = out;
    }
}

// ---------------------------------------------------------------- phi

__global__ void __launch_bounds__(256) dirich_space_kernel(const double2* __restrict__ Ds, int Mx, int My, int Px,
                                                            int Py, int Px1, int Py1, double* __restrict__ out) {
    extern __shared__ double smem[];
    const int Kx = 2 * Mx + 1, Ky = 2 * My + 1;
    double2* Q = reinterpret_cast<double2*>(smem);  // Ky x Px : sum over mx
    double2* ey = Q + Ky * Px;                       // Ky x Py
    const int n = blockIdx.x;
    const int tid = threadIdx.x;
    const int xd = (Px1 - Px) / 2, yd = (Py1 - Py) / 2;
    const double2* D = Ds + (int64_t)n * Kx * Ky;
    for (int o = tid; o < Ky * Px; o += blockDim.x) {
        const int myi = o / Px, px = o % Px;
        const int my = myi - My;
        double sr = 0.0, si = 0.0;
        for (int mx = -Mx; mx <= Mx; ++mx) {
            const double2 d = D[(My - my) * Kx + (mx + Mx)];
            const double sg = (((mx + my) % 2) == 0) ? 1.0 : -1.0;
            const int64_t r = ((((int64_t)mx * (px + xd)) % Px1) + Px1) % Px1;
            double s, c;
            sincospi(2.0 * r / Px1, &s, &c);
            sr += sg * (d.x * c - d.y * s);
            si += sg * (d.x * s + d.y * c);
        }
        Q[o] = make_double2(sr, si);
    }
    for (int o = tid; o < Ky * Py; o += blockDim.x) {
        const int myi = o / Py, py = o % Py;
        const int my = myi - My;
        const int64_t r = ((((int64_t)my * (py + yd)) % Py1) + Py1) % Py1;
        double s, c;
        sincospi(2.0 * r / Py1, &s, &c);
        ey[o] = make_double2(c, s);
    }
    __syncthreads();
    for (int p = tid; p < Px * Py; p += blockDim.x) {
        const int py = p / Px, px = p % Px;
        double acc = 0.0;
        for (int myi = 0; myi < Ky; ++myi) {
            const double2 q = Q[myi * Px + px];
            const double2 e = ey[myi * Py + py];
            acc = fma(q.x, e.x, fma(-q.y, e.y, acc));
        }
        out[(int64_t)n * Px * Py + p] = acc;
    }
}

// ---------------------------------------------------------------- Dsw

__global__ void put_norm_kernel(double* __restrict__ W, int64_t ld, int N, const double* __restrict__ norm) {
    const int a = blockIdx.y;
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= N) return;
    W[(int64_t)a * ld + b] *= norm[a] * norm[b];
}

// ---------------------------------------------------------------- q, G

__global__ void compute_q_kernel(const double* __restrict__ tk1, const double* __restrict__ tk2,
                                 const int32_t* __restrict__ ind, int n, const double* __restrict__ kappa,
                                 const double* __restrict__ delta, const double* __restrict__ bias,
                                 const double* __restrict__ norm, double* __restrict__ q) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int nr = ind[i];
        q[i] = (kappa[nr] * delta[nr] - bias[nr] * (tk2[i] - tk1[i])) * norm[nr];
    }
}

__device__ __forceinline__ double g_time(double tk1, double tk2, double tl1, double tl2, int M, double WM) {
    double sum = 0;
    for (int m = 1; m <= M; ++m) {
        sum += (cos(m * WM * (tk2 - tl2)) - cos(m * WM * (tk2 - tl1)) - cos(m * WM * (tk1 - tl2)) +
                cos(m * WM * (tk1 - tl1))) /
               (m * m);
    }
    sum = sum * 2 / (WM * WM) + (tk2 - tk1) * (tl2 - tl1);
    return sum;
}

// 32x32 output tile per block of 256 threads (each thread 4 rows of one column).
__global__ void __launch_bounds__(256) compute_G_kernel(const double* __restrict__ tk1, const double* __restrict__ tk2,
                                                        const int32_t* __restrict__ ind, int n, double WM, int Mt,
                                                        const double* __restrict__ Dsw, int64_t dsw_ld, double lamb,
                                                        int lower_only, double* __restrict__ G, int64_t G_ld) {
    __shared__ double r1[32], r2[32], c1[32], c2[32];
    __shared__ int ri[32], ci[32];
    const int row0 = blockIdx.y * 32, col0 = blockIdx.x * 32;
    if (lower_only && col0 > row0 + 31) return;
    const int tid = threadIdx.x;
    if (tid < 32) {
        const int r = row0 + tid;
        r1[tid] = r < n ? tk1[r] : 0.0;
        r2[tid] = r < n ? tk2[r] : 0.0;
        ri[tid] = r < n ? ind[r] : 0;
    } else if (tid < 64) {
        const int c = col0 + tid - 32;
        c1[tid - 32] = c < n ? tk1[c] : 0.0;
        c2[tid - 32] = c < n ? tk2[c] : 0.0;
        ci[tid - 32] = c < n ? ind[c] : 0;
    }
    __syncthreads();
    const int lc = tid % 32;
    const int col = col0 + lc;
    if (col >= n) return;
    for (int rr = tid / 32; rr < 32; rr += 8) {
        const int row = row0 + rr;
        if (row >= n) break;
        if (lower_only && col > row) continue;
        double v = g_time(r1[rr], r2[rr], c1[lc], c2[lc], Mt, WM) * Dsw[(int64_t)ri[rr] * dsw_ld + ci[lc]];
        if (row == col && lamb != 0.0) v += lamb;
        G[(int64_t)row * G_ld + col] = v;
    }
}

}  // namespace vtb

using namespace vtb;

VTB_API int vtb_dirichlet_coeffs(const double* rf, int N, int LPy, int LPx, int64_t rf_ld, int Mx, int My,
                                 double dxdy, double* Ds, void* stream) {
    VTB_CHECK_ARG(N >= 0 && LPy > 0 && LPx > 0 && Mx >= 0 && My >= 0 && rf_ld >= (int64_t)LPx * LPy);
    if (N == 0) return VTB_OK;
    VTB_CHECK_ARG(rf && Ds);
    const int Kx = 2 * Mx + 1, Ky = 2 * My + 1;
    VTB_CHECK_ARG(Kx * Ky <= 256);
    const size_t sm = (size_t)(LPx + LPy) * sizeof(double2) + (size_t)kDsRows * LPx * sizeof(double) +
                      (size_t)kDsRows * Kx * sizeof(double2);
    VTB_CHECK_ARG(sm <= 200 * 1024);
    if (sm > 48 * 1024)
        VTB_CUDA_TRY(cudaFuncSetAttribute(ds_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    ds_kernel<<<N, 256, sm, as_stream(stream)>>>(rf, rf_ld, LPy, LPx, Mx, My, dxdy,
                                                 reinterpret_cast<double2*>(Ds));
    return launch_status();
}

VTB_API int vtb_dirich_space(const double* Ds, int N, int Mx, int My, int Px, int Py, int Px1, int Py1,
                             double* out, void* stream) {
    VTB_CHECK_ARG(N >= 0 && Mx >= 0 && My >= 0 && Px > 0 && Py > 0 && Px1 >= Px && Py1 >= Py);
    // the reference's FFT placement folds bins that alias on the period grid
    VTB_CHECK_ARG(2 * Mx + 1 <= Px1 && 2 * My + 1 <= Py1);
    if (N == 0) return VTB_OK;
    VTB_CHECK_ARG(Ds && out);
    const int Ky = 2 * My + 1;
    const size_t sm = (size_t)Ky * (Px + Py) * sizeof(double2);
    VTB_CHECK_ARG(sm <= 200 * 1024);
    if (sm > 48 * 1024)
        VTB_CUDA_TRY(
            cudaFuncSetAttribute(dirich_space_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    dirich_space_kernel<<<N, 256, sm, as_stream(stream)>>>(reinterpret_cast<const double2*>(Ds), Mx, My, Px, Py,
                                                          Px1, Py1, out);
    return launch_status();
}

VTB_API int vtb_dsw(const double* Ds, int N, int Ks, const double* norm, double* Dsw, int64_t ld, void* stream) {
    VTB_CHECK_ARG(N >= 0 && Ks >= 0 && ld >= N);
    if (N == 0) return VTB_OK;
    VTB_CHECK_ARG(Ds && norm && Dsw);
    // Re(conj(a) b) = a.re b.re + a.im b.im: a real GEMM over the interleaved planes
    GemmF64Args g{N, N, 2 * Ks, Ds, 2 * (int64_t)Ks, 1, Ds, 2 * (int64_t)Ks, 1, Dsw, ld, 1, 1.0, 0.0};
    int st = gemm_f64(g, as_stream(stream));
    if (st) return st;
    dim3 grid(ceil_div(N, 256), N);
    put_norm_kernel<<<grid, 256, 0, as_stream(stream)>>>(Dsw, ld, N, norm);
    return launch_status();
}

VTB_API int vtb_compute_q(const double* tk1, const double* tk2, const int32_t* ind, int n, const double* kappa,
                          const double* delta, const double* bias, const double* norm, double* q, void* stream) {
    VTB_CHECK_ARG(n >= 0);
    if (n == 0) return VTB_OK;
    VTB_CHECK_ARG(tk1 && tk2 && ind && kappa && delta && bias && norm && q);
    const int blocks = min(ceil_div(n, 256), 6 * kNumSMs);
    compute_q_kernel<<<blocks, 256, 0, as_stream(stream)>>>(tk1, tk2, ind, n, kappa, delta, bias, norm, q);
    return launch_status();
}

VTB_API int vtb_compute_G(const double* tk1, const double* tk2, const int32_t* ind, int n, double Wt, int Mt,
                          const double* Dsw, int64_t dsw_ld, double lamb, int lower_only, double* G, int64_t G_ld,
                          void* stream) {
    VTB_CHECK_ARG(n >= 0 && Mt >= 0 && G_ld >= n);
    if (n == 0) return VTB_OK;
    VTB_CHECK_ARG(tk1 && tk2 && ind && Dsw && G && Mt > 0);
    dim3 grid(ceil_div(n, 32), ceil_div(n, 32));
    VTB_CHECK_ARG(grid.y <= 65535);
    compute_G_kernel<<<grid, 256, 0, as_stream(stream)>>>(tk1, tk2, ind, n, Wt / Mt, Mt, Dsw, dsw_ld, lamb,
                                                         lower_only, G, G_ld);
    return launch_status();
}
