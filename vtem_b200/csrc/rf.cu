// Receptive-field banks and the float64 RF projection.
//
//  vtb_rf_gabor / vtb_rf_cs : the RF formulas of gabor_Kernel / cs_Kernel
//      (vtem/vrf.py:1197-1291, :1120-1193) on a pixel grid, one thread per
//      pixel, grid (pixels/256, filters).
//  vtb_rf_filter : L[f, n] = scale * sum_p V[f, p] RF[n, p] (the DGEMM of
//      vrf.py:291 / :871), written straight into the layout the IAF scan
//      reads (no separate transpose pass, unlike vrf.py:292).
#include "common.cuh"
#include "gemm_f64.cuh"

namespace vtb {

__device__ __forceinline__ void pixel_xy(int pix, int Px, int Py, double Sx, double Sy, double x_start,
                                         double y_start, double& x, double& y) {
    int px = pix % Px;
    int py = pix / Px;
    double d = Sx / Px;
    x = (double)px * d + x_start;
    d = Sy / Py;
    y = -((double)py * d + y_start);
}

__global__ void rf_gabor_kernel(const double* __restrict__ h_alpha, const double* __restrict__ h_l,
                                const double* __restrict__ h_x0, const double* __restrict__ h_y0,
                                const int32_t* __restrict__ h_ab, const double* __restrict__ gain, int Px,
                                int Py, double Sx, double Sy, double x_start, double y_start, double kappa,
                                double* __restrict__ out, int64_t out_ld) {
    const int n = blockIdx.y;
    const int pix = blockIdx.x * blockDim.x + threadIdx.x;
    if (pix >= Px * Py) return;
    const double alpha = 1.0 / h_alpha[n];
    double x, y;
    pixel_xy(pix, Px, Py, Sx, Sy, x_start, y_start, x, y);
    x = alpha * (x - h_x0[n]);
    y = alpha * (y - h_y0[n]);
    double st, ct;
    sincos(h_l[n], &st, &ct);
    const double X = x * ct + y * st;
    const double Y = -x * st + y * ct;
    const double first = alpha * (1.0 / sqrt(2.0 * 3.141592653589793)) * exp(-((4 * X * X) + (Y * Y)) / 8);
    double sk, ck;
    sincos(kappa * X, &sk, &ck);
    double g = first * (h_ab[n] == 0 ? ck : sk);
    if (gain) g *= gain[n];
    out[(int64_t)n * out_ld + pix] = g;
}

__global__ void rf_cs_kernel(const double* __restrict__ h_alpha, const double* __restrict__ h_x0,
                             const double* __restrict__ h_y0, const double* __restrict__ gain, int Px, int Py,
                             double Sx, double Sy, double x_start, double y_start, double sc2, double ss2,
                             double* __restrict__ out, int64_t out_ld) {
    const int n = blockIdx.y;
    const int pix = blockIdx.x * blockDim.x + threadIdx.x;
    if (pix >= Px * Py) return;
    const double alpha = 1.0 / h_alpha[n];
    double x, y;
    pixel_xy(pix, Px, Py, Sx, Sy, x_start, y_start, x, y);
    x = alpha * (x - h_x0[n]);
    y = alpha * (y - h_y0[n]);
    const double XY = -(x * x + y * y);
    double g = alpha * (exp(XY / (2 * sc2)) / sc2 - 0.9 * exp(XY / (2 * ss2)) / ss2);
    g = g / 6.283185307179586;
    if (gain) g *= gain[n];
    out[(int64_t)n * out_ld + pix] = g;
}

}  // namespace vtb

using namespace vtb;

VTB_API int vtb_rf_gabor(const double* h_alpha, const double* h_l, const double* h_x0, const double* h_y0,
                         const int32_t* h_ab, const double* gain, int n_filters, int Px, int Py, double Sx,
                         double Sy, double x_start, double y_start, double KAPPA, double* out, int64_t out_ld,
                         void* stream) {
    VTB_CHECK_ARG(n_filters >= 0 && Px > 0 && Py > 0 && out_ld >= (int64_t)Px * Py);
    if (n_filters == 0) return VTB_OK;
    VTB_CHECK_ARG(h_alpha && h_l && h_x0 && h_y0 && h_ab && out && n_filters <= 65535);
    dim3 grid(ceil_div((int64_t)Px * Py, 256), n_filters);
    rf_gabor_kernel<<<grid, 256, 0, as_stream(stream)>>>(h_alpha, h_l, h_x0, h_y0, h_ab, gain, Px, Py, Sx, Sy,
                                                         x_start, y_start, KAPPA, out, out_ld);
    return launch_status();
}

VTB_API int vtb_rf_cs(const double* h_alpha, const double* h_x0, const double* h_y0, const double* gain,
                      int n_filters, int Px, int Py, double Sx, double Sy, double x_start, double y_start,
                      double sigma_center, double sigma_surround, double* out, int64_t out_ld, void* stream) {
    VTB_CHECK_ARG(n_filters >= 0 && Px > 0 && Py > 0 && out_ld >= (int64_t)Px * Py);
    if (n_filters == 0) return VTB_OK;
    VTB_CHECK_ARG(h_alpha && h_x0 && h_y0 && out && n_filters <= 65535);
    dim3 grid(ceil_div((int64_t)Px * Py, 256), n_filters);
    rf_cs_kernel<<<grid, 256, 0, as_stream(stream)>>>(h_alpha, h_x0, h_y0, gain, Px, Py, Sx, Sy, x_start,
                                                      y_start, sigma_center * sigma_center,
                                                      sigma_surround * sigma_surround, out, out_ld);
    return launch_status();
}

VTB_API int vtb_rf_filter(const double* video, int F, int P, int64_t video_ld, const double* rf, int N,
                          int64_t rf_ld, double scale, double* out, int64_t out_t_stride, int64_t out_n_stride,
                          void* stream) {
    VTB_CHECK_ARG(F >= 0 && P >= 0 && N >= 0 && video_ld >= P && rf_ld >= P);
    if (F == 0 || N == 0) return VTB_OK;
    VTB_CHECK_ARG(video && rf && out);
    GemmF64Args a{F, N, P, video, video_ld, 1, rf, rf_ld, 1, out, out_t_stride, out_n_stride, scale, 0.0};
    return gemm_f64(a, as_stream(stream));
}

VTB_API int vtb_gemm_f64(int M, int N, int K, const double* A, int64_t a_m, int64_t a_k, const double* B,
                         int64_t b_n, int64_t b_k, double* C, int64_t c_m, int64_t c_n, double alpha, double beta,
                         void* stream) {
    VTB_CHECK_ARG(M >= 0 && N >= 0 && K >= 0);
    if (M == 0 || N == 0) return VTB_OK;
    VTB_CHECK_ARG(A && B && C);
    GemmF64Args a{M, N, K, A, a_m, a_k, B, b_n, b_k, C, c_m, c_n, alpha, beta};
    return gemm_f64(a, as_stream(stream));
}
