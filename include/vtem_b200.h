/*
 * vtem_b200 C ABI: the B200 (sm_100a) kernels behind vtem's video
 * time-encode/decode path.
 *
 * The reference (bionet/vtem) has no native ABI: its Python objects launch
 * inline CUDA strings through PyCUDA.  Each entry point below replaces the
 * kernel or library call cited beside it (file:line inside the reference
 * project); the Python package vtem_b200 keeps the reference's class and
 * function names on top of these.
 *
 * Conventions for every entry point:
 *   - all array arguments are DEVICE pointers owned by the caller (the
 *     library allocates nothing on the device, except cuSOLVER's own handle);
 *   - `stream` is a cudaStream_t passed as void*; work is stream-ordered and
 *     the call returns without synchronising unless stated otherwise;
 *   - the return value is a status code (VTB_OK = 0); no C++ exception
 *     crosses the ABI.  A launch failure returns VTB_CUDA_ERR and
 *     vtb_last_cuda_error() gives the cudaError_t.
 *   - matrices are row-major with an explicit leading dimension; complex
 *     arrays are interleaved (re, im) doubles.
 */
#ifndef VTEM_B200_H
#define VTEM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VTB_ABI_VERSION 1

enum {
    VTB_OK = 0,
    VTB_BAD_ARG = 1,        /* ValueError/TypeError in the reference */
    VTB_OVERFLOW = 2,       /* spike buffer full: ensemble_encode.py:163-164 */
    VTB_OOM = 3,
    VTB_TIMEOUT = 4,
    VTB_CUDA_ERR = 5,
    VTB_NOT_CONVERGED = 6,  /* eigensolver failed */
    VTB_NO_DATA = 7,        /* "no spikes to decode": dirichlet.py:39-40 */
    VTB_BLOCK_LIMIT = 8     /* a frame block reached the per-call spike limit: ensemble_encode.py:163-164 */
};

int vtb_version(void);
const char* vtb_status_string(int status);
int vtb_last_cuda_error(void);

/* Every spin-wait inside this library's kernels (flag hand-offs between
 * CTAs, grid barriers, mbarrier waits) is bounded: after a number of polls
 * the waiting CTA records VTB_TIMEOUT in the call's status word, stops
 * waiting and returns.  polls > 0 makes every kernel launched afterwards (by
 * any thread of the process) give up after `polls` polls; 0 restores each
 * kernel's default (well under a second).  *previous (may be NULL) receives
 * the value replaced.  No counterpart in the reference (its kernels never
 * wait on one another); meant for tests and diagnostics. */
int vtb_set_wait_limit(int64_t polls, int64_t* previous);

/* ------------------------------------------------------------ RF banks */

/* Gabor RF bank on a pixel grid, out[n*out_ld + py*Px + px].
 * Replaces gabor_Kernel + generate_visual_receptive_fields
 * (vtem/vrf.py:1197-1291, :296-331).  h_alpha is the dilation as the user
 * gives it (the reference uploads 1/h_alpha, vrf.py:258); gain (may be NULL)
 * scales each RF (extension, 1 = reference). */
int vtb_rf_gabor(const double* h_alpha, const double* h_l, const double* h_x0, const double* h_y0,
                 const int32_t* h_ab, const double* gain, int n_filters, int Px, int Py, double Sx,
                 double Sy, double x_start, double y_start, double KAPPA, double* out, int64_t out_ld,
                 void* stream);

/* Centre-surround RF bank.  Replaces cs_Kernel (vtem/vrf.py:1120-1193,
 * :876-913). */
int vtb_rf_cs(const double* h_alpha, const double* h_x0, const double* h_y0, const double* gain,
              int n_filters, int Px, int Py, double Sx, double Sy, double x_start, double y_start,
              double sigma_center, double sigma_surround, double* out, int64_t out_ld, void* stream);

/* RF projection out(f, n) = scale * sum_p video[f*video_ld + p] rf[n*rf_ld + p],
 * written at out[f*out_t_stride + n*out_n_stride] (either time- or
 * neuron-major).  Replaces cublasDgemm + .T() of vrf_gabor.filter /
 * vrf_cs.filter (vtem/vrf.py:264-292, :845-872). */
int vtb_rf_filter(const double* video, int F, int P, int64_t video_ld, const double* rf, int N,
                  int64_t rf_ld, double scale, double* out, int64_t out_t_stride, int64_t out_n_stride,
                  void* stream);

/* Plain FP64 GEMM C(m,n) = alpha sum_k A(m,k) B(n,k) + beta C(m,n), all
 * element-strided.  Replaces the cuBLAS DGEMM calls of vtem/utils/linalg.py:32-338
 * (linalg.dot) on this path. */
int vtb_gemm_f64(int M, int N, int K, const double* A, int64_t a_m, int64_t a_k, const double* B,
                 int64_t b_n, int64_t b_k, double* C, int64_t c_m, int64_t c_n, double alpha, double beta,
                 void* stream);

/* ------------------------------------------------------------ tensor cores (tcgen05) */

/* Split a float64 (src_f32 = 0) or float32 matrix src(r, k) = src[r*ld + k*k_stride]
 * (rows x K, times scale) into bf16 hi/lo parts laid out along K as
 * dst[r][0:3Kp] = [hi | hi | lo] (pattern 0, the A side) or [hi | lo | hi]
 * (pattern 1, the B side), Kp = K rounded up to 64, zero padded.  With
 * vtb_tc_gemm_bf16 over K = 3Kp this gives the split-bf16 product
 * hi*hi + hi*lo + lo*hi accumulated in fp32.  The mixed-precision form of
 * the DGEMMs of vtem/vrf.py:291 (RF filter) and the Gram products. */
int vtb_split_bf16x3(const void* src, int src_f32, int rows, int K, int64_t ld, int64_t k_stride, double scale,
                     int pattern, void* dst, void* stream);

/* C(m, n) = alpha * sum_k A[m*K + k] B[n*K + k] (+ C when accumulate), A (M x K)
 * and B (N x K) bf16 row-major (K-major), K a multiple of 64, on the sm_100a
 * tensor cores (TMA + tcgen05.mma, fp32 accumulator in tensor memory), stored
 * at C[m*c_m + n*c_n] as float64 (out_f64 = 1) or float32.  *err (device int,
 * caller-zeroed) receives VTB_TIMEOUT if a pipeline wait ever gave up. */
int vtb_tc_gemm_bf16(const void* A, int M, const void* B, int N, int K, void* C, int64_t c_m, int64_t c_n,
                     int out_f64, double alpha, int accumulate, int32_t* err, void* stream);
/* vtb_tc_gemm_bf16 with output tiles 128 x bn, bn in {64, 96, 128, 160, 192,
 * 256} (vtb_tc_gemm_bf16 is bn = 128); the autotuner picks bn per problem
 * shape.  VTB_BAD_ARG for any other bn. */
int vtb_tc_gemm_bf16_bn(const void* A, int M, const void* B, int N, int K, void* C, int64_t c_m, int64_t c_n,
                        int out_f64, double alpha, int accumulate, int32_t* err, int bn, void* stream);
/* Split-bf16 operands of the three-product mode: dst[r][0:2Kp] = [hi | lo],
 * Kp = K rounded up to 64, zero padded. */
int vtb_split_bf16x2(const void* src, int src_f32, int rows, int K, int64_t ld, int64_t k_stride, double scale,
                     void* dst, void* stream);
/* Three-product split-bf16 GEMM: A (M x 2K) = [A_hi | A_lo], B (N x 2K) =
 * [B_hi | B_lo] (vtb_split_bf16x2; K, the width of one part, a multiple of
 * 64); C = alpha (A_hi B_hi^T + A_hi B_lo^T + A_lo B_hi^T), every k-block's
 * three products issued from the same shared-memory tiles: the result of
 * vtb_tc_gemm_bf16_bn on the three-part layouts with two thirds of their
 * operand bytes (the fp32 sums run in another order).  Same tile widths. */
int vtb_tc_gemm_bf16x3_bn(const void* A, int M, const void* B, int N, int K, void* C, int64_t c_m, int64_t c_n,
                          int out_f64, double alpha, int accumulate, int32_t* err, int bn, void* stream);

/* ------------------------------------------------------------ IAF encoder */

/* IAF time encoding of input(t, n) = input[t*in_t_stride + n*in_n_stride],
 * F samples, in blocks of `block_frames` frames sharing one boundary frame
 * with time_count reset to 0 at each block start (VTEM_IAF's loop,
 * vtem/vtem.py:165-200; block_frames = F gives one IAF_encode.encode call).
 * Replaces the IAF kernels of vtem/ensemble_encode.py:438-552 (randn == NULL)
 * and :555-674 (random thresholds: randn(block, slot, n) holds the N(0,1)
 * draws, block_cap slots per block, threshold = randn*sigma + delta).
 * v0, time_count (and delta_value) are read and written back.  Spikes go to
 * spike_time/spike_step[n*cap + j] (block-relative time, global step index
 * of the interval that holds the crossing), spike_count[n] their number.
 * A neuron that fills its `cap` slots stops and *status is set to
 * VTB_OVERFLOW.  With block_rate > 0, a neuron whose spike count inside
 * frame block b (starting at frame s = b*(block_frames-1)) reaches
 * ceil(min(block_frames, F - s) / block_rate) sets *status to
 * VTB_BLOCK_LIMIT: the reference's per-call buffer limit of each block's
 * IAF_encode.encode (ensemble_encode.py:163-164, avg_rate = block_rate).
 * near_count (may be NULL) accumulates the threshold comparisons whose
 * margin is below near_eps. */
int vtb_iaf_encode(const double* input, int64_t in_t_stride, int64_t in_n_stride, int N, int F,
                   int block_frames, double dt, const double* kappa, const double* bias, const double* delta,
                   double* v0, double* time_count, const double* randn, int64_t randn_block_stride,
                   int64_t randn_slot_stride, int64_t randn_n_stride, int randn_block_cap, const double* sigma,
                   double* delta_value, double* spike_time, int32_t* spike_step, int32_t* spike_count, int cap,
                   unsigned long long* near_count, double near_eps, int32_t* status, double block_rate,
                   void* stream);

/* Consecutive spike pairs of every neuron over the whole encoded clip, the
 * window [t0, T) of read_select_spikes (vtem/spike_store.py:279-351) when it
 * holds every spike: absolute time t = spike_time + (spike_step /
 * (block_frames-1)) * refresh_interval - t0 (the reference's expression,
 * same rounding), then tk1/tk2 = (t_j, t_{j+1}) and ind = n, grouped by
 * neuron.  offsets[n] = sum over m < n of max(spike_count[m] - 1, 0) (the
 * caller's exclusive scan).  *outside is set to 1 when a spike lies outside
 * (0, T), in which case the caller must use the general reader. */
int vtb_spike_pairs(const double* spike_time, const int32_t* spike_step, const int32_t* spike_count, int N, int cap,
                    int block_frames, double refresh_interval, double t0, double T, const int64_t* offsets,
                    double* tk1, double* tk2, int32_t* ind, int32_t* outside, void* stream);

/* ------------------------------------------------------------ Dirichlet space */

/* Dirichlet coefficients Ds (N, 2My+1, 2Mx+1) complex from RFs sampled on
 * an (LPy, LPx) grid over one spatial period.  Replaces compute_Ds + cuFFT +
 * fft2Ds_kernel (vtem/vrf.py:333-377, :1293-1350). */
int vtb_dirichlet_coeffs(const double* rf, int N, int LPy, int LPx, int64_t rf_ld, int Mx, int My,
                         double dxdy, double* Ds, void* stream);

/* Spatial reconstruction functions out (N, Py, Px) from Ds on a (Py1, Px1)
 * period grid, centre-cropped.  Replaces compute_dirich_space_fft +
 * Ds2fft_kernel + cuFFT inverse + filter2rec_kernel (vtem/vrf.py:437-499,
 * :585-677). */
int vtb_dirich_space(const double* Ds, int N, int Mx, int My, int Px, int Py, int Px1, int Py1,
                     double* out, void* stream);

/* Dsw[a*ld + b] = Re sum_s conj(Ds[a,s]) Ds[b,s] * norm[a] norm[b].
 * Replaces compute_Dsw (cublasZgemm + real + put_norm, vtem/vrf.py:502-559). */
int vtb_dsw(const double* Ds, int N, int Ks, const double* norm, double* Dsw, int64_t ld, void* stream);

/* ------------------------------------------------------------ decoder */

/* q[i] = (kappa delta - bias (tk2-tk1)) norm at neuron ind[i].
 * Replaces compute_q_Kernel (vtem/dirichlet.py:55-60, :204-222). */
int vtb_compute_q(const double* tk1, const double* tk2, const int32_t* ind, int n, const double* kappa,
                  const double* delta, const double* bias, const double* norm, double* q, void* stream);

/* Analytic Gram G[k*G_ld + l] = Gt(k,l) Dsw[ind_k, ind_l] (+ lamb on the
 * diagonal).  lower_only = 1 writes only l <= k.  Replaces compute_G_Kernel
 * + diag_add_Kernel (vtem/dirichlet.py:62-85, :272-350). */
int vtb_compute_G(const double* tk1, const double* tk2, const int32_t* ind, int n, double Wt, int Mt,
                  const double* Dsw, int64_t dsw_ld, double lamb, int lower_only, double* G, int64_t G_ld,
                  void* stream);

/* Workspace bytes of vtb_solve_eq_sym for order n. */
int vtb_solve_eq_sym_workspace(int n, int64_t* bytes);

/* Pseudoinverse solve c = G^+ q keeping |eigenvalues| > rcond * max; G (its
 * lower triangle is read) is destroyed.  *kept (may be NULL) receives the
 * number of values kept.  Synchronises the stream once (eigensolver status).
 * Replaces solve_eq_sym (vtem/utils/linalg.py:591-631, CULA gesvd +
 * sq_Kernel :791-833). */
int vtb_solve_eq_sym(double* G, int64_t ld, const double* q, double* c, int n, double rcond, void* work,
                     int64_t work_bytes, int32_t* kept, void* stream);

/* RNN decoder: c = 0, then steps+1 updates c += dt_alpha (q - G c).  y (may
 * be NULL) receives the last residual, c_tmp is an n-double scratch vector,
 * ynorm_trace (may be NULL) the squared residual norm every trace_every
 * steps.  Replaces rnn3 + rnn3_update (vtem/neural_network.py:15-128). */
int vtb_rnn(const double* G, int64_t ld, const double* q, double* c, double* y, double* c_tmp, int n,
            double dt_alpha, int steps, double* ynorm_trace, int trace_every, void* stream);

/* Workspace bytes of vtb_reconstruct. */
int vtb_reconstruct_workspace(int N, int Nt, int Mt, int64_t* bytes);

/* Reconstruction u (Nt, P) = sum_k c_k norm_{ind_k} dirich[ind_k] psi_k(t)
 * at the Nt times t[].  The spike list must be sorted by ind.  Replaces
 * reconstruct + reconstruct_Kernel (vtem/dirichlet.py:165-189, :354-420). */
int vtb_reconstruct(const double* dirich, int N, int P, const double* tk1, const double* tk2,
                    const double* c, const int32_t* ind, const double* norm, int nspk, const double* t, int Nt,
                    int Mt, double WM, double* u, void* work, int64_t work_bytes, void* stream);

/* ------------------------------------------------------------ coefficient-space decoder
 *
 * The same reconstruction as compute_q + compute_G + solve_eq_sym +
 * reconstruct (vtem/dirichlet.py:55-85, :165-189; vtem/utils/linalg.py:591-631)
 * computed in the Dirichlet coefficient space: with Phi[k,(s,m)] =
 * norm conj(Ds[n_k,s]) T_k(m) and G = Phi Phi^H, the reconstruction's
 * coefficients are Phi^H G^+ q = M^+ b with M = Phi^H Phi (K x K, K =
 * ellipse size * (2Mt+1)) and b = Phi^H q; the nonzero spectra of G and M
 * coincide, so the reference's rcond truncation selects the same subspace.
 * Spike lists must be sorted by neuron index. */

/* d[n*Ks + s] = norm[n] Ds[n*Kfull + smap[s]] (complex), the ellipse entries. */
int vtb_coeff_pack(const double* Ds, int N, int Kfull, const int32_t* smap, int Ks, const double* norm, double* d,
                   void* stream);

/* Per-neuron temporal Gram Wn[n][m][m'] = sum_k conj(T_k(m)) T_k(m') and
 * gn[n][m] = sum_k conj(T_k(m)) q_k (q_k as compute_q_Kernel), m in [-Mt, Mt],
 * W = Wt/Mt, Mt <= 21. */
int vtb_coeff_temporal_gram(const double* tk1, const double* tk2, const int32_t* ind, int nspk, int N,
                            const double* kappa, const double* delta, const double* bias, const double* norm, int Mt,
                            double W, double* Wn, double* gn, void* stream);

/* M = sum_n (d_n d_n^H) kron Wn (column-major, K x K complex, ld ldm) and
 * b = sum_n d_n kron gn. */
int vtb_coeff_gram(const double* d, int N, int Ks, const double* Wn, const double* gn, int Kt, double* M,
                   int64_t ldm, double* b, void* stream);

/* Workspace bytes of vtb_herm_solve (mode 0 eigen, 1 Cholesky). */
int vtb_herm_solve_workspace(int K, int mode, int64_t* bytes);

/* Solve M a = b for Hermitian PSD M (column-major, destroyed).  mode 0:
 * pseudoinverse keeping |eigenvalues| > rcond * max (the rule of
 * solve_eq_sym); mode 1: Cholesky + `refine` float64 refinement sweeps,
 * VTB_NOT_CONVERGED when the factorisation fails or the spread of its
 * squared pivots (only a lower bound of the condition number) reaches
 * 1/rcond; mode 1 uses rcond only as that acceptance threshold, and callers
 * pass one well below the pseudoinverse's own rcond.  pivots (HOST, may be NULL) receives
 * (min, max) eigenvalue (mode 0) or squared Cholesky pivot (mode 1).
 * Synchronises the stream. */
int vtb_herm_solve(double* M, int64_t ld, const double* b, double* a, int K, double rcond, int mode, int refine,
                   void* work, int64_t work_bytes, int32_t* kept, double* pivots, void* stream);

/* u[t][py][px] = Re sum_{s,m} a[s][m] e^{jmW(t0 + t dt)} E_s(px, py) on the
 * decode grid (the spatial functions of vtb_dirich_space), Nt frames,
 * float64 (out_f32 = 0) or float32 output.  For 2My+1 <= 13 one fused kernel
 * pairs each spatial frequency with its mirror (the real part of the sum over
 * half the spectrum) and A_work may be NULL; otherwise A_work holds Nt*Ks
 * complex (the per-frame temporal expansion). */
int vtb_coeff_synthesize(const double* a, const int32_t* smap, int Ks, int Mx, int My, int Mt, double W, double t0,
                         double dt, int Nt, int Px, int Py, int Px1, int Py1, double* A_work, void* u, int out_f32,
                         void* stream);
/* The same video as a rank-(2Mt+1) product: u[f][p] = sum_k C[f][k] H[p][k]
 * with C[f] = [1, cos(mWt), sin(mWt) for m = 1..Mt] at t = t0 + f dt and the
 * per-pixel weights H of vtb_coeff_basis (column 0 = Re B_0, 2m-1 = Re P_m,
 * 2m = -Im P_m, where B_m(p) = sum_s a[s][m] E_s(p) and P_m = B_m +
 * conj B_{-m}): the frames are taken in pairs symmetric about each block's
 * centre frame, 2Mt+1 float64 FMAs per pair of voxels, the coefficients'
 * spatial sum done once per window instead of once per frame.  H: P x ldh doubles, P =
 * Px*Py pixels in row-major frame order, ldh >= 2Mt+1 <= 33 (basis) or <= 21
 * (harmonics).  Replaces reconstruct_Kernel (vtem/dirichlet.py:354-420) on
 * the coefficient space, as vtb_coeff_synthesize does. */
int vtb_coeff_basis(const double* a, const int32_t* smap, int Ks, int Mx, int My, int Mt, int Px, int Py, int Px1,
                    int Py1, double* H, int ldh, void* stream);
int vtb_synth_harmonics(const double* H, int ldh, int P, int Mt, double W, double t0, double dt, int Nt, void* u,
                        int out_f32, void* stream);
/* vtb_coeff_basis followed by vtb_synth_harmonics in one call (Mt in
 * 1..10), so that no host round trip separates the two kernels.
 * H is caller-owned scratch of P x ldh doubles.  Replaces reconstruct_Kernel
 * (vtem/dirichlet.py:354-420) on the coefficient space. */
int vtb_coeff_synth_rank(const double* a, const int32_t* smap, int Ks, int Mx, int My, int Mt, int Px, int Py,
                         int Px1, int Py1, double* H, int ldh, double W, double t0, double dt, int Nt, void* u,
                         int out_f32, void* stream);

/* Grouped tensor-core GEMM: nprob independent problems C_p = A_p B_p^T (bf16
 * K-major operands as vtb_tc_gemm_bf16's, float32 row-major C_p with leading
 * dimension ldc_p, alpha 1) in ONE launch, the Gram GEMMs of a batch of clips
 * of uneven size.  vtb_tc_group_build fills a HOST descriptor array
 * (vtb_tc_group_bytes(nprob) bytes; the arrays passed are host arrays of the
 * problems' device pointers and sizes) and returns the grid size; the caller
 * copies it to 64-byte-aligned device memory and launches
 * vtb_tc_gemm_grouped with the same tile width bn (64, 128 or 256). */
int64_t vtb_tc_group_bytes(int nprob);
int vtb_tc_group_build(void* host_desc, int nprob, const uint64_t* A, const int* M, const uint64_t* B, const int* N,
                       const int* K, const uint64_t* C, const int64_t* ldc, const uint64_t* err, int bn,
                       int* total_tiles);
int vtb_tc_gemm_grouped(const void* dev_desc, int nprob, int total_tiles, int bn, void* stream);
/* The same for the three-product mode (K_p the width of one operand part). */
int vtb_tc_group_build_x3(void* host_desc, int nprob, const uint64_t* A, const int* M, const uint64_t* B,
                          const int* N, const int* K, const uint64_t* C, const int64_t* ldc, const uint64_t* err,
                          int bn, int* total_tiles);
int vtb_tc_gemm_grouped_x3(const void* dev_desc, int nprob, int total_tiles, int bn, void* stream);

/* Mixed-precision Kronecker Gram (tensor cores).  ps/ps2 list the npairs
 * spatial index pairs s <= s'; Kh = N rounded up to 64.  L receives the
 * RF-bank operand (2*npairs rows x 2Kh bf16, [hi | lo] of the real and the
 * imaginary part of a_n[p] = d_n[s_p] conj(d_n[s'_p]) over n; once per
 * decoder), R the per-decode operand (Kt(Kt+1) rows x 2Kh: the real and the
 * imaginary part of W_n[m][m'] for m <= m').  vtb_tc_gemm_bf16x3_bn(L, R)
 * over K = Kh gives the four real sums per (pair, (m, m')) from which
 * vtb_coeff_real_scatter forms both M((s,m),(s',m')) and M((s,m'),(s',m)):
 * half the products of the complex GEMM's real form (W_n is Hermitian). */
int vtb_coeff_lhs_sym(const double* d, int N, int Ks, const int32_t* ps, const int32_t* ps2, int npairs, void* L,
                      void* stream);
int vtb_coeff_wn_sym(const double* Wn, int N, int Kt, void* R, void* stream);

/* b[(s,m)] = sum_n d[n][s] gn[n][m] (the right-hand side Phi^H q). */
int vtb_coeff_rhs(const double* d, int N, int Ks, const double* gn, int Kt, double* b, void* stream);

/* Exact float64 residual r = Phi^H (q - Phi a) through the Kronecker factors
 * (gres: N x (2Mt+1) complex scratch).  Refinement sweeps of the mixed
 * decoder. */
int vtb_coeff_residual(const double* tk1, const double* tk2, const int32_t* ind, int nspk, int N, const double* kappa,
                       const double* delta, const double* bias, const double* norm, int Mt, double W, const double* d,
                       int Ks, const double* a, double* gres, double* r, void* stream);

/* a = Phi^H w for per-interval weights w (g: N x (2Mt+1) complex scratch):
 * the reconstruction coefficients of a spike-space solution c = w, e.g.
 * vtb_solve_eq_sym's pseudoinverse of the n x n Gram (vtem/dirichlet.py:165-189
 * regrouped) when a window has fewer intervals than coefficients. */
int vtb_coeff_from_spike_weights(const double* tk1, const double* tk2, const int32_t* ind, int nspk, int N,
                                 const double* w, int Mt, double W, const double* d, int Ks, double* g, double* a,
                                 void* stream);

/* x = M^-1 x with M factorised in place by vtb_herm_solve(mode 1); work >= 256 bytes. */
int vtb_herm_potrs(const double* Mfac, int64_t ld, double* x, int K, void* work, int64_t work_bytes, void* stream);

/* Batched Cholesky solve of `batch` equally sized Hermitian systems (a group
 * of clips with the same K): Mptrs/bptrs are device arrays of device
 * pointers (column-major M factorised in place, b overwritten by the
 * solution), infos[i] != 0 flags a clip whose factorisation failed or whose
 * pivot spread exceeds 1/rcond (it then needs vtb_herm_solve mode 0).  The
 * batched form of the per-window solve of vtem/vtdm.py:645-648. */
int vtb_herm_chol_batched(double** Mptrs, int64_t ld, double** bptrs, int K, int batch, double rcond,
                          int32_t* infos, int32_t* solve_info, void* stream);

/* Batched pseudoinverse solve of `batch` Hermitian systems of one size K by
 * eigendecomposition (cuSOLVER XsyevBatched): a_z = V diag(1/w_i if
 * |w_i| > rcond*max|w| else 0) V^H b_z, the truncation of solve_eq_sym
 * (vtem/utils/linalg.py:591-631) applied per system, as vtb_herm_solve
 * mode 0 does for one.  M holds the column-major matrices contiguously
 * (stride K*K complex) and is overwritten; b and a are contiguous (stride K);
 * kept[z] (optional) receives the number of kept eigenvalues and infos[z]
 * the eigensolver's status per system.  The grouped counterpart of the
 * per-window solve of vtem/vtdm.py:645-648 for systems whose pseudoinverse
 * truncates. */
int vtb_herm_pinv_batched_workspace(int K, int batch, int64_t* bytes);
int vtb_herm_pinv_batched(double* M, const double* b, double* a, int K, int batch, double rcond, void* work,
                          int64_t work_bytes, int32_t* kept, int32_t* infos, void* stream);

/* a += d (n complex). */
int vtb_zadd(double* a, const double* d, int n, void* stream);

/* ------------------------------------------------------------ real form
 *
 * A real video has Hermitian-symmetric coefficients (a[K-1-j] = conj a[j]
 * for the index j = s*(2Mt+1) + m + Mt), and on those vectors the unitary map
 * x_j = sqrt2 Re a_j, x_{h+1+j} = sqrt2 Im a_j (j < h = (K-1)/2), x_h = a_h
 * turns the Hermitian M a = b into the real symmetric Mr x = br with the same
 * eigenvalues: the solve of vtem/vtdm.py:645-648 (solve_eq_sym,
 * vtem/utils/linalg.py:591-631) in a quarter of the complex arithmetic.
 * Mr is written row-major and full (it is symmetric, so also column-major). */

/* Mr (K x K, K = Ks*Kt, float32 or float64 when out_f64) from the tensor-core
 * Gram output C (2*npairs x Kt(Kt+1), leading dimension ldc) of
 * vtb_coeff_lhs_sym/vtb_coeff_wn_sym/vtb_tc_gemm_bf16x3_bn. */
int vtb_coeff_real_scatter(const float* C, int64_t ldc, int Ks, int Kt, void* Mr, int64_t ldr, int out_f64,
                           void* stream);
/* Mr from the complex column-major M of vtb_coeff_gram. */
int vtb_coeff_realify(const double* M, int64_t ldm, int K, void* Mr, int64_t ldr, int out_f64, void* stream);
/* br from b, and a (= or += when accumulate) from x; `batch` vectors at stride K. */
int vtb_coeff_realify_vec(const double* b, int K, int batch, double* br, void* stream);
int vtb_coeff_unrealify_vec(const double* x, int K, int batch, double* a, int accumulate, void* stream);

/* Workspace bytes of the real symmetric solver: mode 0 eigen-pseudoinverse
 * (float64), 1 float64 Cholesky, 2 float32 Cholesky. */
int vtb_sym_workspace(int K, int mode, int64_t* bytes);
/* Cholesky factorisation in place (lower factor), mode 1 (double M) or 2
 * (float M).  Does not synchronise: flag (device int32) receives 0, 1 when
 * the factorisation failed, or 2 when the spread of the squared pivots (a
 * lower bound of cond(M)) times rcond reaches 1; pivots (device, 2 doubles,
 * may be NULL) the (min, max) squared pivot. */
int vtb_sym_factor(void* M, int64_t ld, int K, int mode, double rcond, void* work, int64_t work_bytes,
                   int32_t* flag, double* pivots, void* stream);
/* x = M^-1 x (float64 x) with a factor of vtb_sym_factor of the same mode. */
int vtb_sym_potrs(const void* Mfac, int64_t ld, double* x, int K, int mode, void* work, int64_t work_bytes,
                  void* stream);
/* One system, multi-CTA: x = L^-T L^-1 x (x float64, float32 arithmetic) with
 * a float32 factor of vtb_sym_factor (mode 2).  CTA j owns rows 64j..64j+63;
 * the forward and backward solves hand rows on through per-CTA flags
 * (bounded waits; err (device int32) is set to 3 if one runs out, and the
 * result is then invalid).  Cooperative launch of ceil(K/64) CTAs, which must
 * all be resident (else VTB_BAD_ARG).  Replaces cusolverDnSpotrs in the
 * mixed decoder's solve; the reference's counterpart is the solve of
 * linalg.py:591-631.  Dinv: vtb_sym_dinv (vtb_sym_dinv_floats(K) floats);
 * work: vtb_sym_potrs_flags_bytes(K) bytes. */
int vtb_sym_dinv(const float* L, int64_t ld, int K, float* Dinv, void* stream);
int64_t vtb_sym_potrs_flags_bytes(int K);
int vtb_sym_potrs_flags(const float* L, int64_t ld, const float* Dinv, int K, double* x, void* work,
                        int64_t work_bytes, int32_t* err, void* stream);
/* Float32 Cholesky of ONE symmetric positive definite K x K matrix A
 * (column-major, leading dimension ld; the factor L overwrites the lower
 * triangle), written for the B200: one cooperative launch, 64 x 64 tiles as
 * a data-flow graph (one CTA walks the diagonal: the panel [A_kk; I] ->
 * [L_kk; L_kk^-T], the sub-diagonal tile as a product with L_kk^-T, SYRK of
 * the next diagonal tile; every other CTA accumulates the trailing updates
 * of its tiles in registers and runs their TRSMs as products with the
 * published L_JJ^-T), release/acquire flags between CTAs with bounded
 * waits.  Dinv (vtb_chol_dinv_floats(K) floats, 16-byte aligned) receives
 * the inverses of the 64 x 64 diagonal tiles of L, each ROW-major (tile k
 * at k*4096); work: vtb_chol_work_bytes(K) bytes, 256-byte aligned.
 * status (device int32, zeroed by the caller) receives 1 (a pivot <= 0), 2
 * (max/min squared pivot times rcond >= 1: the pseudoinverse might truncate)
 * or 3 (a wait between CTAs ran out; the factor is then invalid); pivots
 * (device, 2 doubles, may be NULL) the (min, max) squared pivot.  Replaces
 * cuSOLVER's spotrf in the mixed decoder's solve of G c = q, whose
 * reference counterpart is solve_eq_sym (vtem/utils/linalg.py:591-631) as
 * called per window at vtem/vtdm.py:645-648. */
int64_t vtb_chol_dinv_floats(int K);
int64_t vtb_chol_work_bytes(int K);
int vtb_chol_factor(float* A, int64_t ld, int K, float* Dinv, void* work, int64_t work_bytes, int32_t* status,
                    double* pivots, double rcond, void* stream);
/* x = L^-T L^-1 x (x float64 in and out, float32 arithmetic) with the factor
 * and Dinv of vtb_chol_factor, in one thread-block cluster (16 CTAs where the
 * GPU can schedule them, else 8): block-row substitution over the 64-row
 * tiles, each solved block handed to every CTA through distributed shared
 * memory, one cluster barrier per block.  K <= 10240.  Replaces spotrs in the
 * same solve (linalg.py:591-631).  vtb_chol_solve_cluster() gives the
 * cluster size in use (0 before the first call). */
int vtb_chol_solve(const float* L, int64_t ld, const float* Dinv, int K, double* x, void* stream);
int vtb_chol_solve_cluster(void);
/* vtb_chol_factor that also forms X = L^-1 in the same launch: the CTAs
 * that are not busy with the factorisation compute X_ii = L_ii^-1 and
 * X_ij = -X_ii sum_{k=j}^{i-1} L_ik X_kj as soon as their operands are
 * published.  Linv (vtb_chol_inverse_floats(K) floats, 16-byte aligned)
 * receives the tiles (i, j), i >= j, of X, each 64 x 64 row-major, tile
 * (i, j) at offset (i(i+1)/2 + j) * 4096.  Dinv is filled as by
 * vtb_chol_factor. */
int64_t vtb_chol_inverse_floats(int K);
int vtb_chol_factor_inverse(float* A, int64_t ld, int K, float* Dinv, float* Linv, void* work, int64_t work_bytes,
                            int32_t* status, double* pivots, double rcond, void* stream);
/* x = L^-T L^-1 x (x float64 in and out, float32 arithmetic) with the packed
 * inverse of vtb_chol_factor_inverse: two triangular matrix-vector products
 * (y = X b, then x = X^T y), one block per tile, every tile read once; the
 * last block of each block row (column), found by an atomic ticket, sums
 * the partials in a fixed order.  work: vtb_chol_solve_inverse_bytes(K)
 * bytes, zeroed before the first call and left zeroed by every call.
 * Replaces spotrs in the solve of linalg.py:591-631. */
int64_t vtb_chol_solve_inverse_bytes(int K);
int vtb_chol_solve_inverse(const float* Linv, int K, double* x, void* work, int64_t work_bytes, void* stream);
/* Pseudoinverse solve x = V diag(1/w if |w| > rcond*max|w| else 0) V^T b of
 * a float64 symmetric M (destroyed), the rule of solve_eq_sym
 * (vtem/utils/linalg.py:591-631, sq_Kernel :791-833).  kept (device) the
 * number of kept eigenvalues; eig_range (HOST, may be NULL) the smallest
 * and largest eigenvalue.  Synchronises the stream. */
int vtb_sym_pinv(double* M, int64_t ld, const double* b, double* x, int K, double rcond, void* work,
                 int64_t work_bytes, int32_t* kept, double* eig_range, void* stream);
/* Batched float32 Cholesky of `batch` real systems of one size K (a group of
 * clips with equal K; Mptrs: device array of device pointers, factorised in
 * place): cusolverDnSpotrfBatched, the pivot test of vtb_sym_factor per
 * system (flags[z]; pivots, may be NULL, 2 doubles per system) and the
 * inverses of each factor's 32 x 32 diagonal blocks for vtb_sym_potrs_batched
 * (Dinv + z * vtb_sym_dinv_floats(K)).  infos (device) receives cuSOLVER's
 * per-system status.  The grouped counterpart of the per-window solve of
 * vtem/vtdm.py:645-648.  Does not synchronise. */
int vtb_sym_factor_batched(float** Mptrs, int64_t ld, int K, int batch, double rcond, float* Dinv, int32_t* infos,
                           int32_t* flags, double* pivots, void* stream);
int64_t vtb_sym_dinv_floats(int K);

/* One system of vtb_sym_potrs_batched: x = L^-T L^-1 x (x float64, in place). */
typedef struct vtb_trsv_desc {
    const float* L;     /* float32 factor, column-major, leading dimension ld */
    const float* Dinv;  /* inverses of its 32 x 32 diagonal blocks */
    double* x;
    int64_t ld;
    int32_t K;
    int32_t pad;
} vtb_trsv_desc;
/* Solves of `batch` systems (descs: device array), one CTA each; Kmax >= every K. */
int vtb_sym_potrs_batched(const void* descs, int batch, int Kmax, void* stream);

/* Batched eigen-pseudoinverse of `batch` real symmetric systems of one size K
 * (cuSOLVER XsyevBatched): per system the rule of vtb_sym_pinv.  M holds the
 * matrices contiguously (stride K*K, destroyed), b and x at stride K; kept
 * (device, may be NULL) and infos (device) per system.  The grouped
 * counterpart of solve_eq_sym (vtem/utils/linalg.py:591-631) for windows whose
 * pseudoinverse truncates.  Synchronises the stream. */
int vtb_sym_pinv_batched_workspace(int K, int batch, int64_t* bytes);
int vtb_sym_pinv_batched(double* M, const double* b, double* x, int K, int batch, double rcond, void* work,
                         int64_t work_bytes, int32_t* kept, int32_t* infos, void* stream);

/* RNN decoder on the real coefficient system: from x = 0, steps+1 updates
 * x <- x + dt_alpha (br - Mr x), float64.  The same iterates as rnn3 on the
 * spike Gram (vtem/neural_network.py:15-128) mapped by a = Phi^H c
 * (Phi^H c_{i+1} = Phi^H c_i + dt_alpha (Phi^H q - Phi^H Phi Phi^H c_i)), on
 * K x K instead of n x n.  One cooperative launch runs every update (rows of
 * Mr cached in shared memory); x_tmp (K doubles) and bar (16 bytes) are
 * scratch.  After the stream reaches the call's end, the int32 at byte
 * offset 8 of bar is nonzero if a grid-barrier wait exceeded its limit (the
 * result is then invalid). */
int vtb_rnn_coeff(const double* Mr, int64_t ld, const double* br, double* x, double* x_tmp, int K, double dt_alpha,
                  int steps, void* bar, void* stream);

/* out (device) = ||dx|| / ||x||: the relative size of a refinement correction. */
int vtb_norm_ratio(const double* dx, const double* x, int n, double* out, void* stream);
/* y += x (n doubles). */
int vtb_daxpy1(double* y, const double* x, int n, void* stream);

/* vtb_coeff_synthesize without the caller's A_work buffer, for callers that
 * cannot allocate device memory (a plugin confined to another runtime's
 * memory pool, code that may only use a framework's allocator, replay inside
 * an already-built execution graph).  No counterpart in the reference: its
 * reconstruction always allocates through PyCUDA.  The scratch is a fixed
 * 4 MiB device array inside the library, present on every GPU that loads it
 * until the process exits; frames are processed in chunks that fit, so Nt is
 * unbounded but Ks * 16 bytes must be at most 4 MiB (Ks <= 262144), else
 * VTB_BAD_ARG.  The call allocates nothing (no cudaMalloc/cudaFree, no
 * allocating library).  Every call looks up the array's device address on
 * the current device (so a device reset leaves no stale address); the first
 * call on a device also loads the library's module there, so make that first
 * call before any stream capture.  All calls share the one array: calls that overlap on the
 * GPU (other streams, other threads) race, so serialise them.  Output equals
 * vtb_coeff_synthesize's. */
int vtb_coeff_synthesize_noalloc(const double* a, const int32_t* smap, int Ks, int Mx, int My, int Mt, double W,
                                 double t0, double dt, int Nt, int Px, int Py, int Px1, int Py1, void* u,
                                 int out_f32, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* VTEM_B200_H */
