// Synthesis as a rank-(2Mt+1) product of temporal harmonics and per-pixel
// weights.
//
// The reconstruction of one window is (vtem/dirichlet.py:165-189 rewritten
// in the coefficient space, as csrc/coeff.cu derives it)
//     u(t, p) = Re sum_{s, m} a[s][m] phi_s(p) e^{j m W t},
// phi_s the spatial Dirichlet function of ellipse entry s on the decode grid.
// Gathering the spatial sum first, B_m(p) = sum_s a[s][m] phi_s(p), and
// pairing m with -m,
//     u(t, p) = Re B_0(p) + sum_{m=1}^{Mt} [cos(mWt) Re P_m(p) - sin(mWt) Im P_m(p)],
//     P_m = B_m + conj(B_{-m})
// (exact for any coefficients; P_m = 2 B_m for the Hermitian-symmetric ones
// of a real video).  So the video is U = C H^T with C[t] = [1, cos Wt,
// sin Wt, ..., cos MtWt, sin MtWt] (Nt x Kt) and H (P x Kt) the per-pixel
// weights: 2Mt+1 = 17 float64 FMAs per voxel at the GPU configuration,
// against the 8 bytes the voxel costs in HBM.
//
//   basis_kernel: H, a block per m and 64 x 4 pixel tile: the row sums of
//     the coefficient grid over the tile's columns, then 2(2My+1) complex
//     MACs per pixel (ex/ey of the period grid in shared memory, with the
//     (-1)^(mx+my) signs and crop offsets of the decode grid).
//   harmonics_kernel: U.  A block owns 256 * kHPix consecutive pixels and a
//     range of frames; each thread keeps its kHPix pixels' Kt weights in
//     registers, the block's frames' harmonics C (by powers of e^{jWt}) sit
//     in shared memory and are read as broadcasts, and each warp writes 32
//     consecutive voxels per store (streaming stores, the video exceeds L2).
#include <algorithm>

#include "common.cuh"

namespace vtb {

constexpr int kHMaxKt = 33;       // Mt <= 16
constexpr int kHPix = 2;          // pixels per thread
constexpr int kHThreads = 256;
constexpr int kHFrames = 64;      // frames per pass of a block

__device__ __forceinline__ double2 c_mul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// H[p * ldh + k]: k = 0 -> Re B_0, k = 2m-1 -> Re P_m, k = 2m -> -Im P_m.
// The spatial sum is separable over the rows of the coefficient grid:
//   P_m(px, py) = sum_rr [ey[rr][py] Gp[rr][px] + conj(ey[rr][py]) Gn[rr][px]],
//   Gp[rr][px] = sum_{s in row rr} a[s][m] ex[c(s)][px],
//   Gn[rr][px] = sum_{s in row rr} conj(a[s][-m]) conj(ex[c(s)][px]),
// so a block (one m, a tile of kBX x kBY pixels) first forms the row sums of
// its columns, then two complex MACs per pixel and row.
constexpr int kBX = 64;           // pixel columns per block
constexpr int kBY = 4;            // pixel rows per block

__global__ void __launch_bounds__(kBX * kBY) basis_kernel(const double2* __restrict__ a,
                                                          const int32_t* __restrict__ smap, int Ks, int Mx, int My,
                                                          int Mt, int Px, int Py, int Px1, int Py1,
                                                          double* __restrict__ H, int ldh) {
    extern __shared__ double2 bs[];
    const int Kx = 2 * Mx + 1, Ky = 2 * My + 1, Kt = 2 * Mt + 1;
    const int m = blockIdx.y;                       // 0..Mt
    const int tilesx = (Px + kBX - 1) / kBX;
    const int x0 = (blockIdx.x % tilesx) * kBX, y0 = (blockIdx.x / tilesx) * kBY;
    double2* ex = bs;                               // Kx x kBX
    double2* gp = ex + Kx * kBX;                    // Ky x kBX
    double2* gn = gp + Ky * kBX;                    // Ky x kBX
    double2* ey = gn + Ky * kBX;                    // Ky x kBY
    double2* am = ey + Ky * kBY;                    // Ks: a[s][m]
    double2* an = am + Ks;                          // Ks: conj a[s][-m]
    int* srow = reinterpret_cast<int*>(an + Ks);    // Ks: row of entry s
    int* scol = srow + Ks;                          // Ks: column of entry s
    int* rlo = scol + Ks;                           // Ky: first / last entry of each row
    int* rhi = rlo + Ky;
    const int tid = threadIdx.x, nt = blockDim.x;
    const int xd = (Px1 - Px) / 2, yd = (Py1 - Py) / 2;
    for (int r = tid; r < Ky; r += nt) {
        rlo[r] = Ks;
        rhi[r] = -1;
    }
    __syncthreads();
    // threads 0..kBX-1: one pixel column each, ex[Mx +- m] = (-1)^m (e^{2 pi i (px+xd)/Px1})^(+-m)
    // by powers of one sincospi; threads kBX..kBX+kBY-1: the same for the rows (ey); threads
    // from 128: the coefficients of this m and the grid row / column of every entry
    if (tid < kBX) {
        const int px = x0 + tid;
        double sn, co;
        sincospi(2.0 * (double)(((px + xd) % Px1 + Px1) % Px1) / Px1, &sn, &co);
        const double2 base = make_double2(co, sn);
        double2 pw = make_double2(1.0, 0.0);
        for (int mm = 0; mm <= Mx; ++mm) {
            const double sg = (mm & 1) ? -1.0 : 1.0;
            ex[(Mx + mm) * kBX + tid] = make_double2(sg * pw.x, sg * pw.y);
            ex[(Mx - mm) * kBX + tid] = make_double2(sg * pw.x, -sg * pw.y);
            pw = c_mul(pw, base);
        }
    } else if (tid < kBX + kBY) {
        const int y = tid - kBX, py = y0 + y;
        double sn, co;
        sincospi(2.0 * (double)(((py + yd) % Py1 + Py1) % Py1) / Py1, &sn, &co);
        const double2 base = make_double2(co, sn);
        double2 pw = make_double2(1.0, 0.0);
        for (int mm = 0; mm <= My; ++mm) {       // storage row rr holds my = My - rr
            const double sg = (mm & 1) ? -1.0 : 1.0;
            ey[(My - mm) * kBY + y] = make_double2(sg * pw.x, sg * pw.y);
            ey[(My + mm) * kBY + y] = make_double2(sg * pw.x, -sg * pw.y);
            pw = c_mul(pw, base);
        }
    } else if (tid >= 128) {
        for (int s = tid - 128; s < Ks; s += nt - 128) {
            am[s] = a[(int64_t)s * Kt + Mt + m];
            const double2 v = a[(int64_t)s * Kt + Mt - m];
            an[s] = make_double2(v.x, -v.y);
            const int g = __ldg(smap + s), rr = g / Kx;
            const bool ok = g >= 0 && rr < Ky;          // an index outside the grid contributes nothing
            srow[s] = ok ? rr : -1;
            scol[s] = ok ? g - rr * Kx : 0;
            if (ok) {
                atomicMin(rlo + rr, s);
                atomicMax(rhi + rr, s);
            }
        }
    }
    __syncthreads();
    // row sums of this block's columns
    for (int e = tid; e < Ky * kBX; e += nt) {
        const int rr = e / kBX, x = e % kBX;
        double2 sp = make_double2(0.0, 0.0), sq = make_double2(0.0, 0.0);
        for (int s = rlo[rr]; s <= rhi[rr]; ++s) {
            if (srow[s] != rr) continue;
            const double2 e1 = ex[scol[s] * kBX + x];
            const double2 t1 = c_mul(am[s], e1);
            sp.x += t1.x;
            sp.y += t1.y;
            const double2 t2 = c_mul(an[s], make_double2(e1.x, -e1.y));
            sq.x += t2.x;
            sq.y += t2.y;
        }
        gp[e] = sp;
        gn[e] = sq;
    }
    __syncthreads();
    const int x = tid % kBX, y = tid / kBX;
    const int px = x0 + x, py = y0 + y;
    if (px >= Px || py >= Py) return;
    double2 acc = make_double2(0.0, 0.0);
    for (int rr = 0; rr < Ky; ++rr) {
        const double2 e2 = ey[rr * kBY + y];
        const double2 t1 = c_mul(e2, gp[rr * kBX + x]);
        acc.x += t1.x;
        acc.y += t1.y;
        if (m > 0) {
            const double2 t2 = c_mul(make_double2(e2.x, -e2.y), gn[rr * kBX + x]);
            acc.x += t2.x;
            acc.y += t2.y;
        }
    }
    double* h = H + ((int64_t)py * Px + px) * ldh;
    if (m == 0) {
        h[0] = acc.x;
    } else {
        h[2 * m - 1] = acc.x;
        h[2 * m] = -acc.y;
    }
}

template <typename OutT>
__device__ __forceinline__ void stream_store(OutT* p, double v) {
    __stcs(p, (OutT)v);
}

// U[f][p] = sum_k C[f][k] H[p][k], f = fb..fe of this block, pixels
// pbase + t + 256 j (j < kHPix)
template <typename OutT, int KT>
__global__ void __launch_bounds__(kHThreads) harmonics_kernel(const double* __restrict__ H, int ldh, int P,
                                                              double W, double t0, double dt, int Nt, int fchunks,
                                                              OutT* __restrict__ u) {
    __shared__ __align__(16) double Cs[kHFrames + 1][KT + 1];   // one spare row for an odd frame count
    constexpr int MT = (KT - 1) / 2;
    const int tid = threadIdx.x;
    const int ptile = blockIdx.x / fchunks, fc = blockIdx.x % fchunks;
    const int fb = (int)((int64_t)fc * Nt / fchunks), fe = (int)((int64_t)(fc + 1) * Nt / fchunks);
    const int pbase = ptile * kHThreads * kHPix;
    double h[kHPix][KT];
#pragma unroll
    for (int j = 0; j < kHPix; ++j) {
        const int p = pbase + tid + kHThreads * j;
#pragma unroll
        for (int k = 0; k < KT; ++k) h[j][k] = p < P ? __ldg(H + (int64_t)p * ldh + k) : 0.0;
    }
    for (int f0 = fb; f0 < fe; f0 += kHFrames) {
        const int nf = min(kHFrames, fe - f0);
        __syncthreads();
        if (tid < nf) {
            double sn, co;
            sincos(W * (t0 + (f0 + tid) * dt), &sn, &co);
            const double2 base = make_double2(co, sn);
            double2 pw = make_double2(1.0, 0.0);
            Cs[tid][0] = 1.0;
#pragma unroll
            for (int m = 1; m <= MT; ++m) {
                pw = c_mul(pw, base);
                Cs[tid][2 * m - 1] = pw.x;
                Cs[tid][2 * m] = pw.y;
            }
        }
        __syncthreads();
        // two frames at a time: 2 x kHPix independent FMA chains per thread
        for (int q = 0; q < nf; q += 2) {
            const bool two = q + 1 < nf;
            double acc0[kHPix], acc1[kHPix];
#pragma unroll
            for (int j = 0; j < kHPix; ++j) acc0[j] = acc1[j] = 0.0;
#pragma unroll
            for (int k = 0; k < KT; ++k) {
                const double c0 = Cs[q][k], c1 = Cs[q + 1][k];
#pragma unroll
                for (int j = 0; j < kHPix; ++j) {
                    acc0[j] = fma(c0, h[j][k], acc0[j]);
                    acc1[j] = fma(c1, h[j][k], acc1[j]);
                }
            }
            OutT* uf = u + (int64_t)(f0 + q) * P;
#pragma unroll
            for (int j = 0; j < kHPix; ++j) {
                const int p = pbase + tid + kHThreads * j;
                if (p < P) {
                    stream_store(uf + p, acc0[j]);
                    if (two) stream_store(uf + P + p, acc1[j]);
                }
            }
        }
    }
}

template <typename OutT, int KT>
static void launch_harm(const double* H, int ldh, int P, double W, double t0, double dt, int Nt, OutT* u,
                        cudaStream_t s) {
    const int ptiles = ceil_div(P, kHThreads * kHPix);
    // about four blocks per SM in all, at least one frame block per pass
    int fchunks = std::max(1, std::min(ceil_div(Nt, 8), ceil_div(4 * kNumSMs, ptiles)));
    harmonics_kernel<OutT, KT><<<ptiles * fchunks, kHThreads, 0, s>>>(H, ldh, P, W, t0, dt, Nt, fchunks, u);
}

template <typename OutT>
static int dispatch_harm(int Kt, const double* H, int ldh, int P, double W, double t0, double dt, int Nt, OutT* u,
                         cudaStream_t s) {
    switch (Kt) {
        case 3: launch_harm<OutT, 3>(H, ldh, P, W, t0, dt, Nt, u, s); break;
        case 5: launch_harm<OutT, 5>(H, ldh, P, W, t0, dt, Nt, u, s); break;
        case 7: launch_harm<OutT, 7>(H, ldh, P, W, t0, dt, Nt, u, s); break;
        case 9: launch_harm<OutT, 9>(H, ldh, P, W, t0, dt, Nt, u, s); break;
        case 11: launch_harm<OutT, 11>(H, ldh, P, W, t0, dt, Nt, u, s); break;
        case 13: launch_harm<OutT, 13>(H, ldh, P, W, t0, dt, Nt, u, s); break;
        case 15: launch_harm<OutT, 15>(H, ldh, P, W, t0, dt, Nt, u, s); break;
        case 17: launch_harm<OutT, 17>(H, ldh, P, W, t0, dt, Nt, u, s); break;
        case 19: launch_harm<OutT, 19>(H, ldh, P, W, t0, dt, Nt, u, s); break;
        case 21: launch_harm<OutT, 21>(H, ldh, P, W, t0, dt, Nt, u, s); break;
        default: return VTB_BAD_ARG;
    }
    return launch_status();
}

}  // namespace vtb

using namespace vtb;

// Per-pixel weights H (P x ldh doubles, P = Px*Py pixels in row-major frame
// order, ldh >= 2Mt+1) of the coefficients a[s][m] (Ks x (2Mt+1) complex,
// the decoder's layout; smap: storage index of each ellipse entry s in the
// (2My+1) x (2Mx+1) grid): column 0 = Re B_0, 2m-1 = Re P_m, 2m = -Im P_m.
// Replaces the spatial half of reconstruct_Kernel (vtem/dirichlet.py:354-420)
// on the coefficient space: B_m(p) = sum_s a[s][m] phi_s(p), phi_s the
// decode-grid Dirichlet functions of compute_dirich_space_fft
// (vtem/vrf.py:437-499, period Px1 x Py1 cropped to Px x Py).
VTB_API int vtb_coeff_basis(const double* a, const int32_t* smap, int Ks, int Mx, int My, int Mt, int Px, int Py,
                            int Px1, int Py1, double* H, int ldh, void* stream) {
    VTB_CHECK_ARG(Ks > 0 && Mx >= 0 && My >= 0 && Mt >= 0 && Px > 0 && Py > 0 && Px1 >= Px && Py1 >= Py);
    VTB_CHECK_ARG(a && smap && H && ldh >= 2 * Mt + 1 && 2 * Mt + 1 <= kHMaxKt);
    VTB_CHECK_ARG((int64_t)Mx * Px1 < (1LL << 30) && (int64_t)My * Py1 < (1LL << 30));
    const int Kx = 2 * Mx + 1, Ky = 2 * My + 1;
    const size_t sm = (size_t)(Kx * kBX + 2 * Ky * kBX + Ky * kBY + 2 * Ks) * sizeof(double2) +
                      (size_t)(2 * Ks + 2 * Ky) * sizeof(int);
    VTB_CHECK_ARG(sm <= 200 * 1024);
    if (sm > 48 * 1024)
        VTB_CUDA_TRY(cudaFuncSetAttribute(basis_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    dim3 grid(ceil_div(Px, kBX) * ceil_div(Py, kBY), Mt + 1);
    basis_kernel<<<grid, kBX * kBY, sm, as_stream(stream)>>>(reinterpret_cast<const double2*>(a), smap, Ks, Mx, My, Mt,
                                                            Px, Py, Px1, Py1, H, ldh);
    return launch_status();
}

// Video u[f][p] (Nt frames of P pixels, float64 or float32 when out_f32) at
// t = t0 + f dt from the weights H of vtb_coeff_basis: u[f][p] = H[p][0] +
// sum_{m=1}^{Mt} (cos(mWt) H[p][2m-1] + sin(mWt) H[p][2m]).  2Mt+1 in
// {3, 5, ..., 21}.  Replaces the temporal half of reconstruct_Kernel
// (vtem/dirichlet.py:354-420) as the coefficient space writes it.
VTB_API int vtb_synth_harmonics(const double* H, int ldh, int P, int Mt, double W, double t0, double dt, int Nt,
                                void* u, int out_f32, void* stream) {
    VTB_CHECK_ARG(P > 0 && Mt >= 1 && Nt >= 0 && ldh >= 2 * Mt + 1);
    if (Nt == 0) return VTB_OK;
    VTB_CHECK_ARG(H && u);
    cudaStream_t s = as_stream(stream);
    if (out_f32) return dispatch_harm<float>(2 * Mt + 1, H, ldh, P, W, t0, dt, Nt, reinterpret_cast<float*>(u), s);
    return dispatch_harm<double>(2 * Mt + 1, H, ldh, P, W, t0, dt, Nt, reinterpret_cast<double*>(u), s);
}
