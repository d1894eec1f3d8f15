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
//   basis_kernel: H, a block per m and 64 x 4 pixel tile: the coefficients
//     of m and -m placed on the dense (2My+1) x (2Mx+1) grid (zero outside
//     the ellipse), the grid's row sums over the tile's columns, then
//     2(2My+1) complex MACs per pixel (ex/ey of the period grid in shared
//     memory, with the (-1)^(mx+my) signs and crop offsets of the decode
//     grid).
//   harmonics_kernel: U.  A block owns 256 consecutive pixels (one per
//     thread; 64 registers, four blocks per SM) and a range of frames; each
//     thread keeps its pixel's Kt weights in registers, rotated to the
//     block's centre frame, and takes the frames in pairs symmetric about
//     that centre (2Mt+1 FMAs per PAIR of voxels, see the kernel); the pair
//     harmonics (by powers of e^{j W dt (j + 1/2)}) sit in shared memory and
//     are read as broadcasts, and each warp writes 256 consecutive bytes per
//     store (streaming stores, the video exceeds L2).
#include <algorithm>

#include "common.cuh"

namespace vtb {

constexpr int kHMaxKt = 33;       // Mt <= 16
constexpr int kHThreads = 256;    // two adjacent pixels per thread

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
    double2* ap = ey + Ky * kBY;                    // Ky x Kx grid: a[s][m] at entry s's place, 0 elsewhere
    double2* an = ap + Ky * Kx;                     // Ky x Kx grid: conj a[s][-m]
    const int tid = threadIdx.x, nt = blockDim.x;
    const int xd = (Px1 - Px) / 2, yd = (Py1 - Py) / 2;
    for (int g = tid; g < Ky * Kx; g += nt) {
        ap[g] = make_double2(0.0, 0.0);
        an[g] = make_double2(0.0, 0.0);
    }
    __syncthreads();
    // threads 0..kBX-1: one pixel column each, ex[Mx +- m] = (-1)^m (e^{2 pi i (px+xd)/Px1})^(+-m)
    // by powers of one sincospi; threads kBX..kBX+kBY-1: the same for the rows (ey); threads
    // from 128: the coefficients of this m, placed on the grid
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
            const int g = __ldg(smap + s);
            if (g < 0 || g >= Ky * Kx) continue;    // an index outside the grid contributes nothing
            ap[g] = a[(int64_t)s * Kt + Mt + m];
            const double2 v = a[(int64_t)s * Kt + Mt - m];
            an[g] = make_double2(v.x, -v.y);
        }
    }
    __syncthreads();
    // row sums of this block's columns over the grid's columns (zero outside the ellipse);
    // two partial sums per output halve the dependent chain
    for (int e = tid; e < Ky * kBX; e += nt) {
        const int rr = e / kBX, x = e % kBX;
        const double2* apr = ap + rr * Kx;
        const double2* anr = an + rr * Kx;
        double2 sp0 = make_double2(0.0, 0.0), sq0 = sp0, sp1 = sp0, sq1 = sp0;
        int c = 0;
        for (; c + 1 < Kx; c += 2) {
            const double2 e0 = ex[c * kBX + x], e1 = ex[(c + 1) * kBX + x];
            const double2 p0 = apr[c], p1 = apr[c + 1], n0 = anr[c], n1 = anr[c + 1];
            sp0.x = fma(p0.x, e0.x, fma(-p0.y, e0.y, sp0.x));
            sp0.y = fma(p0.x, e0.y, fma(p0.y, e0.x, sp0.y));
            sq0.x = fma(n0.x, e0.x, fma(n0.y, e0.y, sq0.x));      // n0 conj(e0)
            sq0.y = fma(n0.y, e0.x, fma(-n0.x, e0.y, sq0.y));
            sp1.x = fma(p1.x, e1.x, fma(-p1.y, e1.y, sp1.x));
            sp1.y = fma(p1.x, e1.y, fma(p1.y, e1.x, sp1.y));
            sq1.x = fma(n1.x, e1.x, fma(n1.y, e1.y, sq1.x));
            sq1.y = fma(n1.y, e1.x, fma(-n1.x, e1.y, sq1.y));
        }
        if (c < Kx) {
            const double2 e0 = ex[c * kBX + x], p0 = apr[c], n0 = anr[c];
            sp0.x = fma(p0.x, e0.x, fma(-p0.y, e0.y, sp0.x));
            sp0.y = fma(p0.x, e0.y, fma(p0.y, e0.x, sp0.y));
            sq0.x = fma(n0.x, e0.x, fma(n0.y, e0.y, sq0.x));
            sq0.y = fma(n0.y, e0.x, fma(-n0.x, e0.y, sq0.y));
        }
        gp[e] = make_double2(sp0.x + sp1.x, sp0.y + sp1.y);
        gn[e] = make_double2(sq0.x + sq1.x, sq0.y + sq1.y);
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

// two adjacent pixels of one frame with one 16-byte (float64) or 8-byte
// (float32) streaming store when the row allows it
template <typename OutT>
__device__ __forceinline__ void store_pair(OutT* row, int p, int P, bool vec, double v0, double v1) {
    if (vec) {
        if constexpr (sizeof(OutT) == 8) {
            __stcs(reinterpret_cast<double2*>(row + p), make_double2(v0, v1));
        } else {
            __stcs(reinterpret_cast<float2*>(row + p), make_float2((float)v0, (float)v1));
        }
    } else {
        if (p < P) stream_store(row + p, v0);
        if (p + 1 < P) stream_store(row + p + 1, v1);
    }
}

// U[f][p] = sum_k C[f][k] H[p][k] for the frames fb..fe-1 of this block and
// the pixels pbase + 2 t + {0, 1}.  The frames are taken in pairs placed
// symmetrically about the block's centre angle th_c = W (t0 + c dt): with
// A_m = a_m cos(m th_c) + b_m sin(m th_c), B_m = b_m cos(m th_c) - a_m sin(m th_c)
// (a_m = H[p][2m-1], b_m = H[p][2m], A_0 = H[p][0]), the two frames at th_c -+ phi are
//     u = E -+ O,  E = sum_{m=0}^{Mt} A_m cos(m phi),  O = sum_{m=1}^{Mt} B_m sin(m phi),
// so a pair of voxels costs 2Mt+1 FMAs and two adds instead of 2(2Mt+1) FMAs.
// The rotation to A, B is done once per pixel and block.
constexpr int kHPairs = 160;      // frame pairs per pass of a block (even)

#ifndef VTB_HARM_PIX
#define VTB_HARM_PIX 1            // pixels per thread (1, or 2 adjacent with vector stores)
#endif
#ifndef VTB_HARM_QP
#define VTB_HARM_QP 2             // frame pairs per inner iteration
#endif
constexpr int kHPix = VTB_HARM_PIX;
constexpr int kHQp = VTB_HARM_QP;
static_assert(kHPix == 1 || kHPix == 2, "one or two pixels per thread");
static_assert(kHPairs % kHQp == 0, "whole groups of pairs per pass");

template <typename OutT, int KT>
__global__ void __launch_bounds__(kHThreads) harmonics_kernel(const double* __restrict__ H, int ldh, int P,
                                                              double W, double t0, double dt, int Nt, int fchunks,
                                                              int vec, OutT* __restrict__ u) {
    constexpr int MT = (KT - 1) / 2;
    // (cos m phi_j, sin m phi_j), m = 1..MT; spare rows for a pass whose pair count is not a multiple of kHQp
    __shared__ __align__(16) double2 Cs[kHPairs + kHQp][MT];
    __shared__ __align__(16) double2 Rc[MT];                // (cos m th_c, sin m th_c)
    const int tid = threadIdx.x;
    const int ptile = blockIdx.x / fchunks, fc = blockIdx.x % fchunks;
    const int fb = (int)((int64_t)fc * Nt / fchunks), fe = (int)((int64_t)(fc + 1) * Nt / fchunks);
    const int nfr = fe - fb, half = nfr >> 1, odd = nfr & 1;
    const int npairs = half + odd;
    // pair j: frames lo = fb + half - 1 + odd - j and hi = fb + half + j, at th_c -+ (j + h) W dt
    const double h = odd ? 0.0 : 0.5;
    const double wdt = W * dt;
    auto fill_pairs = [&](int j0) {
        const int j = j0 + tid;
        if (tid < kHPairs && j < npairs) {
            double sn, co;
            sincos(wdt * ((double)j + h), &sn, &co);
            const double2 base = make_double2(co, sn);
            double2 pw = base;
#pragma unroll
            for (int m = 0; m < MT; ++m) {
                Cs[tid][m] = pw;
                pw = c_mul(pw, base);
            }
        }
    };
    if (nfr > 0) {
        fill_pairs(0);
        if (tid == kHThreads - 1) {
            double sn, co;
            sincos(W * (t0 + ((double)fb + 0.5 * (double)(nfr - 1)) * dt), &sn, &co);
            const double2 base = make_double2(co, sn);
            double2 pw = base;
#pragma unroll
            for (int m = 0; m < MT; ++m) {
                Rc[m] = pw;
                pw = c_mul(pw, base);
            }
        }
    }
    if (nfr <= 0) return;
    __syncthreads();
    const int p = ptile * kHThreads * kHPix + kHPix * tid;
    double A[kHPix][MT + 1], B[kHPix][MT];
#pragma unroll
    for (int i = 0; i < kHPix; ++i) {
        const bool in = p + i < P;
        const double* hp = H + (int64_t)(p + i) * ldh;
        A[i][0] = in ? __ldg(hp) : 0.0;
#pragma unroll
        for (int m = 1; m <= MT; ++m) {
            const double a = in ? __ldg(hp + 2 * m - 1) : 0.0, b = in ? __ldg(hp + 2 * m) : 0.0;
            const double2 r = Rc[m - 1];
            A[i][m] = fma(a, r.x, b * r.y);
            B[i][m - 1] = fma(b, r.x, -(a * r.y));
        }
    }
    const bool active = p < P;
    for (int j0 = 0; j0 < npairs; j0 += kHPairs) {
        const int np = min(kHPairs, npairs - j0);
        if (j0 > 0) {
            __syncthreads();
            fill_pairs(j0);
            __syncthreads();
        }
        if (active) {
            // kHQp pairs at a time: kHQp x kHPix x (E, O) independent FMA chains
            for (int q = 0; q < np; q += kHQp) {
                double E[kHQp][kHPix], O[kHQp][kHPix];
#pragma unroll
                for (int k = 0; k < kHQp; ++k) {
#pragma unroll
                    for (int i = 0; i < kHPix; ++i) {
                        E[k][i] = A[i][0];
                        O[k][i] = 0.0;
                    }
                }
#pragma unroll
                for (int m = 0; m < MT; ++m) {
#pragma unroll
                    for (int k = 0; k < kHQp; ++k) {
                        const double2 c = Cs[q + k][m];
#pragma unroll
                        for (int i = 0; i < kHPix; ++i) {
                            E[k][i] = fma(c.x, A[i][m + 1], E[k][i]);
                            O[k][i] = fma(c.y, B[i][m], O[k][i]);
                        }
                    }
                }
#pragma unroll
                for (int k = 0; k < kHQp; ++k) {
                    if (q + k >= np) break;
                    const int j = j0 + q + k;
                    const int lo = fb + half - 1 + odd - j, hi = fb + half + j;
                    OutT* rh = u + (int64_t)hi * P;
                    OutT* rl = u + (int64_t)lo * P;
                    if constexpr (kHPix == 2) {
                        store_pair(rh, p, P, vec, E[k][0] + O[k][0], E[k][1] + O[k][1]);
                        if (lo != hi) store_pair(rl, p, P, vec, E[k][0] - O[k][0], E[k][1] - O[k][1]);
                    } else {
                        stream_store(rh + p, E[k][0] + O[k][0]);
                        if (lo != hi) stream_store(rl + p, E[k][0] - O[k][0]);
                    }
                }
            }
        }
    }
}

// fchunks: frame ranges per pixel tile, about four blocks per SM in all and
// at least two frames per range
static int harm_fchunks(int P, int Nt) {
    const int ptiles = ceil_div(P, kHThreads * kHPix);
    return std::max(1, std::min(ceil_div(Nt, 8), ceil_div(4 * kNumSMs, ptiles)));
}

template <typename OutT, int KT>
static void launch_harm(const double* H, int ldh, int P, double W, double t0, double dt, int Nt, OutT* u,
                        cudaStream_t s) {
    const int ptiles = ceil_div(P, kHThreads * kHPix);
    const int fchunks = harm_fchunks(P, Nt);
    const int vec = (P % 2 == 0 && reinterpret_cast<uintptr_t>(u) % (2 * sizeof(OutT)) == 0) ? 1 : 0;
    harmonics_kernel<OutT, KT><<<ptiles * fchunks, kHThreads, 0, s>>>(H, ldh, P, W, t0, dt, Nt, fchunks, vec, u);
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
static int launch_basis(const double* a, const int32_t* smap, int Ks, int Mx, int My, int Mt, int Px, int Py,
                        int Px1, int Py1, double* H, int ldh, cudaStream_t stream) {
    VTB_CHECK_ARG(Ks > 0 && Mx >= 0 && My >= 0 && Mt >= 0 && Px > 0 && Py > 0 && Px1 >= Px && Py1 >= Py);
    VTB_CHECK_ARG(a && smap && H && ldh >= 2 * Mt + 1 && 2 * Mt + 1 <= kHMaxKt);
    VTB_CHECK_ARG((int64_t)Mx * Px1 < (1LL << 30) && (int64_t)My * Py1 < (1LL << 30));
    const int Kx = 2 * Mx + 1, Ky = 2 * My + 1;
    const size_t sm = (size_t)(Kx * kBX + 2 * Ky * kBX + Ky * kBY + 2 * Ky * Kx) * sizeof(double2);
    VTB_CHECK_ARG(sm <= 200 * 1024);
    if (sm > 48 * 1024)
        VTB_CUDA_TRY(cudaFuncSetAttribute(basis_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    dim3 grid(ceil_div(Px, kBX) * ceil_div(Py, kBY), Mt + 1);
    basis_kernel<<<grid, kBX * kBY, sm, stream>>>(reinterpret_cast<const double2*>(a), smap, Ks, Mx, My, Mt, Px, Py,
                                                  Px1, Py1, H, ldh);
    return launch_status();
}

VTB_API int vtb_coeff_basis(const double* a, const int32_t* smap, int Ks, int Mx, int My, int Mt, int Px, int Py,
                            int Px1, int Py1, double* H, int ldh, void* stream) {
    return launch_basis(a, smap, Ks, Mx, My, Mt, Px, Py, Px1, Py1, H, ldh, as_stream(stream));
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

// The whole rank-(2Mt+1) synthesis in one call: the weights H (P x ldh,
// caller-owned scratch) of vtb_coeff_basis, then the video u as
// vtb_synth_harmonics writes it, both kernels queued by this call so that no
// host round trip separates them.  Mt in 1..10.  Replaces reconstruct_Kernel (vtem/dirichlet.py:354-420)
// on the coefficient space.
VTB_API int vtb_coeff_synth_rank(const double* a, const int32_t* smap, int Ks, int Mx, int My, int Mt, int Px, int Py,
                                 int Px1, int Py1, double* H, int ldh, double W, double t0, double dt, int Nt, void* u,
                                 int out_f32, void* stream) {
    VTB_CHECK_ARG(Mt >= 1 && Nt >= 0 && (int64_t)Px * Py < (1LL << 31));
    if (Nt == 0) return VTB_OK;
    VTB_CHECK_ARG(u && 2 * Mt + 1 <= 21);
    cudaStream_t s = as_stream(stream);
    const int st = launch_basis(a, smap, Ks, Mx, My, Mt, Px, Py, Px1, Py1, H, ldh, s);
    if (st != VTB_OK) return st;
    const int P = Px * Py;
    if (out_f32) return dispatch_harm<float>(2 * Mt + 1, H, ldh, P, W, t0, dt, Nt, reinterpret_cast<float*>(u), s);
    return dispatch_harm<double>(2 * Mt + 1, H, ldh, P, W, t0, dt, Nt, reinterpret_cast<double*>(u), s);
}
