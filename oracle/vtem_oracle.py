"""CPU oracle of the vtem video time-encode/decode path (test infrastructure).

This module is the checker, not the product: only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` import
it.  The product path (``vtem_b200``) never calls into it.

Every function is a float64 NumPy (or C, for the IAF scan) restatement of one
piece of the reference, cited by file:line inside the reference project.  The
third-party arithmetic the reference delegates to closed libraries is restated
from its published definition:

* cuBLAS DGEMM/ZGEMM (scikits.cuda) -> ``numpy.matmul`` (same sums, other order)
* cuFFT Z2Z forward/inverse        -> ``numpy.fft.fft2`` / ``ifft2 * size``
  (cuFFT's inverse is unnormalised; NumPy's divides by the size)
* CULA ``culaDeviceDgesvd``          -> ``numpy.linalg.eigh`` of the symmetric
  PSD Gram (its singular values are |eigenvalues|), cross-checked against
  ``numpy.linalg.svd`` in the tests.

The restatement is pinned against the reference's own inline CUDA kernels
compiled for the host (``oracle/_ref``, built by ``oracle/build_ref.py``) and
against the golden fixtures under ``tests/golden/`` that were generated from
them.
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))

# ---------------------------------------------------------------------------
# Receptive fields  (vtem/vrf.py)
# ---------------------------------------------------------------------------


def pixel_coords(Px, Py, Sx, Sy, x_start, y_start):
    """Pixel-grid coordinates of the RF kernels (vrf.py:1254-1257, :1169-1172).

    ``x = pix_x * (Sx/Px) + x_start`` and ``y = -(pix_y * (Sy/Py) + y_start)``
    (the y axis points up while rows go down).
    """
    px = np.arange(Px, dtype=np.float64)
    py = np.arange(Py, dtype=np.float64)
    x = px * (Sx / Px) + x_start
    y = -(py * (Sy / Py) + y_start)
    return x[None, :], y[:, None]


def gabor_rf(h_alpha, h_l, h_x0, h_y0, h_ab, Px, Py, Sx, Sy, x_start, y_start,
             KAPPA, gain=None):
    """Gabor RF bank on a pixel grid -> (N, Py, Px).

    gabor_Kernel, vrf.py:1197-1291; the device holds ``1/h_alpha``
    (vrf.py:258).  ``gain`` is the per-RF amplitude extension (default 1, the
    reference behaviour).
    """
    x, y = pixel_coords(Px, Py, Sx, Sy, x_start, y_start)
    N = len(h_alpha)
    out = np.empty((N, Py, Px))
    for n in range(N):
        alpha = 1.0 / h_alpha[n]
        xs = alpha * (x - h_x0[n])
        ys = alpha * (y - h_y0[n])
        st, ct = math.sin(h_l[n]), math.cos(h_l[n])
        X = xs * ct + ys * st
        Y = -xs * st + ys * ct
        first = alpha * (1 / math.sqrt(2 * math.pi)) * np.exp(-((4 * X * X) + (Y * Y)) / 8)
        car = np.cos(KAPPA * X) if int(h_ab[n]) == 0 else np.sin(KAPPA * X)
        out[n] = first * car
        if gain is not None:
            out[n] *= gain[n]
    return out


def cs_rf(h_alpha, h_x0, h_y0, Px, Py, Sx, Sy, x_start, y_start, sigma_center,
          sigma_surround, gain=None):
    """Centre-surround (difference of Gaussians) RF bank -> (N, Py, Px).

    cs_Kernel, vrf.py:1120-1193 (surround weight 0.9 at :1180, the 2*pi
    divisor at :1187).
    """
    x, y = pixel_coords(Px, Py, Sx, Sy, x_start, y_start)
    sc2 = sigma_center ** 2
    ss2 = sigma_surround ** 2
    N = len(h_alpha)
    out = np.empty((N, Py, Px))
    for n in range(N):
        alpha = 1.0 / h_alpha[n]
        xs = alpha * (x - h_x0[n])
        ys = alpha * (y - h_y0[n])
        XY = -(xs * xs + ys * ys)
        gb = alpha * (np.exp(XY / (2 * sc2)) / sc2 - 0.9 * np.exp(XY / (2 * ss2)) / ss2)
        out[n] = gb / (2 * math.pi)
        if gain is not None:
            out[n] *= gain[n]
    return out


def rf_filter(video, rf, dx, dy):
    """RF projection ``L[f, n] = dx*dy * sum_p V[f, p] RF[n, p]`` -> (F, N).

    cublasDgemm('t','n', F, N, P, dx*dy, video, RFs) then ``.T()``,
    vrf.py:264-292 (Gabor) and vrf.py:845-872 (centre-surround).
    """
    F = video.shape[0]
    V = video.reshape(F, -1)
    R = rf.reshape(rf.shape[0], -1)
    return (dx * dy) * (V @ R.T)


# ---------------------------------------------------------------------------
# IAF encoder  (vtem/ensemble_encode.py, vtem/vtem.py)
# ---------------------------------------------------------------------------

_iaf_lib = None


def _iaf():
    """Load (building on first use) the C restatement of the IAF scan."""
    global _iaf_lib
    if _iaf_lib is None:
        so = os.path.join(_HERE, "libiaf_oracle.so")
        src = os.path.join(_HERE, "iaf_oracle.c")
        if not os.path.exists(so) or os.path.getmtime(so) < os.path.getmtime(src):
            build_c_oracle()
        lib = ctypes.CDLL(so)
        f = lib.iaf_oracle_encode_block
        P = ctypes.c_void_p
        i64 = ctypes.c_longlong
        f.argtypes = [P, i64, i64, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                      P, P, P, P, P, P, i64, i64, P, P, P, P, ctypes.c_int, P,
                      ctypes.c_double, P]
        f.restype = ctypes.c_int
        _iaf_lib = lib
    return _iaf_lib


def build_c_oracle():
    """Compile oracle/iaf_oracle.c without FP contraction (checker build)."""
    so = os.path.join(_HERE, "libiaf_oracle.so")
    src = os.path.join(_HERE, "iaf_oracle.c")
    subprocess.check_call(["gcc", "-O2", "-ffp-contract=off", "-fno-fast-math",
                           "-fPIC", "-shared", "-o", so, src, "-lm"])
    return so


def _ptr(a):
    return None if a is None else a.ctypes.data


@dataclass
class IAFBlockResult:
    spikes: list            # per neuron, block-relative spike times (float64)
    steps: list             # per neuron, step index i of each spike (int32)
    spike_count: np.ndarray  # int32 (N,)
    overflow: int
    near_threshold: int


def iaf_encode_block(inputs, dt, kappa, bias, delta, v0, time_count,
                     max_spike, randn=None, sigma=None, delta_value=None,
                     near_eps=1e-12):
    """One ``IAF_encode.encode`` / ``IAF_encode_rt.encode`` call.

    ``inputs`` is (size, N) time-major, as the reference kernel reads it
    (ensemble_encode.py:490-491).  ``v0``, ``time_count`` (and
    ``delta_value`` for random thresholds) are updated in place, as the
    kernel writes them back (:543-545, :665-668).  ``randn`` (slots, N) holds
    the N(0,1) draws the reference pre-fills the spike buffer with
    (ensemble_encode.py:304-306).
    """
    lib = _iaf()
    inputs = np.ascontiguousarray(inputs, dtype=np.float64)
    size, N = inputs.shape
    st = np.zeros((N, max_spike), np.float64)
    ss = np.zeros((N, max_spike), np.int32)
    cnt = np.zeros(N, np.int32)
    near = np.zeros(1, np.int64)
    f64 = lambda a: np.ascontiguousarray(a, dtype=np.float64)
    kappa, bias, delta = f64(kappa), f64(bias), f64(delta)
    assert v0.dtype == np.float64 and time_count.dtype == np.float64
    if randn is not None:
        randn = f64(randn)
        sigma = f64(sigma)
        assert delta_value.dtype == np.float64
        rs, rn = randn.shape[1], 1
    else:
        rs, rn = 0, 0
    ov = lib.iaf_oracle_encode_block(
        _ptr(inputs), N, 1, N, size, float(dt), _ptr(kappa), _ptr(bias), _ptr(delta),
        _ptr(v0), _ptr(time_count), _ptr(randn), rs, rn, _ptr(sigma),
        _ptr(delta_value), _ptr(st), _ptr(ss), max_spike, _ptr(cnt),
        float(near_eps), _ptr(near))
    spikes = [st[n, :min(cnt[n], max_spike)].copy() for n in range(N)]
    steps = [ss[n, :min(cnt[n], max_spike)].copy() for n in range(N)]
    return IAFBlockResult(spikes, steps, cnt, int(ov), int(near[0]))


def block_schedule(F, block_frames=101, start_frame=0):
    """Frame blocks of VTEM_IAF: ``range(start, end, B-1)`` windows of B
    frames sharing one boundary frame (vtem.py:167-180)."""
    return [(s, min(s + block_frames, F)) for s in range(start_frame, F, block_frames - 1)]


def default_block_frames(F):
    """ONE_TIME_FRAMES on a GPU with ample memory: ``min(101, F+1)``
    (vtem.py:167-169)."""
    return min(101, F + 1)


@dataclass
class EncodeResult:
    """Per-block spike store contents, as vtem_storage keeps them
    (spike_store.py:147-156): block-relative times and per-block counts."""
    block_counts: list      # list over blocks of int32 (N,)
    block_spikes: list      # list over blocks of float64 flat neuron-major
    block_steps: list       # list over blocks of int32 flat (global step index)
    refresh_interval: float
    block_frames: int
    overflow: int
    near_threshold: int
    v0: np.ndarray
    delta_value: np.ndarray | None = None


def vtem_encode(L, dt, kappa, bias, delta, v0, time_count=None, block_frames=None,
                max_spike_per_block=None, randn_blocks=None, sigma=None,
                delta_value=None, avg_rate=0.1):
    """VTEM_IAF's block loop over a filtered signal ``L`` (F, N)
    (vtem.py:165-200): blocks of B frames stepping by B-1, ``reset_timer``
    after every block (vtem.py:197, ensemble_encode.py:170-172), v0 carried
    over.  The spike buffer per block holds ``ceil(B/avg_rate)`` slots
    (ensemble_encode.py:146).
    """
    F, N = L.shape
    B = default_block_frames(F) if block_frames is None else block_frames
    v0 = np.array(v0, dtype=np.float64, copy=True)
    tc = np.zeros(N) if time_count is None else np.array(time_count, np.float64, copy=True)
    dv = None if delta_value is None else np.array(delta_value, np.float64, copy=True)
    res = EncodeResult([], [], [], (B - 1) * dt, B, 0, 0, v0, dv)
    for bi, (s, e) in enumerate(block_schedule(F, B)):
        size = e - s
        cap = int(np.ceil(size / avg_rate)) if max_spike_per_block is None else max_spike_per_block
        rb = None if randn_blocks is None else randn_blocks[bi]
        r = iaf_encode_block(L[s:e], dt, kappa, bias, delta, v0, tc, cap,
                             randn=rb, sigma=sigma, delta_value=dv)
        res.block_counts.append(r.spike_count.copy())
        res.block_spikes.append(np.concatenate(r.spikes) if N else np.zeros(0))
        res.block_steps.append((np.concatenate(r.steps) + s).astype(np.int32) if N else np.zeros(0, np.int32))
        res.overflow += r.overflow
        res.near_threshold += r.near_threshold
        tc[:] = 0.0
    return res


# ---------------------------------------------------------------------------
# Dirichlet space  (vtem/vrf.py, vtem/vtdm.py)
# ---------------------------------------------------------------------------


def ellipse_mask(Mx, My):
    """Spatial basis kept by the reference: ``mx^2 My^2 + my^2 Mx^2 <=
    Mx^2 My^2`` (vrf.py:1331, :1419).  Indexed [my + My, mx + Mx]."""
    my = np.arange(-My, My + 1)[:, None]
    mx = np.arange(-Mx, Mx + 1)[None, :]
    return (mx * mx * My * My + my * my * Mx * Mx) <= Mx * Mx * My * My


def _fftind(mx, my, LPx, LPy):
    """Quadrant index map of fft2Ds_kernel / Ds2fft_kernel (vrf.py:1307-1319,
    :598-610): (my mod LPy) * LPx + (mx mod LPx)."""
    if mx < 0 and my < 0:
        return LPx * (LPy + my) + (LPx + mx)
    if my < 0 and mx >= 0:
        return mx + (LPx * (LPy + my))
    if mx >= 0 and my >= 0:
        return my * LPx + mx
    return my * LPx + (LPx + mx)


def compute_Ds(rf_fine, Mx, My, dxdy):
    """Dirichlet coefficients ``Ds`` (N, 2My+1, 2Mx+1) complex128.

    compute_Ds + fft2Ds_kernel, vrf.py:333-377 and :1293-1350: forward FFT of
    each RF on its (LPy, LPx) grid, ``Ds[n, My-my, mx+Mx] =
    dxdy*(-1)^(mx+my)*FFT[my mod LPy, mx mod LPx]`` inside the ellipse, 0
    outside.
    """
    N, LPy, LPx = rf_fine.shape
    Fk = np.fft.fft2(rf_fine, axes=(1, 2)).reshape(N, -1)
    Ds = np.zeros((N, 2 * My + 1, 2 * Mx + 1), np.complex128)
    for my in range(-My, My + 1):
        for mx in range(-Mx, Mx + 1):
            if mx * mx * My * My + my * my * Mx * Mx <= Mx * Mx * My * My:
                sgn = dxdy if (mx + my) % 2 == 0 else -dxdy
                Ds[:, My - my, mx + Mx] = sgn * Fk[:, _fftind(mx, my, LPx, LPy)]
    return Ds


def compute_dirich_space_fft(Ds, Mx, My, Px, Py, Px1, Py1):
    """Spatial reconstruction functions on the decode grid -> (N, Py, Px).

    compute_dirich_space_fft, Ds2fft_kernel, filter2rec_kernel
    (vrf.py:437-499, :585-632, :635-677): place ``(-1)^(mx+my) Ds[My-my,
    mx+Mx]`` at the (Py1, Px1) FFT index, unnormalised inverse FFT, real part
    of the centred (Py, Px) crop.
    """
    N = Ds.shape[0]
    grid = np.zeros((N, Py1 * Px1), np.complex128)
    for my in range(-My, My + 1):
        for mx in range(-Mx, Mx + 1):
            sgn = 1.0 if (mx + my) % 2 == 0 else -1.0
            grid[:, _fftind(mx, my, Px1, Py1)] = sgn * Ds[:, My - my, mx + Mx]
    f = np.fft.ifft2(grid.reshape(N, Py1, Px1), axes=(1, 2)) * (Px1 * Py1)
    xd = (Px1 - Px) // 2
    yd = (Py1 - Py) // 2
    return np.ascontiguousarray(f[:, yd:yd + Py, xd:xd + Px].real)


def compute_dirich_space_direct(Ds, Mx, My, Px, Py, Sx, Sy, Wx, Wy, x_start=None, y_start=None):
    """Direct-sum form of the spatial functions (psi_dirich_space_Kernel,
    vrf.py:1353-1443): ``Re sum_{ellipse} Ds[my+My, mx+Mx] e^{j(mx Wx/Mx x +
    my Wy/My y)}``."""
    if x_start is None:
        x_start = -Sx / 2
    if y_start is None:
        y_start = -Sy / 2
    x, y = pixel_coords(Px, Py, Sx, Sy, x_start, y_start)
    msk = ellipse_mask(Mx, My)
    out = np.zeros((Ds.shape[0], Py, Px))
    for my in range(-My, My + 1):
        for mx in range(-Mx, Mx + 1):
            if msk[my + My, mx + Mx]:
                e = np.exp(1j * (mx * (Wx / Mx) * x + my * (Wy / My) * y))
                out += (Ds[:, my + My, mx + Mx][:, None, None] * e[None]).real
    return out


def compute_Dsw(Ds, h_norm):
    """RF cross-weights ``Dsw[a, b] = Re sum_s conj(Ds[a,s]) Ds[b,s] *
    norm[a] norm[b]`` (compute_Dsw + put_norm, vrf.py:502-559; the same
    matrix as compute_Gb's two DGEMMs, dirichlet.py:87-126)."""
    D = Ds.reshape(Ds.shape[0], -1)
    W = (np.conj(D) @ D.T).real
    W = W.T.copy()  # d_weight[i][j] holds column-major C[j][i]
    return W * (h_norm[:, None] * h_norm[None, :])


# ---------------------------------------------------------------------------
# Spike store  (vtem/utils/spike_store.py)
# ---------------------------------------------------------------------------


def select_neurons(h_x0, h_y0, domain):
    """Neurons whose centre lies in the domain (+-0.01), spike_store.py:243-277.
    Returns (choose, shiftx, shifty)."""
    Sx = domain[1] - domain[0]
    Sy = domain[3] - domain[2]
    shiftx = domain[0] + Sx / 2
    shifty = domain[2] + Sy / 2
    allind = np.arange(len(h_x0))
    choose = allind[(h_x0 > domain[0] - 0.01) & (h_x0 < domain[1] + 0.01) &
                    (h_y0 > domain[2] - 0.01) & (h_y0 < domain[3] + 0.01)]
    return choose, shiftx, shifty


def read_select_spikes(block_counts, block_spikes, refresh_interval, choose, time_frame):
    """Consecutive spike pairs inside a time window, with one spike either
    side (read_select_spikes, spike_store.py:279-351).

    Returns ``tk1, tk2`` (relative to ``time_frame[0]``) and ``neuron_ind``
    (index into ``choose``).
    """
    total_intervals = len(block_counts)
    start_interval = int(np.floor(time_frame[0] / refresh_interval))
    end_interval = int(np.floor(time_frame[1] / refresh_interval))
    intervals = np.arange(max(0, start_interval - 1), min(total_intervals, end_interval + 2))
    D = len(choose)
    spike_tmp = [np.zeros(0) for _ in range(D)]
    for i in intervals:
        sc = block_counts[i]
        cum = np.concatenate((np.zeros(1, np.int64), np.cumsum(sc)))
        spikes = block_spikes[i] + i * refresh_interval - time_frame[0]
        for j in range(D):
            spike_tmp[j] = np.concatenate((spike_tmp[j], spikes[cum[choose[j]]:cum[choose[j] + 1]]))
    tk = []
    count = np.zeros(D, np.int32)
    for i in range(D):
        a = np.nonzero((spike_tmp[i] > 0) & (spike_tmp[i] < time_frame[1] - time_frame[0]))[0]
        if a.size > 0:
            tk.append(spike_tmp[i][max(0, a[0] - 1):min(a[-1] + 2, spike_tmp[i].size)])
        else:
            tk.append(np.zeros(0))
        count[i] = max(0, tk[i].size - 1)
    cc = np.concatenate((np.zeros(1, np.int64), np.cumsum(count)))
    tk1 = np.empty(cc[-1], np.float64)
    tk2 = np.empty(cc[-1], np.float64)
    ind = np.empty(cc[-1], np.int32)
    for i in range(D):
        tk1[cc[i]:cc[i + 1]] = tk[i][:-1]
        tk2[cc[i]:cc[i + 1]] = tk[i][1:]
        ind[cc[i]:cc[i + 1]] = i
    return tk1, tk2, ind


def h_norm_from_sigma(kappa, sigma):
    """``norm = 1/(kappa sigma)`` normalised to its max, 1 where sigma == 0
    (vtdm.py:408-413, :634-638)."""
    h = np.ones(len(kappa), np.float64)
    nz = np.nonzero(sigma != 0)
    h[nz] = 1.0 / (kappa[nz] * sigma[nz])
    return h / h.max()


# ---------------------------------------------------------------------------
# Decoder  (vtem/dirichlet.py, vtem/utils/linalg.py, vtem/neural_network.py)
# ---------------------------------------------------------------------------


def compute_q(tk1, tk2, ind, kappa, delta, bias, norm):
    """``q_k = (kappa delta - b (t_k2 - t_k1)) norm`` (compute_q_Kernel,
    dirichlet.py:204-222)."""
    return (kappa[ind] * delta[ind] - bias[ind] * (tk2 - tk1)) * norm[ind]


def G_time(tk1, tk2, tl1, tl2, M, WM):
    """Temporal Gram factor (G_dirichlet_time, dirichlet.py:274-285)."""
    s = np.zeros(np.broadcast(tk1, tl1).shape)
    for m in range(1, M + 1):
        s += (np.cos(m * WM * (tk2 - tl2)) - np.cos(m * WM * (tk2 - tl1))
              - np.cos(m * WM * (tk1 - tl2)) + np.cos(m * WM * (tk1 - tl1))) / (m * m)
    return s * 2 / (WM * WM) + (tk2 - tk1) * (tl2 - tl1)


def compute_G(tk1, tk2, ind, Dsw, Wt, Mt, lamb=0.0, rows=None):
    """Analytic Gram ``G[k,l] = Gt(k,l) Dsw[n_k, n_l] (+ lamb I)``
    (compute_G_Kernel + diag_add_Kernel, dirichlet.py:62-85, :272-350).
    ``rows`` restricts to a subset of rows (for large n)."""
    r = np.arange(len(tk1)) if rows is None else np.asarray(rows)
    G = G_time(tk1[r][:, None], tk2[r][:, None], tk1[None, :], tk2[None, :], Mt, Wt / Mt)
    G *= Dsw[ind[r][:, None], ind[None, :]]
    if lamb != 0:
        for i, k in enumerate(r):
            G[i, k] += lamb
    return G


def _threads(threads):
    return max(1, int(threads or os.cpu_count() or 1))


def compute_G_threaded(tk1, tk2, ind, Dsw, Wt, Mt, lamb=0.0, threads=None, rows_per_task=256):
    """:func:`compute_G` with its rows split over host threads: the same
    entries, each computed by the same expression (NumPy releases the GIL
    inside the element-wise ufuncs)."""
    from concurrent.futures import ThreadPoolExecutor
    n = len(tk1)
    G = np.empty((n, n))
    starts = list(range(0, n, rows_per_task))

    def task(r0):
        r = np.arange(r0, min(n, r0 + rows_per_task))
        G[r0:r0 + len(r)] = compute_G(tk1, tk2, ind, Dsw, Wt, Mt, lamb, rows=r)

    with ThreadPoolExecutor(_threads(threads)) as ex:
        list(ex.map(task, starts))
    return G


def reconstruct_factored_threaded(dirich, tk1, tk2, c, t, ind, norm, Mt, WM, threads=None, frames_per_task=64):
    """:func:`reconstruct_factored` with the frames split over host threads."""
    from concurrent.futures import ThreadPoolExecutor
    t = np.asarray(t, np.float64)
    out = np.empty((len(t),) + tuple(dirich.shape[1:]))
    starts = list(range(0, len(t), frames_per_task))

    def task(f0):
        f1 = min(len(t), f0 + frames_per_task)
        out[f0:f1] = reconstruct_factored(dirich, tk1, tk2, c, t[f0:f1], ind, norm, Mt, WM)

    with ThreadPoolExecutor(_threads(threads)) as ex:
        list(ex.map(task, starts))
    return out


def solve_eq_sym(G, q, rcond=1e-8):
    """Pseudoinverse solve of ``G c = q`` for symmetric PSD G with singular
    values below ``rcond * s_0`` dropped (solve_eq_sym + sq_Kernel,
    linalg.py:591-631, :791-833).  Returns (c, number of kept values)."""
    lam, U = np.linalg.eigh(G)
    s = np.abs(lam)
    s0 = s.max()
    qq = U.T @ q
    keep = s > s0 * rcond
    qq = np.where(keep, qq / np.where(keep, s, 1.0), 0.0)
    return U @ qq, int(keep.sum())


def rnn3(G, q, dt=1e-6, alpha=5000, steps=4000):
    """Gradient-flow decoder ``c += dt alpha (q - G c)``, steps+1 updates
    from c = 0 (rnn3 + rnn3_update, neural_network.py:15-128)."""
    c = np.zeros_like(q)
    da = float(dt) * float(alpha)
    for _ in range(steps + 1):
        y = q - G @ c
        c = c + da * y
    return c


def reconstruct_direct(dirich, tk1, tk2, c, t, ind, norm, Mt, WM, pix=None):
    """Reference reconstruction formula (reconstruct_Kernel,
    dirichlet.py:354-420), evaluated literally: O(T * P * n * Mt).
    ``pix`` restricts to flat pixel indices."""
    N = dirich.shape[0]
    D = dirich.reshape(N, -1)
    if pix is not None:
        D = D[:, pix]
    out = np.zeros((len(t), D.shape[1]))
    dt_k = tk2 - tk1
    for it, tt in enumerate(t):
        phi = np.zeros(len(tk1))
        for m in range(1, Mt + 1):
            phi += (np.sin(m * WM * (tt - tk1)) - np.sin(m * WM * (tt - tk2))) / m
        w = c * (phi * 2 / WM + dt_k) * norm[ind]
        out[it] = w @ D[ind]
    return out


def reconstruct_factored(dirich, tk1, tk2, c, t, ind, norm, Mt, WM):
    """The same sum regrouped per neuron: ``u = H @ dirich`` with
    ``H[t, n] = sum_{k in n} c_k norm_n psi_k(t)``.  Equal to
    :func:`reconstruct_direct` up to rounding."""
    N = dirich.shape[0]
    H = np.zeros((len(t), N))
    dt_k = tk2 - tk1
    for it, tt in enumerate(t):
        phi = np.zeros(len(tk1))
        for m in range(1, Mt + 1):
            phi += (np.sin(m * WM * (tt - tk1)) - np.sin(m * WM * (tt - tk2))) / m
        w = c * (phi * 2 / WM + dt_k) * norm[ind]
        H[it] = np.bincount(ind, weights=w, minlength=N)
    return (H @ dirich.reshape(N, -1)).reshape(len(t), *dirich.shape[1:])


def default_Mt(Wt):
    """``Mt = round(Wt / pi)`` when not given (vtdm.py:568-571)."""
    return int(round(Wt * 2 / 2 / np.pi))


def rf_period_grid(Mx, My, Wx, Wy, dx, dy):
    """RF grid over one spatial period (vtdm.py:385-388)."""
    rfSx = (2 * np.pi) * (Mx / Wx)
    rfSy = (2 * np.pi) * (My / Wy)
    rfPx = int(np.ceil(rfSx / dx / 16) * 16)
    rfPy = int(np.ceil(rfSy / dy / 16) * 16)
    return rfSx, rfSy, rfPx, rfPy


# ---------------------------------------------------------------------------
# Synthetic stimulus (seeded Dirichlet-bandlimited video)
# ---------------------------------------------------------------------------


def bandlimited_coeffs(Mx, My, Mt, seed):
    """iid complex N(0,1) coefficients inside the spatial ellipse, made
    Hermitian (a[-m] = conj a[m]) so the video is real.  Shape
    (2My+1, 2Mx+1, 2Mt+1), indexed [my+My, mx+Mx, mt+Mt]."""
    rng = np.random.default_rng(seed)
    shp = (2 * My + 1, 2 * Mx + 1, 2 * Mt + 1)
    a = rng.standard_normal(shp) + 1j * rng.standard_normal(shp)
    a = 0.5 * (a + np.conj(a[::-1, ::-1, ::-1]))
    a *= ellipse_mask(Mx, My)[:, :, None]
    return a


def bandlimited_video(a, Mx, My, Mt, Wx, Wy, Wt, Px, Py, Sx, Sy, F, dt):
    """Evaluate ``u(x, y, t) = sum a e^{j(mx Wx/Mx x + my Wy/My y + mt
    Wt/Mt t)}`` on the reference's pixel grid (centred, y up) at ``t = f dt``.
    Returns the (F, Py, Px) real video, unscaled."""
    x, y = pixel_coords(Px, Py, Sx, Sy, -Sx / 2, -Sy / 2)
    ex = np.exp(1j * np.outer(np.arange(-Mx, Mx + 1), x.ravel()) * (Wx / Mx))   # (2Mx+1, Px)
    ey = np.exp(1j * np.outer(np.arange(-My, My + 1), y.ravel()) * (Wy / My))   # (2My+1, Py)
    et = np.exp(1j * np.outer(np.arange(F) * dt, np.arange(-Mt, Mt + 1)) * (Wt / Mt))  # (F, 2Mt+1)
    A = np.einsum("ymt,ft->fym", a, et)           # (F, 2My+1, 2Mx+1)
    B = np.einsum("fym,mx->fyx", A, ex)           # (F, 2My+1, Px)
    u = np.einsum("fyx,yp->fpx", B, ey)           # (F, Py, Px)
    return u.real.copy()


# ---------------------------------------------------------------------------
# End-to-end drivers (the call order of VTEM_IAF / VTDM_prep / VTDM)
# ---------------------------------------------------------------------------


def prep_decoder_gabor(h_alpha, h_l, h_x0, h_y0, h_ab, KAPPA, gain, Mx, My, Wx, Wy, dx, dy, decPx, decPy,
                       h_norm, cs=None):
    """VTDM_prep (vtdm.py:311-447) for a Gabor bank (plus, optionally, a
    centre-surround bank ``cs = (h_alpha, h_x0, h_y0, sigma_c, sigma_s,
    gain)`` appended after it): RFs at 4x on one spatial period, Ds, phi on
    the decode grid, Dsw.  Returns (Ds, dirich, Dsw)."""
    rfSx, rfSy, rfPx, rfPy = rf_period_grid(Mx, My, Wx, Wy, dx, dy)
    LPx, LPy = rfPx * 4, rfPy * 4
    fdx, fdy = (rfSx / rfPx) / 4, (rfSy / rfPy) / 4
    Sxall, Syall = LPx * fdx, LPy * fdy
    rfs = []
    if h_alpha is not None and len(h_alpha):
        rfs.append(gabor_rf(h_alpha, h_l, h_x0, h_y0, h_ab, LPx, LPy, Sxall, Syall, -Sxall / 2, -Syall / 2,
                            KAPPA, gain))
    if cs is not None:
        ca, cx, cy, sc, ssr, cg = cs
        rfs.append(cs_rf(ca, cx, cy, LPx, LPy, Sxall, Syall, -Sxall / 2, -Syall / 2, sc, ssr, cg))
    rf = np.concatenate(rfs, 0)
    Ds = compute_Ds(rf, Mx, My, fdx * fdy)
    decSx, decSy = decPx * dx, decPy * dy
    Px1 = int(np.round(Sxall / (decSx / decPx)))
    Py1 = int(np.round(Syall / (decSy / decPy)))
    dirich = compute_dirich_space_fft(Ds, Mx, My, decPx, decPy, Px1, Py1)
    Dsw = compute_Dsw(Ds, h_norm)
    return Ds, dirich, Dsw


def decode_window(tk1, tk2, ind, kappa, delta, bias, norm, Dsw, dirich, Wt, Mt, T, dt, rcond=1e-8,
                  lamb=0.0, rnn=None, threads=1):
    """One VTDM window (vtdm.py:631-652): q, G, pinv (or rnn3 with
    ``rnn = (dt, alpha, steps)``), reconstruction at t = arange(0, T, dt).
    ``threads`` > 1 splits the Gram's rows and the frames over host threads."""
    q = compute_q(tk1, tk2, ind, kappa, delta, bias, norm)
    if threads == 1:
        G = compute_G(tk1, tk2, ind, Dsw, Wt, Mt, lamb)
    else:
        G = compute_G_threaded(tk1, tk2, ind, Dsw, Wt, Mt, lamb, threads=threads)
    if rnn is None:
        c, kept = solve_eq_sym(G, q, rcond)
    else:
        c = rnn3(G, q, *rnn)
        kept = None
    t = np.arange(0, T, dt)
    if threads == 1:
        u = reconstruct_factored(dirich, tk1, tk2, c, t, ind, norm, Mt, Wt / Mt)
    else:
        u = reconstruct_factored_threaded(dirich, tk1, tk2, c, t, ind, norm, Mt, Wt / Mt, threads=threads)
    return u, c, q, G, kept


# ---------------------------------------------------------------------------
# Stitching  (vtem/vtdm.py)
# ---------------------------------------------------------------------------


def temporal_stitch(decode, start_time, end_time, dt, stitching, stitch_interval):
    """VTDM's window loop (vtdm.py:573-699): ``decode(start, end)`` returns
    the (frames, Py, Px) reconstruction of one window; consecutive windows
    overlap by 20 % of the interval (at least 4 samples when the interval has
    8 or more) and are cross-faded with a Hann ramp.  Returns the video and
    the list of (start, end) windows decoded."""
    end = float(end_time)
    if stitching:
        if stitch_interval is None:
            stitch_interval = 20 * dt
        stitch_interval = min(stitch_interval, end_time)
        end = round(float(min(start_time + stitch_interval, end_time)) / dt) * dt
        overlap = 0.2 * stitch_interval
    else:
        stitch_interval = float(end_time)
        overlap = 0
    start = float(start_time)
    total_l = round((end_time - start_time) / dt)
    overlap_l = round(overlap / dt)
    if overlap_l < 3:
        if round(stitch_interval / dt) >= 8:
            overlap_l, overlap = 4, 4 * dt
        else:
            overlap_l, overlap = 0, 0
    interval_l = round(stitch_interval / dt)
    lw = np.hanning(2 * overlap_l)[:overlap_l].reshape(-1, 1, 1)
    u = None
    prev = None
    windows = []
    i = 0
    while True:
        windows.append((start, end))
        ur = np.asarray(decode(start, end))
        if u is None:
            u = np.empty((total_l,) + ur.shape[1:], np.float64)
        if overlap_l:
            if i == 0:
                if end_time - end < dt:
                    u = ur
                    break
                u[:interval_l - overlap_l] = ur[:-overlap_l]
                prev = ur[-overlap_l:]
            else:
                a = i * (interval_l - overlap_l)
                b = (i + 1) * (interval_l - overlap_l)
                u[a:a + overlap_l] = ur[:overlap_l] * lw + prev * (1.0 - lw)
                if end_time - end < dt:
                    u[a + overlap_l:] = ur[-u.shape[0] + a + overlap_l:]
                    break
                u[a + overlap_l:b] = ur[overlap_l:interval_l - overlap_l]
                prev = ur[-overlap_l:]
        else:
            u[i * interval_l:i * interval_l + ur.shape[0]] = ur
            if end_time - end < dt:
                break
        start = start + round(stitch_interval / dt) * dt - round(overlap / dt) * dt
        end = min(start + round(stitch_interval / dt) * dt, float(end_time))
        if float(end_time) - end < overlap:
            end = end_time
        i += 1
    return u, windows


def _edge_window(n, lo_edge, hi_edge, over):
    """1-D tile weight of decode_video (vtdm.py:246-262): a rising Hann half
    over the first ``over`` pixels unless the tile starts on the domain edge,
    a falling one over the last ``over`` unless it ends there."""
    left = 0 if lo_edge else over
    right = 0 if hi_edge else over
    return np.concatenate((np.hanning(2 * left)[:left], np.ones(n - left - right),
                           1 - np.hanning(2 * right)[:right]))


def spatial_tile_walk(domain, decPx, decPy, spatial_interval, dx, dy):
    """decode_video's tile walk (vtdm.py:214-302), row by row from the top
    (pixel row 0 = the domain's largest y), each row from the right edge.
    Returns [(tile domain, row0, row1, col0, col1, weight)]."""
    ivx = min(spatial_interval[0], decPx)
    ivy = min(spatial_interval[1], decPy)
    ovx, ovy = round(.2 * ivx), round(.2 * ivy)
    tiles = []
    start_y = max(domain[3] - ivy * dy, domain[2])
    end_y = domain[3]
    sy, ey = 0, ivy
    while True:
        start_x = max(domain[1] - ivx * dx, domain[0])
        end_x = domain[1]
        sx, ex = decPx - ivx, decPx
        while True:
            wy = _edge_window(ey - sy, sy == 0, ey == decPy, ovy)
            wx = _edge_window(ex - sx, sx == 0, ex == decPx, ovx)
            tiles.append(([start_x, end_x, start_y, end_y], sy, ey, sx, ex, np.outer(wy, wx)))
            if start_x == domain[0]:
                break
            start_x = max(start_x - ivx * dx + ovx * dx, domain[0])
            end_x = end_x - ivx * dx + ovx * dx
            sx = max(sx - ivx + ovx, 0)
            ex = ex - ivx + ovx
        if start_y == domain[2]:
            break
        start_y = max(start_y - ivy * dy + ovy * dy, domain[2])
        end_y = end_y - ivy * dy + ovy * dy
        sy = ey - ovy
        ey = min(sy + ivy, decPy)
    return tiles


def spatial_stitch(decode_tile, domain, decPx, decPy, spatial_interval, dx, dy):
    """decode_video with spatial stitching (vtdm.py:181-309): the sum over
    tiles of ``decode_tile(tile domain)`` (frames, rows, cols) times the
    tile's weight."""
    u = None
    for dom, sy, ey, sx, ex, w in spatial_tile_walk(domain, decPx, decPy, spatial_interval, dx, dy):
        ut = np.asarray(decode_tile(dom))
        if u is None:
            u = np.zeros((ut.shape[0], decPy, decPx), np.float64)
        u[:, sy:ey, sx:ex] += ut * w
    return u
