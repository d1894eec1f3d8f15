"""Runs the reference's own kernels on the host (``oracle/_ref``), glued
together the way the reference's Python drivers glue them (test
infrastructure: the checker of the restatement in ``vtem_oracle.py``).

The library calls the drivers make on the GPU are restated with NumPy: cuBLAS
GEMM/GEMV -> ``@``, cuFFT -> ``numpy.fft`` (inverse scaled by the size, as
cuFFT's inverse is unnormalised), CULA gesvd -> ``numpy.linalg.svd``.
Launch shapes are the reference's own.  Buffers the reference kernels write
past their logical end (the IAF kernel's unguarded write-back,
ensemble_encode.py:541-545; reconstruct's ``pix < ld`` guard,
dirichlet.py:411-414) are padded here so the host run stays in bounds.
"""
from __future__ import annotations

import ctypes
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libvtem_ref.so")

_lib = None
_manifest = None


def available() -> bool:
    return os.path.exists(LIB)


def _load():
    global _lib, _manifest
    if _lib is None:
        if not available():
            raise RuntimeError("oracle/_ref not built: run python oracle/build_ref.py")
        _lib = ctypes.CDLL(LIB)
        with open(os.path.join(HERE, "_ref", "manifest.json")) as f:
            _manifest = json.load(f)
    return _lib


def launch(sym, grid, block, *args, os_threads=0):
    """Launch reference kernel ``sym`` with a CUDA-style grid/block."""
    lib = _load()
    spec = _manifest[sym]["args"]
    assert len(spec) == len(args), (sym, len(spec), len(args))
    store = []
    for s, a in zip(spec, args):
        kind = s.split(":")[0]
        if kind == "p":
            store.append(ctypes.c_void_p(a.ctypes.data if isinstance(a, np.ndarray) else a))
        elif kind == "i":
            store.append(ctypes.c_int(int(a)))
        elif kind == "u":
            store.append(ctypes.c_uint(int(a)))
        elif kind == "d":
            store.append(ctypes.c_double(float(a)))
        elif kind == "f":
            store.append(ctypes.c_float(float(a)))
        else:
            raise TypeError(s)
    arr = (ctypes.c_void_p * len(store))(*[ctypes.addressof(x) for x in store])
    gx, gy = (grid + (1,))[:2] if isinstance(grid, tuple) else (grid, 1)
    bx, by = (block + (1,))[:2] if isinstance(block, tuple) else (block, 1)
    getattr(lib, "ref_launch_" + sym)(ctypes.c_uint(gx), ctypes.c_uint(gy), ctypes.c_uint(bx),
                                       ctypes.c_uint(by), arr, ctypes.c_int(os_threads))


def _pad(a, n, dtype):
    out = np.zeros(n, dtype)
    out[:len(a)] = a
    return out


# ----------------------------------------------------------------- encoder

def iaf_encode(inputs, dt, kappa, bias, delta, v0, time_count, avg_rate=0.1,
               randn=None, sigma=None, delta_value=None):
    """IAF_encode.encode / IAF_encode_rt.encode (ensemble_encode.py:106-168,
    :265-329) on host.  ``inputs`` (size, N).  ``v0``/``time_count`` (and
    ``delta_value``) are updated in place.  Returns (list of per-neuron
    spike times, counts)."""
    size, N = inputs.shape
    npb = 64
    grid = int(np.ceil(N / npb))
    Np = grid * npb
    max_spike = int(np.ceil(size / avg_rate))
    inp = np.ascontiguousarray(inputs, np.float64)
    if randn is None:
        spk = np.zeros((max_spike, N), np.float64)
    else:
        spk = np.ascontiguousarray(randn, np.float64).copy()
    pv0 = _pad(v0, Np, np.float64)
    ptc = _pad(time_count, Np, np.float64)
    cnt = np.zeros(Np, np.int32)
    kap = np.ascontiguousarray(kappa, np.float64)
    bia = np.ascontiguousarray(bias, np.float64)
    dlt = np.ascontiguousarray(delta, np.float64)
    if randn is None:
        launch("iaf_linear", grid, npb, inp, N, N, size, spk, N, pv0, kap, bia, dlt, ptc, cnt,
               max_spike, dt)
    else:
        pdv = _pad(delta_value, Np, np.float64)
        sig = np.ascontiguousarray(sigma, np.float64)
        launch("iaf_linear_rt", grid, npb, inp, N, N, size, spk, N, pv0, kap, bia, dlt, ptc, cnt,
               max_spike, dt, pdv, sig)
        delta_value[:] = pdv[:N]
    v0[:] = pv0[:N]
    time_count[:] = ptc[:N]
    cnt = cnt[:N].copy()
    if cnt.max(initial=0) >= max_spike:
        raise ValueError("number of spikes exceeded the limit of buffer")
    return [spk[:cnt[i], i].copy() for i in range(N)], cnt


# ----------------------------------------------------------------- RF / Dirichlet

def gabor(h_alpha, h_l, h_x0, h_y0, h_ab, Px, Py, Sx, Sy, x_start, y_start, KAPPA):
    """generate_visual_receptive_fields + gabor_Kernel (vrf.py:296-331)."""
    N = len(h_alpha)
    out = np.zeros((N, Py * Px), np.float64)
    tiles = ((Px - 1) // 16 + 1) * ((Py - 1) // 16 + 1)
    launch("gabor", (tiles, N), (16, 16), out, Py * Px, np.ascontiguousarray(1.0 / np.asarray(h_alpha)),
           np.ascontiguousarray(h_l, np.float64), np.ascontiguousarray(h_x0, np.float64),
           np.ascontiguousarray(h_y0, np.float64), np.ascontiguousarray(h_ab, np.int32),
           Px, Py, Sx, Sy, x_start, y_start, KAPPA)
    return out.reshape(N, Py, Px)


def cs(h_alpha, h_x0, h_y0, Px, Py, Sx, Sy, x_start, y_start, sigma_center, sigma_surround):
    """generate_visual_receptive_fields + cs_Kernel (vrf.py:876-913)."""
    N = len(h_alpha)
    out = np.zeros((N, Py * Px), np.float64)
    tiles = ((Px - 1) // 16 + 1) * ((Py - 1) // 16 + 1)
    launch("cs", (tiles, N), (16, 16), out, Py * Px, np.ascontiguousarray(1.0 / np.asarray(h_alpha)),
           np.ascontiguousarray(h_x0, np.float64), np.ascontiguousarray(h_y0, np.float64),
           Px, Py, Sx, Sy, x_start, y_start, sigma_center ** 2, sigma_surround ** 2)
    return out.reshape(N, Py, Px)


def compute_Ds(rf_fine, Mx, My, dxdy):
    """compute_Ds: cuFFT forward (numpy) + fft2Ds_kernel (vrf.py:333-377)."""
    N, LPy, LPx = rf_fine.shape
    fk = np.ascontiguousarray(np.fft.fft2(rf_fine, axes=(1, 2)).reshape(N, -1), np.complex128)
    Ks = (2 * Mx + 1) * (2 * My + 1)
    Ds = np.zeros((N, Ks), np.complex128)
    launch("fft2Ds", (2 * Mx + 1, 2 * My + 1), 256, Ds, fk, Mx, My, LPx, LPy, N, Ks, dxdy)
    return Ds.reshape(N, 2 * My + 1, 2 * Mx + 1)


def dirich_space_fft(Ds, Mx, My, Px, Py, Px1, Py1):
    """compute_dirich_space_fft: Ds2fft_kernel, cuFFT inverse (numpy, scaled
    by the size), filter2rec_kernel (vrf.py:437-499)."""
    N = Ds.shape[0]
    Ks = (2 * Mx + 1) * (2 * My + 1)
    D = np.ascontiguousarray(Ds.reshape(N, Ks), np.complex128)
    filt = np.zeros((N, Px1 * Py1), np.complex128)
    launch("Ds2fft", (2 * Mx + 1, 2 * My + 1), 256, D, Ks, filt, Px1 * Py1, Mx, My, Px1, Py1, N)
    filt = np.ascontiguousarray(np.fft.ifft2(filt.reshape(N, Py1, Px1), axes=(1, 2)).reshape(N, -1)
                                * (Px1 * Py1))
    out = np.zeros((N, Py * Px), np.float64)
    tiles = ((Px - 1) // 16 + 1) * ((Py - 1) // 16 + 1)
    launch("filter2rec", (tiles, N), (16, 16), out, Py * Px, filt, Px1 * Py1, N, Px, Py, Px1, Py1)
    return out.reshape(N, Py, Px)


def compute_Dsw(Ds, h_norm):
    """compute_Dsw: ZGEMM('c','n') (numpy), real part, put_norm kernel
    (vrf.py:502-559)."""
    N = Ds.shape[0]
    D = Ds.reshape(N, -1)
    C = np.conj(D) @ D.T            # column-major C = D^H D, read row-major below
    W = np.ascontiguousarray(C.T.real)
    launch("put_norm", N, 256, W, np.ascontiguousarray(h_norm, np.float64), N)
    return W


# ----------------------------------------------------------------- decoder

def compute_q(tk1, tk2, ind, kappa, delta, bias, norm):
    n = len(tk1)
    q = np.zeros(n, np.float64)
    launch("compute_q", 6 * 8, 256, q, np.ascontiguousarray(tk1), np.ascontiguousarray(tk2),
           np.ascontiguousarray(ind, np.int32), np.ascontiguousarray(kappa, np.float64),
           np.ascontiguousarray(delta, np.float64), np.ascontiguousarray(bias, np.float64),
           np.ascontiguousarray(norm, np.float64), n)
    return q


def compute_G(tk1, tk2, ind, Dsw, Wt, Mt, lamb=0.0):
    """dirichlet.compute_G (dirichlet.py:62-85): one block per row."""
    n = len(tk1)
    G = np.zeros((n, n), np.float64)
    D = np.ascontiguousarray(Dsw, np.float64)
    launch("compute_G", n, 256, G, n, np.ascontiguousarray(tk1), np.ascontiguousarray(tk2), Wt, Mt,
           D, D.shape[1], np.ascontiguousarray(ind, np.int32))
    if lamb != 0:
        launch("diag_add", 6 * 8, 256, G, n, n, lamb)
    return G


def solve_eq_sym(G, q, rcond=1e-8):
    """linalg.solve_eq_sym (linalg.py:591-631): SVD (numpy for CULA),
    ``qq = U^H q``, sq_Kernel, ``c = U qq``."""
    U, S, _ = np.linalg.svd(G)
    qq = np.ascontiguousarray(U.T @ q)
    S = np.ascontiguousarray(S)
    launch("sq", 6 * 8, 256, S, qq, rcond, len(S))
    return U @ qq


def rnn3(G, q, dt=1e-6, alpha=5000, steps=4000):
    """neural_network.rnn3 (neural_network.py:15-99): GEMV (numpy) +
    rnn3_update kernel, steps+1 times."""
    n = len(q)
    c = np.zeros(n, np.float64)
    y = np.zeros(n, np.float64)
    qv = np.ascontiguousarray(q, np.float64)
    for _ in range(steps + 1):
        Gc = np.ascontiguousarray(G @ c)
        launch("rnn3_update", 6 * 8, 256, c, float(dt) * float(alpha), qv, Gc, y, n, 1, os_threads=1)
    return c


def reconstruct(dirich, tk1, tk2, c, t, ind, norm, Mt, WM):
    """dirichlet.reconstruct (dirichlet.py:165-189): reconstruct_Kernel over
    (ceil(P/128), len(t)) blocks of 128 threads."""
    N = dirich.shape[0]
    P = dirich[0].size
    gx = (P - 1) // 128 + 1
    ld = gx * 128                   # padded: the kernel reads dirich up to gx*128
    D = np.zeros((N, ld), np.float64)
    D[:, :P] = dirich.reshape(N, P)
    u = np.zeros((len(t), P), np.float64)
    launch("reconstruct", (gx, len(t)), 128, u, P, D, ld, np.ascontiguousarray(tk1),
           np.ascontiguousarray(tk2), np.ascontiguousarray(c, np.float64),
           np.ascontiguousarray(t, np.float64), np.ascontiguousarray(ind, np.int32),
           np.ascontiguousarray(norm, np.float64), Mt, WM, len(tk1))
    return u.reshape(len(t), *dirich.shape[1:])
