"""Visual receptive fields (Gabor and centre-surround) on the B200.

Same classes, methods and argument meanings as the reference's
``vtem/vrf.py`` (``vrf`` :13-82, ``vrf_gabor`` :88-536, ``vrf_cs``
:681-1117); device buffers are torch tensors instead of PitchArrays and the
kernels are the sm_100a ones in ``csrc/rf.cu`` and ``csrc/dirichlet.cu``.

Coordinate system (as in the reference): pixel (row py, column px) sits at
``x = px*dx + x_start``, ``y = -(py*dy + y_start)``; x grows along a row,
y grows upwards.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _abi
from ._abi import call, dptr, stream_ptr

F64 = torch.float64


def _dev(a, dtype=F64, device="cuda"):
    if isinstance(a, torch.Tensor):
        return a.to(device=device, dtype=dtype).contiguous()
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device=device)


class vrf(object):
    """Visual receptive field base (vrf.py:13-82)."""

    def __init__(self, shape, dtype=np.float64, dx=1.0 / 16, dy=1.0 / 16, scale=1, domain=None):
        self.shape = shape
        self.dtype = np.dtype(dtype)
        self.Pyall = shape[-2] * scale
        self.Pxall = shape[-1] * scale
        self.dx = float(np.real(self.dtype.type(dx))) / scale
        self.dy = float(np.real(self.dtype.type(dy))) / scale
        self.Sxall = self.Pxall * self.dx
        self.Syall = self.Pyall * self.dy
        if domain is None:
            self.Sx = self.Pxall * self.dx
            self.Sy = self.Pyall * self.dy
        else:
            self.Sx = float(domain[0])
            self.Sy = float(domain[1])
        self.Px = int(np.round(self.Sx / self.dx))
        self.Py = int(np.round(self.Sy / self.dy))
        self.device = torch.device("cuda", torch.cuda.current_device()) if torch.cuda.is_available() else None
        self.h_gain = None

    # ------------------------------------------------------------ shared
    def _grid_args(self, x_start, y_start):
        if x_start is None:
            x_start = -self.Sxall / 2
        if y_start is None:
            y_start = -self.Syall / 2
        return x_start, y_start

    def filter(self, V, out_layout="time", precision="f64"):
        """Filter a video ``V`` (frames, Py, Px) with every RF.

        Returns the (frames, N) projection ``dx*dy*sum_p V RF`` as a CUDA
        tensor (vrf.py:264-292); ``out_layout="neuron"`` returns the same
        values laid out (N, frames), the layout the IAF scan reads fastest.
        ``precision="bf16x3"`` (extension) computes it on the tensor cores
        from split-bf16 operands (relative error ~1e-5) instead of float64.
        """
        return _project(V, self._rf_full(), self.dx * self.dy, self.Pxall * self.Pyall, out_layout, precision)

    def _rf_full(self):
        if getattr(self, "_rf_cache", None) is None or self._rf_cache.shape[0] != self.num_neurons:
            self.generate_visual_receptive_fields()
            self._rf_cache = self._rfs()
        return self._rf_cache.reshape(self.num_neurons, -1)

    def compute_Ds(self, Mx, My):
        """Dirichlet coefficients (N, 2My+1, 2Mx+1) complex128 of every RF
        (vrf.py:333-377): RFs generated on this object's grid, which must
        span one spatial period."""
        self.generate_visual_receptive_fields()
        rf = self._rfs().reshape(self.num_neurons, -1)
        N = self.num_neurons
        Ds = torch.empty((N, 2 * My + 1, 2 * Mx + 1), dtype=torch.complex128, device=rf.device)
        call("vtb_dirichlet_coeffs", dptr(rf), N, self.Pyall, self.Pxall, self.Pxall * self.Pyall, int(Mx),
             int(My), self.dx * self.dy, dptr(Ds), stream_ptr())
        return Ds

    def compute_dirich_space_fft(self, d_Ds, Mx, My, Px, Py, Sx, Sy, Wx, Wy):
        """Spatial reconstruction functions (N, Py, Px) on the decode grid
        (vrf.py:437-499): the period grid is ``round(self.Sx / (Sx/Px))``
        pixels wide, centre-cropped to (Py, Px)."""
        dx = Sx / Px
        dy = Sy / Py
        Px1 = int(np.round(self.Sx / dx))
        Py1 = int(np.round(self.Sy / dy))
        Ds = d_Ds.contiguous()
        N = Ds.shape[0]
        out = torch.empty((N, Py, Px), dtype=F64, device=Ds.device)
        call("vtb_dirich_space", dptr(Ds), N, int(Mx), int(My), int(Px), int(Py), Px1, Py1, dptr(out),
             stream_ptr())
        return out

    def compute_Dsw(self, d_Ds, Mx, My, h_norm):
        """RF cross-weights Re(Ds Ds^H) * norm norm^T, (N, N) (vrf.py:502-536)."""
        Ds = d_Ds.contiguous()
        N = Ds.shape[0]
        Ks = (2 * Mx + 1) * (2 * My + 1)
        norm = _dev(np.asarray(h_norm, np.float64), device=Ds.device)
        W = torch.empty((N, N), dtype=F64, device=Ds.device)
        call("vtb_dsw", dptr(Ds), N, Ks, dptr(norm), dptr(W), N, stream_ptr())
        return W


class vrf_gabor(vrf):
    """Gabor RFs (vrf.py:88-536)."""

    def get_gabor_parameters(self, dilations=[1, 0, -1, -2, -3], num_rotations=8, alpha0=np.float64(2),
                             b0=np.float64(1.5), b0scalebase=np.sqrt(2), KAPPA=2.5):
        """The reference's default Gabor family (vrf.py:136-205): for each
        dilation m, num_rotations angles and a translation lattice covering
        the domain, a cos/sin quadrature pair."""
        b0 = np.float64(b0)
        b0scalebase = np.float64(b0scalebase)
        alpha0 = np.float64(alpha0)
        self.KAPPA = float(KAPPA)
        l0 = (num_rotations - 1) * np.pi / num_rotations
        bi = np.empty(len(dilations), np.float64)
        trans_x = np.empty(len(dilations), np.int32)
        trans_y = np.empty(len(dilations), np.int32)
        for i in range(bi.size):
            bi[i] = b0 * np.power(alpha0, dilations[i]) * np.power(b0scalebase, -dilations[i])
            trans_x[i] = int(np.floor(self.Sx / 2 / bi[i]))
            trans_y[i] = int(np.floor(self.Sy / 2 / bi[i]))
        self.num_neurons = int(sum((trans_x[i] * 2 + 1) * (trans_y[i] * 2 + 1) * num_rotations * 2
                                   for i in range(len(dilations))))
        self.h_alpha = np.empty(self.num_neurons, np.float64)
        self.h_l = np.empty(self.num_neurons, np.float64)
        self.h_y0 = np.empty(self.num_neurons, np.float64)
        self.h_x0 = np.empty(self.num_neurons, np.float64)
        self.h_ab = np.empty(self.num_neurons, np.int32)
        a = 0
        for i, m in enumerate(dilations):
            for l in range(num_rotations):
                ll = l * l0
                for k in np.arange(-trans_y[i], trans_y[i] + 1, 1):
                    for n in np.arange(-trans_x[i], trans_x[i] + 1, 1):
                        self.h_alpha[a] = self.h_alpha[a + 1] = alpha0 ** (m)
                        self.h_l[a] = self.h_l[a + 1] = ll
                        self.h_y0[a] = self.h_y0[a + 1] = k * bi[i]
                        self.h_x0[a] = self.h_x0[a + 1] = n * bi[i]
                        self.h_ab[a] = 0
                        self.h_ab[a + 1] = 1
                        a += 2

    def load_parameters(self, num_neurons=None, h_alpha=None, h_l=None, h_x0=None, h_y0=None, h_ab=None,
                        KAPPA=2.5, set=0, h_gain=None):
        """Load Gabor parameters to the GPU (vrf.py:209-262).  ``h_gain`` is
        an optional per-RF amplitude (extension; None = reference)."""
        if num_neurons is not None:
            self.num_neurons = int(num_neurons)
            if h_alpha is None or h_l is None or h_x0 is None or h_y0 is None or h_ab is None:
                raise ValueError("must specify the gabor parameters")
            self.h_alpha, self.h_l, self.h_x0, self.h_y0, self.h_ab = h_alpha, h_l, h_x0, h_y0, h_ab
            self.KAPPA = float(KAPPA)
        elif not set:
            self.get_gabor_parameters(KAPPA=KAPPA)
        self.h_gain = h_gain
        self.d_alpha = _dev(self.h_alpha)
        self.d_l = _dev(self.h_l)
        self.d_x0 = _dev(self.h_x0)
        self.d_y0 = _dev(self.h_y0)
        self.d_ab = _dev(np.asarray(self.h_ab, np.int32), dtype=torch.int32)
        self.d_gain = None if h_gain is None else _dev(h_gain)
        self._rf_cache = None

    def generate_visual_receptive_fields(self, startbias=0, N_filters=None, x_start=None, y_start=None):
        """Gabor RFs startbias..startbias+N_filters on the full grid into
        ``self.gabors`` (N_filters, Pyall, Pxall) (vrf.py:296-331)."""
        if N_filters is None:
            N_filters = self.num_neurons - startbias
        x_start, y_start = self._grid_args(x_start, y_start)
        self.gabors = torch.empty((N_filters, self.Pyall, self.Pxall), dtype=F64, device=self.d_alpha.device)
        sl = slice(startbias, startbias + N_filters)
        g = None if self.d_gain is None else self.d_gain[sl]
        call("vtb_rf_gabor", dptr(self.d_alpha[sl]), dptr(self.d_l[sl]), dptr(self.d_x0[sl]),
             dptr(self.d_y0[sl]), dptr(self.d_ab[sl]), dptr(g), int(N_filters), self.Pxall, self.Pyall,
             self.Sxall, self.Syall, float(x_start), float(y_start), float(self.KAPPA), dptr(self.gabors),
             self.Pxall * self.Pyall, stream_ptr())

    def _rfs(self):
        return self.gabors


class vrf_cs(vrf):
    """Centre-surround RFs (vrf.py:681-1117)."""

    def get_cs_parameters(self, dilations=[1, 0, -1, -2, -3], alpha0=np.float64(2), b0=np.float64(1.0),
                          b0scalebase=np.float64(1.0), sigma_center=0.5, sigma_surround=0.8):
        """The reference's default centre-surround family (vrf.py:726-790)."""
        b0 = np.float64(b0)
        b0scalebase = np.float64(b0scalebase)
        alpha0 = np.float64(alpha0)
        self.sigma_center = float(sigma_center)
        self.sigma_surround = float(sigma_surround)
        bi = np.empty(len(dilations), np.float64)
        trans_x = np.empty(len(dilations), np.int32)
        trans_y = np.empty(len(dilations), np.int32)
        for i in range(bi.size):
            bi[i] = b0 * np.power(alpha0, dilations[i]) * np.power(b0scalebase, -dilations[i])
            trans_x[i] = int(np.floor(self.Sx / 2 / bi[i]))
            trans_y[i] = int(np.floor(self.Sy / 2 / bi[i]))
        self.num_neurons = int(sum((trans_x[i] * 2 + 1) * (trans_y[i] * 2 + 1) for i in range(len(dilations))))
        self.h_alpha = np.empty(self.num_neurons, np.float64)
        self.h_y0 = np.empty(self.num_neurons, np.float64)
        self.h_x0 = np.empty(self.num_neurons, np.float64)
        a = 0
        for i, m in enumerate(dilations):
            for k in np.arange(-trans_y[i], trans_y[i] + 1, 1):
                for n in np.arange(-trans_x[i], trans_x[i] + 1, 1):
                    self.h_alpha[a] = alpha0 ** (m)
                    self.h_y0[a] = k * bi[i]
                    self.h_x0[a] = n * bi[i]
                    a += 1

    def load_parameters(self, num_neurons=None, h_alpha=None, h_x0=None, h_y0=None, set=0, sigma_center=0.5,
                        sigma_surround=0.8, h_gain=None):
        """Load centre-surround parameters to the GPU (vrf.py:794-843)."""
        if num_neurons is not None:
            self.num_neurons = int(num_neurons)
            if h_alpha is None or h_x0 is None or h_y0 is None:
                raise ValueError("must specify the gabor parameters")
            self.h_alpha, self.h_x0, self.h_y0 = h_alpha, h_x0, h_y0
            self.sigma_center = float(sigma_center)
            self.sigma_surround = float(sigma_surround)
        elif not set:
            self.get_cs_parameters()
        self.h_gain = h_gain
        self.d_alpha = _dev(self.h_alpha)
        self.d_x0 = _dev(self.h_x0)
        self.d_y0 = _dev(self.h_y0)
        self.d_gain = None if h_gain is None else _dev(h_gain)
        self._rf_cache = None

    def generate_visual_receptive_fields(self, startbias=0, N_filters=None, x_start=None, y_start=None):
        """Centre-surround RFs into ``self.filters`` (vrf.py:876-913)."""
        if N_filters is None:
            N_filters = self.num_neurons - startbias
        x_start, y_start = self._grid_args(x_start, y_start)
        self.filters = torch.empty((N_filters, self.Pyall, self.Pxall), dtype=F64, device=self.d_alpha.device)
        sl = slice(startbias, startbias + N_filters)
        g = None if self.d_gain is None else self.d_gain[sl]
        call("vtb_rf_cs", dptr(self.d_alpha[sl]), dptr(self.d_x0[sl]), dptr(self.d_y0[sl]), dptr(g),
             int(N_filters), self.Pxall, self.Pyall, self.Sxall, self.Syall, float(x_start), float(y_start),
             self.sigma_center, self.sigma_surround, dptr(self.filters), self.Pxall * self.Pyall, stream_ptr())

    def _rfs(self):
        return self.filters


def _project(V, rf, alpha, P_expected, out_layout, precision):
    """alpha * V rf^T, (frames, N) or (N, frames) (vrf.py:264-292)."""
    V = _dev(V).reshape(V.shape[0], -1)
    F, P = V.shape
    if P != P_expected:
        raise ValueError("video frame size does not match the RF grid")
    N = rf.shape[0]
    if precision == "bf16x3":
        from . import tc
        return tc.gemm_split_bf16(V, rf, alpha=alpha, out_layout="row" if out_layout == "time" else "col")
    if precision != "f64":
        raise ValueError("precision must be 'f64' or 'bf16x3'")
    if V.dtype != F64:
        V = V.to(F64)
    if out_layout == "time":
        out = torch.empty((F, N), dtype=F64, device=V.device)
        ts, ns = N, 1
    else:
        out = torch.empty((N, F), dtype=F64, device=V.device)
        ts, ns = 1, F
    call("vtb_rf_filter", dptr(V), F, P, P, dptr(rf), N, P, alpha, dptr(out), ts, ns, stream_ptr())
    return out


class vrf_bank(object):
    """Concatenation of several RF objects sharing one pixel grid, seen as
    one encoder of ``sum(num_neurons)`` neurons (extension: the reference
    encodes one RF family per VTEM call, vtem.py:144-149)."""

    def __init__(self, banks):
        self.banks = list(banks)
        b0 = self.banks[0]
        for b in self.banks:
            if (b.Pxall, b.Pyall) != (b0.Pxall, b0.Pyall):
                raise ValueError("RF banks must share the pixel grid")
        for k in ("Pxall", "Pyall", "dx", "dy", "Sxall", "Syall", "Sx", "Sy", "Px", "Py"):
            setattr(self, k, getattr(b0, k))
        self.num_neurons = sum(b.num_neurons for b in self.banks)

    def filter(self, V, out_layout="time", precision="f64"):
        """Every bank's projection, in bank order, as ONE product of the video
        with the banks' stacked RFs (one pass over the video, no
        concatenation of outputs) when the banks share the pixel area."""
        b0 = self.banks[0]
        if any((b.dx, b.dy) != (b0.dx, b0.dy) for b in self.banks):
            outs = [b.filter(V, out_layout, precision) for b in self.banks]
            return torch.cat(outs, dim=1 if out_layout == "time" else 0)
        parts = [b._rf_full() for b in self.banks]
        # the stacked RFs are rebuilt when any bank regenerated its RFs (the
        # held references keep a regenerated array from reusing an address)
        src = [b._rf_cache for b in self.banks]
        held = getattr(self, "_rf_src", None)
        if held is None or len(held) != len(src) or any(a is not b for a, b in zip(held, src)):
            self._rf_all = torch.cat(parts, dim=0).contiguous()
            self._rf_src = src
        return _project(V, self._rf_all, b0.dx * b0.dy, self.Pxall * self.Pyall, out_layout, precision)
