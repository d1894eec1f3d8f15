"""Seeded synthetic workloads of the encode/decode path.

The reference ships no data (its demos read external files), so every run
uses a Dirichlet-bandlimited video: complex N(0,1) coefficients inside the
reference's spatial ellipse (mx^2 My^2 + my^2 Mx^2 <= Mx^2 My^2, vrf.py:1331),
made Hermitian so the video is real, scaled to max|u| = 1, evaluated on the
reference's pixel grid (domain [-1/2, 1/2]^2 centred, y up) at t = f*dt.

Configurations:
  small  (32x32, 2000 samples, Mx=My=3, Mt=4, 128 Gabor RFs, IAF b=3,
          delta~N(0.04, 0.004) clipped > 0)
  gpu    (64x64, 10000 samples, Mx=My=6, Mt=8, 768 Gabor + 256 centre-
          surround RFs, IAF b~U(2,4), delta~N(0.12, 0.012); the threshold
          mean is chosen so the clip yields ~25k spikes, the size the
          workload is specified at; a mean of 0.03 would give ~100k)
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import torch


@dataclass
class GaborParams:
    h_alpha: np.ndarray
    h_l: np.ndarray
    h_x0: np.ndarray
    h_y0: np.ndarray
    h_ab: np.ndarray
    KAPPA: float
    gain: np.ndarray


@dataclass
class CSParams:
    h_alpha: np.ndarray
    h_x0: np.ndarray
    h_y0: np.ndarray
    sigma_center: float
    sigma_surround: float
    gain: np.ndarray


@dataclass
class Workload:
    name: str
    Px: int
    Py: int
    F: int
    dt: float
    Mx: int
    My: int
    Mt: int
    Wx: float
    Wy: float
    Wt: float
    coeffs: np.ndarray          # (2My+1, 2Mx+1, 2Mt+1) complex, unscaled
    scale: float                # 1 / max|u|
    gabor: GaborParams | None
    cs: CSParams | None
    kappa: np.ndarray
    bias: np.ndarray
    delta: np.ndarray
    v0: np.ndarray
    rcond: float
    extra: dict = field(default_factory=dict)

    @property
    def dx(self):
        return 1.0 / self.Px

    @property
    def dy(self):
        return 1.0 / self.Py

    @property
    def N(self):
        return (0 if self.gabor is None else len(self.gabor.h_alpha)) + (0 if self.cs is None else len(self.cs.h_alpha))

    @property
    def T(self):
        return self.F * self.dt

    def video(self, device="cpu"):
        """(F, Py, Px) float64 video, max|u| = 1."""
        u = bandlimited_video(self.coeffs, self.Mx, self.My, self.Mt, self.Wx, self.Wy, self.Wt, self.Px,
                              self.Py, self.F, self.dt, device)
        if self.scale is None:
            self.scale = 1.0 / float(u.abs().max())
        return u * self.scale


def ellipse_mask(Mx, My):
    my = np.arange(-My, My + 1)[:, None]
    mx = np.arange(-Mx, Mx + 1)[None, :]
    return (mx * mx * My * My + my * my * Mx * Mx) <= Mx * Mx * My * My


def bandlimited_coeffs(Mx, My, Mt, seed):
    rng = np.random.default_rng(seed)
    shp = (2 * My + 1, 2 * Mx + 1, 2 * Mt + 1)
    a = rng.standard_normal(shp) + 1j * rng.standard_normal(shp)
    a = 0.5 * (a + np.conj(a[::-1, ::-1, ::-1]))
    return a * ellipse_mask(Mx, My)[:, :, None]


def bandlimited_video(a, Mx, My, Mt, Wx, Wy, Wt, Px, Py, F, dt, device="cpu"):
    """sum_m a[my,mx,mt] e^{j(mx Wx/Mx x + my Wy/My y + mt Wt/Mt t)} on the
    centred pixel grid; separable evaluation, float64 real part."""
    c128 = torch.complex128
    dev = torch.device(device)
    x = torch.arange(Px, dtype=torch.float64, device=dev) * (1.0 / Px) - 0.5
    y = -(torch.arange(Py, dtype=torch.float64, device=dev) * (1.0 / Py) - 0.5)
    t = torch.arange(F, dtype=torch.float64, device=dev) * dt
    mx = torch.arange(-Mx, Mx + 1, dtype=torch.float64, device=dev)
    my = torch.arange(-My, My + 1, dtype=torch.float64, device=dev)
    mt = torch.arange(-Mt, Mt + 1, dtype=torch.float64, device=dev)
    ex = torch.exp(1j * torch.outer(mx, x) * (Wx / Mx)).to(c128)        # (Kx, Px)
    ey = torch.exp(1j * torch.outer(my, y) * (Wy / My)).to(c128)        # (Ky, Py)
    et = torch.exp(1j * torch.outer(t, mt) * (Wt / Mt)).to(c128)        # (F, Kt)
    A = torch.as_tensor(a, dtype=c128, device=dev)
    B = torch.einsum("ymt,ft->fym", A, et)
    C = torch.einsum("fym,mx->fyx", B, ex)
    u = torch.einsum("fyx,yp->fpx", C, ey)
    return u.real.contiguous()


def gabor_grid_values(p: GaborParams, Px, Py, gain=True):
    """Gabor RFs (N, Py, Px) on the video grid (formula of vrf.py:1254-1285),
    used to set unit-norm gains."""
    x = (np.arange(Px) * (1.0 / Px) - 0.5)[None, None, :]
    y = (-(np.arange(Py) * (1.0 / Py) - 0.5))[None, :, None]
    al = (1.0 / p.h_alpha)[:, None, None]
    xs = al * (x - p.h_x0[:, None, None])
    ys = al * (y - p.h_y0[:, None, None])
    st, ct = np.sin(p.h_l)[:, None, None], np.cos(p.h_l)[:, None, None]
    X = xs * ct + ys * st
    Y = -xs * st + ys * ct
    first = al * (1 / math.sqrt(2 * math.pi)) * np.exp(-((4 * X * X) + (Y * Y)) / 8)
    v = np.where(p.h_ab[:, None, None] == 0, np.cos(p.KAPPA * X), np.sin(p.KAPPA * X)) * first
    return v * p.gain[:, None, None] if gain else v


def cs_grid_values(p: CSParams, Px, Py, gain=True):
    x = (np.arange(Px) * (1.0 / Px) - 0.5)[None, None, :]
    y = (-(np.arange(Py) * (1.0 / Py) - 0.5))[None, :, None]
    al = (1.0 / p.h_alpha)[:, None, None]
    xs = al * (x - p.h_x0[:, None, None])
    ys = al * (y - p.h_y0[:, None, None])
    XY = -(xs * xs + ys * ys)
    sc2, ss2 = p.sigma_center ** 2, p.sigma_surround ** 2
    v = al * (np.exp(XY / (2 * sc2)) / sc2 - 0.9 * np.exp(XY / (2 * ss2)) / ss2) / (2 * math.pi)
    return v * p.gain[:, None, None] if gain else v


def _unit_gain(vals, dx, dy):
    nrm = np.sqrt((vals.reshape(len(vals), -1) ** 2).sum(1) * dx * dy)
    return 1.0 / nrm


def small(seed=0):
    """32x32, 0.2 s at dt=1e-4, Mx=My=3, Mt=4, Wx=Wy=2pi*3, Wt=2pi*20,
    128 Gabor RFs (4 orientations x 2 scales x 4x4 centres), IAF b=3, k=1,
    delta~N(0.04, 0.004) clipped > 0, pseudoinverse rcond 1e-10."""
    Px = Py = 32
    Mx = My = 3
    Mt = 4
    a = bandlimited_coeffs(Mx, My, Mt, seed)
    orients = np.arange(4) * np.pi / 4
    sigmas = np.array([0.1, 0.2])
    cent = (np.arange(4) + 0.5) / 4 - 0.5
    al, th, x0, y0, ab = [], [], [], [], []
    i = 0
    for s in sigmas:
        for o in orients:
            for cy in cent:
                for cx in cent:
                    al.append(s)
                    th.append(o)
                    x0.append(cx)
                    y0.append(cy)
                    ab.append(i % 2)
                    i += 1
    g = GaborParams(np.array(al), np.array(th), np.array(x0), np.array(y0), np.array(ab, np.int32), 2.5,
                    np.ones(len(al)))
    g.gain = _unit_gain(gabor_grid_values(g, Px, Py, gain=False), 1.0 / Px, 1.0 / Py)
    rng = np.random.default_rng(seed + 100)
    N = len(al)
    delta = np.abs(rng.normal(0.04, 0.004, N))
    delta = np.where(delta <= 0, 0.04, delta)
    v0 = rng.uniform(0, 1, N) * delta
    w = Workload("small", Px, Py, 2000, 1e-4, Mx, My, Mt, 2 * np.pi * 3, 2 * np.pi * 3, 2 * np.pi * 20, a, 1.0,
                 g, None, np.ones(N), np.full(N, 3.0), delta, v0, 1e-10)
    w.scale = 1.0 / float(w.video().abs().max())
    return w


def gpu_scale(seed=0, rf_seed=1, frames=10000):
    """64x64, 1 s at dt=1e-4, Mx=My=6, Mt=8, Wx=Wy=2pi*6, Wt=2pi*20; 768
    Gabor (8 orientations x 3 scales x 32 uniform centres, seed 1) + 256
    centre-surround (sigma_c 0.05, sigma_s 0.15, surround weight 0.9)."""
    Px = Py = 64
    Mx = My = 6
    Mt = 8
    a = bandlimited_coeffs(Mx, My, Mt, seed)
    rng = np.random.default_rng(rf_seed)
    orients = np.arange(8) * np.pi / 8
    sigmas = np.array([0.05, 0.1, 0.2])
    al, th, x0, y0, ab = [], [], [], [], []
    i = 0
    for s in sigmas:
        for o in orients:
            c = rng.uniform(-0.5, 0.5, (32, 2))
            for cx, cy in c:
                al.append(s)
                th.append(o)
                x0.append(cx)
                y0.append(cy)
                ab.append(i % 2)
                i += 1
    g = GaborParams(np.array(al), np.array(th), np.array(x0), np.array(y0), np.array(ab, np.int32), 2.5,
                    np.ones(len(al)))
    g.gain = _unit_gain(gabor_grid_values(g, Px, Py, gain=False), 1.0 / Px, 1.0 / Py)
    c = rng.uniform(-0.5, 0.5, (256, 2))
    cs = CSParams(np.ones(256), c[:, 0].copy(), c[:, 1].copy(), 0.05, 0.15, np.ones(256))
    cs.gain = _unit_gain(cs_grid_values(cs, Px, Py, gain=False), 1.0 / Px, 1.0 / Py)
    N = 1024
    rng2 = np.random.default_rng(seed + 200)
    bias = rng2.uniform(2, 4, N)
    delta = np.abs(rng2.normal(0.12, 0.012, N))
    v0 = rng2.uniform(0, 1, N) * delta
    w = Workload("gpu", Px, Py, frames, 1e-4, Mx, My, Mt, 2 * np.pi * 6, 2 * np.pi * 6, 2 * np.pi * 20, a, 1.0, g,
                 cs, np.ones(N), bias, delta, v0, 1e-8)
    w.scale = 1.0 / float(w.video().abs().max())
    return w


def batch_clips(count=256, seed=2, rf_scale=1.0):
    """Independent clips of uneven size for batched decoding: frame side in
    {16, 32, 48, 64}, duration U(0.05, 0.5) s at dt=1e-4, Mt in {3..8},
    Mx=My in {2..6}, RF count in {32..1024} (3/4 Gabor, 1/4 centre-surround
    as in the GPU configuration), IAF b~U(2,4), delta~N(0.075, 0.0075) (~40 Hz).
    The video scale (max|u| = 1) is set on the device at encode time."""
    rng = np.random.default_rng(seed)
    clips = []
    for i in range(count):
        side = int(rng.choice([16, 32, 48, 64]))
        dur = float(rng.uniform(0.05, 0.5))
        F = int(round(dur / 1e-4))
        Mt = int(rng.integers(3, 9))
        M = int(rng.integers(2, 7))
        N = int(rng.integers(32, 1025))
        Ng = max(1, (3 * N) // 4)
        Nc = N - Ng
        sub = np.random.default_rng(rng.integers(1 << 62))
        a = bandlimited_coeffs(M, M, Mt, int(sub.integers(1 << 31)))
        sig = sub.choice([0.05, 0.1, 0.2], Ng)
        g = GaborParams(sig, sub.uniform(0, np.pi, Ng), sub.uniform(-0.5, 0.5, Ng), sub.uniform(-0.5, 0.5, Ng),
                        (np.arange(Ng) % 2).astype(np.int32), 2.5, np.ones(Ng))
        g.gain = _unit_gain(gabor_grid_values(g, side, side, gain=False), 1.0 / side, 1.0 / side)
        cs = None
        if Nc > 0:
            c = sub.uniform(-0.5, 0.5, (Nc, 2))
            cs = CSParams(np.ones(Nc), c[:, 0].copy(), c[:, 1].copy(), 0.05, 0.15, np.ones(Nc))
            cs.gain = _unit_gain(cs_grid_values(cs, side, side, gain=False), 1.0 / side, 1.0 / side)
        bias = sub.uniform(2, 4, N)
        delta = np.abs(sub.normal(0.075, 0.0075, N))
        v0 = sub.uniform(0, 1, N) * delta
        w = Workload("batch%03d" % i, side, side, F, 1e-4, M, M, Mt, 2 * np.pi * M, 2 * np.pi * M, 2 * np.pi * 20, a,
                     None, g, cs, np.ones(N), bias, delta, v0, 1e-8)
        clips.append(w)
    return clips
