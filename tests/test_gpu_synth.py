"""Coefficient-space synthesis against the direct sum (GPU).

vtb_coeff_synthesize renders u[f][py][px] = Re sum_s A_t[s] ey_s[py] ex_s[px]
with A_t[s] = sum_m a[s][m] e^{j m W t_f} over the reference's spatial
ellipse (the Dirichlet reconstruction of dirichlet.py:354-420 and
vrf.py:437-499 in coefficient form).  It has three kernels: the
warp-specialised one (frames up to 64 px wide, Mx, My <= 6), the
half-spectrum one (2 My + 1 <= 13) and the general two-pass one; each is
checked on odd sizes, crop offsets, frame counts that leave partial chunks,
and non-Hermitian coefficients (the kernels may not assume the symmetry the
decoders produce)."""
import numpy as np
import pytest
import torch

from vtem_b200 import _abi
from vtem_b200.fast import ellipse_storage_index

pytestmark = pytest.mark.gpu


def _direct(a, Mx, My, Mt, W, t0, dt, Nt, Px, Py, Px1, Py1):
    smap = ellipse_storage_index(Mx, My)
    Kx, Kt = 2 * Mx + 1, 2 * Mt + 1
    my = My - smap // Kx
    mx = smap % Kx - Mx
    px = (np.arange(Px) + (Px1 - Px) // 2) % Px1
    py = (np.arange(Py) + (Py1 - Py) // 2) % Py1
    ex = ((-1.0) ** mx)[:, None] * np.exp(2j * np.pi * np.outer(mx, px) / Px1)
    ey = ((-1.0) ** my)[:, None] * np.exp(2j * np.pi * np.outer(my, py) / Py1)
    E = np.exp(1j * W * np.outer(t0 + np.arange(Nt) * dt, np.arange(-Mt, Mt + 1)))
    A = E @ a.reshape(len(smap), Kt).T
    return np.einsum("fs,sy,sx->fyx", A, ey, ex).real


CASES = [
    # Mx, My, Mt, Px, Py, Px1, Py1, Nt          kernel
    (6, 6, 8, 64, 64, 64, 64, 37),              # warp-specialised (the decoder's configuration)
    (3, 3, 4, 32, 32, 32, 32, 16),              # warp-specialised, whole chunks
    (2, 5, 3, 17, 70, 20, 75, 53),              # warp-specialised, odd sizes, crop offsets, two row tiles
    (0, 2, 1, 9, 5, 9, 5, 3),                   # warp-specialised, Mx = 0
    (7, 4, 2, 40, 24, 48, 30, 21),              # half-spectrum (Mx > 6)
    (3, 3, 4, 80, 50, 96, 60, 19),              # half-spectrum (wider than 64)
    (4, 7, 2, 20, 20, 20, 20, 11),              # general (2 My + 1 > 13)
]


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_synthesis_matches_direct_sum(case, dtype):
    Mx, My, Mt, Px, Py, Px1, Py1, Nt = case
    rng = np.random.default_rng(Mx * 100 + My * 10 + Mt)
    smap = torch.as_tensor(ellipse_storage_index(Mx, My), device="cuda")
    Ks, Kt = int(smap.numel()), 2 * Mt + 1
    a = rng.standard_normal(Ks * Kt) + 1j * rng.standard_normal(Ks * Kt)
    W, t0, dt = 2 * np.pi * 20 / Mt, 0.013, 1e-3
    ad = torch.as_tensor(a, dtype=torch.complex128, device="cuda")
    A = torch.empty((Nt, Ks), dtype=torch.complex128, device="cuda")
    u = torch.full((Nt, Py, Px), float("nan"), dtype=dtype, device="cuda")
    st = _abi.lib().vtb_coeff_synthesize(ad.data_ptr(), smap.data_ptr(), Ks, Mx, My, Mt, W, t0, dt, Nt, Px, Py, Px1,
                                         Py1, A.data_ptr(), u.data_ptr(), int(dtype == torch.float32),
                                         _abi.stream_ptr())
    assert st == 0, _abi.status_string(st)
    ref = _direct(a, Mx, My, Mt, W, t0, dt, Nt, Px, Py, Px1, Py1)
    got = u.double().cpu().numpy()
    assert np.isfinite(got).all()
    tol = 1e-12 if dtype == torch.float64 else 1e-6
    err = np.abs(got - ref).max() / np.abs(ref).max()
    assert err <= tol, err


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_rank_synthesis_matches_direct_sum(case, dtype):
    """vtb_coeff_basis + vtb_synth_harmonics: the same video as a product of
    the frames' temporal harmonics and per-pixel weights (non-Hermitian
    coefficients, so the m / -m pairing is exercised), frame ranges rendered
    separately as the chunked download does."""
    Mx, My, Mt, Px, Py, Px1, Py1, Nt = case
    rng = np.random.default_rng(Mx * 100 + My * 10 + Mt + 7)
    smap = torch.as_tensor(ellipse_storage_index(Mx, My), device="cuda")
    Ks, Kt = int(smap.numel()), 2 * Mt + 1
    a = rng.standard_normal(Ks * Kt) + 1j * rng.standard_normal(Ks * Kt)
    W, t0, dt = 2 * np.pi * 20 / Mt, 0.013, 1e-3
    ad = torch.as_tensor(a, dtype=torch.complex128, device="cuda")
    P = Px * Py
    H = torch.empty((P, Kt), dtype=torch.float64, device="cuda")
    lib = _abi.lib()
    st = lib.vtb_coeff_basis(ad.data_ptr(), smap.data_ptr(), Ks, Mx, My, Mt, Px, Py, Px1, Py1, H.data_ptr(), Kt,
                             _abi.stream_ptr())
    assert st == 0, _abi.status_string(st)
    u = torch.full((Nt, Py, Px), float("nan"), dtype=dtype, device="cuda")
    half = Nt // 2
    for f0, f1 in ((0, half), (half, Nt)):
        st = lib.vtb_synth_harmonics(H.data_ptr(), Kt, P, Mt, W, t0 + f0 * dt, dt, f1 - f0, u[f0:f1].data_ptr(),
                                     int(dtype == torch.float32), _abi.stream_ptr())
        assert st == 0, _abi.status_string(st)
    ref = _direct(a, Mx, My, Mt, W, t0, dt, Nt, Px, Py, Px1, Py1)
    got = u.double().cpu().numpy()
    assert np.isfinite(got).all()
    tol = 1e-12 if dtype == torch.float64 else 1e-6
    err = np.abs(got - ref).max() / np.abs(ref).max()
    assert err <= tol, err


def test_rank_synthesis_rejects_unsupported_orders():
    lib = _abi.lib()
    assert lib.vtb_synth_harmonics(None, 0, 10, 0, 1.0, 0.0, 1e-3, 5, None, 0, None) == _abi.VTB_BAD_ARG
    x = torch.zeros(64, dtype=torch.float64, device="cuda")
    # Mt = 11: 23 harmonics, beyond the kernel's 21
    assert lib.vtb_synth_harmonics(x.data_ptr(), 23, 2, 11, 1.0, 0.0, 1e-3, 1, x.data_ptr(), 0,
                                   _abi.stream_ptr()) == _abi.VTB_BAD_ARG


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_synth_rank_one_call_matches_direct_sum(case, dtype):
    """vtb_coeff_synth_rank: weights and harmonics in one call, the harmonics
    kernel launched programmatically behind the weights kernel."""
    Mx, My, Mt, Px, Py, Px1, Py1, Nt = case
    rng = np.random.default_rng(Mx * 100 + My * 10 + Mt + 11)
    smap = torch.as_tensor(ellipse_storage_index(Mx, My), device="cuda")
    Ks, Kt = int(smap.numel()), 2 * Mt + 1
    a = rng.standard_normal(Ks * Kt) + 1j * rng.standard_normal(Ks * Kt)
    W, t0, dt = 2 * np.pi * 20 / Mt, 0.021, 1e-3
    ad = torch.as_tensor(a, dtype=torch.complex128, device="cuda")
    H = torch.empty((Px * Py, Kt), dtype=torch.float64, device="cuda")
    u = torch.full((Nt, Py, Px), float("nan"), dtype=dtype, device="cuda")
    st = _abi.lib().vtb_coeff_synth_rank(ad.data_ptr(), smap.data_ptr(), Ks, Mx, My, Mt, Px, Py, Px1, Py1,
                                         H.data_ptr(), Kt, W, t0, dt, Nt, u.data_ptr(), int(dtype == torch.float32),
                                         _abi.stream_ptr())
    assert st == 0, _abi.status_string(st)
    ref = _direct(a, Mx, My, Mt, W, t0, dt, Nt, Px, Py, Px1, Py1)
    got = u.double().cpu().numpy()
    assert np.isfinite(got).all()
    tol = 1e-12 if dtype == torch.float64 else 1e-6
    err = np.abs(got - ref).max() / np.abs(ref).max()
    assert err <= tol, err


@pytest.mark.parametrize("Nt", [1100, 1101])
def test_synth_rank_long_frame_ranges(Nt):
    """Frame ranges longer than one pass of frame pairs (a wide frame, so few
    ranges per pixel tile), even and odd range lengths: the same video as
    the per-frame fused kernel."""
    Mx, My, Mt, Px, Py = 3, 3, 4, 296, 256
    rng = np.random.default_rng(Nt)
    smap = torch.as_tensor(ellipse_storage_index(Mx, My), device="cuda")
    Ks, Kt = int(smap.numel()), 2 * Mt + 1
    a = rng.standard_normal(Ks * Kt) + 1j * rng.standard_normal(Ks * Kt)
    W, t0, dt = 2 * np.pi * 20 / Mt, 0.37, 1e-4
    ad = torch.as_tensor(a, dtype=torch.complex128, device="cuda")
    H = torch.empty((Px * Py, Kt), dtype=torch.float64, device="cuda")
    u = torch.full((Nt, Py, Px), float("nan"), dtype=torch.float64, device="cuda")
    ref = torch.empty_like(u)
    lib = _abi.lib()
    st = lib.vtb_coeff_synth_rank(ad.data_ptr(), smap.data_ptr(), Ks, Mx, My, Mt, Px, Py, Px, Py, H.data_ptr(), Kt,
                                  W, t0, dt, Nt, u.data_ptr(), 0, _abi.stream_ptr())
    assert st == 0, _abi.status_string(st)
    st = lib.vtb_coeff_synthesize(ad.data_ptr(), smap.data_ptr(), Ks, Mx, My, Mt, W, t0, dt, Nt, Px, Py, Px, Py,
                                  None, ref.data_ptr(), 0, _abi.stream_ptr())
    assert st == 0, _abi.status_string(st)
    assert torch.isfinite(u).all()
    err = float((u - ref).abs().max() / ref.abs().max())
    assert err <= 1e-12, err
