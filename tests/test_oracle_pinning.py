"""The CPU oracle against the reference itself (CPU, no GPU).

Golden fixtures in tests/golden/ are outputs of the reference's own kernels
compiled for the host (tests/golden/make_golden.py).  When the host build of
the reference (oracle/_ref) is present, the restatement is also checked live
against it on fresh random inputs.
"""
import os

import numpy as np
import pytest

from oracle import ref_runner as R
from oracle import vtem_oracle as O


def load(golden_dir, name):
    return np.load(os.path.join(golden_dir, name))


def test_rf_dirichlet_golden(golden_dir):
    g = load(golden_dir, "rf_dirichlet.npz")
    ha, hl, hx, hy, hab = g["h_alpha"], g["h_l"], g["h_x0"], g["h_y0"], g["h_ab"]
    gab = O.gabor_rf(ha, hl, hx, hy, hab, 24, 20, 1.0, 0.9, -0.5, -0.45, 2.5)
    np.testing.assert_allclose(gab.reshape(g["gabor"].shape), g["gabor"], rtol=0, atol=1e-13)
    cs = O.cs_rf(ha, hx, hy, 24, 20, 1.0, 0.9, -0.5, -0.45, 0.05, 0.15)
    np.testing.assert_allclose(cs.reshape(g["cs"].shape), g["cs"], rtol=1e-13, atol=1e-12)
    fine = O.gabor_rf(ha, hl, hx, hy, hab, 64, 64, 1.0, 1.0, -0.5, -0.5, 2.5)
    Ds = O.compute_Ds(fine, 3, 2, (1 / 64) ** 2)
    np.testing.assert_allclose(Ds, g["Ds"], rtol=0, atol=1e-14)
    dirich = O.compute_dirich_space_fft(g["Ds"], 3, 2, 16, 14, 16, 16)
    np.testing.assert_allclose(dirich, g["dirich"], rtol=0, atol=1e-13)
    Dsw = O.compute_Dsw(g["Ds"], g["norm"])
    np.testing.assert_allclose(Dsw, g["Dsw"], rtol=1e-14, atol=1e-16)


def test_iaf_golden_bitexact(golden_dir):
    g = load(golden_dir, "iaf.npz")
    L, dt = g["L"], float(g["dt"])
    F, N = L.shape
    cap = int(np.ceil(F / 0.1))
    v0, tc = g["v0"].copy(), np.zeros(N)
    r = O.iaf_encode_block(L, dt, g["kappa"], g["bias"], g["delta"], v0, tc, cap)
    assert np.array_equal(r.spike_count, g["lin_counts"])
    assert np.array_equal(np.concatenate(r.spikes), g["lin_spikes"])  # bit-exact
    assert np.array_equal(v0, g["lin_v0"]) and np.array_equal(tc, g["lin_tc"])
    v0, tc, dv = g["v0"].copy(), np.zeros(N), g["delta_value0"].copy()
    r = O.iaf_encode_block(L, dt, g["kappa"], g["bias"], g["delta"], v0, tc, cap, randn=g["randn"],
                           sigma=g["sigma"], delta_value=dv)
    assert np.array_equal(r.spike_count, g["rt_counts"])
    assert np.array_equal(np.concatenate(r.spikes), g["rt_spikes"])
    assert np.array_equal(v0, g["rt_v0"]) and np.array_equal(dv, g["rt_dv"])


def test_iaf_golden_blocks(golden_dir):
    g = load(golden_dir, "iaf.npz")
    enc = O.vtem_encode(g["L"], float(g["dt"]), g["kappa"], g["bias"], g["delta"], g["v0"], block_frames=101)
    assert np.array_equal(np.stack(enc.block_counts), g["blk_counts"])
    assert np.array_equal(np.concatenate(enc.block_spikes), g["blk_spikes"])
    assert np.array_equal(enc.v0, g["blk_v0"])


def test_negative_branch_exercised(golden_dir):
    g = load(golden_dir, "iaf.npz")
    y = (g["L"] + g["bias"]) / g["kappa"]
    neg = (y[1:] < 0) & (y[:-1] > 0)
    assert neg.any()


def test_decode_golden(golden_dir):
    g = load(golden_dir, "decode.npz")
    tk1, tk2, ind = g["tk1"], g["tk2"], g["ind"]
    q = O.compute_q(tk1, tk2, ind, g["kappa"], g["delta"], g["bias"], g["norm"])
    np.testing.assert_array_equal(q, g["q"])
    G = O.compute_G(tk1, tk2, ind, g["Dsw"], float(g["Wt"]), int(g["Mt"]))
    np.testing.assert_allclose(G, g["G"], rtol=1e-13, atol=1e-18)
    Gl = O.compute_G(tk1, tk2, ind, g["Dsw"], float(g["Wt"]), int(g["Mt"]), lamb=0.05)
    np.testing.assert_allclose(Gl, g["G_lamb"], rtol=1e-13, atol=1e-18)
    c, kept = O.solve_eq_sym(g["G"], g["q"], 1e-8)
    # reference pinv (SVD) vs eigh restatement: same truncated solution
    assert np.linalg.norm(c - g["c"]) / np.linalg.norm(g["c"]) < 1e-6
    cr = O.rnn3(g["G"], g["q"], 1e-6, 5000, 60)
    np.testing.assert_allclose(cr, g["c_rnn"], rtol=1e-12, atol=1e-15)
    Mt, Wt = int(g["Mt"]), float(g["Wt"])
    u = O.reconstruct_direct(g["dirich"], tk1, tk2, g["c"], g["t"], ind, g["norm"], Mt, Wt / Mt)
    ur = g["u"].reshape(u.shape)
    assert np.abs(u - ur).max() <= 1e-12 * np.abs(ur).max()
    uf = O.reconstruct_factored(g["dirich"], tk1, tk2, g["c"], g["t"], ind, g["norm"], Mt, Wt / Mt)
    assert np.abs(uf.reshape(u.shape) - ur).max() <= 1e-12 * np.abs(ur).max()


def test_pinv_matches_svd_definition():
    rng = np.random.default_rng(5)
    A = rng.standard_normal((40, 12))
    G = A @ A.T
    q = G @ rng.standard_normal(40)
    c, kept = O.solve_eq_sym(G, q, 1e-8)
    assert kept == 12
    U, S, _ = np.linalg.svd(G)
    keep = S > S[0] * 1e-8
    c2 = U[:, keep] @ ((U[:, keep].T @ q) / S[keep])
    assert np.linalg.norm(c - c2) / np.linalg.norm(c2) < 1e-10


@pytest.mark.skipif(not R.available(), reason="host build of the reference (oracle/_ref) not present")
def test_live_against_reference_kernels():
    rng = np.random.default_rng(11)
    N, F = 10, 700
    L = rng.standard_normal((F, N)) * 0.8
    kap = rng.uniform(0.7, 1.3, N)
    bia = rng.uniform(0.6, 1.0, N)
    dl = rng.uniform(0.005, 0.02, N)
    v0 = rng.uniform(0, 1, N) * dl
    a, b = v0.copy(), np.zeros(N)
    r = O.iaf_encode_block(L, 1e-3, kap, bia, dl, a, b, int(np.ceil(F / 0.1)))
    c, d = v0.copy(), np.zeros(N)
    sp, cnt = R.iaf_encode(L, 1e-3, kap, bia, dl, c, d)
    assert np.array_equal(r.spike_count, cnt)
    for x, y in zip(r.spikes, sp):
        assert np.array_equal(x, y)
    assert np.array_equal(a, c) and np.array_equal(b, d)
