"""Per-kernel parity of the CUDA path against the oracle and the golden
fixtures (GPU).  Integer and index outputs are compared bit for bit; float64
outputs within the tolerances stated per test (they come from different
summation orders and libm implementations only)."""
import os

import numpy as np
import pytest
import torch

from oracle import vtem_oracle as O
from vtem_b200 import _abi, dirichlet, ensemble_encode, linalg, neural_network, vrf

pytestmark = pytest.mark.gpu

dev = "cuda"


def g_load(golden_dir, name):
    return np.load(os.path.join(golden_dir, name))


def t(a, dtype=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device=dev)


def relerr(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


# ------------------------------------------------------------------ RF banks

def test_rf_gabor_cs_golden(golden_dir):
    g = g_load(golden_dir, "rf_dirichlet.npz")
    gb = vrf.vrf_gabor((20, 24), dx=1.0 / 24, dy=0.9 / 20)
    gb.load_parameters(num_neurons=6, h_alpha=g["h_alpha"], h_l=g["h_l"], h_x0=g["h_x0"], h_y0=g["h_y0"],
                       h_ab=g["h_ab"], KAPPA=2.5)
    gb.generate_visual_receptive_fields(x_start=-0.5, y_start=-0.45)
    got = gb.gabors.cpu().numpy().reshape(g["gabor"].shape)
    # tolerance: CUDA and glibc exp/sincos differ in the last ulps
    np.testing.assert_allclose(got, g["gabor"], rtol=0, atol=1e-13 * np.abs(g["gabor"]).max())
    cs = vrf.vrf_cs((20, 24), dx=1.0 / 24, dy=0.9 / 20)
    cs.load_parameters(num_neurons=6, h_alpha=g["h_alpha"], h_x0=g["h_x0"], h_y0=g["h_y0"], sigma_center=0.05,
                       sigma_surround=0.15)
    cs.generate_visual_receptive_fields(x_start=-0.5, y_start=-0.45)
    got = cs.filters.cpu().numpy().reshape(g["cs"].shape)
    np.testing.assert_allclose(got, g["cs"], rtol=0, atol=1e-13 * np.abs(g["cs"]).max())


def test_rf_filter_layouts():
    rng = np.random.default_rng(1)
    V = rng.standard_normal((37, 16, 20))
    gb = vrf.vrf_gabor((16, 20), dx=1 / 20, dy=1 / 16)
    N = 45
    gb.load_parameters(num_neurons=N, h_alpha=rng.uniform(0.05, 0.2, N), h_l=rng.uniform(0, 3, N),
                       h_x0=rng.uniform(-.4, .4, N), h_y0=rng.uniform(-.4, .4, N),
                       h_ab=rng.integers(0, 2, N).astype(np.int32), KAPPA=2.5, h_gain=rng.uniform(0.5, 2, N))
    rf = O.gabor_rf(gb.h_alpha, gb.h_l, gb.h_x0, gb.h_y0, gb.h_ab, 20, 16, 1.0, 1.0, -0.5, -0.5, 2.5, gb.h_gain)
    ref = O.rf_filter(V, rf, 1 / 20, 1 / 16)
    a = gb.filter(V).cpu().numpy()
    b = gb.filter(V, out_layout="neuron").cpu().numpy()
    assert relerr(a, ref) < 1e-13
    assert np.array_equal(a, b.T)


# ------------------------------------------------------------------ IAF

def _iaf(N, dt, kap, bia, dl, v0, rt=None):
    enc = ensemble_encode.IAF_encode(N, dt) if rt is None else ensemble_encode.IAF_encode_rt(N, dt)
    if rt is None:
        enc.load_parameters(h_kappa=kap, h_bias=bia, h_delta=dl, h_v0=v0)
    else:
        sig, dv, randn = rt
        enc.load_parameters(h_kappa=kap, h_bias=bia, h_delta=dl, h_sigma=sig, h_delta_value=dv, h_v0=v0)
        enc.randn_source = lambda shape: randn.reshape(shape)
    return enc


def test_iaf_golden_bitexact(golden_dir):
    g = g_load(golden_dir, "iaf.npz")
    L, dt = g["L"], float(g["dt"])
    F, N = L.shape
    enc = _iaf(N, dt, g["kappa"], g["bias"], g["delta"], g["v0"])
    spk, cnt = enc.encode(L)
    assert np.array_equal(cnt, g["lin_counts"])
    assert np.array_equal(np.concatenate(spk), g["lin_spikes"])          # bit-exact spike times
    assert np.array_equal(enc.d_v0.cpu().numpy(), g["lin_v0"])
    assert np.array_equal(enc.d_time_count.cpu().numpy(), g["lin_tc"])
    # time-major and neuron-major inputs give identical results
    enc2 = _iaf(N, dt, g["kappa"], g["bias"], g["delta"], g["v0"])
    spk2, cnt2 = enc2.encode(np.ascontiguousarray(L.T), layout="neuron")
    assert np.array_equal(np.concatenate(spk2), g["lin_spikes"])


def test_iaf_rt_golden_bitexact(golden_dir):
    g = g_load(golden_dir, "iaf.npz")
    L, dt = g["L"], float(g["dt"])
    F, N = L.shape
    enc = _iaf(N, dt, g["kappa"], g["bias"], g["delta"], g["v0"], rt=(g["sigma"], g["delta_value0"], g["randn"]))
    spk, cnt = enc.encode(L)
    assert np.array_equal(cnt, g["rt_counts"])
    assert np.array_equal(np.concatenate(spk), g["rt_spikes"])
    assert np.array_equal(enc.d_delta_value.cpu().numpy(), g["rt_dv"])


def test_iaf_blocks_match_reference_block_loop(golden_dir):
    g = g_load(golden_dir, "iaf.npz")
    L, dt = g["L"], float(g["dt"])
    F, N = L.shape
    enc = _iaf(N, dt, g["kappa"], g["bias"], g["delta"], g["v0"])
    sp = enc.encode_blocks(L, block_frames=101)
    per = ensemble_encode.spikes_per_block(sp, F)
    assert np.array_equal(per, g["blk_counts"])
    times, steps, cnt = sp.to_host_lists()
    flat = []
    for b in range(per.shape[0]):
        for n in range(N):
            sel = (steps[n] // 100) == b
            flat.append(times[n][sel])
    assert np.array_equal(np.concatenate(flat), g["blk_spikes"])
    assert np.array_equal(enc.d_v0.cpu().numpy(), g["blk_v0"])
    assert (enc.d_time_count.cpu().numpy() == 0).all()


@pytest.mark.parametrize("N,F,seed", [(1, 5, 0), (33, 1000, 1), (130, 3001, 2)])
def test_iaf_steps_bitexact_random(N, F, seed):
    rng = np.random.default_rng(seed)
    L = rng.standard_normal((F, N)) * 0.5
    L[F // 3:F // 3 + 7] -= 3.0                       # negative-slope crossings
    kap = rng.uniform(0.7, 1.3, N)
    bia = rng.uniform(0.5, 1.5, N)
    dl = rng.uniform(0.002, 0.02, N)
    v0 = rng.uniform(0, 1, N) * dl
    dt = 1e-3
    enc = O.vtem_encode(L, dt, kap, bia, dl, v0, block_frames=101)
    e = _iaf(N, dt, kap, bia, dl, v0)
    sp = e.encode_blocks(L, block_frames=101)
    times, steps, cnt = sp.to_host_lists()
    ref_steps = np.concatenate(enc.block_steps) if enc.block_steps else np.zeros(0, np.int32)
    got_steps = []
    for b in range(len(enc.block_counts)):
        for n in range(N):
            got_steps.append(steps[n][(steps[n] // 100) == b])
    assert np.array_equal(np.concatenate(got_steps), ref_steps)            # sample indices bit-exact
    assert sp.near_threshold == enc.near_threshold


def test_iaf_overflow_reported():
    N, F = 4, 200
    L = np.full((F, N), 50.0)
    e = _iaf(N, 1e-3, np.ones(N), np.ones(N), np.full(N, 1e-4), np.zeros(N))
    with pytest.raises(ValueError, match="exceeded"):
        e.encode(L)


# ------------------------------------------------------------------ Dirichlet

def test_ds_dirich_dsw_golden(golden_dir):
    g = g_load(golden_dir, "rf_dirichlet.npz")
    gb = vrf.vrf_gabor((16, 16), dx=1 / 16, dy=1 / 16, scale=4)
    gb.load_parameters(num_neurons=6, h_alpha=g["h_alpha"], h_l=g["h_l"], h_x0=g["h_x0"], h_y0=g["h_y0"],
                       h_ab=g["h_ab"], KAPPA=2.5)
    Ds = gb.compute_Ds(3, 2)
    np.testing.assert_allclose(Ds.cpu().numpy(), g["Ds"], rtol=0, atol=1e-13 * np.abs(g["Ds"]).max())
    dirich = gb.compute_dirich_space_fft(t(g["Ds"], torch.complex128), 3, 2, 16, 14, 1.0, 14 / 16, 0, 0)
    np.testing.assert_allclose(dirich.cpu().numpy(), g["dirich"], rtol=0, atol=1e-13 * np.abs(g["dirich"]).max())
    Dsw = gb.compute_Dsw(t(g["Ds"], torch.complex128), 3, 2, g["norm"])
    np.testing.assert_allclose(Dsw.cpu().numpy(), g["Dsw"], rtol=1e-13, atol=1e-15 * np.abs(g["Dsw"]).max())


def test_q_G_golden(golden_dir):
    g = g_load(golden_dir, "decode.npz")
    N = len(g["kappa"])
    cp = dirichlet.dirichlet(N, g["tk1"], g["tk2"], g["ind"], g["kappa"], g["delta"], g["bias"], g["norm"],
                             float(g["Wt"]), int(g["Mt"]))
    cp.compute_q()
    # q = kappa*delta - bias*dt cancels; FMA contraction moves it by a few ulps of its terms
    np.testing.assert_allclose(cp.d_q.cpu().numpy().ravel(), g["q"], rtol=0, atol=1e-15 * np.abs(g["q"]).max())
    cp.compute_G(g["Dsw"])
    G = cp.d_G.cpu().numpy()
    np.testing.assert_allclose(G, g["G"], rtol=0, atol=1e-13 * np.abs(g["G"]).max())
    cp.compute_G(g["Dsw"], lamb=0.05)
    np.testing.assert_allclose(cp.d_G.cpu().numpy(), g["G_lamb"], rtol=0, atol=1e-13 * np.abs(g["G"]).max())
    cp.compute_G(g["Dsw"], lower_only=True)
    Gl = cp.d_G.cpu().numpy()
    il = np.tril_indices(len(g["q"]))
    np.testing.assert_allclose(Gl[il], g["G"][il], rtol=0, atol=1e-13 * np.abs(g["G"]).max())


def test_pinv_rnn_reconstruct_golden(golden_dir):
    g = g_load(golden_dir, "decode.npz")
    Gt = t(g["G"])
    q = t(g["q"]).reshape(-1, 1)
    c = linalg.solve_eq_sym(Gt.clone(), q, rcond=1e-8)
    assert relerr(c.cpu().numpy().ravel(), g["c"]) < 1e-6      # pinv of an ill-conditioned G
    co, _ = O.solve_eq_sym(g["G"], g["q"], 1e-8)
    assert relerr(c.cpu().numpy().ravel(), co) < 1e-6
    cr = neural_network.rnn3(t(g["G"]), q, dt=1e-6, alpha=5000, steps=60)
    np.testing.assert_allclose(cr.cpu().numpy().ravel(), g["c_rnn"], rtol=1e-11, atol=1e-14)
    N = len(g["kappa"])
    cp = dirichlet.dirichlet(N, g["tk1"], g["tk2"], g["ind"], g["kappa"], g["delta"], g["bias"], g["norm"],
                             float(g["Wt"]), int(g["Mt"]))
    cp.d_q = t(g["c"]).reshape(-1, 1)
    u = cp.reconstruct(g["dirich"], [0, 0.02], 2e-3).cpu().numpy()
    ur = g["u"].reshape(u.shape)
    assert np.abs(u - ur).max() <= 1e-11 * np.abs(ur).max()


def test_reconstruct_unsorted_spikes():
    rng = np.random.default_rng(4)
    N, n, Mt = 9, 300, 6
    tk1 = rng.uniform(0, 0.3, n)
    tk2 = tk1 + rng.uniform(0.004, 0.02, n)
    ind = rng.integers(0, N, n).astype(np.int32)
    c = rng.standard_normal(n)
    norm = rng.uniform(0.5, 1, N)
    dirich = rng.standard_normal((N, 6, 5))
    tt = np.arange(0, 0.05, 1e-3)
    W = 2 * np.pi * 20 / Mt
    ref = O.reconstruct_direct(dirich, tk1, tk2, c, tt, ind, norm, Mt, W)
    cp = dirichlet.dirichlet(N, tk1, tk2, ind, np.ones(N), np.ones(N), np.ones(N), norm, 2 * np.pi * 20, Mt)
    cp.d_q = t(c).reshape(-1, 1)
    u = cp.reconstruct(dirich, [0, 0.05], 1e-3).cpu().numpy().reshape(ref.shape)
    assert np.abs(u - ref).max() <= 1e-11 * np.abs(ref).max()


def test_bad_shapes_raise():
    with pytest.raises(ValueError):
        dirichlet.dirichlet(3, np.zeros(0), np.zeros(0), np.zeros(0, np.int32), 1, 1, 1, 1, 1.0, 2)
    G = torch.zeros((3, 4), dtype=torch.float64, device=dev)
    with pytest.raises(ValueError):
        linalg.solve_eq_sym(G, torch.zeros((3, 1), dtype=torch.float64, device=dev))
    with pytest.raises(TypeError):
        linalg.solve_eq_sym(torch.zeros((3, 3), dtype=torch.float32, device=dev),
                            torch.zeros((3, 1), dtype=torch.float64, device=dev))


def _block_counts_oracle(L, dt, kap, bia, dl, v0, B):
    r = O.vtem_encode(L, dt, kap, bia, dl, v0, block_frames=B, max_spike_per_block=100000)
    return np.array(r.block_counts)          # (blocks, N)


@pytest.mark.parametrize("rate_scale", [0.9, 1.1])
def test_iaf_block_limit_matches_reference_rule(rate_scale):
    """The kernel's per-block spike limit raises exactly when a block's count
    reaches ceil(block length / avg_rate) (ensemble_encode.py:163-164)."""
    rng = np.random.default_rng(5)
    N, F, B, dt = 6, 1210, 101, 1e-4
    L = rng.standard_normal((F, N)) * 0.2
    kap, bia = np.ones(N), np.full(N, 2.0)
    dl = np.full(N, 2.0 * dt * 3)            # about one spike every 3 samples
    v0 = rng.uniform(0, 1, N) * dl
    cnt = _block_counts_oracle(L, dt, kap, bia, dl, v0, B)
    sizes = np.array([min(B, F - s) for s in range(0, F, B - 1)])[:cnt.shape[0]]
    # an avg_rate whose limit sits just above / below the busiest block
    worst = np.max(cnt.max(axis=1) / sizes)
    avg_rate = 1.0 / (worst * rate_scale)
    expect_raise = bool((cnt.max(axis=1) >= np.ceil(sizes / avg_rate)).any())
    enc = _iaf(N, dt, kap, bia, dl, v0)
    if expect_raise:
        with pytest.raises(ValueError):
            enc.encode_blocks(L, block_frames=B, avg_rate=avg_rate)
    else:
        sp = enc.encode_blocks(L, block_frames=B, avg_rate=avg_rate)
        assert np.array_equal(ensemble_encode.spikes_per_block(sp, F), cnt)


def test_iaf_small_buffer_retry_is_exact():
    """A neuron that outgrows the first-try buffer triggers the full-buffer
    rerun from the saved state: same spikes, same v0 as one full-buffer run."""
    rng = np.random.default_rng(8)
    N, F, B, dt = 40, 3000, 101, 1e-4
    L = rng.standard_normal((F, N)) * 0.3
    kap, bia = np.ones(N), np.full(N, 3.0)
    dl = np.full(N, 0.02)
    dl[7] = 3.0 * dt * 4                     # ~750 spikes: beyond the first-try buffer
    v0 = rng.uniform(0, 1, N) * dl
    small = 64 + -(-F // ensemble_encode.SMALL_CAP_STRIDE)
    a = _iaf(N, dt, kap, bia, dl, v0)
    sa = a.encode_blocks(L, block_frames=B)
    b = _iaf(N, dt, kap, bia, dl, v0)
    sb = b.encode_blocks(L, block_frames=B, cap=int(np.ceil(F / 0.1)))
    ca, cb = sa.count.cpu().numpy(), sb.count.cpu().numpy()
    assert ca[7] > small and np.array_equal(ca, cb)
    ta, tb = sa.to_host_lists(), sb.to_host_lists()
    for n in range(N):
        assert np.array_equal(ta[0][n], tb[0][n]) and np.array_equal(ta[1][n], tb[1][n])
    assert torch.equal(a.d_v0, b.d_v0)


@pytest.mark.parametrize("N,F,seed,dmin,dmax", [(64, 10000, 5, 0.01, 0.04), (40, 4000, 6, 0.002, 0.01),
                                                (96, 10000, 7, 0.03, 0.2)])
def test_iaf_long_scan_bitexact(N, F, seed, dmin, dmax):
    """Long scans at dt = 1e-4 with sparse spiking: whole 32-step chunks
    without a crossing (the register-chain path, with frame-block
    boundaries inside chunks) and chunks with crossings; spike times, steps,
    final membrane values and near-threshold counts bit-exact against the
    reference-order C oracle."""
    rng = np.random.default_rng(seed)
    L = rng.standard_normal((F, N)) * 0.5
    kap = rng.uniform(0.7, 1.3, N)
    bia = rng.uniform(2.0, 4.0, N)
    dl = rng.uniform(dmin, dmax, N)
    v0 = rng.uniform(0, 1, N) * dl
    dt = 1e-4
    enc = O.vtem_encode(L, dt, kap, bia, dl, v0, block_frames=101)
    e = _iaf(N, dt, kap, bia, dl, v0)
    sp = e.encode_blocks(L, block_frames=101)
    times, steps, cnt = sp.to_host_lists()
    got_t, got_s = [], []
    for b in range(len(enc.block_counts)):
        for n in range(N):
            sel = (steps[n] // 100) == b
            got_t.append(times[n][sel])
            got_s.append(steps[n][sel])
    assert np.array_equal(np.concatenate(got_s), np.concatenate(enc.block_steps))
    assert np.array_equal(np.concatenate(got_t), np.concatenate(enc.block_spikes))
    assert np.array_equal(e.d_v0.cpu().numpy(), enc.v0)
    assert sp.near_threshold == enc.near_threshold
