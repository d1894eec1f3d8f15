"""Parity at the shape the headline is measured on (GPU).

The GPU configuration (64x64 px, Mx=My=6, Mt=8, K=1921, 768 Gabor + 256
centre-surround RFs, IAF b~U(2,4)) over 0.4 s: one full temporal period of
the Dirichlet space (2 pi Mt / Wt), so the window's coefficient system has
full rank (1921 kept) as the 1 s clip's does, with ~9.4k spike intervals,
small enough for the oracle's n x n pseudoinverse on the host.

Checked against the oracle (vtem/ensemble_encode.py:438-552 for the scan;
vtem/vtdm.py:630-652 and vtem/utils/linalg.py:591-631 for the decode):
  * spike times of the mixed bank, bit-exact, on the same projection;
  * the decoder preparation (Ds, phi) of the mixed bank;
  * the plain n x n decode and the coefficient-space float64 decode,
    rel-L2 <= 1e-8;
  * the mixed-precision decoder exactly as the benchmark runs it (one
    float64 refinement sweep), >= 40 dB, and the same decoder when its
    single sweep is refused, which must fall back to float64 (<= 1e-8).
"""
import os

import numpy as np
import pytest
import torch

from oracle import vtem_oracle as O
from vtem_b200 import ensemble_encode, fast, spike_store, vrf, vtdm, vtem, workloads

pytestmark = pytest.mark.gpu

FRAMES = 4000          # 0.4 s at dt = 1e-4: one temporal period at Mt = 8, Wt = 2 pi 20


def _banks(w, shape, dx, dy, scale=1):
    g, c = w.gabor, w.cs
    gb = vrf.vrf_gabor(shape, dx=dx, dy=dy, scale=scale)
    gb.load_parameters(num_neurons=len(g.h_alpha), h_alpha=g.h_alpha, h_l=g.h_l, h_x0=g.h_x0, h_y0=g.h_y0,
                       h_ab=g.h_ab, KAPPA=g.KAPPA, h_gain=g.gain)
    cb = vrf.vrf_cs(shape, dx=dx, dy=dy, scale=scale)
    cb.load_parameters(num_neurons=len(c.h_alpha), h_alpha=c.h_alpha, h_x0=c.h_x0, h_y0=c.h_y0,
                       sigma_center=c.sigma_center, sigma_surround=c.sigma_surround, h_gain=c.gain)
    return vrf.vrf_bank([gb, cb])


@pytest.fixture(scope="module")
def c1():
    w = workloads.gpu_scale(frames=FRAMES)
    V = w.video(device="cuda")
    bank = _banks(w, (w.Py, w.Px), w.dx, w.dy)
    iaf = ensemble_encode.IAF_encode(w.N, w.dt)
    iaf.load_parameters(h_kappa=w.kappa, h_bias=w.bias, h_delta=w.delta, h_v0=w.v0)
    store, sp = vtem.VTEM_IAF(V, None, w.Wt, bank, w.Wx, w.Wy, dx=w.dx, dy=w.dy, fps=1.0 / w.dt, npinput=True,
                              iaf=iaf, return_spikes=True)
    L = bank.filter(V).cpu().numpy()                 # (F, N) float64 projection the scan read
    prep = vtdm.VTDM_prep(store, None, None, w.Mx, w.My)
    rd = spike_store.vtem_storage_read(store)
    rd.read_vrf_type()
    rd.read_num_neurons()
    rd.select_neurons([-0.5, 0.5, -0.5, 0.5])
    tk1, tk2, ind, kap, dl, bia, sig = rd.read_select_spikes([0.0, w.T])
    g, c = w.gabor, w.cs
    norm = np.ones(w.N)
    Ds, dirich, Dsw = O.prep_decoder_gabor(g.h_alpha, g.h_l, g.h_x0, g.h_y0, g.h_ab, g.KAPPA, g.gain, w.Mx, w.My,
                                           w.Wx, w.Wy, w.dx, w.dy, w.Px, w.Py, norm,
                                           cs=(c.h_alpha, c.h_x0, c.h_y0, c.sigma_center, c.sigma_surround, c.gain))
    uo, co, qo, Go, kept = O.decode_window(tk1, tk2, ind, kap, dl, bia, norm, Dsw, dirich, w.Wt, w.Mt, w.T, w.dt,
                                           rcond=w.rcond, threads=os.cpu_count())
    del Go
    return dict(w=w, store=store, sp=sp, L=L, prep=prep, spikes=(tk1, tk2, ind, kap, dl, bia),
                oracle=dict(Ds=Ds, dirich=dirich, u=uo, kept=kept))


def test_spikes_bitexact_mixed_bank(c1):
    w, store, sp = c1["w"], c1["store"], c1["sp"]
    enc = O.vtem_encode(c1["L"], w.dt, w.kappa, w.bias, w.delta, w.v0)
    assert store.refresh_interval == len(enc.block_counts)
    for b in range(len(enc.block_counts)):
        assert np.array_equal(store.spike_count[b], enc.block_counts[b])
        assert np.array_equal(store.spikes[b], enc.block_spikes[b])
    assert sp.near_threshold == enc.near_threshold
    print("intervals %d, near-threshold events %d" % (len(c1["spikes"][0]), enc.near_threshold))


def test_prep_mixed_bank_matches_oracle(c1):
    prep, o = c1["prep"], c1["oracle"]
    assert np.abs(prep.Ds.cpu().numpy() - o["Ds"]).max() < 1e-12 * np.abs(o["Ds"]).max()
    assert np.abs(prep.dirich.cpu().numpy() - o["dirich"]).max() < 1e-12 * np.abs(o["dirich"]).max()
    assert o["kept"] == fast.coefficient_count(c1["w"].Mx, c1["w"].My, c1["w"].Mt) == 1921


def _rel(u, uo):
    u = u.cpu().numpy() if isinstance(u, torch.Tensor) else u
    return float(np.linalg.norm(u.reshape(uo.shape) - uo) / np.linalg.norm(uo))


def test_plain_decode_matches_oracle(c1):
    w = c1["w"]
    u = vtdm.VTDM(c1["store"], None, None, 0.0, w.T, w.dt, w.Mx, Mt=w.Mt, rcond=w.rcond, output_format=2,
                  prep=c1["prep"])
    rel = _rel(u, c1["oracle"]["u"])
    assert rel <= 1e-8, rel


def test_coeff_f64_decode_matches_oracle(c1):
    w = c1["w"]
    u = vtdm.VTDM(c1["store"], None, None, 0.0, w.T, w.dt, w.Mx, Mt=w.Mt, rcond=w.rcond, output_format=2,
                  prep=c1["prep"], decoder="coeff", coeff_solver="auto")
    rel = _rel(u, c1["oracle"]["u"])
    assert rel <= 1e-8, rel


def _bench_decode(c1, sweeps):
    """The decoder as the benchmark drives it: device-resident spikes sorted
    by neuron, one ``decode`` call (the synthesis queued before the
    acceptance read, done again after a fallback)."""
    w, prep = c1["w"], c1["prep"]
    dec = fast.from_prep(prep, w.Wt, w.Mt, rcond=w.rcond, solver="mixed", mixed_sweeps=sweeps)
    d = tuple(torch.as_tensor(x, device="cuda") for x in c1["spikes"])
    u = dec.decode(*d, w.T, w.dt, assume_sorted=True)
    return dec, u


def test_mixed_one_sweep_as_benchmarked(c1):
    dec, u = _bench_decode(c1, 1)
    rel = _rel(u, c1["oracle"]["u"])
    snr = -20 * np.log10(rel)
    print("mixed, 1 sweep: %s, ratios %s, rel-L2 %.3g (%.1f dB)" % (dec.last_solver, dec.last_ratios, rel, snr))
    assert dec.last_solver == "mixed"
    assert snr >= 40.0, snr
    # the accepted single sweep leaves at most ~r^2 of the solution: well inside float64-level parity
    assert rel <= 1e-6, rel


def test_mixed_refused_sweep_falls_back(c1, monkeypatch):
    # an acceptance bar no single sweep can meet: the window must go to the float64 path
    monkeypatch.setattr(fast, "MIXED_TOL", 1e-60)
    dec, u = _bench_decode(c1, 1)
    assert dec.last_solver.startswith("mixed->"), dec.last_solver
    rel = _rel(u, c1["oracle"]["u"])
    assert rel <= 1e-8, rel
