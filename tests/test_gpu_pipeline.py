"""End-to-end parity on the small configuration (32x32, 2000 samples, 128
Gabor RFs): VTEM_IAF -> VTDM_prep -> VTDM on the GPU against the oracle's
restatement of the same calls (GPU)."""
import numpy as np
import pytest
import torch

from oracle import vtem_oracle as O
from vtem_b200 import ensemble_encode, vrf, vtdm, vtem, workloads

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small():
    return workloads.small()


def _encode(w, V):
    g = w.gabor
    rf = vrf.vrf_gabor((w.Py, w.Px), dx=w.dx, dy=w.dy)
    rf.load_parameters(num_neurons=w.N, h_alpha=g.h_alpha, h_l=g.h_l, h_x0=g.h_x0, h_y0=g.h_y0, h_ab=g.h_ab,
                       KAPPA=g.KAPPA, h_gain=g.gain)
    iaf = ensemble_encode.IAF_encode(w.N, w.dt)
    iaf.load_parameters(h_kappa=w.kappa, h_bias=w.bias, h_delta=w.delta, h_v0=w.v0)
    store, sp = vtem.VTEM_IAF(V, None, w.Wt, rf, w.Wx, w.Wy, dx=w.dx, dy=w.dy, fps=1.0 / w.dt, npinput=True,
                              iaf=iaf, return_spikes=True)
    return store, sp, rf


def test_encode_matches_oracle_on_same_projection(small):
    w = small
    V = w.video(device="cuda")
    store, sp, rf = _encode(w, V)
    L = rf.filter(V).cpu().numpy()                            # GPU projection
    g = w.gabor
    rfo = O.gabor_rf(g.h_alpha, g.h_l, g.h_x0, g.h_y0, g.h_ab, w.Px, w.Py, 1.0, 1.0, -0.5, -0.5, g.KAPPA, g.gain)
    Lo = O.rf_filter(V.cpu().numpy(), rfo, w.dx, w.dy)
    assert np.linalg.norm(L - Lo) / np.linalg.norm(Lo) < 1e-13
    enc = O.vtem_encode(L, w.dt, w.kappa, w.bias, w.delta, w.v0)   # oracle IAF on the same input
    rd = store
    assert rd.refresh_interval == len(enc.block_counts)
    for b in range(len(enc.block_counts)):
        assert np.array_equal(rd.spike_count[b], enc.block_counts[b])
        assert np.array_equal(rd.spikes[b], enc.block_spikes[b])       # bit-exact spike times
    assert sp.near_threshold == enc.near_threshold
    # oracle IAF on the oracle projection: identical spike counts unless a
    # crossing sits within rounding of a sample boundary (counted above)
    enc2 = O.vtem_encode(Lo, w.dt, w.kappa, w.bias, w.delta, w.v0)
    s1 = np.concatenate(enc.block_steps)
    s2 = np.concatenate(enc2.block_steps)
    assert len(s1) == len(s2) and (s1 != s2).sum() <= enc2.near_threshold


@pytest.mark.parametrize("rcond", [1e-10, 1e-8])
def test_decode_matches_oracle(small, rcond):
    w = small
    V = w.video(device="cuda")
    store, sp, rf = _encode(w, V)
    prep = vtdm.VTDM_prep(store, None, None, w.Mx, w.My)
    u = vtdm.VTDM(store, None, None, 0.0, w.T, w.dt, w.Mx, Mt=w.Mt, rcond=rcond, output_format=2, prep=prep)
    # oracle decode of the very same spikes
    rd = vtem_read(store)
    rd.select_neurons([-0.5, 0.5, -0.5, 0.5])
    tk1, tk2, ind, kap, dl, bia, sig = rd.read_select_spikes([0.0, w.T])
    g = w.gabor
    norm = np.ones(w.N)
    Ds, dirich, Dsw = O.prep_decoder_gabor(g.h_alpha, g.h_l, g.h_x0, g.h_y0, g.h_ab, g.KAPPA, g.gain, w.Mx, w.My,
                                           w.Wx, w.Wy, w.dx, w.dy, w.Px, w.Py, norm)
    assert np.abs(prep.Ds.cpu().numpy() - Ds).max() < 1e-12 * np.abs(Ds).max()
    assert np.abs(prep.dirich.cpu().numpy() - dirich).max() < 1e-12 * np.abs(dirich).max()
    uo, c, q, G, kept = O.decode_window(tk1, tk2, ind, kap, dl, bia, norm, Dsw, dirich, w.Wt, w.Mt, w.T, w.dt,
                                        rcond=rcond)
    rel = np.linalg.norm(u - uo) / np.linalg.norm(uo)
    assert rel <= 1e-8, rel
    Vh = V.cpu().numpy()
    snr = -20 * np.log10(np.linalg.norm(u - Vh) / np.linalg.norm(Vh))
    # the encoder samples the RFs on the video grid, the decoder on a 4x grid over one period; RFs
    # touching the domain edge differ by a few percent between the two sums, which caps the SNR
    assert snr > 20


def test_rnn_decode_matches_oracle(small):
    w = small
    V = w.video(device="cuda")
    store, sp, rf = _encode(w, V)
    prep = vtdm.VTDM_prep(store, None, None, w.Mx, w.My)
    T = 0.05
    u = vtdm.VTDM(store, None, None, 0.0, T, w.dt, w.Mx, Mt=w.Mt, rnn=True, alpha=5000, steps=200,
                  output_format=2, prep=prep)
    rd = vtem_read(store)
    rd.select_neurons([-0.5, 0.5, -0.5, 0.5])
    tk1, tk2, ind, kap, dl, bia, sig = rd.read_select_spikes([0.0, T])
    norm = np.ones(w.N)
    Dsw = prep.Dsw.cpu().numpy()
    dirich = prep.dirich.cpu().numpy()
    uo, *_ = O.decode_window(tk1, tk2, ind, kap, dl, bia, norm, Dsw, dirich, w.Wt, w.Mt, T, w.dt,
                             rnn=(1e-6, 5000, 200))
    assert np.linalg.norm(u - uo) / np.linalg.norm(uo) < 1e-10


@pytest.mark.parametrize("decoder", ["plain", "coeff", "batch"])
def test_stitched_decode_matches_oracle(small, decoder):
    """Temporal stitching (vtdm.py:573-699): three overlapping windows, each
    decoded alone and cross-faded, against the oracle's window loop.  The
    pseudoinverse cut is the reference's own (rcond 1e-8, vtdm.py:648): the
    short windows' Grams are ill-conditioned enough that a 1e-10 cut lets
    rounding through at the 1e-7 level."""
    w = small
    V = w.video(device="cuda")
    store, sp, rf = _encode(w, V)
    prep = vtdm.VTDM_prep(store, None, None, w.Mx, w.My)
    u = vtdm.VTDM(store, None, None, 0.0, 0.1, w.dt, w.Mx, Mt=w.Mt, stitching=True, stitch_interval=0.04,
                  output_format=2, prep=prep, decoder=decoder)
    rd = vtem_read(store)
    rd.select_neurons([-0.5, 0.5, -0.5, 0.5])
    norm = np.ones(w.N)
    Dsw = prep.Dsw.cpu().numpy()
    dirich = prep.dirich.cpu().numpy()

    def window(s, e):
        tk1, tk2, ind, kap, dl, bia, sig = rd.read_select_spikes([s, e])
        return O.decode_window(tk1, tk2, ind, kap, dl, bia, norm, Dsw, dirich, w.Wt, w.Mt,
                               round((e - s) / w.dt) * w.dt, w.dt, rcond=1e-8)[0]

    uo, wins = O.temporal_stitch(window, 0.0, 0.1, w.dt, True, 0.04)
    assert len(wins) == 3 and u.shape == uo.shape == (1000, 32, 32)
    rel = np.linalg.norm(u - uo) / np.linalg.norm(uo)
    assert rel <= 1e-8, rel


@pytest.mark.parametrize("decoder", ["plain", "coeff", "batch"])
def test_spatial_stitching_matches_oracle(small, decoder):
    """decode_video with spatial stitching (vtdm.py:181-309): 2 x 2 tiles of
    20 x 20 pixels over the 32 x 32 frame, each prepared on its own domain
    (neurons centred in it, positions relative to its centre) and decoded
    alone, blended with the tiles' Hann weights; against the oracle's tile
    walk over the oracle's per-tile preparation and decode."""
    w = small
    V = w.video(device="cuda")
    store, sp, rf = _encode(w, V)
    T = 0.05
    u = vtdm.decode_video(store, None, None, 0.0, T, w.dt, w.Mx, Mt=w.Mt, spatial_stitching=True,
                          spatial_interval=[20, 20], output_format=2, decoder=decoder)
    rd = vtem_read(store)
    g = w.gabor
    dom = [-0.5, 0.5, -0.5, 0.5]

    def tile(d):
        choose, sx, sy = O.select_neurons(g.h_x0, g.h_y0, d)
        tPx = int(np.round((d[1] - d[0]) / w.dx))
        tPy = int(np.round((d[3] - d[2]) / w.dy))
        norm = np.ones(len(choose))
        Ds, dirich, Dsw = O.prep_decoder_gabor(g.h_alpha[choose], g.h_l[choose], g.h_x0[choose] - sx,
                                               g.h_y0[choose] - sy, g.h_ab[choose], g.KAPPA, g.gain[choose],
                                               w.Mx, w.My, w.Wx, w.Wy, w.dx, w.dy, tPx, tPy, norm)
        rd.select_neurons(d)
        assert np.array_equal(rd.choose, choose)
        tk1, tk2, ind, kap, dl, bia, sig = rd.read_select_spikes([0.0, T])
        return O.decode_window(tk1, tk2, ind, kap, dl, bia, norm, Dsw, dirich, w.Wt, w.Mt, T, w.dt,
                               rcond=1e-8)[0]

    uo = O.spatial_stitch(tile, dom, 32, 32, [20, 20], w.dx, w.dy)
    assert u.shape == uo.shape == (500, 32, 32)
    rel = np.linalg.norm(u - uo) / np.linalg.norm(uo)
    assert rel <= 1e-8, rel


def test_vtdmb_matches_vtdm(small, tmp_path):
    """VTDM_prepb + VTDMb (vtdm.py:701-1071: Ds written by the prep, the
    cross-weights formed per window by compute_Gb) reproduce VTDM_prep +
    VTDM, through the files the preps write; decode_video's precompute=False
    takes that path."""
    w = small
    V = w.video(device="cuda")
    store, sp, rf = _encode(w, V)
    T = 0.05
    prep = vtdm.VTDM_prep(store, str(tmp_path / "dsw.npy"), str(tmp_path / "dirich.npy"), w.Mx, w.My)
    u = vtdm.VTDM(store, str(tmp_path / "dsw.npy"), str(tmp_path / "dirich.npy"), 0.0, T, w.dt, w.Mx, Mt=w.Mt,
                  output_format=2)
    vtdm.VTDM_prepb(store, str(tmp_path / "ds.npy"), str(tmp_path / "dirich_b.npy"), w.Mx, w.My)
    ub = vtdm.VTDMb(store, str(tmp_path / "ds.npy"), str(tmp_path / "dirich_b.npy"), 0.0, T, w.dt, w.Mx, Mt=w.Mt,
                    output_format=2)
    assert np.abs(ub - u).max() <= 1e-12 * np.abs(u).max()
    kw = dict(Mt=w.Mt, spatial_stitching=True, spatial_interval=[24, 24], output_format=2)
    ua = vtdm.decode_video(store, None, None, 0.0, T, w.dt, w.Mx, **kw)
    uc = vtdm.decode_video(store, None, None, 0.0, T, w.dt, w.Mx, precompute=False, **kw)
    assert np.abs(uc - ua).max() <= 1e-12 * np.abs(ua).max()


@pytest.mark.parametrize("decoder", ["plain", "coeff"])
def test_random_threshold_decode_matches_oracle(small, decoder):
    """Random-threshold IAF (ensemble_encode.py:175-333) with per-neuron
    sigma, decoded with the reference's weighting norm = 1/(kappa sigma)
    normalised to its maximum (vtdm.py:408-413, :634-638): the decoder's
    cross-weights and q carry the non-uniform norm; against the oracle's
    decode of the same spikes with the oracle's norm."""
    w = small
    V = w.video(device="cuda")
    g = w.gabor
    rf = vrf.vrf_gabor((w.Py, w.Px), dx=w.dx, dy=w.dy)
    rf.load_parameters(num_neurons=w.N, h_alpha=g.h_alpha, h_l=g.h_l, h_x0=g.h_x0, h_y0=g.h_y0, h_ab=g.h_ab,
                       KAPPA=g.KAPPA, h_gain=g.gain)
    rng = np.random.default_rng(11)
    sigma = w.delta * rng.uniform(0.01, 0.03, w.N)
    iaf = ensemble_encode.IAF_encode_rt(w.N, w.dt)
    iaf.randn_source = lambda shape: rng.standard_normal(shape)
    iaf.load_parameters(h_kappa=w.kappa, h_bias=w.bias, h_delta=w.delta, h_sigma=sigma,
                        h_delta_value=w.delta + sigma * rng.standard_normal(w.N), h_v0=w.v0)
    store = vtem.VTEM_IAF(V, None, w.Wt, rf, w.Wx, w.Wy, dx=w.dx, dy=w.dy, fps=1.0 / w.dt, npinput=True, iaf=iaf)
    T = 0.05
    prep = vtdm.VTDM_prep(store, None, None, w.Mx, w.My)
    u = vtdm.VTDM(store, None, None, 0.0, T, w.dt, w.Mx, Mt=w.Mt, output_format=2, prep=prep, decoder=decoder)
    norm = O.h_norm_from_sigma(w.kappa, sigma)
    assert norm.min() < 0.9                       # the weighting is not uniform
    np.testing.assert_allclose(prep.h_norm, norm, rtol=1e-15)
    rd = vtem_read(store)
    rd.select_neurons([-0.5, 0.5, -0.5, 0.5])
    tk1, tk2, ind, kap, dl, bia, sig = rd.read_select_spikes([0.0, T])
    Ds, dirich, Dsw = O.prep_decoder_gabor(g.h_alpha, g.h_l, g.h_x0, g.h_y0, g.h_ab, g.KAPPA, g.gain, w.Mx, w.My,
                                           w.Wx, w.Wy, w.dx, w.dy, w.Px, w.Py, norm)
    uo = O.decode_window(tk1, tk2, ind, kap, dl, bia, norm, Dsw, dirich, w.Wt, w.Mt, T, w.dt, rcond=1e-8)[0]
    rel = np.linalg.norm(u - uo) / np.linalg.norm(uo)
    assert rel <= 1e-8, rel


def vtem_read(store):
    from vtem_b200 import spike_store as ss
    rd = ss.vtem_storage_read(store)
    rd.read_vrf_type()
    rd.read_num_neurons()
    return rd
