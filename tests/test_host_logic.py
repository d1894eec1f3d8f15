"""Host-side logic of the path against the oracle (CPU)."""
import numpy as np

from oracle import vtem_oracle as O
from vtem_b200 import spike_store as ss
from vtem_b200 import vtdm, vtem, workloads


def _store_from_blocks(counts, spikes, R, N):
    st = ss.vtem_storage(None, N, "gabor")
    st.write_video_attributes(1.0, 2.0, 3.0, 8, 8, 0.1, 0.1)
    st.vrf["alpha"].append(np.ones(N))
    st.vrf["x0"].append(np.linspace(-0.3, 0.3, N))
    st.vrf["y0"].append(np.linspace(0.2, -0.2, N))
    st.vrf["l"].append(np.zeros(N))
    st.vrf["ab"].append(np.zeros(N, np.int32))
    st.data["vrf/KAPPA"] = np.array(2.5)
    st.iaf["kappa"].append(np.ones(N))
    st.iaf["delta"].append(np.ones(N))
    st.iaf["bias"].append(np.ones(N))
    st.iaf["sigma"].append(np.zeros(N))
    st.write_refresh_interval(R)
    for c, s in zip(counts, spikes):
        st.write_spike_in_timebin(c, s)
    st.close()
    return st


def _random_blocks(rng, N, nb, R):
    counts, spikes = [], []
    for b in range(nb):
        c = rng.integers(0, 5, N).astype(np.int32)
        s = np.concatenate([np.sort(rng.uniform(0, R, k)) for k in c]) if c.sum() else np.zeros(0)
        counts.append(c)
        spikes.append(s)
    return counts, spikes


def test_read_select_spikes_matches_oracle():
    rng = np.random.default_rng(3)
    N, nb, R = 7, 9, 0.01
    counts, spikes = _random_blocks(rng, N, nb, R)
    st = _store_from_blocks(counts, spikes, R, N)
    rd = ss.vtem_storage_read(st)
    rd.read_vrf_type()
    rd.read_num_neurons()
    for dom in ([-0.5, 0.5, -0.5, 0.5], [-0.1, 0.35, -0.5, 0.5]):
        rd.select_neurons(dom)
        choose, sx, sy = O.select_neurons(rd.d["vrf/x0"], rd.d["vrf/y0"], dom)
        assert np.array_equal(rd.choose, choose)
        for tf in ([0.0, 0.09], [0.013, 0.05], [0.02, 0.021]):
            a = rd.read_select_spikes(tf)
            b = O.read_select_spikes(counts, spikes, R, choose, tf)
            for x, y in zip(a[:3], b):
                assert np.array_equal(x, y)


def test_wx_wy_swapped_in_store():
    st = ss.vtem_storage(None, 1, "cs")
    st.write_video_attributes(1.0, 2.0, 3.0, 8, 8, 0.1, 0.1)
    st.close()
    rd = ss.vtem_storage_read(st)
    Wt, Wx, Wy = rd.read_video_attributes()[:3]
    assert (Wt, Wx, Wy) == (1.0, 3.0, 2.0)


def test_block_schedule_and_frames():
    assert vtem.one_time_frames(2000) == 101
    assert vtem.one_time_frames(50) == 51
    assert O.block_schedule(2000)[-1] == (1900, 2000)
    assert len(O.block_schedule(2000)) == 20
    assert len(O.block_schedule(2001)) == 21


def test_norm_and_period_grid():
    h = vtdm._norm_from_sigma(np.array([1.0, 2.0, 1.0]), np.array([0.0, 0.5, 0.25]))
    np.testing.assert_allclose(h, O.h_norm_from_sigma(np.array([1.0, 2.0, 1.0]), np.array([0.0, 0.5, 0.25])))
    assert vtdm.period_grid(3, 3, 2 * np.pi * 3, 2 * np.pi * 3, 1 / 32, 1 / 32) == O.rf_period_grid(
        3, 3, 2 * np.pi * 3, 2 * np.pi * 3, 1 / 32, 1 / 32)
    assert O.default_Mt(2 * np.pi * 20) == 40


def test_small_workload_video_and_bank():
    w = workloads.small()
    V = w.video().numpy()
    assert V.shape == (2000, 32, 32)
    assert abs(np.abs(V).max() - 1.0) < 1e-12
    a = w.coeffs
    # Hermitian coefficients inside the ellipse give a real video
    assert np.allclose(a, np.conj(a[::-1, ::-1, ::-1]))
    Vo = O.bandlimited_video(a * w.scale, w.Mx, w.My, w.Mt, w.Wx, w.Wy, w.Wt, w.Px, w.Py, 1.0, 1.0, 50, w.dt)
    np.testing.assert_allclose(V[:50], Vo, atol=1e-12)
    g = w.gabor
    rf = O.gabor_rf(g.h_alpha, g.h_l, g.h_x0, g.h_y0, g.h_ab, w.Px, w.Py, 1.0, 1.0, -0.5, -0.5, g.KAPPA, g.gain)
    np.testing.assert_allclose(np.sqrt((rf ** 2).sum((1, 2)) * w.dx * w.dy), 1.0, rtol=1e-12)
    assert w.N == 128 and (w.delta > 0).all()


TEMPORAL_CASES = [
    (0.0, 1.0, 0.001, True, 0.2),
    (0.0, 0.1, 0.001, True, 0.04),
    (0.0, 0.1, 0.001, False, None),     # one window (4-sample overlap unused)
    (0.0, 0.5, 0.01, True, None),       # default interval 20 dt
    (0.1, 0.7, 0.001, True, 0.13),      # offset start, ragged last window
    (0.0, 0.05, 0.01, True, 0.05),      # 5-sample interval: no overlap
    (0.0, 0.2, 0.01, True, 0.07),
    (0.0, 0.33, 0.001, True, 0.1),
]


def test_temporal_plan_matches_oracle():
    """Window schedule and Hann cross-fade of VTDM's temporal stitching
    (vtdm.py:573-699) against the oracle's loop, on random window contents."""
    import torch
    rng = np.random.default_rng(3)
    for st, et, dt, stitching, si in TEMPORAL_CASES:
        recs = {}

        def dec(s, e):
            if (s, e) not in recs:
                recs[(s, e)] = rng.standard_normal((int(round((e - s) / dt)), 3, 2))
            return recs[(s, e)]

        uo, wins = O.temporal_stitch(dec, st, et, dt, stitching, si)
        plan = vtdm.temporal_plan(st, et, dt, stitching, si)
        assert plan.windows == wins
        u = torch.empty((plan.total_l, 3, 2), dtype=torch.float64)
        prev = None
        for i, (s, e) in enumerate(plan.windows):
            u, prev = vtdm.place_window(u, plan, i, torch.as_tensor(dec(s, e)), prev)
        np.testing.assert_allclose(u.numpy(), uo, rtol=0, atol=1e-15)


def test_spatial_tiles_match_oracle():
    """decode_video's tile walk and 2-D Hann weights (vtdm.py:214-302)
    against the oracle's, and the weights' partition of unity over the
    domain, including tiles wider than the domain and ragged last tiles."""
    for Px, Py, ix, iy in [(32, 32, 20, 20), (64, 48, 30, 20), (97, 33, 30, 7), (128, 100, 96, 96),
                           (48, 24, 200, 8), (33, 100, 30, 96), (64, 64, 64, 64)]:
        dx = dy = 1.0 / Px
        dom = [-Px * dx / 2, Px * dx / 2, -Py * dy / 2, Py * dy / 2]
        a = O.spatial_tile_walk(dom, Px, Py, [ix, iy], dx, dy)
        b = vtdm.spatial_tiles(Px, Py, (ix, iy), dom, dx, dy)
        assert len(a) == len(b)
        cover = np.zeros((Py, Px))
        for (da, r0, r1, c0, c1, wa), (db, rows, wb) in zip(a, b):
            assert da == db and (r0, r1, c0, c1) == rows
            np.testing.assert_array_equal(wa, wb)
            cover[r0:r1, c0:c1] += wa
        np.testing.assert_allclose(cover, 1.0, rtol=0, atol=1e-12)


def test_frame_pair_synthesis_identity():
    """The harmonics kernel's frame-pair form (csrc/synth_rank.cu): with the
    weights rotated to a block's centre angle th_c, A_m = a_m cos(m th_c) +
    b_m sin(m th_c) and B_m = b_m cos(m th_c) - a_m sin(m th_c), the frames
    at th_c -+ phi are E -+ O (E = sum_m A_m cos(m phi), O = sum_m B_m
    sin(m phi)).  Checked against u[f] = H_0 + sum_m (cos(m W t_f) a_m +
    sin(m W t_f) b_m) for even and odd frame ranges, with the kernel's
    pairing of frames lo = fb + half - 1 + odd - j and hi = fb + half + j."""
    rng = np.random.default_rng(5)
    Mt, W, t0, dt = 8, 2 * np.pi * 2.5, 0.013, 1e-4
    H = rng.standard_normal((7, 2 * Mt + 1))
    m = np.arange(1, Mt + 1)
    for fb, nfr in ((0, 10), (3, 11), (17, 1), (5, 2)):
        f = np.arange(fb, fb + nfr)
        th = W * (t0 + f * dt)
        direct = H[:, 0][None, :] + np.cos(np.outer(th, m)) @ H[:, 1::2].T + np.sin(np.outer(th, m)) @ H[:, 2::2].T
        half, odd = nfr >> 1, nfr & 1
        thc = W * (t0 + (fb + 0.5 * (nfr - 1)) * dt)
        a, b = H[:, 1::2], H[:, 2::2]
        A = a * np.cos(m * thc) + b * np.sin(m * thc)
        B = b * np.cos(m * thc) - a * np.sin(m * thc)
        got = np.full((nfr, H.shape[0]), np.nan)
        for j in range(half + odd):
            phi = W * dt * (j + (0.0 if odd else 0.5))
            E = H[:, 0] + A @ np.cos(m * phi)
            Od = B @ np.sin(m * phi)
            lo, hi = fb + half - 1 + odd - j, fb + half + j
            got[hi - fb] = E + Od
            got[lo - fb] = E - Od
        assert np.isfinite(got).all()
        assert np.abs(got - direct).max() <= 1e-12 * np.abs(direct).max()


def test_pinv_buckets_partition_sizes():
    """Padded-size buckets of the batched eigen-pseudoinverse: every system
    in exactly one bucket, padded to the bucket's largest size, and no
    system smaller than PINV_BUCKET_RATIO of it (bounded padding work)."""
    from vtem_b200 import batch
    rng = np.random.default_rng(11)
    for Ks in ([1921], [91, 91, 91], list(rng.integers(91, 1922, 97)), [100, 69, 70, 49, 48, 1000]):
        out = batch.pinv_buckets(Ks)
        seen = sorted(i for _, idx in out for i in idx)
        assert seen == list(range(len(Ks)))
        for top, idx in out:
            assert top == max(Ks[i] for i in idx)
            assert all(Ks[i] >= batch.PINV_BUCKET_RATIO * top for i in idx)
        tops = [t for t, _ in out]
        assert tops == sorted(tops, reverse=True)
