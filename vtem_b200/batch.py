"""Batched decoding of many independent clips (uneven durations, RF counts
and Dirichlet orders) on one GPU.

Each clip is decoded in the Dirichlet coefficient space exactly as
:class:`vtem_b200.fast.CoeffDecoder` does alone; the batch only changes how
the work is scheduled:

* per-clip temporal/Kronecker Gram kernels are issued round-robin on
  several CUDA streams so that small clips overlap on the device;
* clips whose systems have the same size K are factorised and solved by one
  batched Cholesky call per group (``vtb_herm_chol_batched``), the grouped
  counterpart of the reference's per-window ``solve_eq_sym``
  (vtem/vtdm.py:645-648); a clip whose factorisation fails (its
  pseudoinverse would truncate) is solved alone by the eigen-pseudoinverse;
* synthesis kernels are again spread over the streams.

The result of every clip equals its stand-alone decode (tests check it).
"""
from __future__ import annotations

from collections import defaultdict

import numpy as np
import torch

from . import fast
from ._abi import call, dptr, stream_ptr


class ClipProblem(object):
    """One clip to decode: decoder prep (Ds, norm, grid), orders, spike
    intervals (sorted by neuron) and IAF parameters, all on the device."""

    def __init__(self, prep, Wt, Mt, tk1, tk2, ind, kappa, delta, bias, T, dt, rcond=1e-8):
        self.prep, self.Wt, self.Mt = prep, float(Wt), int(Mt)
        self.tk1, self.tk2, self.ind = tk1, tk2, ind
        self.kappa, self.delta, self.bias = kappa, delta, bias
        self.T, self.dt, self.rcond = float(T), float(dt), float(rcond)
        self.Nt = len(np.arange(0, T, dt))

    @property
    def voxels(self):
        return self.Nt * self.prep.decPx * self.prep.decPy


class BatchDecoder(object):
    def __init__(self, problems, streams=8):
        self.problems = list(problems)
        self.decs = [fast.from_prep(p.prep, p.Wt, p.Mt, rcond=p.rcond, solver="chol") for p in self.problems]
        dev = self.decs[0].M.device
        self.streams = [torch.cuda.Stream(device=dev) for _ in range(streams)]
        self.groups = defaultdict(list)
        for i, (p, d) in enumerate(zip(self.problems, self.decs)):
            if int(p.tk1.numel()) >= d.K:
                self.groups[d.K].append(i)
        self.ptrs = {}
        for K, idx in self.groups.items():
            mp = torch.as_tensor([self.decs[i].M.data_ptr() for i in idx], dtype=torch.int64, device=dev)
            bp = torch.as_tensor([self.decs[i].a.data_ptr() for i in idx], dtype=torch.int64, device=dev)
            infos = torch.zeros(len(idx), dtype=torch.int32, device=dev)
            sinfo = torch.zeros(1, dtype=torch.int32, device=dev)
            self.ptrs[K] = (mp, bp, infos, sinfo)
        self.outs = [torch.empty((p.Nt, p.prep.decPy, p.prep.decPx), dtype=torch.float64, device=dev)
                     for p in self.problems]
        self.fallbacks = 0

    def run(self, timing=False):
        """Decode every clip; returns the list of videos.  With ``timing`` the
        device time of the three phases is left in ``self.phase_ms`` (the
        caller synchronises before reading it)."""
        main = torch.cuda.current_stream()
        start = torch.cuda.Event(enable_timing=timing)
        start.record(main)
        for s in self.streams:
            s.wait_event(start)
        # phase 1: per-clip Gram and right-hand side, round-robin over the
        # streams; clips with fewer intervals than coefficients are solved in
        # the (smaller) spike space right away
        for i, (p, d) in enumerate(zip(self.problems, self.decs)):
            st = self.streams[i % len(self.streams)]
            with torch.cuda.stream(st):
                s = stream_ptr()
                n = int(p.tk1.numel())
                if n < d.K:
                    d._solve_spike_space(s, (p.tk1, p.tk2, p.ind, n, p.kappa, p.delta, p.bias))
                    continue
                call("vtb_coeff_temporal_gram", dptr(p.tk1), dptr(p.tk2), dptr(p.ind), n, d.N, dptr(p.kappa),
                     dptr(p.delta), dptr(p.bias), dptr(d.norm), d.Mt, d.W, dptr(d.Wn), dptr(d.gn), s)
                d._build_M(s)
                d.a.copy_(d.b)
                d.last_solver = "chol-batched"
        joins = []
        for st in self.streams:
            e = torch.cuda.Event()
            e.record(st)
            joins.append(e)
        for e in joins:
            main.wait_event(e)
        t1 = torch.cuda.Event(enable_timing=timing)
        t1.record(main)
        # phase 2: one batched Cholesky per group of equally sized systems
        # (clips with fewer intervals than unknowns are singular: eigen path)
        s = stream_ptr()
        for K, idx in self.groups.items():
            mp, bp, infos, sinfo = self.ptrs[K]
            rc = self.problems[idx[0]].rcond * fast.CHOL_MARGIN
            call("vtb_herm_chol_batched", mp.data_ptr(), K, bp.data_ptr(), K, len(idx), rc, dptr(infos), dptr(sinfo),
                 s)
        # clips whose factorisation was refused (their pseudoinverse truncates):
        # batched eigen-pseudoinverse per system size (one host check)
        keys = list(self.groups)
        if keys:
            flags = torch.cat([self.ptrs[K][2] for K in keys]).ne(0).cpu().tolist()
            bad_by_K, o = defaultdict(list), 0
            for K in keys:
                idx = self.groups[K]
                bad_by_K[K] = [self.decs[idx[j]] for j in range(len(idx)) if flags[o + j]]
                o += len(idx)
            eig_infos = [fast.pinv_batched(ds) for ds in bad_by_K.values() if ds]
            self.fallbacks = sum(len(ds) for ds in bad_by_K.values())
            if eig_infos and int(torch.cat(eig_infos).ne(0).sum()) != 0:
                raise fast.VtbError("vtb_herm_pinv_batched", fast.VTB_NOT_CONVERGED)
        done = torch.cuda.Event(enable_timing=timing)
        done.record(main)
        # phase 3: synthesis
        for i, (p, d) in enumerate(zip(self.problems, self.decs)):
            st = self.streams[i % len(self.streams)]
            st.wait_event(done)
            with torch.cuda.stream(st):
                d.synthesize(d.a, p.T, p.dt, out=self.outs[i])
        for st in self.streams:
            e = torch.cuda.Event()
            e.record(st)
            main.wait_event(e)
        if timing:
            end = torch.cuda.Event(enable_timing=True)
            end.record(main)
            self._phase_events = (start, t1, done, end)
        return self.outs

    @property
    def phase_ms(self):
        """(Gram/right-hand sides, solves, synthesis) device milliseconds of
        the last ``run(timing=True)``."""
        e = self._phase_events
        return tuple(e[i].elapsed_time(e[i + 1]) for i in range(3))


def encode_clip_problem(w, device="cuda", keep_video=False, video=None, precision="f64"):
    """Encode workload ``w`` on the GPU (RF projection + IAF block loop) and
    prepare its coefficient-space decode: the ClipProblem of the clip (and
    the video when ``keep_video``).  ``video`` (a device tensor, float64 or
    float32) replaces the clip's generated video; ``precision`` is the RF
    projection's ("f64", or "bf16x3" on the tensor cores)."""
    from . import ensemble_encode, spike_store, vrf, vtdm
    V = w.video(device=device) if video is None else video
    banks, dbanks = [], []
    rfSx, rfSy, rfPx, rfPy = vtdm.period_grid(w.Mx, w.My, w.Wx, w.Wy, w.dx, w.dy)
    if w.gabor is not None:
        g = w.gabor
        for shape, kw, lst in (((w.Py, w.Px), dict(dx=w.dx, dy=w.dy), banks),
                               ((rfPy, rfPx), dict(dx=rfSx / rfPx, dy=rfSy / rfPy, scale=4), dbanks)):
            b = vrf.vrf_gabor(shape, **kw)
            b.load_parameters(num_neurons=len(g.h_alpha), h_alpha=g.h_alpha, h_l=g.h_l, h_x0=g.h_x0, h_y0=g.h_y0,
                              h_ab=g.h_ab, KAPPA=g.KAPPA, h_gain=g.gain)
            lst.append(b)
    if w.cs is not None:
        c = w.cs
        for shape, kw, lst in (((w.Py, w.Px), dict(dx=w.dx, dy=w.dy), banks),
                               ((rfPy, rfPx), dict(dx=rfSx / rfPx, dy=rfSy / rfPy, scale=4), dbanks)):
            b = vrf.vrf_cs(shape, **kw)
            b.load_parameters(num_neurons=len(c.h_alpha), h_alpha=c.h_alpha, h_x0=c.h_x0, h_y0=c.h_y0,
                              sigma_center=c.sigma_center, sigma_surround=c.sigma_surround, h_gain=c.gain)
            lst.append(b)
    bank = vrf.vrf_bank(banks) if len(banks) > 1 else banks[0]
    L = bank.filter(V, out_layout="neuron", precision=precision)
    iaf = ensemble_encode.IAF_encode(w.N, w.dt)
    iaf.load_parameters(h_kappa=w.kappa, h_bias=w.bias, h_delta=w.delta, h_v0=w.v0)
    B = min(101, w.F + 1)
    sp = iaf.encode_blocks(L, block_frames=B, layout="neuron")
    tk1, tk2, ind = spike_store.device_pairs(sp, w.T)
    Ds = torch.cat([b.compute_Ds(w.Mx, w.My) for b in dbanks], 0)
    Px1 = int(np.round(dbanks[0].Sx / w.dx))
    Py1 = int(np.round(dbanks[0].Sy / w.dy))
    prep = vtdm.PrepResult(Ds, None, None, np.ones(w.N), w.Mx, w.My, w.Px, w.Py, Px1, Py1)
    dev = V.device
    t = lambda x: torch.as_tensor(x, device=dev)
    prob = ClipProblem(prep, w.Wt, w.Mt, tk1, tk2, ind, t(w.kappa), t(w.delta), t(w.bias), w.T, w.dt, w.rcond)
    if keep_video:
        return prob, V
    return prob
