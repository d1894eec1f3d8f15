"""Batched decoding of many independent clips (uneven durations, RF counts
and Dirichlet orders) on one GPU, in mixed precision.

Each clip is decoded in the Dirichlet coefficient space as
:class:`vtem_b200.fast.CoeffDecoder` (``solver="mixed"``) does alone; the
batch changes how the work is scheduled:

* per clip, the temporal Gram and the right-hand side are issued
  round-robin on several CUDA streams; the tensor-core Kronecker Grams of all
  clips run as ONE grouped GEMM launch (``GroupedGram``, tile width chosen by
  timing), then each is scattered into its real symmetric float32 system;
* clips whose systems have the same size K are factorised by one batched
  float32 Cholesky per group (``vtb_sym_factor_batched``), and every clip's
  triangular solves run in one launch (``vtb_sym_potrs_batched``, one CTA per
  clip), the grouped counterpart of the reference's per-window solve
  (vtem/vtdm.py:645-648); float64 refinement sweeps against each clip's
  exact residual follow;
* that whole sequence, up to the acceptance check, is captured once as a
  CUDA graph and replayed per run (``graph=True``);
* one host check then reads every clip's flags: a clip whose pseudoinverse
  might truncate (factorisation refused, or refinement not contracting) is
  decoded by the float64 path -- Cholesky, else the eigen-pseudoinverse --
  on a pool of host threads with their own streams, so that the
  latency-bound eigensolvers of different clips overlap on the device;
  clips with fewer intervals than coefficients take the spike-space
  pseudoinverse the same way;
* synthesis kernels are again spread over the streams (a second graph).

The result of every clip equals its stand-alone decode within the mixed
decoder's tolerance, and the reference's pseudoinverse within 1e-8 (tests).
"""
from __future__ import annotations

from collections import defaultdict
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import torch

from . import autotune, fast
from ._abi import call, dptr, lib, stream_ptr

TRSV_DESC = np.dtype([("L", "<u8"), ("Dinv", "<u8"), ("x", "<u8"), ("ld", "<i8"), ("K", "<i4"), ("pad", "<i4")])


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

    @property
    def spikes(self):
        return (self.tk1, self.tk2, self.ind, int(self.tk1.numel()), self.kappa, self.delta, self.bias)


class GroupedGram(object):
    """The tensor-core Kronecker Gram GEMMs of many mixed decoders
    (C_p = the three split-bf16 products of L_p and R_p, uneven sizes) as
    ONE grouped launch (``vtb_tc_gemm_grouped_x3``); its tile width is
    chosen by timing the candidates on the first eager run (``autotune``)."""

    WIDTHS = (64, 128, 256)

    def __init__(self, decs):
        self.decs = list(decs)
        self.n = len(self.decs)
        dev = self.decs[0].M.device
        u64 = np.uint64
        self.args = [
            np.array([d.Lsplit.data_ptr() for d in self.decs], u64), np.array([2 * d.npairs for d in self.decs], np.int32),
            np.array([d.Rsplit.data_ptr() for d in self.decs], u64), np.array([d.NE for d in self.decs], np.int32),
            np.array([d.Kh for d in self.decs], np.int32), np.array([d.C.data_ptr() for d in self.decs], u64),
            np.array([d.ldc for d in self.decs], np.int64),
            np.array([d._stat_ptr(7) for d in self.decs], u64)]
        self.desc = {}
        self.tiles = {}
        nbytes = int(lib().vtb_tc_group_bytes(self.n))
        for bn in self.WIDTHS:
            host = np.zeros(nbytes, np.uint8)
            tiles = np.zeros(1, np.int32)
            a = self.args
            call("vtb_tc_group_build_x3", host.ctypes.data, self.n, a[0].ctypes.data, a[1].ctypes.data, a[2].ctypes.data,
                 a[3].ctypes.data, a[4].ctypes.data, a[5].ctypes.data, a[6].ctypes.data, a[7].ctypes.data, bn,
                 tiles.ctypes.data)
            self.desc[bn] = torch.as_tensor(host).to(dev)
            self.tiles[bn] = int(tiles[0])
        self.bn = None

    def _launch(self, bn, s):
        call("vtb_tc_gemm_grouped_x3", dptr(self.desc[bn]), self.n, self.tiles[bn], bn, s)

    def launch(self, s):
        if self.bn is None:
            if torch.cuda.is_current_stream_capturing():
                self.bn = 64
            else:
                times = {}
                for bn in self.WIDTHS:
                    self._launch(bn, s)
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record()
                    for _ in range(3):
                        self._launch(bn, s)
                    e1.record()
                    e1.synchronize()
                    times[bn] = e0.elapsed_time(e1) / 3
                self.bn = min(times, key=times.get)
                self.timings = times
        self._launch(self.bn, s)


def stage_mixed_pre(d, p, s):
    """Device work of one clip before its Gram GEMM: W_n, g_n, b and its real
    form br, and the split-bf16 operand of the temporal Grams."""
    tk1, tk2, ind, n, kap, dl, bi = p.spikes
    d.stat.zero_()
    call("vtb_coeff_temporal_gram", dptr(tk1), dptr(tk2), dptr(ind), n, d.N, dptr(kap), dptr(dl), dptr(bi),
         dptr(d.norm), d.Mt, d.W, dptr(d.Wn), dptr(d.gn), s)
    call("vtb_coeff_rhs", dptr(d.d), d.N, d.Ks, dptr(d.gn), d.Kt, dptr(d.b), s)
    call("vtb_coeff_realify_vec", dptr(d.b), d.K, 1, dptr(d.br), s)
    call("vtb_coeff_wn_sym", dptr(d.Wn), d.N, d.Kt, dptr(d.Rsplit), s)


def stage_mixed_post(d, s):
    """After the Gram GEMM: the float32 real system and xr = br."""
    call("vtb_coeff_real_scatter", dptr(d.C), d.ldc, d.Ks, d.Kt, dptr(d.Mr32), d.ld32, 0, s)
    d.xr.copy_(d.br)


def stage_mixed(d, p, s):
    """Device work of one clip up to its factorisation (no synchronisation):
    W_n, g_n, b and its real form br, the tensor-core Gram scattered into the
    float32 real system Mr32, and xr = br."""
    tk1, tk2, ind, n, kap, dl, bi = p.spikes
    K = d.K
    d.stat.zero_()
    call("vtb_coeff_temporal_gram", dptr(tk1), dptr(tk2), dptr(ind), n, d.N, dptr(kap), dptr(dl), dptr(bi),
         dptr(d.norm), d.Mt, d.W, dptr(d.Wn), dptr(d.gn), s)
    call("vtb_coeff_rhs", dptr(d.d), d.N, d.Ks, dptr(d.gn), d.Kt, dptr(d.b), s)
    call("vtb_coeff_realify_vec", dptr(d.b), K, 1, dptr(d.br), s)
    call("vtb_coeff_wn_sym", dptr(d.Wn), d.N, d.Kt, dptr(d.Rsplit), s)
    autotune.gemm_bf16_tuned(dptr(d.Lsplit), 2 * d.npairs, dptr(d.Rsplit), d.NE, d.Kh, dptr(d.C), d.ldc, 1, 0, 1.0, 0,
                             d._stat_ptr(7), s, x3=True)
    call("vtb_coeff_real_scatter", dptr(d.C), d.ldc, d.Ks, d.Kt, dptr(d.Mr32), d.ld32, 0, s)
    d.xr.copy_(d.br)


def sweep_residual(d, p, s):
    """One clip's part of a refinement sweep before its solve: a from xr, the
    exact float64 residual, and its real form rr."""
    tk1, tk2, ind, n, kap, dl, bi = p.spikes
    K = d.K
    call("vtb_coeff_unrealify_vec", dptr(d.xr), K, 1, dptr(d.a), 0, s)
    call("vtb_coeff_residual", dptr(tk1), dptr(tk2), dptr(ind), n, d.N, dptr(kap), dptr(dl), dptr(bi),
         dptr(d.norm), d.Mt, d.W, dptr(d.d), d.Ks, dptr(d.a), dptr(d.gres), dptr(d.r), s)
    call("vtb_coeff_realify_vec", dptr(d.r), K, 1, dptr(d.rr), s)


def sweep_update(d, i, s):
    """After the solve of rr: record ||rr|| / ||xr|| and xr += rr."""
    call("vtb_norm_ratio", dptr(d.rr), dptr(d.xr), d.K, d._stat_ptr(3 + min(i, 3)), s)
    call("vtb_daxpy1", dptr(d.xr), dptr(d.rr), d.K, s)


def trsv_descs(entries, device):
    """Device array of vtb_trsv_desc for (L, Dinv, x, ld, K) tuples."""
    a = np.zeros(len(entries), TRSV_DESC)
    for i, (L, Dinv, x, ld, K) in enumerate(entries):
        a[i] = (L, Dinv, x, ld, K, 0)
    return torch.as_tensor(np.frombuffer(a.tobytes(), np.uint8).copy()).to(device)


class MixedSolvePlan(object):
    """Grouped float32 Cholesky, batched triangular solves and float64
    refinement sweeps of a set of mixed decoders whose systems were staged by
    :func:`stage_mixed` (each with at least K intervals).  ``launch`` only
    enqueues device work (capturable in a CUDA graph); ``check`` reads every
    system's flags and correction ratios in one synchronising copy and
    returns the indices (into ``decs``) that need the float64 path."""

    def __init__(self, decs, probs, sweeps, streams):
        self.decs, self.probs = list(decs), list(probs)
        self.sweeps = int(sweeps)
        self.streams = streams
        dev = self.decs[0].M.device
        self.device = dev
        by_K = defaultdict(list)
        for i, d in enumerate(self.decs):
            by_K[d.K].append(i)
        self.groups = []
        l = lib()
        dinv_of = {}
        for K, idx in sorted(by_K.items()):
            B = len(idx)
            nf = int(l.vtb_sym_dinv_floats(K))
            g = {
                "K": K, "idx": idx, "ld": self.decs[idx[0]].ld32,
                "mptrs": torch.as_tensor([self.decs[i].Mr32.data_ptr() for i in idx], dtype=torch.int64, device=dev),
                "dinv": torch.empty((B, nf), dtype=torch.float32, device=dev),
                "infos": torch.zeros(B, dtype=torch.int32, device=dev),
                "flags": torch.zeros(B, dtype=torch.int32, device=dev),
                "piv": torch.zeros(2 * B, dtype=torch.float64, device=dev),
            }
            for j, i in enumerate(idx):
                dinv_of[i] = g["dinv"][j]
            self.groups.append(g)
        self.Kmax = max(d.K for d in self.decs)
        self.desc_x = trsv_descs([(d.Mr32.data_ptr(), dinv_of[i].data_ptr(), d.xr.data_ptr(), d.ld32, d.K)
                                  for i, d in enumerate(self.decs)], dev)
        self.desc_r = trsv_descs([(d.Mr32.data_ptr(), dinv_of[i].data_ptr(), d.rr.data_ptr(), d.ld32, d.K)
                                  for i, d in enumerate(self.decs)], dev)
        self.order = [i for g in self.groups for i in g["idx"]]

    def _fork(self):
        main = torch.cuda.current_stream(self.device)
        ev = torch.cuda.Event()
        ev.record(main)
        for st in self.streams:
            st.wait_event(ev)
        return main

    def _join(self, main):
        for st in self.streams:
            ev = torch.cuda.Event()
            ev.record(st)
            main.wait_event(ev)

    def launch(self):
        s = stream_ptr()
        for g in self.groups:
            rc = self.probs[g["idx"][0]].rcond * fast.CHOL_MARGIN
            call("vtb_sym_factor_batched", g["mptrs"].data_ptr(), g["ld"], g["K"], len(g["idx"]), rc,
                 dptr(g["dinv"]), dptr(g["infos"]), dptr(g["flags"]), dptr(g["piv"]), s)
        n = len(self.decs)
        call("vtb_sym_potrs_batched", dptr(self.desc_x), n, self.Kmax, s)
        for i in range(self.sweeps):
            main = self._fork()
            for c, (d, p) in enumerate(zip(self.decs, self.probs)):
                with torch.cuda.stream(self.streams[c % len(self.streams)]):
                    sweep_residual(d, p, stream_ptr())
            self._join(main)
            call("vtb_sym_potrs_batched", dptr(self.desc_r), n, self.Kmax, stream_ptr())
            main = self._fork()
            for c, d in enumerate(self.decs):
                with torch.cuda.stream(self.streams[c % len(self.streams)]):
                    sweep_update(d, i, stream_ptr())
            self._join(main)
        s = stream_ptr()
        for d in self.decs:
            call("vtb_coeff_unrealify_vec", dptr(d.xr), d.K, 1, dptr(d.a), 0, s)

    def gather(self):
        """Device tensors (flags, pivots, per-system status words) for
        :meth:`evaluate`; copying them to the host is the caller's choice
        (synchronous in :meth:`check`, asynchronous in the serving loop)."""
        flags = torch.cat([g["flags"] for g in self.groups])
        piv = torch.cat([g["piv"] for g in self.groups])
        stats = torch.stack([d.stat for d in self.decs])
        return flags, piv, stats

    def evaluate(self, flags, piv, stats):
        """Indices of the systems the float64 path must decode, from host
        copies of :meth:`gather`'s tensors; records pivots and correction
        ratios on each decoder."""
        flags, piv, stats = (np.asarray(x) for x in (flags, piv, stats))
        bad = []
        fl = dict(zip(self.order, flags))
        pv = {i: (float(piv[2 * j]), float(piv[2 * j + 1])) for j, i in enumerate(self.order)}
        for i, d in enumerate(self.decs):
            tc_err = int(stats[i].view(np.int32)[14])
            if tc_err != 0:
                raise fast.VtbError("vtb_tc_gemm_bf16", tc_err)
            d.last_pivots = pv[i]
            d.last_ratios = [float(x) for x in stats[i][3:3 + min(self.sweeps, 4)]]
            if fl[i] != 0 or not d._mixed_converged(d.last_ratios):
                bad.append(i)
            else:
                d.last_solver = "mixed-batched"
        return bad

    def check(self):
        """Indices of the systems the float64 path must decode (one
        synchronising read)."""
        return self.evaluate(*(t.cpu().numpy() for t in self.gather()))


# Eigen-pseudoinverses of systems of different sizes are grouped into batches
# of one padded size: a system of size K joins a batch of size K' >= K when
# K >= PINV_BUCKET_RATIO * K'.  Scratch per batched call is bounded.
PINV_BUCKET_RATIO = 0.7
PINV_BATCH_BYTES = 2 << 30


def pinv_buckets(Ks, ratio=PINV_BUCKET_RATIO):
    """Greedy grouping of system sizes (indices into Ks) by padded size."""
    order = sorted(range(len(Ks)), key=lambda i: -Ks[i])
    out = []
    while order:
        top = Ks[order[0]]
        take = [i for i in order if Ks[i] >= ratio * top]
        out.append((top, take))
        order = [i for i in order if Ks[i] < ratio * top]
    return out


def pinv_bucketed(decs, s):
    """Truncated eigen-pseudoinverse (float64, the rule of solve_eq_sym) of
    the real systems of ``decs`` (their complex M and b already built), in
    batched eigensolver calls of one padded size.  A system of size K is
    embedded in a K' x K' matrix whose extra diagonal entries equal Mr's
    largest diagonal entry d: the padded eigenvalues (= d, with
    lambda_max / K <= d <= lambda_max) change neither lambda_max nor which of
    the system's own eigenvalues pass rcond * lambda_max, and with a zero
    right-hand side there the solution is zero in the padding, so every
    system gets exactly its stand-alone pseudoinverse."""
    if not decs:
        return
    if len({d.rcond for d in decs}) > 1:
        by_r = defaultdict(list)
        for d in decs:
            by_r[d.rcond].append(d)
        for group in by_r.values():
            pinv_bucketed(group, s)
        return
    dev = decs[0].M.device
    for Kp, idx in pinv_buckets([d.K for d in decs]):
        per = max(1, int(PINV_BATCH_BYTES // (Kp * Kp * 8)))
        for c0 in range(0, len(idx), per):
            chunk = [decs[i] for i in idx[c0:c0 + per]]
            B = len(chunk)
            Mb = torch.zeros((B, Kp, Kp), dtype=torch.float64, device=dev)
            bb = torch.zeros((B, Kp), dtype=torch.float64, device=dev)
            for z, d in enumerate(chunk):
                K = d.K
                call("vtb_coeff_realify", dptr(d.M), K, K, dptr(d.Mr), K, 1, s)
                Mb[z, :K, :K].copy_(d.Mr)
                if K < Kp:
                    Mb[z].diagonal()[K:] = d.Mr.diagonal().max()
                bb[z, :K].copy_(d.br)
            xb = torch.empty_like(bb)
            nb = np.zeros(1, np.int64)
            call("vtb_sym_pinv_batched_workspace", Kp, B, nb.ctypes.data)
            work = torch.empty(int(nb[0]), dtype=torch.uint8, device=dev)
            kept = torch.zeros(B, dtype=torch.int32, device=dev)
            infos = torch.zeros(B, dtype=torch.int32, device=dev)
            call("vtb_sym_pinv_batched", dptr(Mb), dptr(bb), dptr(xb), Kp, B, chunk[0].rcond, dptr(work),
                 int(nb[0]), dptr(kept), dptr(infos), s)
            if int(infos.ne(0).sum()) != 0:
                raise fast.VtbError("vtb_sym_pinv_batched", fast.VTB_NOT_CONVERGED)
            for z, d in enumerate(chunk):
                d.xr.copy_(xb[z, :d.K])
                call("vtb_coeff_unrealify_vec", dptr(d.xr), d.K, 1, dptr(d.a), 0, s)
                d.kept.copy_(kept[z:z + 1] - (Kp - d.K))


class BatchDecoder(object):
    """Decode many clips per ``run()``: mixed-precision grouped solves as
    described in the module docstring.  ``graph`` captures the staging,
    factorisation and refinement (and, separately, the synthesis) as CUDA
    graphs on the first run and replays them afterwards; inputs are read
    from the problems' device tensors, so new spikes of the same sizes are
    decoded by copying them into those tensors.  ``workers`` host threads
    run the float64 fallbacks and spike-space solves concurrently.
    ``eig`` chooses how refused systems that the float64 Cholesky refuses
    too are eigen-solved: "bucketed" (batched eigensolver calls of one padded
    size, after every float64 Cholesky has finished) or "threads" (each on
    its worker thread, as a stand-alone decoder would, concurrently over the
    workers' streams)."""

    def __init__(self, problems, streams=8, sweeps=1, graph=True, workers=8, eig="bucketed"):
        if eig not in ("threads", "bucketed"):
            raise ValueError("eig must be 'threads' or 'bucketed'")
        self.eig = eig
        self.problems = list(problems)
        self.decs = [fast.from_prep(p.prep, p.Wt, p.Mt, rcond=p.rcond, solver="mixed", mixed_sweeps=sweeps)
                     for p in self.problems]
        dev = self.decs[0].M.device
        self.device = dev
        self.streams = [torch.cuda.Stream(device=dev) for _ in range(streams)]
        self.coeff = [i for i, (p, d) in enumerate(zip(self.problems, self.decs)) if int(p.tk1.numel()) >= d.K]
        self.spike = [i for i in range(len(self.problems)) if i not in set(self.coeff)]
        self.plan = MixedSolvePlan([self.decs[i] for i in self.coeff], [self.problems[i] for i in self.coeff], sweeps,
                                   self.streams) if self.coeff else None
        self.groups = self.plan.groups if self.plan else []
        self.gram = GroupedGram([self.decs[i] for i in self.coeff]) if self.coeff else None
        self.outs = [torch.empty((p.Nt, p.prep.decPy, p.prep.decPx), dtype=torch.float64, device=dev)
                     for p in self.problems]
        self.use_graph = bool(graph)
        self.graph_error = None
        self._g1 = self._g2 = None
        self._pool = ThreadPoolExecutor(max_workers=max(1, workers))
        self._worker_streams = {}
        self.fallbacks = 0
        self._phase_events = None

    # ---------------------------------------------------------- device work
    def _fork(self):
        main = torch.cuda.current_stream(self.device)
        ev = torch.cuda.Event()
        ev.record(main)
        for st in self.streams:
            st.wait_event(ev)
        return main

    def _join(self, main):
        for st in self.streams:
            ev = torch.cuda.Event()
            ev.record(st)
            main.wait_event(ev)

    def _stage_and_solve(self):
        main = self._fork()
        for c, i in enumerate(self.coeff):
            with torch.cuda.stream(self.streams[c % len(self.streams)]):
                stage_mixed_pre(self.decs[i], self.problems[i], stream_ptr())
        self._join(main)
        # every clip's Kronecker Gram in one grouped tensor-core launch
        self.gram.launch(stream_ptr())
        main = self._fork()
        for c, i in enumerate(self.coeff):
            with torch.cuda.stream(self.streams[c % len(self.streams)]):
                stage_mixed_post(self.decs[i], stream_ptr())
        self._join(main)
        self.plan.launch()

    def _synthesize(self):
        main = self._fork()
        for i, (p, d) in enumerate(zip(self.problems, self.decs)):
            with torch.cuda.stream(self.streams[i % len(self.streams)]):
                d.synthesize(d.a, p.T, p.dt, out=self.outs[i])
        self._join(main)

    def _capture(self, fn):
        fn()                      # eager warm-up: library handles, kernel attributes, allocations
        torch.cuda.synchronize(self.device)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            fn()
        return g

    def _ensure_graphs(self):
        if not self.use_graph or self._g2 is not None:
            return
        try:
            if self.plan is not None:
                self._g1 = self._capture(self._stage_and_solve)
            self._g2 = self._capture(self._synthesize)
        except Exception as e:  # graphs unavailable: the same launches, issued eagerly
            self.graph_error = repr(e)
            self.use_graph = False
            self._g1 = self._g2 = None
            torch.cuda.synchronize(self.device)

    # ---------------------------------------------------------- float64 path
    def _worker_stream(self):
        import threading
        tid = threading.get_ident()
        st = self._worker_streams.get(tid)
        if st is None:
            st = torch.cuda.Stream(device=self.device)
            self._worker_streams[tid] = st
        return st

    def _float64(self, i, after=None, eig=True):
        """Float64 decode of clip i on a worker thread: the spike-space
        pseudoinverse (fewer intervals than coefficients), else Cholesky of
        its real system and, when ``eig``, the eigen-pseudoinverse if the
        Cholesky is refused.  Returns (solved, event)."""
        torch.cuda.set_device(self.device)
        st = self._worker_stream()
        ok = True
        with torch.cuda.stream(st):
            if after is not None:
                st.wait_event(after)
            d, p = self.decs[i], self.problems[i]
            n = int(p.tk1.numel())
            s = stream_ptr()
            if n < d.K:
                d._solve_spike_space(s, p.spikes)
            else:
                d.solver = "auto" if eig else "chol"
                try:
                    d._solve(s, n)
                    d.last_solver = "mixed->" + d.last_solver
                except fast.VtbError as e:
                    if eig or e.status != fast.VTB_NOT_CONVERGED:
                        raise
                    ok = False
                finally:
                    d.solver = "mixed"
            ev = torch.cuda.Event()
            ev.record(st)
        return ok, ev

    # ---------------------------------------------------------- run
    def run(self, timing=False):
        """Decode every clip; returns the list of videos (device).  With
        ``timing`` the device time of (staging + grouped solves, float64
        fallbacks, synthesis) is left in ``self.phase_ms``."""
        self._ensure_graphs()
        main = torch.cuda.current_stream(self.device)
        ev = [torch.cuda.Event(enable_timing=timing) for _ in range(4)]
        ev[0].record(main)
        futs = [self._pool.submit(self._float64, i, ev[0]) for i in self.spike]
        bad, chol = [], []
        if self.plan is not None:
            if self._g1 is not None:
                self._g1.replay()
            else:
                self._stage_and_solve()
            ev[1].record(main)
            bad = [self.coeff[j] for j in self.plan.check()]
            # float64 Cholesky first (concurrently); the systems it refuses are
            # eigen-solved on the same worker thread, or together, grouped by
            # padded size
            threads = self.eig == "threads"
            chol = [(i, self._pool.submit(self._float64, i, ev[1], threads)) for i in bad]
        else:
            ev[1].record(main)
        rest = []
        for i, f in chol:
            ok, e = f.result()
            main.wait_event(e)
            if not ok:
                rest.append(i)
        if rest:
            pinv_bucketed([self.decs[i] for i in rest], stream_ptr())
            for i in rest:
                self.decs[i].last_solver = "mixed->eig-batched"
        for f in futs:
            main.wait_event(f.result()[1])
        self.fallbacks = len(bad)
        ev[2].record(main)
        if self._g2 is not None:
            self._g2.replay()
        else:
            self._synthesize()
        ev[3].record(main)
        self._phase_events = ev
        return self.outs

    @property
    def phase_ms(self):
        """(staging + grouped solves, float64 fallbacks, synthesis) device
        milliseconds of the last ``run(timing=True)`` (synchronise first)."""
        e = self._phase_events
        return tuple(e[i].elapsed_time(e[i + 1]) for i in range(3))

    def solver_counts(self):
        c = {}
        for d in self.decs:
            c[d.last_solver] = c.get(d.last_solver, 0) + 1
        return c

    def close(self):
        self._pool.shutdown(wait=True)
        self._g1 = self._g2 = None


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
