"""Continuous-batching service for encode + decode requests on one GPU.

A request carries a float32 video in pinned host memory and its encoder
description (RF bank, IAF parameters, Dirichlet orders); the service
returns the reconstructed float64 video in pinned host memory.  The loop
runs in ticks of ``tick_s`` (2 ms):

1. arrived requests are admitted in arrival order while the device-memory
   budget allows (video, projection, spikes, RF coefficients, Gram system,
   factor and output stay resident until the result is back on the host);
   an admitted request runs its first phase on a worker thread with its own
   CUDA stream: upload, RF projection on the tensor cores (split-bf16 from
   the float32 video), IAF block loop, spike pairing, Dirichlet coefficients
   and the tensor-core Kronecker Gram of its real coefficient system;
2. at each tick the systems of every request whose first phase has finished
   are solved together in mixed precision (vtem_b200.batch.MixedSolvePlan):
   requests with equal system size K share one batched float32 Cholesky,
   all share one batched triangular-solve launch per refinement sweep; a
   request whose pseudoinverse might truncate goes to a solver thread
   (float64 Cholesky, else the eigen-pseudoinverse batched over padded
   sizes), and one with fewer intervals than coefficients was solved in the
   spike space by its encoder;
3. solved requests run their synthesis and the download of the video on
   their own stream; a request completes when its download has finished,
   and its memory returns to the budget.

Requests arriving while others are on the GPU are admitted at the next tick
and their work overlaps on the device with the in-flight ones.  A result
does not depend on what else is in flight.
"""
from __future__ import annotations

import queue
import sys
import threading
import time
from collections import defaultdict
from dataclasses import dataclass

import numpy as np
import torch

from . import autotune, batch, fast
from ._abi import call, dptr, stream_ptr
from .workloads import ellipse_mask


@dataclass
class Request:
    rid: int
    arrival: float              # seconds after the start of the run
    workload: object            # vtem_b200.workloads.Workload
    video: torch.Tensor         # (F, Py, Px) float32 in pinned host memory
    bytes: int = 0
    admitted: float = -1.0
    encoded: float = -1.0        # first phase finished on its worker
    solved: float = -1.0         # synthesis launched
    done: float = -1.0
    state: str = "queued"
    result: torch.Tensor | None = None
    out: torch.Tensor | None = None   # optional pinned float64 output buffer
    solver: str | None = None
    error: str | None = None

    @property
    def voxels(self):
        w = self.workload
        return w.F * w.Px * w.Py

    @property
    def latency(self):
        return self.done - self.arrival


def request_bytes(w):
    """Upper estimate of the device bytes a request holds while in flight."""
    P = w.Px * w.Py
    K = int(ellipse_mask(w.Mx, w.My).sum()) * (2 * w.Mt + 1)
    Kp = -(-P // 64) * 64
    video = w.F * P * (4 + 2 * 3)                 # float32 upload + split-bf16 operand
    rf = w.N * (P * 8 + Kp * 6 + 16 * P * 8)      # encoder RFs, split operand, period-grid RFs
    proj = w.N * w.F * 8 * 2                      # projection (+ IAF staging)
    spikes = w.N * (int(w.F * w.dt * 200) + 64) * 40
    system = K * K * 16 * 3 + K * 16 * 8          # M, eigen/Cholesky workspace, vectors
    out = w.F * P * 8
    return video + rf + proj + spikes + system + out + (8 << 20)


def output_shape(w):
    """(samples, Py, Px) of a request's reconstruction (t = arange(0, T, dt))."""
    return (len(np.arange(0, w.T, w.dt)), w.Py, w.Px)


def make_requests(clips, rate=200.0, seed=3, device="cuda", preallocate_out=True):
    """Seeded Poisson arrivals at ``rate`` per second; each request carries
    its clip's video as float32 in pinned host memory and, when
    ``preallocate_out``, a pinned float64 buffer for its result (the
    client's registered output; otherwise the server allocates one)."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, len(clips)))
    reqs = []
    for i, (w, ta) in enumerate(zip(clips, t)):
        v = w.video(device=device).to(torch.float32).cpu().pin_memory()
        out = torch.empty(output_shape(w), dtype=torch.float64, pin_memory=True) if preallocate_out else None
        reqs.append(Request(i, float(ta), w, v, request_bytes(w), out=out))
    return reqs


class _InFlight(object):
    __slots__ = ("req", "stream", "problem", "dec", "ev_a", "ev_s", "ev_b", "out_dev")

    def __init__(self, req, stream):
        self.req, self.stream = req, stream
        self.problem = self.dec = self.ev_a = self.ev_s = self.ev_b = self.out_dev = None


class _CholBatch(object):
    """Handle of the grouped mixed solve launched at one tick."""

    def __init__(self, jobs, plan, host, event):
        self.jobs, self._plan, self._host, self._event = jobs, plan, host, event

    def query(self):
        return self._event.query()

    def flags(self):
        bad = set(self._plan.evaluate(*(h.numpy() for h in self._host)))
        return [i in bad for i in range(len(self.jobs))]

    @property
    def event(self):
        return self._event


class Server(object):
    """Request loop over one GPU (see the module docstring)."""

    def __init__(self, budget_bytes=120 * 10 ** 9, workers=2, tick_s=0.002, device="cuda", precision="bf16x3",
                 switch_interval=2e-4, sweeps=1, solvers=2):
        self.budget = int(budget_bytes)
        self.workers = int(workers)
        self.tick_s = float(tick_s)
        dev = torch.device(device)
        if dev.type == "cuda" and dev.index is None:
            dev = torch.device("cuda", torch.cuda.current_device())
        self.device = dev
        self.precision = precision
        self.sweeps = int(sweeps)
        self.solvers = max(1, int(solvers))   # threads for the float64 fallbacks
        # the interpreter's thread switch interval while serving: shorter
        # than a kernel launch sequence, so that a thread with device work to
        # issue does not wait behind another thread's Python
        self.switch_interval = switch_interval
        self.in_flight_bytes = 0
        self.peak_bytes = 0
        self.ticks = 0
        self.batched_solves = 0
        self.max_batch = 0

    def _new_stream(self):
        return torch.cuda.Stream(device=self.device)

    def _solver_stream(self):
        tid = threading.get_ident()
        st = self._eig_streams.get(tid)
        if st is None:
            st = self._eig_streams[tid] = self._new_stream()
        return st

    def _bind_thread(self):
        torch.cuda.set_device(self.device)

    # -- phase 1 (worker thread, own stream) -------------------------------
    def _phase_a(self, job):
        req = job.req
        # no GEMM tile tuning inside the loop (it would time launches under
        # the other threads' load and stall this worker)
        with torch.cuda.stream(job.stream), autotune.frozen():
            V = req.video.to(self.device, non_blocking=True)
            p = batch.encode_clip_problem(req.workload, self.device, video=V, precision=self.precision)
            n = int(p.tk1.numel())
            mixed = n >= fast.coefficient_count(p.prep.Mx, p.prep.My, p.Mt)
            d = fast.from_prep(p.prep, p.Wt, p.Mt, rcond=p.rcond, solver="mixed" if mixed else "auto",
                               mixed_sweeps=self.sweeps)
            s = stream_ptr()
            if n < d.K:
                d._solve_spike_space(s, p.spikes)
                req.solver = d.last_solver
            else:
                batch.stage_mixed(d, p, s)
            job.problem, job.dec = p, d
            job.ev_a = torch.cuda.Event()
            job.ev_a.record(job.stream)

    # -- phase 2: batched Cholesky (loop thread, solve stream) --------------
    def _launch_chol(self, jobs):
        """Launch the grouped mixed-precision solve of ``jobs`` (all with a
        coefficient-space system staged by the encoder): one batched float32
        Cholesky per system size, batched triangular solves, float64
        refinement sweeps; returns a handle whose ``query()`` tells when it
        is done and ``flags()`` then lists, per job, whether the float64 path
        must solve it instead."""
        with torch.cuda.stream(self._solve_stream):
            main = torch.cuda.current_stream(self.device)
            for j in jobs:
                main.wait_event(j.ev_a)
            plan = batch.MixedSolvePlan([j.dec for j in jobs], [j.problem for j in jobs], self.sweeps,
                                        [self._solve_stream])
            plan.launch()
            host = [torch.empty(t.shape, dtype=t.dtype, pin_memory=True) for t in plan.gather()]
            for h, t in zip(host, plan.gather()):
                h.copy_(t, non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(main)
            self.batched_solves += len(plan.groups)
            self.max_batch = max([self.max_batch] + [len(g["idx"]) for g in plan.groups])
        return _CholBatch(jobs, plan, host, ev)

    # -- phase 2b: eigen-pseudoinverse of refused systems (solver thread) ----
    def _eig(self, jobs):
        """Float64 path for systems the mixed solve refused (solver thread):
        float64 Cholesky where its pivot test passes, else the truncated
        eigen-pseudoinverse, batched over padded sizes.  Returns when the
        solutions are on the device."""
        with torch.cuda.stream(self._solver_stream()):
            st = torch.cuda.current_stream(self.device)
            for j in jobs:
                st.wait_event(j.ev_s)
            s = stream_ptr()
            rest = []
            for j in jobs:
                d = j.dec
                d.solver = "chol"
                try:
                    d._solve(s, int(j.problem.tk1.numel()))
                    d.last_solver = "mixed->chol"
                except fast.VtbError as e:
                    if e.status != fast.VTB_NOT_CONVERGED:
                        raise
                    rest.append(d)
                    d.last_solver = "mixed->eig-batched"
                finally:
                    d.solver = "mixed"
            batch.pinv_bucketed(rest, s)
            ev = torch.cuda.Event()
            ev.record(st)
        for j in jobs:
            j.ev_s = ev
            j.req.solver = j.dec.last_solver

    # -- phase 3 (loop thread, the request's stream) -------------------------
    def _phase_b(self, job):
        req = job.req
        with torch.cuda.stream(job.stream):
            if job.ev_s is not None:
                torch.cuda.current_stream(self.device).wait_event(job.ev_s)
            p, d = job.problem, job.dec
            job.out_dev = d.synthesize(d.a, p.T, p.dt)
            if req.out is not None and tuple(req.out.shape) == tuple(job.out_dev.shape) \
                    and req.out.dtype == job.out_dev.dtype:
                req.result = req.out
            else:
                req.result = torch.empty(job.out_dev.shape, dtype=job.out_dev.dtype, pin_memory=True)
            req.result.copy_(job.out_dev, non_blocking=True)
            job.ev_b = torch.cuda.Event()
            job.ev_b.record(job.stream)

    def run(self, requests, max_seconds=600.0, keep_result=None):
        """Serve ``requests`` (arrival times in seconds after the start) and
        return them, completed or failed, with their timestamps.  A completed
        request keeps its pinned host result unless ``keep_result(request)``
        is false; then the buffer returns to the pinned-memory cache once the
        result has arrived (a client that consumed it at completion).

        The loop thread never waits on the device: it launches work and
        polls events.  Encoding runs on ``workers`` threads, eigen-
        pseudoinverses on ``solvers`` solver threads (own streams)."""
        pending = sorted(requests, key=lambda r: r.arrival)
        for r in pending:
            if r.bytes > self.budget:
                raise ValueError("request %d needs %d bytes, above the budget" % (r.rid, r.bytes))
        waiting, ready, checking, in_b = [], [], [], []
        done = []
        lock = threading.Lock()
        encoded, solved = [], []            # filled by the encode workers / the solver threads
        work_q, eig_q = queue.Queue(), queue.Queue()
        thread_errors = []
        streams = [self._new_stream() for _ in range(self.workers)]
        self._solve_stream = self._new_stream()
        self._eig_streams = {}

        def encoder(st):
            try:
                self._bind_thread()
            except Exception as e:
                thread_errors.append(repr(e))
                return
            while True:
                job = work_q.get()
                if job is None:
                    return
                job.stream = st
                try:
                    self._phase_a(job)
                except Exception as e:      # the request completes with its error
                    job.req.error = repr(e)
                job.req.encoded = time.perf_counter() - t0
                with lock:
                    encoded.append(job)

        def solver():
            # one stream per solver thread
            try:
                self._bind_thread()
            except Exception as e:
                thread_errors.append(repr(e))
                return
            while True:
                jobs = eig_q.get()
                if jobs is None:
                    return
                try:
                    self._eig(jobs)
                except Exception as e:
                    for j in jobs:
                        j.req.error = repr(e)
                with lock:
                    solved.extend(jobs)

        old_switch = sys.getswitchinterval()
        if self.switch_interval:
            sys.setswitchinterval(self.switch_interval)
        t0 = time.perf_counter()
        threads = [threading.Thread(target=encoder, args=(st,), daemon=True) for st in streams]
        threads.extend(threading.Thread(target=solver, daemon=True) for _ in range(self.solvers))
        for t in threads:
            t.start()
        nreq = len(pending)

        def finish(j, state):
            j.req.state = state
            j.req.done = time.perf_counter() - t0
            self.in_flight_bytes -= j.req.bytes
            done.append(j.req)

        def to_synthesis(j):
            j.req.state = "synthesis"
            j.req.solved = time.perf_counter() - t0
            self._phase_b(j)
            in_b.append(j)

        try:
            while len(done) < nreq:
                now = time.perf_counter() - t0
                if now > max_seconds:
                    raise RuntimeError("serving loop exceeded %.0f s" % max_seconds)
                if thread_errors or not all(t.is_alive() for t in threads):
                    raise RuntimeError("a worker thread stopped: %s" % "; ".join(thread_errors))
                self.ticks += 1
                # 1. arrivals and admission by memory budget, in arrival order
                while pending and pending[0].arrival <= now:
                    waiting.append(pending.pop(0))
                while waiting and self.in_flight_bytes + waiting[0].bytes <= self.budget:
                    r = waiting.pop(0)
                    r.admitted = now
                    r.state = "encoding"
                    self.in_flight_bytes += r.bytes
                    self.peak_bytes = max(self.peak_bytes, self.in_flight_bytes)
                    work_q.put(_InFlight(r, None))
                with lock:
                    new_enc, new_eig = encoded[:], solved[:]
                    del encoded[:], solved[:]
                for j in new_enc:
                    if j.req.error is not None:
                        finish(j, "failed")
                    else:
                        ready.append(j)
                # 2. every system whose encoding finished: spike-space ones are
                # solved already; the rest share batched Cholesky calls
                solvable = [j for j in ready if j.ev_a.query()]
                if solvable:
                    ready = [j for j in ready if j not in solvable]
                    for j in solvable:
                        if j.req.solver is not None:
                            to_synthesis(j)
                    coeff = [j for j in solvable if j.req.solver is None]
                    if coeff:
                        for j in coeff:
                            j.req.state = "solving"
                        checking.append(self._launch_chol(coeff))
                # 3. finished factorisations: accepted -> synthesis, refused ->
                # a solver thread (grouped by padded size there)
                still = []
                for cb in checking:
                    if not cb.query():
                        still.append(cb)
                        continue
                    refused = []
                    for j, bad in zip(cb.jobs, cb.flags()):
                        j.ev_s = cb.event
                        if bad:
                            refused.append(j)
                        else:
                            j.req.solver = "mixed-batched"
                            to_synthesis(j)
                    if refused:
                        eig_q.put(refused)
                checking = still
                for j in new_eig:
                    if j.req.error is not None:
                        finish(j, "failed")
                    else:
                        to_synthesis(j)
                # 4. completions
                still = []
                for j in in_b:
                    if j.ev_b.query():
                        if keep_result is not None and not keep_result(j.req):
                            j.req.result = None
                        finish(j, "done")
                    else:
                        still.append(j)
                in_b = still
                nxt = (int(now / self.tick_s) + 1) * self.tick_s
                delay = nxt - (time.perf_counter() - t0)
                if delay > 0:
                    time.sleep(delay)
        finally:
            for _ in range(self.workers):
                work_q.put(None)
            for _ in range(self.solvers):
                eig_q.put(None)
            for t in threads:
                t.join()
            sys.setswitchinterval(old_switch)
        self.wall_s = time.perf_counter() - t0
        return done


def plain_fp64(req, device="cuda"):
    """One request executed alone by the plain float64 path of the reference:
    float64 upload and RF projection, IAF block loop, analytic n x n Gram
    (vtem/dirichlet.py compute_G), eigen-pseudoinverse (vtem/linalg.py
    solve_eq_sym), synthesis through the spatial functions on the decode
    grid (vtem/vrf.py compute_dirich_space_fft).  Returns the video on the
    host (float64) and the seconds it took."""
    from . import dirichlet, linalg, vrf, vtdm
    w = req.workload
    dev = torch.device(device)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    V = req.video.to(dev).to(torch.float64)
    p = batch.encode_clip_problem(w, dev, video=V, precision="f64")
    rfSx, rfSy, rfPx, rfPy = vtdm.period_grid(w.Mx, w.My, w.Wx, w.Wy, w.dx, w.dy)
    grid = vrf.vrf_gabor((rfPy, rfPx), dx=rfSx / rfPx, dy=rfSy / rfPy, scale=4)
    Ds = p.prep.Ds
    dirich = grid.compute_dirich_space_fft(Ds, w.Mx, w.My, w.Px, w.Py, 1.0, 1.0, w.Wx, w.Wy)
    Dsw = grid.compute_Dsw(Ds, w.Mx, w.My, np.ones(w.N))
    cp = dirichlet.dirichlet(w.N, p.tk1, p.tk2, p.ind, w.kappa, w.delta, w.bias, np.ones(w.N), w.Wt, w.Mt)
    cp.compute_q()
    cp.compute_G(Dsw, lower_only=True)
    cp.d_q = linalg.solve_eq_sym(cp.d_G, cp.d_q, rcond=w.rcond)
    cp.freeG()
    u = cp.reconstruct(dirich, [0, w.T], w.dt).cpu()
    torch.cuda.synchronize(dev)
    return u, time.perf_counter() - t0


def summary(done, wall_s):
    ok = [r for r in done if r.state == "done"]
    lat = np.array([r.latency for r in ok]) * 1e3
    vox = sum(r.voxels for r in ok)
    first = min(r.arrival for r in done)
    def mean_ms(a, b):
        return float(np.mean([getattr(r, b) - getattr(r, a) for r in ok])) * 1e3

    return {"p50_ms": float(np.percentile(lat, 50)), "p95_ms": float(np.percentile(lat, 95)),
            "p99_ms": float(np.percentile(lat, 99)), "mean_ms": float(lat.mean()), "completed": len(ok),
            "failed": len(done) - len(ok), "voxels_per_s": vox / max(wall_s - first, 1e-9), "wall_s": wall_s,
            "phases_mean_ms": {"queued": mean_ms("arrival", "admitted"), "encode": mean_ms("admitted", "encoded"),
                               "solve": mean_ms("encoded", "solved"), "synthesis": mean_ms("solved", "done")}}
