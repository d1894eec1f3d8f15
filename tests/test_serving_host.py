"""Host logic of the serving loop on the CPU: admission by memory budget,
arrival order, batching of ready systems per tick, completion accounting,
failed requests and a stopped worker.  The device phases are replaced by
timed fakes; the GPU tests run the real ones."""
import time
from types import SimpleNamespace

import numpy as np
import pytest

from vtem_b200 import serving


class _Event(object):
    def __init__(self, at):
        self.at = at

    def query(self):
        return time.perf_counter() >= self.at


class _FakeChol(object):
    def __init__(self, jobs, flags, event):
        self.jobs, self._flags, self.event = jobs, flags, event

    def query(self):
        return self.event.query()

    def flags(self):
        return self._flags


class _Dec(object):
    def __init__(self, K):
        self.K = K


class FakeServer(serving.Server):
    """Phase A takes ``enc_s`` on its worker; the solve and synthesis take
    ``solve_s`` / ``synth_s`` of device time after their launch."""

    def __init__(self, enc_s=0.004, solve_s=0.001, synth_s=0.003, eig_s=0.01, fail=(), refuse=(), eig_fail=(),
                 **kw):
        super().__init__(device="cpu", **kw)
        self.enc_s, self.solve_s, self.synth_s, self.eig_s = enc_s, solve_s, synth_s, eig_s
        self.fail, self.refuse, self.eig_fail = set(fail), set(refuse), set(eig_fail)
        self.batches = []
        self.eig_groups = []

    def _new_stream(self):
        return object()

    def _bind_thread(self):
        pass

    def _phase_a(self, job):
        time.sleep(self.enc_s)
        if job.req.rid in self.fail:
            raise RuntimeError("encode failed")
        job.dec = _Dec(job.req.workload.K)
        job.ev_a = _Event(time.perf_counter() + 0.0005)

    def _launch_chol(self, jobs):
        self.batches.append(sorted(j.req.rid for j in jobs))
        return _FakeChol(jobs, [j.req.rid in self.refuse for j in jobs],
                         _Event(time.perf_counter() + self.solve_s))

    def _eig(self, jobs):
        time.sleep(self.eig_s)
        if any(j.req.rid in self.eig_fail for j in jobs):
            raise RuntimeError("eigensolver failed")
        self.eig_groups.append(sorted(j.req.rid for j in jobs))
        for j in jobs:
            # systems of any size: the solver thread groups them by padded size
            j.req.solver = "eig"

    def _phase_b(self, job):
        assert job.req.solver is not None
        job.req.result = np.full(3, job.req.rid)
        job.ev_b = _Event(time.perf_counter() + self.synth_s)


def _reqs(n, rate, seed=3, nbytes=10, K=None):
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, n))
    return [serving.Request(i, float(t[i]), SimpleNamespace(K=(K[i] if K else 100), F=10, Px=4, Py=4), None, nbytes)
            for i in range(n)]


def test_all_complete_and_budget_returns_to_zero():
    srv = FakeServer(budget_bytes=1000, workers=3)
    reqs = _reqs(40, rate=400.0)
    done = srv.run(reqs, max_seconds=30)
    assert sorted(r.rid for r in done) == list(range(40))
    assert all(r.state == "done" for r in done)
    assert srv.in_flight_bytes == 0
    for r in done:
        assert r.arrival <= r.admitted + 1e-9 <= r.done + 1e-9
        assert r.result[0] == r.rid
    st = serving.summary(done, srv.wall_s)
    assert st["completed"] == 40 and st["failed"] == 0
    assert st["p50_ms"] <= st["p95_ms"] <= st["p99_ms"]


def test_budget_limits_in_flight_and_keeps_arrival_order():
    srv = FakeServer(budget_bytes=25, workers=4)     # room for two requests of 10
    reqs = _reqs(20, rate=2000.0)
    done = srv.run(reqs, max_seconds=30)
    assert srv.peak_bytes <= 25
    adm = sorted(done, key=lambda r: r.rid)
    assert all(a.admitted <= b.admitted for a, b in zip(adm, adm[1:]))
    # at any admission instant at most two requests are between admission and completion
    for r in done:
        live = [x for x in done if x.admitted <= r.admitted < x.done]
        assert len(live) <= 2


def test_requests_ready_in_one_tick_are_solved_together():
    srv = FakeServer(budget_bytes=10 ** 6, workers=8, enc_s=0.01)
    reqs = _reqs(16, rate=1e6)          # all arrive at once
    srv.run(reqs, max_seconds=30)
    assert max(len(b) for b in srv.batches) > 1
    assert sorted(sum(srv.batches, [])) == list(range(16))


def test_failed_request_completes_with_its_error():
    srv = FakeServer(budget_bytes=1000, workers=2, fail={3, 7})
    done = srv.run(_reqs(10, rate=1000.0), max_seconds=30)
    failed = {r.rid for r in done if r.state == "failed"}
    assert failed == {3, 7}
    assert all("encode failed" in r.error for r in done if r.state == "failed")
    assert srv.in_flight_bytes == 0


def test_oversize_request_is_refused():
    srv = FakeServer(budget_bytes=5, workers=1)
    with pytest.raises(ValueError):
        srv.run(_reqs(2, rate=100.0), max_seconds=5)


def test_stopped_worker_is_reported():
    class Broken(FakeServer):
        def _bind_thread(self):
            raise RuntimeError("no device")

    with pytest.raises(RuntimeError, match="worker thread stopped"):
        Broken(budget_bytes=100, workers=1).run(_reqs(2, rate=100.0), max_seconds=5)


def test_keep_result_drops_consumed_buffers():
    srv = FakeServer(budget_bytes=1000, workers=2)
    done = srv.run(_reqs(6, rate=1000.0), max_seconds=30, keep_result=lambda r: r.rid < 2)
    kept = {r.rid for r in done if r.result is not None}
    assert kept == {0, 1}


def test_arrivals_are_seeded_poisson():
    from vtem_b200 import workloads
    rng = np.random.default_rng(3)
    t = np.cumsum(rng.exponential(1.0 / 200.0, 4000))
    assert abs(4000 / t[-1] - 200.0) < 10.0
    w = workloads.batch_clips(count=3, seed=3)
    b = [serving.request_bytes(x) for x in w]
    assert all(x > 0 for x in b)


def test_refused_factorisations_go_to_the_solver_thread():
    K = [100 + (i % 3) for i in range(18)]
    srv = FakeServer(budget_bytes=10 ** 6, workers=4, refuse={1, 4, 5, 7, 10, 13})
    done = srv.run(_reqs(18, rate=3000.0, K=K), max_seconds=30)
    assert all(r.state == "done" for r in done)
    solver = {r.rid: r.solver for r in done}
    assert {i for i, v in solver.items() if v == "eig"} == {1, 4, 5, 7, 10, 13}
    assert sorted(sum(srv.eig_groups, [])) == [1, 4, 5, 7, 10, 13]
    assert srv.in_flight_bytes == 0


def test_solver_failure_fails_only_its_requests():
    srv = FakeServer(budget_bytes=10 ** 6, workers=2, refuse={2, 3}, eig_fail={3})
    done = srv.run(_reqs(6, rate=100.0), max_seconds=30)
    failed = {r.rid for r in done if r.state == "failed"}
    assert 3 in failed and failed <= {2, 3}
    assert all(r.state == "done" for r in done if r.rid not in (2, 3))
    assert srv.in_flight_bytes == 0
