"""Scheduling logic of the serving loop on the CPU (fake device backend):
first-come-first-served admission within the memory budget and the slot
limit, bounded iterations in flight, every request completed, latency
accounting."""

import time

import pytest

from mr_aha_b200 import serve


class FakeBackend(serve.Backend):
    """Each request holds `mem` bytes; an iteration takes `dt` seconds of
    device time, and a request's iterations run back to back."""

    def __init__(self, dt=0.002):
        self.dt = dt
        self.log = []

    def estimate_bytes(self, req):
        return req.cfg["mem"]

    def admit(self, req):
        self.log.append(("admit", req.rid))
        return {"req": req, "until": 0.0, "done": 0}, req.cfg["mem"]

    def step(self, st, n):
        now = time.perf_counter()
        st["until"] = max(st["until"], now) + n * self.dt
        st["done"] += n

    def busy(self, st):
        return time.perf_counter() < st["until"]

    def finish(self, st):
        self.log.append(("finish", st["req"].rid))
        return [float(st["done"])], st["req"].rid


def _reqs(n, mem, iters, gap):
    return [serve.Request(rid=i, arrival=i * gap, cfg={"mem": mem}, SEs=None, phi2=None,
                          traj=None, b=None, n_iter=iters) for i in range(n)]


def test_all_requests_complete_within_limits():
    be = FakeBackend()
    srv = serve.Server(be, hbm_budget=300, max_active=3, chunk=2)
    res = srv.run(_reqs(8, 100, 6, 0.001))
    assert [r.rid for r in res] == list(range(8))
    assert all(r.rr == [6.0] and r.x == r.rid for r in res)
    assert srv.peak_bytes <= 300 and srv.peak_active <= 3
    assert srv.peak_active >= 2  # requests overlapped
    # first come, first served
    admits = [rid for ev, rid in be.log if ev == "admit"]
    assert admits == sorted(admits)
    for r in res:
        assert r.finished >= r.admitted >= r.arrival - 1e-9
        assert r.latency >= 6 * be.dt * 0.9


def test_memory_budget_serialises():
    be = FakeBackend()
    srv = serve.Server(be, hbm_budget=150, max_active=8)
    res = srv.run(_reqs(4, 100, 3, 0.0))
    assert len(res) == 4 and srv.peak_active == 1 and srv.peak_bytes == 100
    # each admission follows the previous finish
    seq = [ev for ev, _ in be.log]
    assert seq == ["admit", "finish"] * 4


def test_oversized_request_rejected():
    srv = serve.Server(FakeBackend(), hbm_budget=50)
    with pytest.raises(ValueError):
        srv.run(_reqs(1, 100, 1, 0.0))


def test_sequential_baseline_and_stats():
    be = FakeBackend()
    res = serve.run_sequential(be, _reqs(3, 10, 4, 0.0))
    assert len(res) == 3
    assert res[1].admitted >= res[0].finished - 1e-9
    st = serve.latency_stats(res)
    assert st["n"] == 3 and st["p99_s"] >= st["p50_s"] > 0


class SlowBuildBackend(FakeBackend):
    """Building an operator takes `build` seconds of host time."""

    def __init__(self, dt=0.002, build=0.05):
        super().__init__(dt)
        self.build = build
        self.events = []

    def admit(self, req):
        self.events.append((time.perf_counter(), "admit-start", req.rid))
        time.sleep(self.build)
        self.events.append((time.perf_counter(), "admit-end", req.rid))
        return super().admit(req)

    def step(self, st, n):
        self.events.append((time.perf_counter(), "step", st["req"].rid))
        super().step(st, n)


def test_background_build_overlaps_running_solves():
    be = SlowBuildBackend()
    reqs = _reqs(2, 10, 40, 0.02)
    srv = serve.Server(be, hbm_budget=100, max_active=4, chunk=1, background=True)
    res = srv.run(reqs)
    assert len(res) == 2
    t_start = next(t for t, e, r in be.events if e == "admit-start" and r == 1)
    t_end = next(t for t, e, r in be.events if e == "admit-end" and r == 1)
    during = [t for t, e, r in be.events if e == "step" and r == 0 and t_start < t < t_end]
    assert during, "request 0 made no progress while request 1 was being built"


def test_shortest_remaining_work_first():
    """A short request arriving while a long one runs finishes first when one
    solve runs at a time, and both complete."""
    be = FakeBackend(dt=0.002)
    reqs = _reqs(2, 10, 5, 0.01)
    reqs[0].n_iter = 60
    srv = serve.Server(be, hbm_budget=100, max_active=4, chunk=1, run_slots=1)
    res = srv.run(reqs)
    assert res[1].finished < res[0].finished
    assert [r.rr for r in res] == [[60.0], [5.0]]
