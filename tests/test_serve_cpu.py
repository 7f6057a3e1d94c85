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
