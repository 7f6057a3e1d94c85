"""The serving loop on the GPU: requests of different sizes arriving over
time are admitted while others run, their iterations share the GPU, and each
result is bit-identical to the same request solved alone (the solver is
deterministic), with the same residual history."""

import numpy as np
import pytest

from mr_aha_b200 import serve, synth
from tests.gpu_util import dev, host

pytestmark = pytest.mark.gpu

SMALL = dict(n=(32, 48), nz=(4, 8), L=(2, 4), coils=(2, 4))


def _requests(n=6, gap=0.0):
    import mr_aha_b200 as mr

    specs = synth.batch_specs(n, seed=9, choices=SMALL, spokes=(24, 64))
    rng = np.random.default_rng(9)
    reqs = []
    for i, sp in enumerate(specs):
        p = synth.spec_inputs(sp, with_x=False)
        cfg = mr.make_config(p["traj_type"], p["n_dim"], p["L"], n_coils=p["n_coils"])
        b = synth.crandn(rng, (p["L"],) + tuple(reversed(p["n_dim"])))
        reqs.append(serve.Request(rid=i, arrival=i * gap, cfg=cfg, SEs=dev(p["SEs"]),
                                  phi2=dev(p["phi2"]), traj=dev(p["traj"]), b=dev(b),
                                  n_iter=int(rng.integers(40, 81))))
    return reqs


@pytest.mark.parametrize("fmt", ["int16", "complex64"])
def test_served_results_equal_alone(fmt):
    import mr_aha_b200 as mr

    reqs = _requests()
    srv = serve.Server(serve.GPUBackend(kernel_format=fmt), hbm_budget=40e9, max_active=4,
                       chunk=2, run_slots=None)
    res = srv.run(reqs)
    assert [r.rid for r in res] == [r.rid for r in reqs]
    # the requests shared the GPU: some request was admitted while another ran
    assert any(a.admitted < b.admitted < a.finished for a in res for b in res if a is not b)
    for r, q in zip(res, reqs):
        op = mr.create_op(q.cfg, q.SEs, q.phi2, q.traj)
        if fmt != "complex64":
            op.set_kernel_format(fmt, keep_complex64=False)
        x, rr = op.cg(q.b, q.n_iter)
        op.close()
        assert np.array_equal(host(r.x), host(x)), r.rid
        assert np.array_equal(r.rr, rr)
        assert np.all(np.isfinite(r.rr))
    st = serve.latency_stats(res)
    assert st["n"] == len(reqs) and st["p99_s"] >= st["p50_s"] > 0


def test_sequential_baseline_matches():
    reqs = _requests(3)
    be = serve.GPUBackend(kernel_format="complex64")
    seq = serve.run_sequential(be, reqs)
    mix = serve.Server(be, hbm_budget=40e9, max_active=3).run(reqs)
    for a, b in zip(seq, mix):
        assert np.array_equal(host(a.x), host(b.x))
