"""Batched apply of uneven operators and the autotuner, through the C ABI.

* Batch (worker streams, eager or one captured CUDA graph): every output is
  bit-identical to the operator applied alone (same kernels, same inputs),
  also after the arrays change (the graph is captured again), and matches
  the FP64 oracle within 1e-5 (relative L2, written here).
* Autotuner: the tuned operator still meets 1e-5 against the oracle.
"""

import numpy as np
import pytest

from mr_aha_b200 import synth
from oracle import aha_oracle as O
from tests.gpu_util import dev, host, random_kernel

pytestmark = pytest.mark.gpu

TOL = 1e-5
GEOMS = [
    ("stack", (64, 64, 8), 4, 4),
    ("2D", (40, 36), 3, 5),
    ("3D", (16, 18, 14), 2, 3),
    ("stack", (48, 40, 6), 8, 2),
    ("stack", (64, 64, 8), 16, 2),
]


def _ops(seed=0):
    import mr_aha_b200 as mr

    rng = np.random.default_rng(seed)
    out = []
    for tt, n_dim, L, nc in GEOMS:
        cfg = mr.make_config(tt, n_dim, L, n_coils=nc)
        img = tuple(reversed(n_dim))
        S = synth.crandn(rng, (nc,) + img)
        K = random_kernel(rng, mr.phi2_toep_shape(cfg))
        x = synth.crandn(rng, (L,) + img)
        op = mr.create_op(cfg, dev(S), None, None, _phi2_toep=dev(K))
        out.append(dict(tt=tt, n_dim=n_dim, L=L, S=S, K=K, x=x, op=op,
                        phi2_dim=synth.default_phi2_dim(tt, n_dim)))
    return out


@pytest.mark.parametrize("graph", [True, False])
def test_batch_equals_single_and_oracle(graph):
    import torch

    import mr_aha_b200 as mr

    items = _ops()
    try:
        singles = [host(it["op"](dev(it["x"]))) for it in items]
        with mr.Batch([it["op"] for it in items], n_streams=3, graph=graph) as b:
            xs = [dev(it["x"]) for it in items]
            ys = b(xs)
            torch.cuda.synchronize()
            for it, y, y1 in zip(items, ys, singles):
                assert np.array_equal(host(y), y1)
                ref = O.aha_toeplitz(it["tt"], it["n_dim"], it["phi2_dim"], it["L"], it["x"],
                                     it["S"], it["K"])
                assert O.rel_l2(host(y), ref) <= TOL
            # replay, then new arrays (graph captured again)
            ys2 = b(xs)
            xs3 = [x.clone() for x in xs]
            ys3 = b(xs3)
            torch.cuda.synchronize()
            for y, y2, y3 in zip(ys, ys2, ys3):
                assert torch.equal(y, y2) and torch.equal(y, y3)
    finally:
        for it in items:
            it["op"].close()


def test_batch_rejects_repeated_operator():
    import mr_aha_b200 as mr

    items = _ops(1)[:2]
    try:
        with pytest.raises(mr.MRError):
            mr.Batch([items[0]["op"], items[1]["op"], items[0]["op"]])
    finally:
        for it in items:
            it["op"].close()


def test_autotune_keeps_accuracy():
    import mr_aha_b200 as mr

    items = _ops(2)
    try:
        for it in items[:1] + items[3:]:
            ms = it["op"].autotune(reps=1)
            assert ms > 0
            y = host(it["op"](dev(it["x"])))
            ref = O.aha_toeplitz(it["tt"], it["n_dim"], it["phi2_dim"], it["L"], it["x"],
                                 it["S"], it["K"])
            assert O.rel_l2(y, ref) <= TOL
        with mr.Batch([it["op"] for it in items], tune=True) as b:
            ys = b([dev(it["x"]) for it in items])
            for it, y in zip(items, ys):
                ref = O.aha_toeplitz(it["tt"], it["n_dim"], it["phi2_dim"], it["L"], it["x"],
                                     it["S"], it["K"])
                assert O.rel_l2(host(y), ref) <= TOL
    finally:
        for it in items:
            it["op"].close()
