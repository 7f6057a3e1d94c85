"""Applies from and to host memory (``mr_b200_op_execute_host``,
``AhAOp.apply_host``), through the C ABI.

* Several calls queued back to back, each with its own input and output
  buffer (page-locked and pageable), give after ``host_sync`` exactly the
  device apply of each input (bit-identical: same kernels, same inputs), so
  the two device slots are never overwritten while in use.
* One pair of buffers reused by every call (the bench's end-to-end loop)
  ends with the last call's result.
* After ``host_release`` the next call allocates the slots again.
* The output also meets 1e-5 against the FP64 oracle (relative L2).
"""

import numpy as np
import pytest

from mr_aha_b200 import synth
from oracle import aha_oracle as O
from tests.gpu_util import dev, host, random_kernel

pytestmark = pytest.mark.gpu

N_DIM, L, NC = (64, 64, 8), 4, 4


@pytest.fixture(scope="module")
def case():
    import mr_aha_b200 as mr

    rng = np.random.default_rng(5)
    cfg = mr.make_config("stack", N_DIM, L, n_coils=NC)
    img = tuple(reversed(N_DIM))
    S = synth.crandn(rng, (NC,) + img)
    K = random_kernel(rng, mr.phi2_toep_shape(cfg))
    xs = [synth.crandn(rng, (L,) + img) for _ in range(5)]
    op = mr.create_op(cfg, dev(S), None, None, _phi2_toep=dev(K))
    ys = [host(op(dev(x))) for x in xs]
    yield dict(op=op, S=S, K=K, xs=xs, ys=ys)
    op.close()


@pytest.mark.parametrize("pinned", [True, False], ids=["pinned", "pageable"])
def test_queued_host_applies_match_device_applies(case, pinned):
    import mr_aha_b200 as mr

    op = case["op"]
    if pinned:
        hx = [mr.pinned_empty(x.shape) for x in case["xs"]]
        for h, x in zip(hx, case["xs"]):
            h[...] = x
        hy = [mr.pinned_empty(x.shape) for x in case["xs"]]
    else:
        hx = [x.copy() for x in case["xs"]]
        hy = [np.empty_like(x) for x in case["xs"]]
    for h, o in zip(hx, hy):
        assert op.apply_host(h, o) is o
    op.host_sync()
    for o, y in zip(hy, case["ys"]):
        np.testing.assert_array_equal(o, y)
    assert op.device_status == 0


def test_reused_buffers_release_and_oracle(case):
    import mr_aha_b200 as mr

    op = case["op"]
    hx = mr.pinned_empty(case["xs"][0].shape)
    hy = mr.pinned_empty(case["xs"][0].shape)
    for x in case["xs"][:3]:
        hx[...] = x
        op.apply_host(hx, hy)
        op.host_sync()
    np.testing.assert_array_equal(hy, case["ys"][2])
    for _ in range(4):
        op.apply_host(hx, hy)
    op.host_sync()
    np.testing.assert_array_equal(hy, case["ys"][2])
    op.host_release()
    y = op.apply_host(case["xs"][4])
    op.host_sync()
    np.testing.assert_array_equal(y, case["ys"][4])
    ref = O.aha_toeplitz("stack", N_DIM, synth.default_phi2_dim("stack", N_DIM), L,
                         case["xs"][4], case["S"], case["K"])
    assert O.rel_l2(y, ref) <= 1e-5
