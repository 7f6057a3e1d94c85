"""Pass 3 with its input rows loaded by TMA tensor copies (``k_xbdh<...,
blocked,tma>``) across row lengths, ranks and coils per CTA, both packings,
through operators that own their kernel (built from Gram blocks, so the
blocked kernel copy exists): against the FP64 oracle's apply of the
operator's own kernel (relative L2 <= 1e-5), bit-identical to the same kernel
with per-thread loads (``MR_AHA_B200_NO_TMA=1``), with the device status word
clear (no bounded wait ran out). One case has a coil count that leaves the
last CTA's tile partly past the group's planes (read as zeros by the copy)."""

import numpy as np
import pytest

from mr_aha_b200 import synth
from oracle import aha_oracle as O
from tests.gpu_util import dev, host
from tests.test_gpu_headline import traced

pytestmark = pytest.mark.gpu

CASES = [(64, 4, 5), (128, 8, 3), (192, 16, 2), (256, 32, 2), (320, 16, 3), (320, 8, 3)]


@pytest.mark.parametrize("tri", ["lower", "upper"])
@pytest.mark.parametrize("n,L,nc", CASES, ids=[f"N{n}-L{L}-C{c}" for n, L, c in CASES])
def test_tma_input_rows(n, L, nc, tri, monkeypatch):
    import mr_aha_b200 as mr

    spec = dict(traj_type="stack", n_dim=(n, n, 2), L=L, n_coils=nc, n_traj=max(24, n // 4),
                n_kx=2 * n, n_frames=max(32, L), frame_rule="mod", seed=n + L + (tri == "upper"))
    p = synth.spec_inputs(spec)
    cfg = mr.make_config("stack", p["n_dim"], L, n_coils=nc, triangulation=tri)
    with mr.create_op(cfg, dev(p["SEs"]), dev(p["phi2"]), dev(p["traj"])) as op:
        assert op.blocked_copy(True) is True
        y, trace = traced(lambda: host(op(dev(p["x"]))))
        assert any(t.startswith(f"k_xbdh<N={n},L={L},") and t.endswith("blocked,tma>")
                   for t in trace), trace
        assert op.device_status == 0
        monkeypatch.setenv("MR_AHA_B200_NO_TMA", "1")
        y_regs, trace2 = traced(lambda: host(op(dev(p["x"]))))
        monkeypatch.delenv("MR_AHA_B200_NO_TMA")
        assert not any(t.endswith("tma>") for t in trace2), trace2
        K = host(op.kernel())
    np.testing.assert_array_equal(y, y_regs)
    ref = O.aha_toeplitz_lean("stack", p["n_dim"], p["phi2_dim"], L, p["x"], p["SEs"], K,
                              upper=tri == "upper")
    err = O.rel_l2(y, ref)
    assert err <= 1e-5, err
