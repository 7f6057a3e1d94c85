"""The instantiated specialised kernels of uneven geometries against the FP64
oracle: half-length pass 3 for N in {64, 128, 192, 256} and every rank
configuration (L = 4, 8 with several coils per tile, 16, and 32 with the
split two-thread block multiply), strided passes of 256 / 384 / 512-point y
lines and 16 / 32-point z lines (the pipelined coil sum with a ragged last
tile, and the plain one on an odd plane it cannot align); lower and upper
packings, a coil count that does not fill the last tile, and a masked
rank-32 kernel. Tolerance
(relative L2): 1e-5."""

import numpy as np
import pytest

from mr_aha_b200 import synth
from oracle import aha_oracle as O
from tests.gpu_util import dev, host, random_kernel

pytestmark = pytest.mark.gpu

TOL = 1e-5
CASES = [
    ((64, 64, 2), 32, 2, "lower"),
    ((64, 64, 2), 32, 2, "upper"),
    ((64, 64, 2), 8, 3, "lower"),
    ((64, 64, 2), 16, 2, "upper"),
    ((128, 128, 2), 16, 2, "lower"),
    ((192, 192, 2), 4, 5, "lower"),
    ((256, 256, 2), 8, 2, "upper"),
    ((64, 64, 16), 4, 2, "lower"),
    ((64, 64, 32), 4, 2, "upper"),
    ((30, 22, 16), 4, 3, "lower"),    # ragged last z tile (660 columns), pipelined coil sum
    ((21, 25, 16), 2, 3, "upper"),    # odd plane (525 columns): unaligned, plain coil sum
]
IDS = [f"{n[0]}x{n[1]}x{n[2]}-L{L}-C{c}-{t}" for n, L, c, t in CASES]


@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_uneven_geometry(case):
    import mr_aha_b200 as mr

    n_dim, L, nc, tri = case
    rng = np.random.default_rng(L * 100 + nc)
    img = tuple(reversed(n_dim))
    x = synth.crandn(rng, (L,) + img)
    S = synth.crandn(rng, (nc,) + img)
    cfg = mr.make_config("stack", n_dim, L, n_coils=nc, triangulation=tri)
    K = random_kernel(rng, mr.phi2_toep_shape(cfg))
    y = host(mr.aha_toeplitz(cfg, dev(x), dev(S), dev(K)))
    ref = O.aha_toeplitz("stack", n_dim, synth.default_phi2_dim("stack", n_dim), L, x, S, K,
                         upper=tri == "upper")
    assert O.rel_l2(y, ref) <= TOL, O.rel_l2(y, ref)


def test_masked_rank32():
    import mr_aha_b200 as mr

    n_dim, L, nc = (64, 64, 2), 32, 2
    rng = np.random.default_rng(77)
    img = tuple(reversed(n_dim))
    x = synth.crandn(rng, (L,) + img)
    S = synth.crandn(rng, (nc,) + img)
    phi2_dim = synth.default_phi2_dim("stack", n_dim)
    mask = O.calc_mask("stack", phi2_dim, synth.make_traj("stack", 24, 128), 2)
    cfg = mr.make_config("stack", n_dim, L, n_coils=nc, is_masked=True, num_masked=len(mask))
    K = random_kernel(rng, (O.num_tri(L), len(mask)))
    y = host(mr.aha_toeplitz(cfg, dev(x), dev(S), dev(K), mask=dev(mask)))
    ref = O.aha_toeplitz("stack", n_dim, phi2_dim, L, x, S, K, mask=mask)
    assert O.rel_l2(y, ref) <= TOL


@pytest.mark.parametrize("n_dim,L,nc", [((64, 64, 8), 4, 4), ((64, 64, 2), 32, 2)])
def test_blocked_kernel_copy_equals_reference_layout(n_dim, L, nc, monkeypatch):
    """An operator that owns its kernel reads a blocked copy in pass 3; the
    apply equals the one reading the reference layout bit for bit (same
    values, same arithmetic), for the single-thread and the split rank-32
    block multiply, and stays within 1e-5 of the FP64 oracle."""
    import mr_aha_b200 as mr

    spec = dict(traj_type="stack", n_dim=n_dim, L=L, n_coils=nc, n_traj=24, n_kx=2 * n_dim[0],
                n_frames=max(L, 8), frame_rule="mod", seed=5)
    p = synth.spec_inputs(spec)
    ys, devbytes = [], []
    for off in ("0", "1"):
        monkeypatch.setenv("MR_AHA_B200_NO_BLOCKED", off)
        cfg = mr.make_config("stack", n_dim, L, n_coils=nc)
        with mr.create_op(cfg, dev(p["SEs"]), dev(p["phi2"]), dev(p["traj"])) as op:
            ys.append(host(op(dev(p["x"]))))
            devbytes.append(op.device_bytes)
            K = host(op.kernel())
            if off == "0":
                # freeing the copy switches pass 3 to the reference layout
                assert op.blocked_copy(False) is False
                assert op.device_bytes < devbytes[0]
                assert np.array_equal(host(op(dev(p["x"]))), ys[0])
                assert op.blocked_copy(True) is True
    assert devbytes[0] > devbytes[1]          # the copy was built
    assert np.array_equal(ys[0], ys[1])
    ref = O.aha_toeplitz("stack", n_dim, synth.default_phi2_dim("stack", n_dim), L, p["x"],
                         p["SEs"], K)
    assert O.rel_l2(ys[0], ref) <= TOL


@pytest.mark.parametrize("n_dim,L,nc", [((64, 64, 8), 4, 3), ((64, 64, 2), 32, 2),
                                        ((320, 320, 2), 16, 2)])
def test_masked_blocked_copy_equals_masked_layout(n_dim, L, nc):
    """A masked operator that owns its kernel keeps a grid-order blocked copy
    (zero outside the mask); pass 3 reads it for the locations in the mask
    and still skips the others. Bit-identical to the masked reference layout
    (the same operator after ``blocked_copy(False)``), within 1e-5 of the FP64
    oracle's masked apply (64-point grids)."""
    import mr_aha_b200 as mr
    from tests.test_gpu_headline import traced

    spec = dict(traj_type="stack", n_dim=n_dim, L=L, n_coils=nc, n_traj=24, n_kx=2 * n_dim[0],
                n_frames=max(L, 8), frame_rule="mod", seed=9)
    p = synth.spec_inputs(spec)
    cfg = mr.make_config("stack", n_dim, L, n_coils=nc)
    mask = mr.calc_mask(cfg, dev(p["traj"]))
    mcfg = mr.make_config("stack", n_dim, L, n_coils=nc, is_masked=True,
                          num_masked=int(mask.numel()))
    with mr.create_op(mcfg, dev(p["SEs"]), dev(p["phi2"]), dev(p["traj"]), mask=mask) as op:
        assert op.blocked_copy(True) is True
        y_blk, trace = traced(lambda: host(op(dev(p["x"]))))
        assert any("blocked" in t and t.endswith(",masked>") for t in trace), trace
        assert op.blocked_copy(False) is False
        y_ref, trace2 = traced(lambda: host(op(dev(p["x"]))))
        assert not any("blocked" in t for t in trace2), trace2
        Km = host(op.kernel())
    np.testing.assert_array_equal(y_blk, y_ref)
    if n_dim[0] <= 64:  # the dense FP64 oracle of the 320-point grid needs GBs of host memory
        ref = O.aha_toeplitz("stack", n_dim, synth.default_phi2_dim("stack", n_dim), L,
                             p["x"], p["SEs"], Km, mask=host(mask))
        assert O.rel_l2(y_blk, ref) <= TOL
