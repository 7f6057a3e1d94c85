"""GPU parity of the CUDA library against the FP64 oracle, through the C ABI.

Cases are the reference's own synthetic set (tests/make_reference.py:130-146
of the reference: 2D / 3D / stack, odd sizes, a prime 101 x 81 grid, odd Nz,
L in {1, 3, 4}) plus larger ranks. Tolerances (relative L2, written here):

* apply (FP32 path) vs the FP64 oracle of the same operator: 1e-5;
* kernel build vs the exact FP64 kernel: 1e-6;
* calc_mask: bit-exact;
* operator built from the Gram blocks vs the exact NUFFT-route A^H A: 1e-5.
"""

import numpy as np
import pytest

from mr_aha_b200 import synth
from oracle import aha_oracle as O
from tests.gpu_util import dev, host, random_kernel

pytestmark = pytest.mark.gpu

TOL_APPLY = 1e-5
TOL_TOEP = 1e-6
TOL_OP = 1e-5

CASES = synth.REFERENCE_CASES
IDS = [c["name"] for c in CASES]


def _mr():
    import mr_aha_b200 as mr

    return mr


def _cfg(p, tri="lower", **kw):
    mr = _mr()
    return mr.make_config(p["traj_type"], p["n_dim"], p["L"], phi2_dim=p["phi2_dim"],
                          triangulation=tri, n_coils=p["n_coils"], **kw)


@pytest.mark.parametrize("tri", ["lower", "upper"])
@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_apply_random_kernel(case, tri):
    """mr_aha_toeplitz with a random packed kernel vs the FP64 apply."""
    mr = _mr()
    p = synth.reference_case(case)
    cfg = _cfg(p, tri)
    rng = np.random.default_rng(100 + case["seed"])
    K = random_kernel(rng, mr.phi2_toep_shape(cfg))
    y = host(mr.aha_toeplitz(cfg, dev(p["x"]), dev(p["SEs"]), dev(K)))
    ref = O.aha_toeplitz(p["traj_type"], p["n_dim"], p["phi2_dim"], p["L"], p["x"], p["SEs"], K,
                         upper=tri == "upper")
    assert O.rel_l2(y, ref) <= TOL_APPLY


@pytest.mark.parametrize("case", CASES[:3] + CASES[5:], ids=IDS[:3] + IDS[5:])
def test_apply_masked_random_kernel(case):
    """Masked apply: kernel stored at the calc_mask locations only."""
    mr = _mr()
    p = synth.reference_case(case)
    mask = O.calc_mask(p["traj_type"], p["phi2_dim"], p["traj"], 2)
    cfg = _cfg(p, is_masked=True, num_masked=len(mask))
    rng = np.random.default_rng(200 + case["seed"])
    K = random_kernel(rng, (O.num_tri(p["L"]), len(mask)))
    y = host(mr.aha_toeplitz(cfg, dev(p["x"]), dev(p["SEs"]), dev(K), mask=dev(mask)))
    ref = O.aha_toeplitz(p["traj_type"], p["n_dim"], p["phi2_dim"], p["L"], p["x"], p["SEs"], K,
                         mask=mask)
    assert O.rel_l2(y, ref) <= TOL_APPLY


@pytest.mark.parametrize("L", [1, 2, 5, 7, 12, 16, 17, 20, 33])
def test_apply_ranks(L):
    """Every compiled rank and the runtime-rank path (L > 16)."""
    mr = _mr()
    rng = np.random.default_rng(L)
    n_dim, nc = (20, 18), 3
    cfg = mr.make_config("2D", n_dim, L, n_coils=nc)
    x = synth.crandn(rng, (L, 18, 20))
    S = synth.crandn(rng, (nc, 18, 20))
    K = random_kernel(rng, mr.phi2_toep_shape(cfg))
    for tri in ("lower", "upper"):
        cfg = mr.make_config("2D", n_dim, L, n_coils=nc, triangulation=tri)
        y = host(mr.aha_toeplitz(cfg, dev(x), dev(S), dev(K)))
        ref = O.aha_toeplitz("2D", n_dim, (40, 36), L, x, S, K, upper=tri == "upper")
        assert O.rel_l2(y, ref) <= TOL_APPLY


@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_calc_toep_exact(case):
    """mr_calc_toep vs the exact FP64 kernel (type-1 NUDFT + centred IFFT)."""
    mr = _mr()
    p = synth.reference_case(case)
    for tri in ("lower", "upper"):
        cfg = _cfg(p, tri)
        K = host(mr.calc_toep(cfg, dev(p["phi2"]), dev(p["traj"])))
        ref = O.calc_toep(p["traj_type"], p["phi2_dim"], p["L"], p["phi2"], p["traj"],
                          upper=tri == "upper")
        assert O.rel_l2(K, ref) <= TOL_TOEP, tri


@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_calc_mask_bit_exact(case):
    mr = _mr()
    p = synth.reference_case(case)
    cfg = _cfg(p)
    for r in (0, 1, 2):
        m = host(mr.calc_mask(cfg, dev(p["traj"]), radius=r))
        ref = O.calc_mask(p["traj_type"], p["phi2_dim"], p["traj"], r)
        np.testing.assert_array_equal(m, ref)


@pytest.mark.parametrize("case", [CASES[0], CASES[2], CASES[5], CASES[6]],
                         ids=[IDS[0], IDS[2], IDS[5], IDS[6]])
def test_op_vs_exact_nufft_route(case):
    """create_op from the Gram blocks vs the exact NUFFT-route A^H A."""
    mr = _mr()
    p = synth.reference_case(case)
    cfg = _cfg(p)
    with mr.create_op(cfg, dev(p["SEs"]), dev(p["phi2"]), dev(p["traj"])) as op:
        y = host(op(dev(p["x"])))
        info = op.info
    assert info["toep_source"] == "broadcast" and len(info["devices"]) == 1
    ref = O.aha_nufft(p["traj_type"], p["n_dim"], p["L"], p["x"], p["SEs"], p["phi2"], p["traj"])
    assert O.rel_l2(y, ref) <= TOL_OP


def test_op_injected_kernel_bit_identical():
    """An operator given a kernel equals mr_aha_toeplitz bit for bit
    (reference tests/check_op.py:252-259)."""
    mr = _mr()
    p = synth.reference_case(CASES[5])
    cfg = _cfg(p)
    rng = np.random.default_rng(5)
    K = dev(random_kernel(rng, mr.phi2_toep_shape(cfg)))
    x, S = dev(p["x"]), dev(p["SEs"])
    a = host(mr.aha_toeplitz(cfg, x, S, K))
    for share in (True, False):
        with mr.create_op(cfg, S, None, None, _phi2_toep=K, share_primary=share) as op:
            b = host(op(x))
            assert op.info["toep_source"] == "supplied"
        np.testing.assert_array_equal(a, b)


def test_op_kernel_matches_calc_toep():
    mr = _mr()
    p = synth.reference_case(CASES[6])
    cfg = _cfg(p)
    K = host(mr.calc_toep(cfg, dev(p["phi2"]), dev(p["traj"])))
    with mr.create_op(cfg, dev(p["SEs"]), dev(p["phi2"]), dev(p["traj"])) as op:
        Ko = host(op.kernel(0))
    assert O.rel_l2(Ko, K) <= 1e-6


def test_calc_toep_masked_equals_gathered():
    """Masked kernel = unmasked kernel gathered at the mask (reference
    tests/make_reference.py:484, <= 1e-6)."""
    mr = _mr()
    p = synth.reference_case(CASES[5])
    mask = O.calc_mask(p["traj_type"], p["phi2_dim"], p["traj"], 2)
    cfg = _cfg(p)
    full = host(mr.calc_toep(cfg, dev(p["phi2"]), dev(p["traj"])))
    cfgm = _cfg(p, is_masked=True)
    Km = host(mr.calc_toep(cfgm, dev(p["phi2"]), dev(p["traj"]), mask=dev(mask)))
    assert cfgm.num_masked == len(mask)
    ref = full.reshape(full.shape[0], -1)[:, mask]
    assert O.rel_l2(Km, ref) <= 1e-6


def test_upper_lower_agree():
    """A^H A from the upper and the lower packing agree (make_reference.py:489)."""
    mr = _mr()
    p = synth.reference_case(CASES[6])
    out = []
    for tri in ("lower", "upper"):
        cfg = _cfg(p, tri)
        K = mr.calc_toep(cfg, dev(p["phi2"]), dev(p["traj"]))
        out.append(host(mr.aha_toeplitz(cfg, dev(p["x"]), dev(p["SEs"]), K)))
    assert O.rel_l2(out[1], out[0]) <= 1e-5


def test_calc_toep_from_psf_matches():
    """Two-stage build: exact PSFs (oracle) finished on the GPU."""
    mr = _mr()
    p = synth.reference_case(CASES[5])
    cfg = _cfg(p)
    packed = O.pack_gram(p["phi2"], p["L"], False)
    psf = O.psf_exact(p["traj_type"], p["phi2_dim"], packed, p["traj"]).astype(np.complex64)
    out = dev(np.zeros(mr.phi2_toep_shape(cfg), np.complex64))
    mr.calc_toep_from_psf(cfg, dev(psf[:2]), 0, out)
    mr.calc_toep_from_psf(cfg, dev(psf[2:]), 2, out)
    ref = O.psf_to_kernel(p["traj_type"], psf.astype(np.complex128))
    assert O.rel_l2(host(out), ref) <= 1e-6
