"""CPU tests of the FP64 oracle: pinned to the reference's own outputs and to
an independent known-answer identity.

* Golden outputs made by the reference's CUDA apply compiled from its sources
  (``tests/golden/make_golden.py`` on a B200): the oracle's FP64 apply matches
  them to the reference's single-precision rounding (<= 1e-5), and the
  oracle's mask equals the reference's ``mr_calc_mask`` bit for bit.
* Known answer: with the exact kernel, the Toeplitz route equals the exact
  NUFFT route (the 2x circulant embedding is exact) to FP64 rounding, for
  2D, 3D and stack, odd sizes, a prime grid and both packings.
* The FP32 CPU port timed as the CPU baseline agrees with the oracle.
"""

from pathlib import Path

import numpy as np
import pytest

from mr_aha_b200 import synth
from oracle import aha_oracle as O

GOLDEN = Path(__file__).resolve().parent / "golden"
CASES = synth.REFERENCE_CASES
IDS = [c["name"] for c in CASES]
KERNEL_SEED = 1000  # tests/golden/make_golden.py


def golden_kernel(case, p, n_loc):
    rng = np.random.default_rng(KERNEL_SEED + case["seed"])
    ntri = O.num_tri(p["L"])
    return (rng.standard_normal((ntri, n_loc)) +
            1j * rng.standard_normal((ntri, n_loc))).astype(np.complex64)


@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_mask_matches_reference_bit_exact(case):
    p = synth.reference_case(case)
    g = np.load(GOLDEN / f"ref_{case['name']}.npz")
    for r in (0, 1, 2):
        np.testing.assert_array_equal(
            O.calc_mask(p["traj_type"], p["phi2_dim"], p["traj"], r), g[f"mask_r{r}"])


@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_apply_matches_reference(case):
    p = synth.reference_case(case)
    g = np.load(GOLDEN / f"ref_{case['name']}.npz")
    K = golden_kernel(case, p, int(np.prod(p["phi2_dim"])))
    for upper, name in ((False, "lower"), (True, "upper")):
        y = O.aha_toeplitz(p["traj_type"], p["n_dim"], p["phi2_dim"], p["L"], p["x"],
                           p["SEs"], K, upper=upper)
        assert O.rel_l2(g[f"AhAx_{name}"], y) <= 1e-5
    mask = g["mask_r2"]
    Km = golden_kernel(case, p, len(mask))
    y = O.aha_toeplitz(p["traj_type"], p["n_dim"], p["phi2_dim"], p["L"], p["x"], p["SEs"],
                       Km, mask=mask)
    assert O.rel_l2(g["AhAx_masked"], y) <= 1e-5


@pytest.mark.parametrize("case", [CASES[i] for i in (0, 1, 2, 4, 5, 6)],
                         ids=[IDS[i] for i in (0, 1, 2, 4, 5, 6)])
def test_toeplitz_equals_exact_nufft_route(case):
    p = synth.reference_case(case)
    ref = O.aha_nufft(p["traj_type"], p["n_dim"], p["L"], p["x"], p["SEs"], p["phi2"],
                      p["traj"])
    for upper in (False, True):
        K = O.calc_toep(p["traj_type"], p["phi2_dim"], p["L"], p["phi2"], p["traj"],
                        upper=upper)
        y = O.aha_toeplitz(p["traj_type"], p["n_dim"], p["phi2_dim"], p["L"], p["x"],
                           p["SEs"], K, upper=upper)
        assert O.rel_l2(y, ref) <= 1e-12


def test_index_maps_and_packing():
    for M in (1, 2, 7, 8, 101, 640):
        k = np.arange(M)
        np.testing.assert_array_equal(O.nat2cent(O.cent2nat(k, M), M), k)
        assert O.cent2nat(M // 2, M) == 0
    for L in (1, 2, 5, 16):
        for upper in (False, True):
            rows, cols = O.tri_pairs(L, upper)
            assert len(rows) == O.num_tri(L)
            for t, (r, c) in enumerate(zip(rows, cols)):
                assert O.tri_offset(r, c, L, upper) == (t, False)
                if r != c:
                    assert O.tri_offset(c, r, L, upper) == (t, True)
            rng = np.random.default_rng(L)
            A = rng.standard_normal((L, L)) + 1j * rng.standard_normal((L, L))
            A = A + A.conj().T
            phi2 = A.T[:, :, None]           # phi2[j, i, b] = A[i, j]
            packed = O.pack_gram(phi2, L, upper)
            np.testing.assert_allclose(O.unpack_blocks(packed, L, upper)[0], A)


def test_hermitian_operator():
    """<y, A^H A x> = <A^H A y, x> (reference examples/example_aha.cu:240-242)."""
    p = synth.reference_case(CASES[6])
    K = O.calc_toep(p["traj_type"], p["phi2_dim"], p["L"], p["phi2"], p["traj"])
    rng = np.random.default_rng(3)
    y = synth.crandn(rng, p["x"].shape, np.complex128)
    ax = O.aha_toeplitz(p["traj_type"], p["n_dim"], p["phi2_dim"], p["L"], p["x"], p["SEs"], K)
    ay = O.aha_toeplitz(p["traj_type"], p["n_dim"], p["phi2_dim"], p["L"], y, p["SEs"], K)
    a = np.vdot(y, ax)
    b = np.vdot(ay, p["x"])
    assert abs(a - b) <= 1e-10 * abs(a)


@pytest.mark.parametrize("case", [CASES[0], CASES[3], CASES[6]], ids=[IDS[0], IDS[3], IDS[6]])
def test_cpu_fp32_port(case):
    from oracle import cpu_port

    p = synth.reference_case(case)
    rng = np.random.default_rng(9)
    shape = (O.num_tri(p["L"]),) + O.spatial_axes(p["traj_type"], p["phi2_dim"])
    K = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)
    for upper in (False, True):
        cp = cpu_port.CpuToeplitz(p["traj_type"], p["n_dim"], p["phi2_dim"], p["L"], p["SEs"],
                                  K, upper=upper)
        ref = O.aha_toeplitz(p["traj_type"], p["n_dim"], p["phi2_dim"], p["L"], p["x"],
                             p["SEs"], K, upper=upper)
        assert O.rel_l2(cp.apply(p["x"]), ref) <= 1e-5


def test_oracle_catches_a_planted_error():
    """The checker is sensitive: a wrong conjugation in a copy of the oracle's
    block multiply (planted on the CPU) is far outside the tolerance."""
    p = synth.reference_case(CASES[5])
    rng = np.random.default_rng(4)
    shape = (O.num_tri(p["L"]),) + O.spatial_axes(p["traj_type"], p["phi2_dim"])
    K = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)
    good = O.aha_toeplitz(p["traj_type"], p["n_dim"], p["phi2_dim"], p["L"], p["x"], p["SEs"], K)
    blocks = O.kernel_natural_full(p["traj_type"], p["phi2_dim"], K, p["L"], False)
    bad = O.aha_toeplitz(p["traj_type"], p["n_dim"], p["phi2_dim"], p["L"], p["x"], p["SEs"], K,
                         blocks=np.conj(blocks))
    assert O.rel_l2(bad, good) > 1e-2


def test_oracle_cg_solves_spd_system():
    """The oracle CG reaches the direct solution of a small Hermitian positive
    definite system in n iterations (finite termination), with and without a
    start vector and a Tikhonov term."""
    rng = np.random.default_rng(11)
    n = 24
    Q, _ = np.linalg.qr(synth.crandn(rng, (n, n), np.complex128))
    A = (Q * np.linspace(1.0, 8.0, n)) @ Q.conj().T
    b = synth.crandn(rng, (n,), np.complex128)
    for lam, x0 in ((0.0, None), (0.5, synth.crandn(rng, (n,), np.complex128))):
        x, rr = O.cg(lambda v: A @ v, b, n, lam=lam, x0=x0)
        ref = np.linalg.solve(A + lam * np.eye(n), b)
        assert O.rel_l2(x, ref) <= 1e-9
        assert rr[-1] <= 1e-18 * rr[0]


def test_oracle_cg_on_the_operator():
    """CG on the oracle's own A^H A (a Gram-derived kernel, Hermitian PSD)
    decreases the A^H A-norm error monotonically, as CG must."""
    p = synth.reference_case(CASES[6])
    K = O.calc_toep(p["traj_type"], p["phi2_dim"], p["L"], p["phi2"], p["traj"])

    def A(v):
        return O.aha_toeplitz(p["traj_type"], p["n_dim"], p["phi2_dim"], p["L"], v, p["SEs"], K)

    b = A(p["x"].astype(np.complex128))
    errs = []
    for k in (2, 4, 8):
        x, _ = O.cg(A, b, k)
        e = x - p["x"]
        errs.append(float(np.vdot(e, A(e)).real))
    assert errs[0] > errs[1] > errs[2]


def test_dequantized_kernel_formats():
    """The 16-bit storage restatement: int16 codes within half a step of the
    value, bf16 within 2^-9 relative of the location's largest component, and
    exact round trips of representable values."""
    rng = np.random.default_rng(4)
    K = synth.crandn(rng, (10, 3, 5)).astype(np.complex64)
    K[:, 0, 0] = 0
    for fmt, tol in (("int16", 0.5 / 32767), ("bf16", 2.0 ** -8)):
        Kq = O.dequantized_kernel(K, fmt)
        m = np.maximum(np.abs(K.real), np.abs(K.imag)).max(axis=0)
        d = np.maximum(np.abs((Kq - K).real), np.abs((Kq - K).imag))
        assert np.all(d <= tol * m * 1.0001 + 1e-30)
        assert np.array_equal(O.dequantized_kernel(Kq, fmt) if fmt == "bf16" else Kq, Kq)
        assert np.all(Kq[:, 0, 0] == 0)
