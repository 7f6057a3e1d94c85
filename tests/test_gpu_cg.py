"""Device conjugate gradients against the FP64 oracle CG (``oracle.aha_oracle.cg``).

Problem: the small stack workload (64 x 64 x 8, L = 4, 4 coils) with its
Gram-derived kernel from the library's ``calc_toep``; the oracle applies the
same kernel in FP64. ``b = A^H A x_true + n`` with complex Gaussian noise at
1e-3 of ``|A^H A x_true|`` per element (RMS), 30 iterations from zero.

The oracle of a 16-bit operator applies the values that operator stores
(``O.dequantized_kernel``) in FP64, so every format is held to one bar: the
relative L2 of the iterate after 30 iterations vs the FP64 oracle's iterate
at most 1e-4, the solver's error bar (measured: about 1e-5, FP32 rounding
of 30 iterations). How far a 16-bit operator is from the
complex64 one is the apply-level figure of tests/test_gpu_precision.py; CG
amplifies it by the conditioning (about 5e-3 on the iterate for the int16
kernel here). The solver is deterministic (fixed-order FP64 reductions):
repeated solves, graph replay vs eager launches and 10 + 20 steps vs 30 steps
agree bit for bit.
"""

import functools

import numpy as np
import pytest

from mr_aha_b200 import synth
from oracle import aha_oracle as O
from tests.gpu_util import dev, host

pytestmark = pytest.mark.gpu

N_ITER = 30
TOL = 1e-4


@functools.lru_cache(maxsize=None)
def _problem(fmt="complex64"):
    import mr_aha_b200 as mr

    w = synth.workload("stack64")
    cfg = mr.make_config(w["traj_type"], w["n_dim"], w["L"], n_coils=w["n_coils"])
    K = host(mr.calc_toep(cfg, dev(w["phi2"]), dev(w["traj"])))
    Kq = K if fmt == "complex64" else O.dequantized_kernel(K, fmt)

    def A(v):
        return O.aha_toeplitz(w["traj_type"], w["n_dim"], w["phi2_dim"], w["L"], v, w["SEs"], Kq)

    x_true = w["x"].astype(np.complex128)
    ax = A(x_true)
    rng = np.random.default_rng(123)
    sigma = 1e-3 * np.linalg.norm(ax) / np.sqrt(ax.size)
    b = (ax + sigma * synth.crandn(rng, ax.shape, np.complex128)).astype(np.complex64)
    x_ref, rr_ref = O.cg(A, b, N_ITER)
    return w, cfg, K, b, x_ref, rr_ref, A


def _op(fmt="complex64"):
    import mr_aha_b200 as mr

    w, cfg, K, *_ = _problem()
    return mr.create_op(cfg, dev(w["SEs"]), None, None, _phi2_toep=dev(K), kernel_format=fmt)


@pytest.mark.parametrize("fmt", ["complex64", "int16", "bf16"])
def test_cg_matches_fp64_oracle(fmt):
    w, cfg, K, b, x_ref, rr_ref, A = _problem(fmt)
    with _op(fmt) as op:
        x, rr = op.cg(dev(b), N_ITER)
    err = O.rel_l2(host(x), x_ref)
    assert err <= TOL, err
    # the residual history follows the oracle's while it is far above rounding
    assert np.allclose(rr[:6], rr_ref[:6], rtol=1e-3)
    assert rr[-1] < 1e-3 * rr[0]


def test_cg_deterministic_and_graph_equals_eager():
    *_, b, x_ref, rr_ref, A = _problem()
    with _op() as op:
        x1, r1 = op.cg(dev(b), N_ITER, graph=True)
        x2, r2 = op.cg(dev(b), N_ITER, graph=True)
        x3, r3 = op.cg(dev(b), N_ITER, graph=False)
    assert np.array_equal(host(x1), host(x2)) and np.array_equal(r1, r2)
    assert np.array_equal(host(x1), host(x3)) and np.array_equal(r1, r3)


def test_cg_stepwise_equals_one_call():
    import torch

    *_, b, x_ref, rr_ref, A = _problem()
    with _op() as op:
        x_one, r_one = op.cg(dev(b), N_ITER)
        bd = dev(b)
        x = torch.empty_like(bd)
        with op.cg_solver(bd, x, max_iters=N_ITER) as s:
            s.step(10)
            s.step(N_ITER - 10)
            r = s.residuals()
        assert np.array_equal(host(x), host(x_one))
        assert np.array_equal(r, r_one)


def test_cg_start_vector_and_tikhonov():
    w, cfg, K, b, x_ref, rr_ref, A = _problem()
    rng = np.random.default_rng(5)
    x0 = (0.1 * synth.crandn(rng, b.shape)).astype(np.complex64)
    lam = 0.05
    ref, _ = O.cg(A, b, 12, lam=lam, x0=x0)
    with _op() as op:
        x, rr = op.cg(dev(b), 12, lam=lam, x0=dev(x0))
    assert O.rel_l2(host(x), ref) <= 1e-5


def test_cg_argument_errors():
    import torch

    import mr_aha_b200 as mr

    *_, b, x_ref, rr_ref, A = _problem()
    with _op() as op:
        bd = dev(b)
        with pytest.raises(mr.MRError):
            op.cg(bd, 3, lam=-1.0)
        with pytest.raises(mr.MRError):
            op.cg_solver(bd, bd)
        with pytest.raises(ValueError):
            op.cg(bd[:1], 3)
        x = torch.zeros_like(bd)
        with op.cg_solver(bd, x, max_iters=2) as s:
            s.step(5)  # more steps than the history holds: history stops at 2
            assert len(s.residuals()) == 3


@pytest.mark.parametrize("fmt", ["int16", "bf16"])
def test_16bit_operator_equals_dequantized_kernel(fmt):
    """The device's 16-bit storage holds the values of the oracle's
    restatement: an operator given those values as a complex64 kernel gives
    the same apply up to FP32 rounding (the 16-bit operator multiplies the
    stored codes and scales each location's result once): relative L2 at
    most 1e-6."""
    import mr_aha_b200 as mr

    w, cfg, K, b, *_ = _problem()
    Kq = O.dequantized_kernel(K, fmt)
    with _op(fmt) as op16, mr.create_op(cfg, dev(w["SEs"]), None, None,
                                        _phi2_toep=dev(Kq)) as opq:
        y16 = host(op16(dev(b)))
        yq = host(opq(dev(b)))
    assert O.rel_l2(y16, yq) <= 1e-6
