"""Parity of the exact kernels the headline apply runs (320 x 320 x 56
stack, L = 16, 12 coils, operator built from its Gram blocks and owning its
kernel, so pass 3 reads the blocked kernel copy).

The launch trace (``mr_b200_trace_launches``) shows which template
instantiation ran each pass; every test asserts the headline ones:

* pass 1 ``k_xs_pipe<M=56,XT=32,tma>`` and pass 5
  ``k_coilsum_pipe<M=56,XT=32,tma>`` (56-point z lines, radix 8 x 7, tiles
  loaded by TMA tensor copies; with ``MR_AHA_B200_NO_TMA=1`` by per-thread
  cp.async, bit-identical);
* pass 2 ``k_hf_pipe<N=320,XT=8,tma>`` (tiles loaded by TMA tensor copies)
  and pass 4 ``k_strided_hi<N=320,XT=16>`` (first radix pass reading global
  memory directly: a whole-tile TMA load ahead of it measured slower, 7.0
  against 6.5 ms) -- half-length 320-point y lines;
* pass 3 ``k_xbdh<N=320,L=16,NC=1,F32,256,blocked,tma>`` (half-length x lines
  and the packed 16 x 16 Hermitian block multiply, input rows loaded by TMA
  tensor copies); with ``MR_AHA_B200_NO_TMA=1`` the same kernel with
  per-thread loads, bit-identical.

Checks, relative L2 (tolerances written in each test):

1. ``z56``: a 64 x 64 x 56 stack with L = 16 and 12 coils (the headline z
   kernels) against the FP64 oracle's apply of the operator's own kernel,
   <= 1e-5.
2. ``slab320``: a 320 x 320 x 4 stack with L = 16 and 3 coils (the headline
   y and x kernels, blocked copy) against the FP64 oracle, <= 1e-5; the same
   with the copy released (reference layout); the int16 and bf16 kernel
   formats (their own blocked copies, bit-identical to the reference layout)
   against the FP64 oracle of the values they store (<= 1e-5) and of the
   complex64 kernel (int16 <= 1e-4, bf16 <= 5e-3).
3. ``stack320``: the full headline workload against the reference's own CUDA
   apply (compiled from its sources into ``oracle/_ref`` by
   ``oracle/Makefile``) given the same kernel, <= 1e-5 (both FP32); with the
   blocked copy and without; the 16-bit formats against the complex64
   operator. Prints the agreement and both applies' times (CUDA events).
4. Config-2 solver at a size that runs the headline x / y kernels
   (320 x 320 x 2, L = 16, 2 coils): 10 CG iterations of every kernel format
   against the FP64 oracle CG of the same operator, <= 1e-4, and the
   complex64 iterate's distance from the FP64 CG of the exact kernel.
"""

import ctypes
import json
from pathlib import Path

import numpy as np
import pytest

from mr_aha_b200 import synth
from oracle import aha_oracle as O
from tests.gpu_util import dev, host

pytestmark = pytest.mark.gpu

REF_LIB = Path(__file__).resolve().parent.parent / "oracle" / "_ref" / "libmr_aha_ref.so"

Z_KERNELS = ("k_xs_pipe<M=56,XT=32,tma>", "k_coilsum_pipe<M=56,XT=32,tma>")
XY_KERNELS = ("k_hf_pipe<N=320,XT=8,tma>", "k_strided_hi<N=320,XT=16>")
X_BLOCKED = "k_xbdh<N=320,L=16,NC=1,F32,256,blocked,tma>"
X_BLOCKED_REGS = "k_xbdh<N=320,L=16,NC=1,F32,256,blocked>"
X_PLAIN = "k_xbdh<N=320,L=16,NC=1,F32,256>"


def traced(fn):
    """Run ``fn()`` with the calling thread's launch trace on; returns
    ``(result, [kernel line, ...])``."""
    from mr_aha_b200 import lib

    lib.mr_b200_trace_launches(1)
    try:
        r = fn()
    finally:
        lib.mr_b200_trace_launches(0)
    n = int(lib.mr_b200_trace_read(None, 0))
    buf = ctypes.create_string_buffer(n + 1)
    lib.mr_b200_trace_read(buf, n + 1)
    return r, buf.value.decode().splitlines()


def _spec(n_dim, L, nc, n_traj, seed, n_frames=32):
    return dict(traj_type="stack", n_dim=n_dim, L=L, n_coils=nc, n_traj=n_traj,
                n_kx=2 * n_dim[0], n_frames=n_frames, frame_rule="mod", seed=seed)


def _oracle(p, K, upper=False):
    return O.aha_toeplitz_lean(p["traj_type"], p["n_dim"], p["phi2_dim"], p["L"], p["x"],
                               p["SEs"], K, upper=upper)


def test_z56_kernels_vs_fp64(monkeypatch):
    import mr_aha_b200 as mr

    p = synth.spec_inputs(_spec((64, 64, 56), 16, 12, 48, seed=21))
    cfg = mr.make_config("stack", p["n_dim"], p["L"], n_coils=p["n_coils"])
    with mr.create_op(cfg, dev(p["SEs"]), dev(p["phi2"]), dev(p["traj"])) as op:
        y, trace = traced(lambda: host(op(dev(p["x"]))))
        assert op.device_status == 0
        monkeypatch.setenv("MR_AHA_B200_NO_TMA", "1")
        y_cp, trace_cp = traced(lambda: host(op(dev(p["x"]))))
        monkeypatch.delenv("MR_AHA_B200_NO_TMA")
        K = host(op.kernel())
    for k in Z_KERNELS:
        assert k in trace, trace
        assert k.replace(",tma>", ">") in trace_cp, trace_cp
    np.testing.assert_array_equal(y_cp, y)
    err = O.rel_l2(y, _oracle(p, K))
    print(f"z56 (64x64x56, L=16, 12 coils) vs FP64: {err:.3e}")
    assert err <= 1e-5, err


@pytest.fixture(scope="module")
def slab():
    import mr_aha_b200 as mr

    p = synth.spec_inputs(_spec((320, 320, 4), 16, 3, 160, seed=22))
    cfg = mr.make_config("stack", p["n_dim"], p["L"], n_coils=p["n_coils"])
    op = mr.create_op(cfg, dev(p["SEs"]), dev(p["phi2"]), dev(p["traj"]))
    K = host(op.kernel())
    ref = _oracle(p, K)
    yield p, op, K, ref
    op.close()


def test_slab320_blocked_and_reference_layout_vs_fp64(slab, monkeypatch):
    p, op, K, ref = slab
    assert op.blocked_copy(True) is True
    y, trace = traced(lambda: host(op(dev(p["x"]))))
    assert X_BLOCKED in trace and all(k in trace for k in XY_KERNELS), trace
    assert op.device_status == 0
    err = O.rel_l2(y, ref)
    print(f"slab320 blocked copy vs FP64: {err:.3e}")
    assert err <= 1e-5, err
    monkeypatch.setenv("MR_AHA_B200_NO_TMA", "1")
    y1, trace1 = traced(lambda: host(op(dev(p["x"]))))
    monkeypatch.delenv("MR_AHA_B200_NO_TMA")
    assert X_BLOCKED_REGS in trace1, trace1
    np.testing.assert_array_equal(y1, y)
    assert op.blocked_copy(False) is False
    y2, trace2 = traced(lambda: host(op(dev(p["x"]))))
    assert X_PLAIN in trace2 and X_BLOCKED not in trace2, trace2
    np.testing.assert_array_equal(y2, y)
    assert op.blocked_copy(True) is True


@pytest.mark.parametrize("fmt,tol_exact", [("int16", 1e-4), ("bf16", 5e-3)])
def test_slab320_16bit_vs_fp64(slab, fmt, tol_exact):
    p, op, K, ref = slab
    kf = "I16" if fmt == "int16" else "BF16"
    op.set_kernel_format(fmt)
    try:
        # the 16-bit blocked copy (four codes per 16-byte load), then the
        # reference layout: the same codes, decode and products
        y, trace = traced(lambda: host(op(dev(p["x"]))))
        assert f"k_xbdh<N=320,L=16,NC=1,{kf},256,blocked,tma>" in trace, trace
        assert op.blocked_copy(False) is False
        y1, trace1 = traced(lambda: host(op(dev(p["x"]))))
        assert f"k_xbdh<N=320,L=16,NC=1,{kf},256>" in trace1, trace1
        np.testing.assert_array_equal(y1, y)
    finally:
        op.set_kernel_format("complex64")
    assert op.blocked_copy(True) is True
    same = O.rel_l2(y, _oracle(p, O.dequantized_kernel(K, fmt)))
    exact = O.rel_l2(y, ref)
    print(f"slab320 {fmt}: vs FP64 of the stored values {same:.3e}, "
          f"vs FP64 of the complex64 kernel {exact:.3e}")
    assert same <= 1e-5, same
    assert exact <= tol_exact, exact


def _ref_lib():
    from mr_aha_b200._lib import PROTOTYPES

    lib = ctypes.CDLL(str(REF_LIB))
    for n in ("mr_aha_toeplitz", "mr_aha_plan_create", "mr_aha_plan_execute",
              "mr_aha_plan_destroy", "mr_last_error"):
        res, args = PROTOTYPES[n]
        getattr(lib, n).restype = res
        getattr(lib, n).argtypes = args
    return lib


def _time_ms(fn, reps=3):
    import torch

    fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def _rel_t(a, b):
    import torch

    d = (a - b).to(torch.complex128)
    return float(torch.linalg.vector_norm(d) / torch.linalg.vector_norm(b.to(torch.complex128)))


@pytest.mark.skipif(not REF_LIB.exists(), reason="reference apply not built (oracle/Makefile)")
def test_stack320_vs_reference_cuda_apply():
    import torch

    import mr_aha_b200 as mr
    from mr_aha_b200._lib import MRConfig

    w = synth.workload("stack320")
    cfg = mr.make_config(w["traj_type"], w["n_dim"], w["L"], n_coils=w["n_coils"])
    x, S = dev(w["x"]), dev(w["SEs"])
    ref = _ref_lib()
    out = {}
    with mr.create_op(cfg, S, dev(w["phi2"]), dev(w["traj"])) as op:
        K = op.kernel()
        y, trace = traced(lambda: op(x))
        for k in Z_KERNELS + XY_KERNELS + (X_BLOCKED,):
            assert k in trace, trace
        assert op.device_status == 0
        # the reference's own apply of the same kernel
        rcfg = MRConfig.from_buffer_copy(cfg)
        plan = ctypes.c_void_p()
        assert ref.mr_aha_plan_create(ctypes.byref(rcfg), ctypes.byref(plan)) == 0, \
            ref.mr_last_error()
        y_ref = torch.empty_like(x)

        def run_ref():
            rc = ref.mr_aha_plan_execute(plan, x.data_ptr(), S.data_ptr(), K.data_ptr(), None,
                                         y_ref.data_ptr())
            assert rc == 0, ref.mr_last_error()

        try:
            out["ref_ms"] = _time_ms(run_ref)
        finally:
            torch.cuda.synchronize()
            ref.mr_aha_plan_destroy(plan)
        y_out = torch.empty_like(x)
        out["ours_ms"] = _time_ms(lambda: op(x, out=y_out))
        out["blocked_vs_reference"] = _rel_t(y, y_ref)
        assert op.blocked_copy(False) is False
        y2, trace2 = traced(lambda: op(x))
        assert X_PLAIN in trace2, trace2
        out["reference_layout_vs_reference"] = _rel_t(y2, y_ref)
        assert op.blocked_copy(True) is True
        for fmt in ("int16", "bf16"):
            op.set_kernel_format(fmt)
            out[f"{fmt}_vs_complex64"] = _rel_t(op(x), y)
        op.set_kernel_format("complex64")
    print("stack320:", json.dumps(out))
    assert out["blocked_vs_reference"] <= 1e-5
    assert out["reference_layout_vs_reference"] <= 1e-5
    assert out["int16_vs_complex64"] <= 1e-4
    assert out["bf16_vs_complex64"] <= 5e-3


@pytest.mark.parametrize("fmt", ["complex64", "int16", "bf16"])
def test_config2_cg_at_headline_xy_kernels_vs_fp64(fmt):
    """10 CG iterations on b = A^H A x_true + noise (1e-3 RMS relative),
    from zero. The FP64 oracle CG applies the values the operator stores:
    iterate within 1e-4. The complex64 solve is also compared with the FP64
    CG of the exact kernel (the operator the 16-bit forms approximate)."""
    import mr_aha_b200 as mr

    p = synth.spec_inputs(_spec((320, 320, 2), 16, 2, 120, seed=23))
    cfg = mr.make_config("stack", p["n_dim"], p["L"], n_coils=p["n_coils"])
    with mr.create_op(cfg, dev(p["SEs"]), dev(p["phi2"]), dev(p["traj"])) as op:
        K = host(op.kernel())
        Kq = K if fmt == "complex64" else O.dequantized_kernel(K, fmt)

        def A(v):
            return O.aha_toeplitz_lean("stack", p["n_dim"], p["phi2_dim"], p["L"], v, p["SEs"], Kq)

        x_true = p["x"].astype(np.complex128)
        ax = A(x_true)
        rng = np.random.default_rng(123)
        sigma = 1e-3 * np.linalg.norm(ax) / np.sqrt(ax.size)
        b = (ax + sigma * synth.crandn(rng, ax.shape, np.complex128)).astype(np.complex64)
        x_ref, _ = O.cg(A, b, 10)
        if fmt != "complex64":
            op.set_kernel_format(fmt)
        (x, rr), trace = traced(lambda: op.cg(dev(b), 10, graph=False))
        assert all(k in trace for k in XY_KERNELS), trace
    err = O.rel_l2(host(x), x_ref)
    print(f"config-2 CG ({fmt}, 10 iterations) vs FP64 CG of the same operator: {err:.3e}")
    assert err <= 1e-4, err
