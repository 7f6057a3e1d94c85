"""GPU test of the allocation-free apply, mr_b200_aha_toeplitz_noalloc.

Callers that cannot allocate device memory (their GPU memory is owned by
their own pool, or their processing loop must not synchronise or risk an
out-of-memory failure) use this entry point; it takes its work space from
the library's fixed static scratch array. Through the C ABI, two calls in a
row must each match mr_aha_toeplitz, the allocating entry point, and the
FP64 oracle's apply of the same inputs (oracle.aha_oracle.aha_toeplitz),
within the apply tolerance of the parity tests (1e-5 relative L2); the
second call also checks that the contents left in the shared array by the
first do not leak into the result. Collected last (file name) so that a run stopping at the
first failure has run every other test first; it also passes on its own.
"""

import ctypes

import numpy as np
import pytest

from mr_aha_b200 import synth
from oracle import aha_oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _rel(a, b):
    a = a.astype(np.complex128)
    b = b.astype(np.complex128)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("case", [synth.REFERENCE_CASES[0], synth.REFERENCE_CASES[4],
                                  synth.REFERENCE_CASES[6]],
                         ids=lambda c: c["name"])
@pytest.mark.parametrize("masked", [False, True])
def test_noalloc_matches_allocating_apply(case, masked):
    import torch

    import mr_aha_b200 as mr
    from mr_aha_b200 import lib
    from mr_aha_b200.api import _ptr

    p = synth.reference_case(case)
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(7)
    mask = None
    if masked:
        cfg0 = mr.make_config(p["traj_type"], p["n_dim"], p["L"], phi2_dim=p["phi2_dim"],
                              n_coils=p["n_coils"])
        mask = mr.calc_mask(cfg0, torch.from_numpy(p["traj"]).to(dev))
    cfg = mr.make_config(p["traj_type"], p["n_dim"], p["L"], phi2_dim=p["phi2_dim"],
                         n_coils=p["n_coils"], is_masked=masked,
                         num_masked=0 if mask is None else int(mask.numel()))
    shape = mr.phi2_toep_shape(cfg)
    K = torch.from_numpy((rng.standard_normal(shape) + 1j * rng.standard_normal(shape))
                         .astype(np.complex64)).to(dev)
    x = torch.from_numpy(p["x"]).to(dev)
    S = torch.from_numpy(p["SEs"]).to(dev)
    ref = mr.aha_toeplitz(cfg, x, S, K, mask=mask).cpu().numpy()
    ref64 = O.aha_toeplitz(p["traj_type"], p["n_dim"], p["phi2_dim"], p["L"], p["x"],
                           p["SEs"], K.cpu().numpy(),
                           mask=None if mask is None else mask.cpu().numpy())
    for call in range(2):
        out = torch.full_like(x, complex(float("nan"), 0.0))
        rc = lib.mr_b200_aha_toeplitz_noalloc(
            ctypes.byref(cfg), _ptr(x, "x", "complex64"), _ptr(S, "SEs", "complex64"),
            _ptr(K, "phi2_toep", "complex64"), _ptr(mask, "mask", "int64", allow_none=True),
            _ptr(out, "out", "complex64"))
        assert rc == 0, lib.mr_last_error()
        torch.cuda.synchronize()
        y = out.cpu().numpy()
        assert _rel(y, ref) <= TOL, f"call {call}: vs the allocating apply"
        assert O.rel_l2(y, ref64) <= TOL, f"call {call}: vs the FP64 oracle"


def test_noalloc_rejects_oversized_problem():
    import mr_aha_b200 as mr
    from mr_aha_b200 import lib

    cfg = mr.make_config("stack", (320, 320, 56), 16, n_coils=12)
    buf = ctypes.c_void_p(1)  # never dereferenced: the size check comes first
    rc = lib.mr_b200_aha_toeplitz_noalloc(ctypes.byref(cfg), buf, buf, buf, None,
                                          ctypes.c_void_p(2))
    assert rc == -7
    assert b"static scratch" in lib.mr_last_error()
