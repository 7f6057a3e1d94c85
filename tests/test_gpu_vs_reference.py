"""GPU parity against the reference's OWN CUDA apply (compiled from its
sources into oracle/_ref by oracle/Makefile), at sizes beyond what the FP64
oracle checks in seconds: same inputs through both C ABIs, relative L2
difference <= 1e-5 (both are single precision; measured ~2.5e-7 at
320 x 320 x 56, L = 16, 12 coils).
"""

import ctypes
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REF_LIB = Path(__file__).resolve().parent.parent / "oracle" / "_ref" / "libmr_aha_ref.so"

SIZES = [
    # traj_type, n_dim, L, C, masked, tri
    ("stack", (160, 160, 16), 16, 4, False, "lower"),
    ("stack", (96, 80, 12), 8, 3, True, "upper"),
    ("2D", (256, 192), 12, 5, False, "lower"),
    ("2D", (128, 128), 20, 2, False, "upper"),   # rank above 16: tiled kernels of the reference
    ("3D", (48, 40, 32), 5, 2, False, "lower"),
]


def _ref():
    from mr_aha_b200._lib import PROTOTYPES

    lib = ctypes.CDLL(str(REF_LIB))
    for n in ("mr_aha_toeplitz", "mr_last_error", "mr_calc_mask"):
        res, args = PROTOTYPES[n]
        getattr(lib, n).restype = res
        getattr(lib, n).argtypes = args
    return lib


@pytest.mark.skipif(not REF_LIB.exists(), reason="reference apply not built (oracle/Makefile)")
@pytest.mark.parametrize("size", SIZES, ids=[f"{s[0]}_{'x'.join(map(str, s[1]))}_L{s[2]}" for s in SIZES])
def test_apply_matches_reference_cuda(size):
    import torch

    import mr_aha_b200 as mr
    from mr_aha_b200 import synth

    tt, n_dim, L, C, masked, tri = size
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(sum(n_dim) + L)
    traj = synth.make_traj(tt, 64, 2 * n_dim[0])
    cfg0 = mr.make_config(tt, n_dim, L, n_coils=C, triangulation=tri)
    mask = mr.calc_mask(cfg0, torch.from_numpy(traj).to(dev)) if masked else None
    cfg = mr.make_config(tt, n_dim, L, n_coils=C, triangulation=tri, is_masked=masked,
                         num_masked=0 if mask is None else int(mask.numel()))
    shape = mr.phi2_toep_shape(cfg)
    K = torch.from_numpy((rng.standard_normal(shape) + 1j * rng.standard_normal(shape))
                         .astype(np.complex64)).to(dev)
    img = tuple(reversed(n_dim))
    x = torch.from_numpy(synth.crandn(rng, (L,) + img)).to(dev)
    S = torch.from_numpy(synth.crandn(rng, (C,) + img)).to(dev)
    ours = mr.aha_toeplitz(cfg, x, S, K, mask=mask)
    ref = _ref()
    y = torch.empty_like(x)
    rc = ref.mr_aha_toeplitz(ctypes.byref(cfg), x.data_ptr(), S.data_ptr(), K.data_ptr(),
                             None if mask is None else mask.data_ptr(), y.data_ptr())
    assert rc == 0, ref.mr_last_error()
    torch.cuda.synchronize()
    d = (ours - y).to(torch.complex128)
    rel = float(torch.linalg.vector_norm(d) / torch.linalg.vector_norm(y.to(torch.complex128)))
    assert rel <= 1e-5, rel
