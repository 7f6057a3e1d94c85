"""Checkpoint of a 16-bit kernel (``mr_b200_op_save_kernel16`` /
``mr_b200_op_load_kernel16``), through the C ABI.

* The codes and scales saved from a 16-bit operator, taken through host
  memory and loaded into an operator built from an all-zero kernel, give
  bit-identical applies (same codes, same kernels); that operator reports the
  format and no longer has a complex64 kernel.
* Masked operators: the same round trip over ``num_masked`` locations.
* The saved codes are the oracle's restatement of the quantisation
  (``dequantized_kernel``) up to FP32 rounding of the values they represent,
  and the restored operator meets 1e-5 against the FP64 oracle of those
  values (relative L2).
* Saving a complex64 kernel is refused.
"""

import numpy as np
import pytest

from mr_aha_b200 import synth
from oracle import aha_oracle as O
from tests.gpu_util import dev, host

pytestmark = pytest.mark.gpu

CASE = synth.REFERENCE_CASES[5]  # stack 40 x 36 x 10, L = 3, 3 coils


def _cfg(p, **kw):
    import mr_aha_b200 as mr

    return mr.make_config(p["traj_type"], p["n_dim"], p["L"], phi2_dim=p["phi2_dim"],
                          n_coils=p["n_coils"], **kw)


@pytest.mark.parametrize("fmt", ["int16", "bf16"])
def test_kernel16_roundtrip(fmt):
    import torch

    import mr_aha_b200 as mr

    p = synth.reference_case(CASE)
    cfg = _cfg(p)
    x = dev(p["x"])
    with mr.create_op(cfg, dev(p["SEs"]), dev(p["phi2"]), dev(p["traj"])) as a:
        with pytest.raises(mr.MRError):
            a.save_kernel16()
        K = host(a.kernel())
        a.set_kernel_format(fmt)
        y_a = host(a(x))
        f, codes, scale = a.save_kernel16()
    assert f == fmt and codes.shape == (K.shape[0], K[0].size, 2)
    # through host memory, as a file would
    codes_h, scale_h = codes.cpu().clone(), scale.cpu().clone()
    zero = torch.zeros(mr.phi2_toep_shape(cfg), dtype=torch.complex64, device="cuda")
    with mr.create_op(cfg, dev(p["SEs"]), None, None, _phi2_toep=zero,
                      share_primary=False) as b:
        b.load_kernel16(fmt, codes_h.cuda(), scale_h.cuda())
        assert b.kernel_format == fmt
        with pytest.raises(mr.MRError):
            b.kernel()
        y_b = host(b(x))
    np.testing.assert_array_equal(y_b, y_a)
    # the codes represent the oracle's dequantised kernel
    sc = scale_h.numpy()
    c = codes_h.float().numpy() if fmt == "bf16" else codes_h.numpy().astype(np.float64)
    vals = (c[..., 0] + 1j * c[..., 1]) * sc[None, :]
    Kq = O.dequantized_kernel(K, fmt).reshape(vals.shape)
    assert O.rel_l2(vals, Kq) <= 1e-6
    ref = O.aha_toeplitz(p["traj_type"], p["n_dim"], p["phi2_dim"], p["L"], p["x"], p["SEs"],
                         Kq.reshape(K.shape))
    assert O.rel_l2(y_b, ref) <= 1e-5


def test_kernel16_roundtrip_masked():
    import mr_aha_b200 as mr

    p = synth.reference_case(CASE)
    mask = mr.calc_mask(_cfg(p), dev(p["traj"]))
    cfg = _cfg(p, is_masked=True, num_masked=int(mask.numel()))
    x = dev(p["x"])
    args = (dev(p["SEs"]), dev(p["phi2"]), dev(p["traj"]))
    with mr.create_op(cfg, *args, mask=mask) as a:
        a.set_kernel_format("int16")
        y_a = host(a(x))
        _, codes, scale = a.save_kernel16()
    assert codes.shape[1] == int(mask.numel())
    with mr.create_op(cfg, *args, mask=mask) as b:
        y_c64 = host(b(x))
        b.load_kernel16("int16", codes, scale)
        y_b = host(b(x))
    np.testing.assert_array_equal(y_b, y_a)
    assert not np.array_equal(y_b, y_c64)
