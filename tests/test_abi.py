"""CPU tests of the C ABI boundary and the host-side logic (no GPU calls).

* ``libmr_aha_c.so`` loads and exports every function declared in
  ``include/mr_aha/*.h``.
* Struct layouts match the reference's C structs (field offsets).
* ``mr_config_defaults`` / ``mr_config_validate`` / the size helpers /
  ``mr_status_string`` behave exactly like the reference's own host code
  (``src/common/mr_config.cpp``, compiled into ``oracle/_ref`` by
  ``oracle/Makefile``) on a sweep of valid and invalid configurations.
* The Python binding validates like the reference's ``api.py``.
"""

import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
REF_HOST = ROOT / "oracle" / "_ref" / "libmr_ref_host.so"


def _lib():
    from mr_aha_b200._lib import lib

    return lib


def declared_symbols():
    names = set()
    for h in (ROOT / "include" / "mr_aha").glob("*.h"):
        text = h.read_text()
        for m in re.finditer(r"MR_EXPORT\s+[^;(]*?\b(mr_\w+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    from mr_aha_b200._lib import PROTOTYPES, library_path

    names = declared_symbols()
    reference_abi = {
        "mr_status_string", "mr_last_error", "mr_backend", "mr_config_defaults",
        "mr_config_validate", "mr_num_tri", "mr_image_size", "mr_pad_size",
        "mr_phi2_toep_size", "mr_x_size", "mr_se_size", "mr_aha_plan_create",
        "mr_aha_plan_execute", "mr_aha_plan_destroy", "mr_aha_toeplitz",
        "mr_op_options_defaults", "mr_op_create", "mr_op_execute", "mr_op_info", "mr_op_kernel",
        "mr_op_destroy", "mr_op_abandon", "mr_calc_toep", "mr_calc_toep_from_psf",
        "mr_calc_mask", "mr_version"}
    assert reference_abi <= set(names)
    lib = ctypes.CDLL(str(library_path()))
    for n in names:
        assert hasattr(lib, n), n
        assert n in PROTOTYPES, f"{n} has no ctypes prototype"
    assert _lib().mr_backend() == b"cuda"


def test_struct_layouts():
    from mr_aha_b200._lib import MRConfig, MROpInfo, MROpInputs, MROpOptions

    # offsets of the C structs (x86-64 SysV, natural alignment)
    assert MRConfig.num_masked.offset == 48 and MRConfig.eps.offset == 64
    assert MRConfig.stream.offset == 80 and ctypes.sizeof(MRConfig) == 104
    assert ctypes.sizeof(MROpInputs) == 56 and MROpInputs.d_phi2_toep.offset == 48
    assert ctypes.sizeof(MROpOptions) == 48 and MROpOptions.nufft_upsampfac.offset == 32
    assert MROpInfo.peer_bandwidth_gbs.offset == 272 and ctypes.sizeof(MROpInfo) == 320


def _configs():
    """A sweep of valid and invalid configurations (edge cases of every rule)."""
    out = []
    base = dict(tt=2, ns=3, n=(64, 64, 8), m=(128, 128, 8), L=4, tri=0, masked=0, nm=0, C=4,
                eps=1e-6, r=2)
    out.append(base)
    out.append(dict(base, tt=0, ns=2, n=(50, 40, 1), m=(100, 80, 1)))
    out.append(dict(base, tt=1, n=(24, 20, 16), m=(48, 40, 32)))
    out.append(dict(base, m=(128, 128, 16)))                 # stack with Mz != Nz
    out.append(dict(base, ns=2))                             # wrong n_spatial
    out.append(dict(base, tt=0, ns=2, n=(50, 40, 2), m=(100, 80, 2)))  # unused axis != 1
    out.append(dict(base, m=(63, 128, 8)))                   # M < N
    out.append(dict(base, n=(0, 64, 8)))                     # zero extent
    out.append(dict(base, L=0))
    out.append(dict(base, C=0))
    out.append(dict(base, tri=2))
    out.append(dict(base, eps=0.0))
    out.append(dict(base, eps=1.0))
    out.append(dict(base, r=-1))
    out.append(dict(base, masked=1, nm=0))
    out.append(dict(base, masked=1, nm=128 * 128 * 8 + 1))
    out.append(dict(base, masked=1, nm=128 * 128 * 8))
    out.append(dict(base, tt=5))
    out.append(dict(base, n=(64, 64, 8), m=(64, 64, 8)))      # M == N allowed
    out.append(dict(base, tt=0, ns=3, n=(50, 40, 1), m=(100, 80, 1)))
    return out


def _fill(lib, cfg_cls, d):
    c = cfg_cls()
    lib.mr_config_defaults(ctypes.byref(c), d["tt"] if d["tt"] in (0, 1, 2) else 2)
    c.traj_type = d["tt"]
    c.n_spatial = d["ns"]
    for i in range(3):
        c.n_dim[i] = d["n"][i]
        c.phi2_dim[i] = d["m"][i]
    c.L, c.triangulation, c.is_masked, c.num_masked = d["L"], d["tri"], d["masked"], d["nm"]
    c.n_coils, c.eps, c.mask_radius = d["C"], d["eps"], d["r"]
    return c


@pytest.mark.skipif(not REF_HOST.exists(), reason="reference host code not built here")
def test_config_semantics_match_reference_host_code():
    from mr_aha_b200._lib import PROTOTYPES, MRConfig

    ours = _lib()
    ref = ctypes.CDLL(str(REF_HOST))
    for n in ("mr_config_defaults", "mr_config_validate", "mr_num_tri", "mr_image_size",
              "mr_pad_size", "mr_phi2_toep_size", "mr_x_size", "mr_se_size",
              "mr_status_string", "mr_last_error"):
        res, args = PROTOTYPES[n]
        getattr(ref, n).restype = res
        getattr(ref, n).argtypes = args
    for tt in (0, 1, 2):
        a, b = MRConfig(), MRConfig()
        assert ours.mr_config_defaults(ctypes.byref(a), tt) == ref.mr_config_defaults(
            ctypes.byref(b), tt) == 0
        assert bytes(a) == bytes(b)
    for d in _configs():
        a, b = _fill(ours, MRConfig, d), _fill(ref, MRConfig, d)
        ra = ours.mr_config_validate(ctypes.byref(a))
        rb = ref.mr_config_validate(ctypes.byref(b))
        assert ra == rb, (d, ours.mr_last_error(), ref.mr_last_error())
        for n in ("mr_image_size", "mr_pad_size", "mr_phi2_toep_size", "mr_x_size", "mr_se_size"):
            assert getattr(ours, n)(ctypes.byref(a)) == getattr(ref, n)(ctypes.byref(b)), n
    for L in (-1, 0, 1, 16, 512):
        assert ours.mr_num_tri(L) == ref.mr_num_tri(L)
    for s in range(-12, 2):
        assert ours.mr_status_string(s) == ref.mr_status_string(s)
    assert ours.mr_config_validate(None) == ref.mr_config_validate(None) == -1


def test_last_error_is_thread_local_and_cleared():
    import threading

    from mr_aha_b200._lib import MRConfig

    lib = _lib()
    c = MRConfig()
    lib.mr_config_defaults(ctypes.byref(c), 2)
    c.L = 0
    assert lib.mr_config_validate(ctypes.byref(c)) == -2
    assert b"L = 0" in lib.mr_last_error()
    seen = []
    t = threading.Thread(target=lambda: seen.append(lib.mr_last_error()))
    t.start()
    t.join()
    assert seen == [b""]
    c.L = 1
    assert lib.mr_config_validate(ctypes.byref(c)) == 0
    assert lib.mr_last_error() == b""


def test_python_binding_validation():
    import mr_aha_b200 as mr

    cfg = mr.make_config("stack", (64, 64, 8), 4, n_coils=4)
    assert list(cfg.phi2_dim) == [128, 128, 8]
    assert mr.phi2_toep_shape(cfg) == (10, 8, 128, 128)
    assert mr.num_tri(16) == 136
    with pytest.raises(ValueError):
        mr.make_config("stack", (64, 64), 4)
    with pytest.raises(mr.MRError) as e:
        mr.make_config("stack", (64, 64, 8), 4, phi2_dim=(128, 128, 16))
    assert e.value.status == -2
    with pytest.raises(ValueError):
        mr.make_config("4D", (64, 64, 8), 4)
    m = mr.make_config("2D", (50, 40), 3, is_masked=True)     # num_masked filled later
    assert m.is_masked == 1 and m.num_masked == 0
    with pytest.raises(TypeError):
        mr.aha_toeplitz(cfg, np.zeros((4, 8, 64, 64), np.complex64),
                        np.zeros((4, 8, 64, 64), np.complex64),
                        np.zeros((10, 8, 128, 128), np.complex64))


def test_host_buffer_validation():
    """Host-buffer arguments of ``AhAOp.apply_host``: dtype, layout, size and
    memory kind are checked before any call into the library."""
    import numpy as np
    import torch

    from mr_aha_b200.api import _host_ptr, pinned_empty

    a = np.zeros((2, 3), np.complex64)
    assert _host_ptr(a, "x", 6) == a.ctypes.data
    t = torch.zeros(6, dtype=torch.complex64)
    assert _host_ptr(t, "x", 6) == t.data_ptr()
    with pytest.raises(TypeError):
        _host_ptr(a.astype(np.complex128), "x", 6)
    with pytest.raises(ValueError):
        _host_ptr(np.zeros((3, 4), np.complex64)[:, ::2], "x", 6)
    with pytest.raises(ValueError):
        _host_ptr(a, "x", 7)
    with pytest.raises(TypeError):
        _host_ptr([0j] * 6, "x", 6)
    if torch.cuda.is_available():
        p = pinned_empty((2, 3))
        assert p.dtype == np.complex64 and p.shape == (2, 3)


def test_synthetic_workloads_are_seeded():
    from mr_aha_b200 import synth

    a = synth.workload("stack64")
    b = synth.workload("stack64")
    for k in ("traj", "phi2", "SEs", "x"):
        np.testing.assert_array_equal(a[k], b[k])
    s = np.sum(np.abs(a["SEs"]) ** 2, axis=0)
    np.testing.assert_allclose(s, 1.0, rtol=1e-5)
    Phi = a["Phi"]
    np.testing.assert_allclose(Phi @ Phi.conj().T, np.eye(Phi.shape[0]), atol=1e-12)


def test_added_entry_points_reject_null_arguments():
    """The solver, batch and operator-extension entry points check their
    arguments before any device work: NULL handles give MR_ERR_INVALID_ARG
    (-1) with a message, destroy(NULL) is a no-op (as mr_op_destroy)."""
    lib = _lib()
    h = ctypes.c_void_p(1)
    assert lib.mr_b200_cg_create(None, None, None, 0.0, 0, 10, ctypes.byref(h)) == -1
    assert h.value is None and b"op is NULL" in lib.mr_last_error()
    assert lib.mr_b200_cg_step(None, 1) == -1
    n = ctypes.c_int(0)
    rr = (ctypes.c_double * 2)()
    assert lib.mr_b200_cg_residuals(None, rr, 2, ctypes.byref(n)) == -1
    assert lib.mr_b200_cg_busy(None, ctypes.byref(n)) == -1
    assert lib.mr_b200_cg_iterations(None, ctypes.byref(n)) == -1
    assert lib.mr_b200_cg_destroy(None) == 0
    h = ctypes.c_void_p(1)
    assert lib.mr_b200_batch_create(None, 0, 4, 0, ctypes.byref(h)) == -1
    assert h.value is None and b"no operators" in lib.mr_last_error()
    assert lib.mr_b200_batch_execute(None, None, None, None) == -1
    assert lib.mr_b200_batch_destroy(None) == 0
    assert lib.mr_b200_op_blocked_copy(None, 0, None) == -1
    assert lib.mr_b200_op_autotune(None, 1, None) == -1
    b = ctypes.c_uint64(0)
    assert lib.mr_b200_op_device_bytes(None, ctypes.byref(b)) == -1
    assert lib.mr_b200_op_execute_host(None, None, None) == -1
    assert b"op is NULL" in lib.mr_last_error()
    assert lib.mr_b200_op_host_sync(None) == -1
    assert lib.mr_b200_op_host_release(None) == -1
    f = ctypes.c_int(0)
    assert lib.mr_b200_op_save_kernel16(None, ctypes.byref(f), None, None) == -1
    assert lib.mr_b200_op_load_kernel16(None, 2, None, None) == -1
