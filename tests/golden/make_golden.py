"""Generate golden outputs from the REFERENCE's own CUDA code (run on a B200).

The reference's golden files (data/ref_mlx/*.npz) are not distributed with
its sources, so this script makes them: it loads ``oracle/_ref/libmr_aha_ref.so``
(the reference's apply path compiled from its sources by ``oracle/Makefile``)
through the same C ABI and runs, for every case of the reference's own
synthetic set (``mr_aha_b200.synth.REFERENCE_CASES``, seeded):

* ``mr_calc_mask`` with radius 0, 1, 2;
* ``mr_aha_toeplitz`` with a seeded random packed kernel (the reference's
  tests/check_bd_kernels.py uses random kernels the same way), lower and
  upper packing, and masked (mask radius 2, the kernel's first num_masked
  locations' worth of random values).

Inputs are regenerated from their seeds by the tests; only outputs are
stored (``tests/golden/ref_<case>.npz``). Usage, on the GPU box::

    python tests/golden/make_golden.py [--out DIR]
"""

from __future__ import annotations

import argparse
import ctypes
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from mr_aha_b200._lib import PROTOTYPES, MRConfig  # noqa: E402
from mr_aha_b200 import synth  # noqa: E402

REF_LIB = ROOT / "oracle" / "_ref" / "libmr_aha_ref.so"
KERNEL_SEED = 1000


def load_ref():
    lib = ctypes.CDLL(str(REF_LIB))
    for name, (res, args) in PROTOTYPES.items():
        if name.startswith("mr_b200") or name.startswith("mr_op") or "calc_toep" in name:
            continue
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


def make_cfg(lib, p, tri=0, masked=0, nm=0, radius=2):
    cfg = MRConfig()
    tt = {"2D": 0, "3D": 1, "stack": 2}[p["traj_type"]]
    assert lib.mr_config_defaults(ctypes.byref(cfg), tt) == 0
    for i, v in enumerate(p["n_dim"]):
        cfg.n_dim[i] = v
    for i, v in enumerate(p["phi2_dim"]):
        cfg.phi2_dim[i] = v
    cfg.L = p["L"]
    cfg.n_coils = p["n_coils"]
    cfg.triangulation = tri
    cfg.is_masked = masked
    cfg.num_masked = nm
    cfg.gpu_device_id = -1
    cfg.mask_radius = radius
    assert lib.mr_config_validate(ctypes.byref(cfg)) == 0, lib.mr_last_error()
    return cfg


def golden_kernel(p, n_loc):
    """The seeded random packed kernel the golden outputs were made with."""
    rng = np.random.default_rng(KERNEL_SEED + p["seed"])
    ntri = p["L"] * (p["L"] + 1) // 2
    return (rng.standard_normal((ntri, n_loc)) +
            1j * rng.standard_normal((ntri, n_loc))).astype(np.complex64)


def main(argv=None):
    import torch

    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=str(ROOT / "tests" / "golden"))
    a = ap.parse_args(argv)
    lib = load_ref()
    out_dir = Path(a.out)
    out_dir.mkdir(parents=True, exist_ok=True)
    dev = torch.device("cuda", 0)

    def d(arr):
        return torch.from_numpy(np.ascontiguousarray(arr)).to(dev)

    for case in synth.REFERENCE_CASES:
        p = synth.reference_case(case)
        p["seed"] = case["seed"]
        res = {}
        traj = d(p["traj"])
        Ntrajs, Nkx = p["traj"].shape[2], p["traj"].shape[1]
        for r in (0, 1, 2):
            cfg = make_cfg(lib, p, radius=r)
            buf = torch.empty(int(np.prod(p["phi2_dim"])), dtype=torch.int64, device=dev)
            # (traj is held in a variable above for the same reason)
            n = ctypes.c_int64(0)
            rc = lib.mr_calc_mask(ctypes.byref(cfg), traj.data_ptr(), Ntrajs, Nkx,
                                  buf.data_ptr(), ctypes.byref(n))
            assert rc == 0, lib.mr_last_error()
            torch.cuda.synchronize()
            res[f"mask_r{r}"] = buf[: n.value].cpu().numpy()
        x, S = d(p["x"]), d(p["SEs"])
        vpad = int(np.prod(p["phi2_dim"]))
        # Device tensors are held in variables for the whole (asynchronous)
        # call: a temporary's memory would be recycled by the caching
        # allocator while the library still reads it.
        Kfull = d(golden_kernel(p, vpad))
        for tri, name in ((0, "lower"), (1, "upper")):
            cfg = make_cfg(lib, p, tri=tri)
            y = torch.empty_like(x)
            rc = lib.mr_aha_toeplitz(ctypes.byref(cfg), x.data_ptr(), S.data_ptr(),
                                     Kfull.data_ptr(), None, y.data_ptr())
            assert rc == 0, lib.mr_last_error()
            torch.cuda.synchronize()
            res[f"AhAx_{name}"] = y.cpu().numpy()
        mask = res["mask_r2"]
        nm = len(mask)
        Km = d(golden_kernel(p, nm))
        mask_d = d(mask)
        cfg = make_cfg(lib, p, masked=1, nm=nm)
        y = torch.empty_like(x)
        rc = lib.mr_aha_toeplitz(ctypes.byref(cfg), x.data_ptr(), S.data_ptr(),
                                 Km.data_ptr(), mask_d.data_ptr(), y.data_ptr())
        assert rc == 0, lib.mr_last_error()
        torch.cuda.synchronize()
        res["AhAx_masked"] = y.cpu().numpy()
        np.savez_compressed(out_dir / f"ref_{case['name']}.npz", **res)
        print(case["name"], {k: v.shape for k, v in res.items()}, flush=True)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
