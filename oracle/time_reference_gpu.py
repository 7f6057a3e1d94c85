"""Time the reference's own CUDA apply on a GPU (TEST / MEASUREMENT ONLY).

Loads ``oracle/_ref/libmr_aha_ref.so`` (the reference's apply path compiled
from its sources by ``oracle/Makefile``: per-coil pad / crop kernels, cuFFT,
L-specialised block-diagonal kernels, coil groups of 4) and times
``mr_aha_plan_execute`` with CUDA events on the headline workload, with the
same inputs as ``bench.py`` and a kernel of the right size (the reference's
``mr_calc_toep`` needs cufinufft, which is absent, so the kernel comes from
this library's ``calc_toep``). This is the "plain FP32 Toeplitz apply"
measured on B200.

Usage (on the GPU box)::

    python oracle/time_reference_gpu.py [--workload stack320] [--steps 10] [--warmup 3]
"""

from __future__ import annotations

import argparse
import ctypes
import json
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))

REF_LIB = ROOT / "oracle" / "_ref" / "libmr_aha_ref.so"


def main(argv=None) -> int:
    import torch

    import mr_aha_b200 as mr
    from mr_aha_b200 import synth
    from mr_aha_b200._lib import PROTOTYPES, MRConfig

    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="stack320")
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    a = ap.parse_args(argv)

    ref = ctypes.CDLL(str(REF_LIB))
    for n in ("mr_config_defaults", "mr_config_validate", "mr_aha_plan_create",
              "mr_aha_plan_execute", "mr_aha_plan_destroy", "mr_last_error"):
        res, args = PROTOTYPES[n]
        getattr(ref, n).restype = res
        getattr(ref, n).argtypes = args

    wl = synth.workload(a.workload)
    dev = torch.device("cuda", 0)
    x = torch.from_numpy(wl["x"]).to(dev)
    S = torch.from_numpy(wl["SEs"]).to(dev)
    cfg = mr.make_config(wl["traj_type"], wl["n_dim"], wl["L"], phi2_dim=wl["phi2_dim"],
                         n_coils=wl["n_coils"], mem_fraction=0.9)
    K = mr.calc_toep(cfg, torch.from_numpy(wl["phi2"]).to(dev),
                     torch.from_numpy(wl["traj"]).to(dev))
    rc_cfg = MRConfig.from_buffer_copy(cfg)
    plan = ctypes.c_void_p()
    rc = ref.mr_aha_plan_create(ctypes.byref(rc_cfg), ctypes.byref(plan))
    assert rc == 0, ref.mr_last_error()
    y = torch.empty_like(x)
    ours = torch.empty_like(x)

    def run():
        r = ref.mr_aha_plan_execute(plan, x.data_ptr(), S.data_ptr(), K.data_ptr(), None,
                                    y.data_ptr())
        assert r == 0, ref.mr_last_error()

    for _ in range(a.warmup):
        run()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(a.steps):
        run()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / a.steps
    # agreement with this library on the same inputs
    with mr.create_op(cfg, S, None, None, _phi2_toep=K) as op:
        op(x, out=ours)
    torch.cuda.synchronize()
    rel = float(torch.linalg.vector_norm((ours - y).to(torch.complex128)) /
                torch.linalg.vector_norm(y.to(torch.complex128)))
    ref.mr_aha_plan_destroy(plan)
    print(json.dumps({"impl": "reference CUDA apply (oracle/_ref)", "workload": a.workload,
                      "ms_per_apply": ms, "applies_per_s": 1e3 / ms, "steps": a.steps,
                      "rel_l2_vs_this_library": rel}), flush=True)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
