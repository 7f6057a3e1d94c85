"""The library's own non-uniform FFTs (nufft.cu: ES-kernel spreading and
interpolation on a 2x oversampled grid) through the two places that use
them, on every reference case (2-D, 3-D and stack; odd sizes; the prime
101 x 81 grid):

* the NUFFT-method operator (``method='nufft'``, MR_OP_NUFFT): against the
  FP64 oracle's exact NUFFT-route A^H A (relative L2 <= 1e-5) and against the
  Toeplitz operator of the same inputs (<= 1e-4, the reference's bar between
  the two methods, tests/make_reference.py:504);
* the kernel build by spreading with FP64 accumulation
  (``MR_AHA_B200_TOEP_METHOD=1``): against the exact kernel (type-1 NUDFT +
  centred inverse FFT, oracle.aha_oracle.calc_toep), <= 1e-6, both packings,
  and the masked form against the gathered unmasked one; and against the
  closed-form build on a 3-D kooshball grid too large for the CPU oracle
  (64 x 64 x 64 image, 128^3 grid, 2000 spokes), <= 1e-6, with both builds
  timed (printed).
"""

import time

import numpy as np
import pytest

from mr_aha_b200 import synth
from oracle import aha_oracle as O
from tests.gpu_util import dev, host

pytestmark = pytest.mark.gpu

CASES = synth.REFERENCE_CASES
IDS = [c["name"] for c in CASES]


def _cfg(p, tri="lower", **kw):
    import mr_aha_b200 as mr

    return mr.make_config(p["traj_type"], p["n_dim"], p["L"], phi2_dim=p["phi2_dim"],
                          n_coils=p["n_coils"], triangulation=tri, **kw)


@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_nufft_operator_vs_exact_and_toeplitz(case):
    import mr_aha_b200 as mr

    p = synth.reference_case(case)
    cfg = _cfg(p)
    with mr.create_op(cfg, dev(p["SEs"]), dev(p["phi2"]), dev(p["traj"]), method="nufft") as op:
        assert op.method == "nufft" and op.info["toep_source"] == "none"
        y = host(op(dev(p["x"])))
        with pytest.raises(mr.MRError):
            op.kernel()
    with mr.create_op(cfg, dev(p["SEs"]), dev(p["phi2"]), dev(p["traj"])) as top:
        yt = host(top(dev(p["x"])))
    ref = O.aha_nufft(p["traj_type"], p["n_dim"], p["L"], p["x"], p["SEs"], p["phi2"], p["traj"])
    e_exact, e_toep = O.rel_l2(y, ref), O.rel_l2(y, yt)
    print(f"{case['name']}: NUFFT operator vs exact {e_exact:.2e}, vs Toeplitz {e_toep:.2e}")
    assert e_exact <= 1e-5, e_exact
    assert e_toep <= 1e-4, e_toep


def test_nufft_operator_cg_and_options():
    """The conjugate-gradient solver runs on a NUFFT operator (it only needs
    applies); an upsampling factor of 1.5 keeps 1e-5; a masked configuration
    is rejected (no kernel to mask)."""
    import mr_aha_b200 as mr

    p = synth.reference_case(CASES[6])
    cfg = _cfg(p)
    ref = O.aha_nufft(p["traj_type"], p["n_dim"], p["L"], p["x"], p["SEs"], p["phi2"], p["traj"])
    with mr.create_op(cfg, dev(p["SEs"]), dev(p["phi2"]), dev(p["traj"]), method="nufft",
                      nufft_opts={"upsampfac": 1.5}) as op:
        assert O.rel_l2(host(op(dev(p["x"]))), ref) <= 1e-5
        b = dev(ref.astype(np.complex64))
        x, rr = op.cg(b, 5, graph=False)
        assert rr[-1] < rr[0]
    mcfg = _cfg(p, is_masked=True)
    with pytest.raises(ValueError):
        mr.create_op(mcfg, dev(p["SEs"]), dev(p["phi2"]), dev(p["traj"]), method="nufft")


@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_spread_kernel_build_vs_exact(case, monkeypatch):
    import mr_aha_b200 as mr

    monkeypatch.setenv("MR_AHA_B200_TOEP_METHOD", "1")
    p = synth.reference_case(case)
    for tri in ("lower", "upper"):
        cfg = _cfg(p, tri)
        K = host(mr.calc_toep(cfg, dev(p["phi2"]), dev(p["traj"])))
        ref = O.calc_toep(p["traj_type"], p["phi2_dim"], p["L"], p["phi2"], p["traj"],
                          upper=tri == "upper")
        err = O.rel_l2(K, ref)
        print(f"{case['name']} {tri}: spread build vs exact {err:.2e}")
        assert err <= 1e-6, err


def test_spread_kernel_build_masked(monkeypatch):
    import mr_aha_b200 as mr

    monkeypatch.setenv("MR_AHA_B200_TOEP_METHOD", "1")
    p = synth.reference_case(CASES[3])
    cfg = _cfg(p)
    full = host(mr.calc_toep(cfg, dev(p["phi2"]), dev(p["traj"])))
    mask = mr.calc_mask(cfg, dev(p["traj"]))
    mcfg = _cfg(p, is_masked=True, num_masked=int(mask.numel()))
    Km = host(mr.calc_toep(mcfg, dev(p["phi2"]), dev(p["traj"]), mask=mask))
    gathered = full.reshape(full.shape[0], -1)[:, host(mask)]
    assert O.rel_l2(Km, gathered) <= 1e-6


def test_spread_build_3d_kooshball_vs_closed_form(monkeypatch):
    """64 x 64 x 64 image (grid 128^3), L = 4, 2000 golden-means spokes of
    128 samples: both builds agree to 1e-6; their times are printed."""
    import torch

    import mr_aha_b200 as mr

    spec = dict(traj_type="3D", n_dim=(64, 64, 64), L=4, n_coils=1, n_traj=2000, n_kx=128,
                n_frames=40, frame_rule="div", seed=31)
    p = synth.spec_inputs(spec, with_x=False)
    cfg = mr.make_config("3D", p["n_dim"], 4, n_coils=1)
    phi2, traj = dev(p["phi2"]), dev(p["traj"])
    Ks, times = {}, {}
    for method, code in (("spread", "1"), ("closed", "2")):
        monkeypatch.setenv("MR_AHA_B200_TOEP_METHOD", code)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        Ks[method] = mr.calc_toep(cfg, phi2, traj)
        torch.cuda.synchronize()
        times[method] = time.perf_counter() - t0
    d = (Ks["spread"] - Ks["closed"]).to(torch.complex128)
    rel = float(torch.linalg.vector_norm(d) /
                torch.linalg.vector_norm(Ks["closed"].to(torch.complex128)))
    print(f"3-D 64^3 kooshball build: spread {times['spread']:.2f} s, "
          f"closed form {times['closed']:.2f} s, agreement {rel:.2e}")
    assert rel <= 1e-6, rel
