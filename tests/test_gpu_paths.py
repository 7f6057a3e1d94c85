"""Every kernel generation of the apply against the FP64 oracle.

The plan picks, per pass, the half-length pass 3 (M = 2N), the
compile-time-specialised kernels, the in-place generic ones or the ping-pong
ones, fused or unfused; environment switches read at plan creation force
each of them, so that every path stays parity-green, not only the default
one. Geometries: the small stack workload (64 x 64 x 8, L = 4, 4 coils) and
a 320 x 320 slab with L = 16 (the headline x / y lengths and rank). Tolerance
(relative L2 vs the FP64 oracle): 1e-5.
"""

import functools

import numpy as np
import pytest

from mr_aha_b200 import synth
from oracle import aha_oracle as O
from tests.gpu_util import dev, host, random_kernel

pytestmark = pytest.mark.gpu

TOL_APPLY = 1e-5

VARIANTS = {
    "default": {},
    "no_half": {"MR_AHA_B200_NO_HALF": "1"},
    "no_fixed": {"MR_AHA_B200_NO_FIXED": "1"},
    "fft_v1": {"MR_AHA_B200_FFT_V1": "1"},
    "unfused": {"MR_AHA_B200_UNFUSED_BD": "1"},
    "full_tiles": {"MR_AHA_B200_FULL_TILES": "1"},
    "narrow_tiles": {"MR_AHA_B200_XT_Z": "32", "MR_AHA_B200_XT_Y": "8"},
}

GEOMS = {
    "stack64": dict(n_dim=(64, 64, 8), L=4, nc=4),
    "slab320": dict(n_dim=(320, 320, 2), L=16, nc=2),
}


def _case(name, seed):
    g = GEOMS[name]
    rng = np.random.default_rng(seed)
    nx, ny, nz = g["n_dim"]
    x = synth.crandn(rng, (g["L"], nz, ny, nx))
    S = synth.crandn(rng, (g["nc"], nz, ny, nx))
    return g, rng, x, S


@functools.lru_cache(maxsize=None)
def _inputs(geom, tri):
    """Seeded inputs and the oracle's result, shared by every variant."""
    import mr_aha_b200 as mr

    g, rng, x, S = _case(geom, 7 if tri == "lower" else 9)
    cfg = mr.make_config("stack", g["n_dim"], g["L"], n_coils=g["nc"], triangulation=tri)
    K = random_kernel(rng, mr.phi2_toep_shape(cfg))
    ref = O.aha_toeplitz("stack", g["n_dim"], synth.default_phi2_dim("stack", g["n_dim"]),
                         g["L"], x, S, K, upper=tri == "upper")
    return x, S, K, ref


@pytest.mark.parametrize("tri", ["lower", "upper"])
@pytest.mark.parametrize("variant", list(VARIANTS))
@pytest.mark.parametrize("geom", list(GEOMS))
def test_apply_paths(geom, variant, tri, monkeypatch):
    import mr_aha_b200 as mr

    for k, v in VARIANTS[variant].items():
        monkeypatch.setenv(k, v)
    g = GEOMS[geom]
    x, S, K, ref = _inputs(geom, tri)
    cfg = mr.make_config("stack", g["n_dim"], g["L"], n_coils=g["nc"], triangulation=tri)
    y = host(mr.aha_toeplitz(cfg, dev(x), dev(S), dev(K)))
    assert O.rel_l2(y, ref) <= TOL_APPLY, O.rel_l2(y, ref)


@pytest.mark.parametrize("variant", ["default", "no_half"])
def test_apply_paths_masked(variant, monkeypatch):
    import mr_aha_b200 as mr

    for k, v in VARIANTS[variant].items():
        monkeypatch.setenv(k, v)
    g, rng, x, S = _case("stack64", 8)
    phi2_dim = synth.default_phi2_dim("stack", g["n_dim"])
    traj = synth.make_traj("stack", 48, 128)
    mask = O.calc_mask("stack", phi2_dim, traj, 2)
    cfg = mr.make_config("stack", g["n_dim"], g["L"], n_coils=g["nc"], is_masked=True,
                         num_masked=len(mask))
    K = random_kernel(rng, (O.num_tri(g["L"]), len(mask)))
    y = host(mr.aha_toeplitz(cfg, dev(x), dev(S), dev(K), mask=dev(mask)))
    ref = O.aha_toeplitz("stack", g["n_dim"], phi2_dim, g["L"], x, S, K, mask=mask)
    assert O.rel_l2(y, ref) <= TOL_APPLY
