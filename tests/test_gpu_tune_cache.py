"""On-disk autotune cache (``MR_AHA_B200_TUNE_CACHE``), through the C ABI.

* An autotune writes one line per tuned geometry, ``<device>|<geometry>|``
  followed by 15 integers, and keeps the lines of other devices.
* A fresh process with the cache set launches exactly the kernels of the
  tuned operator (same launch trace); without it, the default kernels.
* A line whose values the autotuner would never choose (edited or stale) is
  ignored: the operator runs its defaults and still meets 1e-5 against the
  FP64 oracle (relative L2).
"""

import json
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

from oracle import aha_oracle as O
from tests.gpu_util import dev, host
from tests.test_gpu_headline import traced

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
GEOM = dict(tt="stack", n_dim=(64, 64, 8), L=4, nc=4, seed=11)

# One operator of GEOM (seeded inputs), one traced apply; writes the output to
# argv[1] and prints the launch trace as JSON.
CHILD = r"""
import json, sys
import numpy as np
sys.path.insert(0, sys.argv[2])
from tests.test_gpu_tune_cache import make_inputs, make_op
from tests.test_gpu_headline import traced
from tests.gpu_util import dev, host
inp = make_inputs()
with make_op(inp) as op:
    y, tr = traced(lambda: host(op(dev(inp["x"]))))
np.save(sys.argv[1], y)
print(json.dumps(tr))
"""


def make_inputs():
    import mr_aha_b200 as mr
    from mr_aha_b200 import synth
    from tests.gpu_util import random_kernel

    rng = np.random.default_rng(GEOM["seed"])
    cfg = mr.make_config(GEOM["tt"], GEOM["n_dim"], GEOM["L"], n_coils=GEOM["nc"])
    img = tuple(reversed(GEOM["n_dim"]))
    return dict(cfg=cfg, S=synth.crandn(rng, (GEOM["nc"],) + img),
                K=random_kernel(rng, mr.phi2_toep_shape(cfg)),
                x=synth.crandn(rng, (GEOM["L"],) + img),
                phi2_dim=synth.default_phi2_dim(GEOM["tt"], GEOM["n_dim"]))


def make_op(inp):
    import mr_aha_b200 as mr

    return mr.create_op(inp["cfg"], dev(inp["S"]), None, None, _phi2_toep=dev(inp["K"]))


def _child(tmp_path, name, cache):
    env = dict(os.environ)
    env.pop("MR_AHA_B200_TUNE_CACHE", None)
    if cache is not None:
        env["MR_AHA_B200_TUNE_CACHE"] = str(cache)
    out = tmp_path / f"{name}.npy"
    r = subprocess.run([sys.executable, "-c", CHILD, str(out), str(ROOT)], env=env, cwd=ROOT,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return np.load(out), json.loads(r.stdout.strip().splitlines()[-1])


def _oracle(inp, y):
    ref = O.aha_toeplitz(GEOM["tt"], GEOM["n_dim"], inp["phi2_dim"], GEOM["L"], inp["x"],
                         inp["S"], inp["K"])
    return O.rel_l2(y, ref)


def test_tune_cache_roundtrip(tmp_path, monkeypatch):
    import torch

    cache = tmp_path / "tune.txt"
    other = "Some Other GPU|t2 n1,2,3 m2,4,6 L1 C1 G1 k0 u0 f1| 0 0 0 0 0 0 0 0 0 0 0 0 0 0 0\n"
    cache.write_text("not a cache line\n" + other)
    monkeypatch.setenv("MR_AHA_B200_TUNE_CACHE", str(cache))
    inp = make_inputs()
    with make_op(inp) as op:
        assert op.autotune(reps=1) > 0
        y_tuned, tr_tuned = traced(lambda: host(op(dev(inp["x"]))))
    assert _oracle(inp, y_tuned) <= 1e-5

    lines = cache.read_text().splitlines()
    assert other.strip() in lines and "not a cache line" not in lines
    name = torch.cuda.get_device_name(0)
    mine = [ln for ln in lines if ln.startswith(name + "|")]
    assert mine, lines
    for ln in mine:
        _, key, vals = ln.split("|")
        assert key.startswith("t") and len(vals.split()) == 15

    y_def, tr_def = _child(tmp_path, "default", None)
    y_hit, tr_hit = _child(tmp_path, "cached", cache)
    assert tr_hit == tr_tuned
    assert _oracle(inp, y_def) <= 1e-5 and _oracle(inp, y_hit) <= 1e-5

    # every value out of any range the autotuner uses: the line is ignored
    bad = tmp_path / "bad.txt"
    bad.write_text("".join(f"{ln.rsplit('|', 1)[0]}|{' 4099' * 15}\n" for ln in mine))
    y_bad, tr_bad = _child(tmp_path, "bad", bad)
    assert tr_bad == tr_def
    assert _oracle(inp, y_bad) <= 1e-5
