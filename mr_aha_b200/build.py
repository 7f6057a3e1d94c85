"""Build ``libmr_aha_c.so`` (sm_100a only) in-tree with nvcc.

Every ``csrc/*.cu`` is compiled to an object under ``mr_aha_b200/_build/``
(in parallel, skipped when up to date) and linked into
``mr_aha_b200/lib/libmr_aha_c.so`` with the CUDA runtime linked statically,
so that the library does not depend on which ``libcudart`` another framework
in the same process has loaded.

Usage::

    python -m mr_aha_b200.build [--force] [--verbose-ptxas]
"""

from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import re
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OBJ = PKG / "_build"
LIBDIR = PKG / "lib"
LIB = LIBDIR / "libmr_aha_c.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC,-fvisibility=hidden", "-DMR_AHA_CUDA_COMPLEX",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libmr_aha_c.so")


_INCLUDE = re.compile(r'^\s*#\s*include\s*"([^"]+)"', re.M)


def _deps(src: Path, seen=None) -> set:
    """Files `src` includes with quotes, recursively (csrc/ and include/)."""
    seen = set() if seen is None else seen
    for name in _INCLUDE.findall(src.read_text()):
        for base in (src.parent, CSRC, ROOT / "include"):
            f = (base / name).resolve()
            if f.exists():
                if f not in seen:
                    seen.add(f)
                    _deps(f, seen)
                break
    return seen


def _compile(src: Path, force: bool, ptxas_v: bool) -> Path:
    obj = OBJ / (src.stem + ".o")
    newest = max([src.stat().st_mtime] + [h.stat().st_mtime for h in _deps(src)])
    if not force and obj.exists() and obj.stat().st_mtime >= newest:
        return obj
    cmd = [nvcc(), *ARCH, *NVCC_FLAGS, "-I", str(ROOT / "include"), "-I", str(CSRC),
           "-c", str(src), "-o", str(obj)]
    if ptxas_v:
        cmd[1:1] = ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{r.stdout}\n{r.stderr}")
    if ptxas_v:
        sys.stderr.write(r.stderr)
    return obj


def build(force: bool = False, ptxas_v: bool = False) -> Path:
    """Compile and link the library; returns its path."""
    OBJ.mkdir(exist_ok=True)
    LIBDIR.mkdir(exist_ok=True)
    srcs = sorted(CSRC.glob("*.cu"))
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, force, ptxas_v), srcs))
    if not force and LIB.exists() and LIB.stat().st_mtime >= max(o.stat().st_mtime for o in objs):
        return LIB
    cmd = [nvcc(), *ARCH, "-shared", "-cudart", "static", "-Xcompiler", "-fPIC",
           *map(str, objs), "-o", str(LIB), "-lpthread", "-ldl", "-lrt"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose-ptxas", action="store_true")
    a = ap.parse_args(argv)
    print(build(force=a.force, ptxas_v=a.verbose_ptxas))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
