"""FP32 CPU restatement of the Toeplitz apply, timed as the CPU baseline.

TEST / MEASUREMENT INFRASTRUCTURE ONLY. The reference's CPU route (FINUFFT
A^H A) is not available here (the finufft package and the third_party/finufft
submodule are absent), so the CPU baseline is this port of the reference's
apply (src/cuda/mr_aha.cu:694-790) in single precision on all host cores:
pad x S_c (mr_kernels.cu:98-142), multi-threaded ``scipy.fft`` over the
upsampled grid, the packed Hermitian block multiply in C/OpenMP
(``bd_cpu.c``), the inverse transform, crop and conj(S_c) coil sum
(mr_kernels.cu:144-176). ``apply_coil`` is one coil's term, the bounded
sample the baseline times.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
BUILD = HERE / "_build"
LIB = BUILD / "libbd_cpu.so"


def build_c(force: bool = False) -> Path:
    """Compile ``bd_cpu.c`` into ``oracle/_build/libbd_cpu.so`` with gcc."""
    BUILD.mkdir(exist_ok=True)
    src = HERE / "bd_cpu.c"
    if not force and LIB.exists() and LIB.stat().st_mtime >= src.stat().st_mtime:
        return LIB
    subprocess.run(["gcc", "-O3", "-mavx2", "-mfma", "-fopenmp", "-shared", "-fPIC",
                    str(src), "-o", str(LIB)], check=True)
    return LIB


_lib = None


def _bd():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build_c()
        _lib = ctypes.CDLL(str(LIB))
        _lib.bd_cpu_apply.restype = None
        _lib.bd_cpu_apply.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                      ctypes.c_int64, ctypes.c_int, ctypes.c_int]
    return _lib


def timing_kernel(shape, seed: int = 0) -> np.ndarray:
    """A complex64 kernel of the given shape for timing only: a seeded random
    1 Mi-element block repeated (the block multiply's cost does not depend on
    the values, and this avoids generating or transferring 25 GB)."""
    rng = np.random.default_rng(seed)
    blk = (rng.standard_normal(1 << 20) + 1j * rng.standard_normal(1 << 20)).astype(np.complex64)
    n = int(np.prod(shape))
    out = np.empty(n, dtype=np.complex64)
    for o in range(0, n, blk.size):
        m = min(blk.size, n - o)
        out[o:o + m] = blk[:m]
    return out.reshape(shape)


def cores() -> int:
    return len(os.sched_getaffinity(0))


class CpuToeplitz:
    """FP32 Toeplitz A^H A on the CPU for one stack / 3D / 2D operator.

    ``kernel`` is ``phi2_toep`` (complex64, ``[ntri, (Mz,) My, Mx]``), shifted
    once to natural order here (outside any timed region).
    """

    def __init__(self, traj_type, n_dim, phi2_dim, L, SEs, kernel, upper=False,
                 natural=False):
        from oracle.aha_oracle import pad_index_maps, spatial_axes

        self.img = spatial_axes(traj_type, n_dim)
        self.mpad = spatial_axes(traj_type, phi2_dim)
        self.L = int(L)
        self.upper = 1 if upper else 0
        self.S = np.asarray(SEs, dtype=np.complex64).reshape((-1,) + self.img)
        K = np.asarray(kernel, dtype=np.complex64).reshape((-1,) + self.mpad)
        if not natural:
            K = np.fft.ifftshift(K, axes=tuple(range(1, K.ndim)))
        self.K = np.ascontiguousarray(K)
        self.ix = np.ix_(*pad_index_maps(self.img, self.mpad))
        self.axes = tuple(range(1, 1 + len(self.img)))
        self.workers = cores()
        self.nloc = int(np.prod(self.mpad))

    def apply_coil(self, x, c):
        import scipy.fft as sfft

        L = self.L
        pad = np.zeros((L,) + self.mpad, dtype=np.complex64)
        pad[(slice(None),) + self.ix] = self.S[c][None] * x
        F = sfft.fftn(pad, axes=self.axes, workers=self.workers, overwrite_x=True)
        F = np.ascontiguousarray(F, dtype=np.complex64)
        Y = np.empty_like(F)
        _bd().bd_cpu_apply(F.ctypes.data, Y.ctypes.data, self.K.ctypes.data, self.nloc, L,
                           self.upper)
        back = sfft.ifftn(Y, axes=self.axes, workers=self.workers, overwrite_x=True,
                          norm="forward")
        return np.conj(self.S[c])[None] * back[(slice(None),) + self.ix]

    def apply(self, x):
        x = np.asarray(x, dtype=np.complex64).reshape((self.L,) + self.img)
        out = np.zeros_like(x)
        for c in range(self.S.shape[0]):
            out += self.apply_coil(x, c)
        return out
