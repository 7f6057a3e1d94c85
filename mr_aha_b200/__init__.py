"""MR_AHA on NVIDIA B200: the Toeplitz-embedded low-rank normal operator A^H A.

A drop-in for the reference MR_AHA Python binding (``import mr_aha_b200 as
mr_aha``): ``make_config``, ``calc_mask``, ``calc_toep``, ``aha_toeplitz``,
``create_op`` / ``AhAOp`` with the same shapes and semantics, over the C ABI
of ``libmr_aha_c.so`` (``include/mr_aha/mr_aha.h``), which runs hand-written
sm_100a CUDA kernels. Arrays are CUDA tensors (torch) or any
``__cuda_array_interface__`` array.
"""

from ._lib import MRConfig, MRError, TrajType, Triangulation, backend, lib  # noqa: F401
from .api import (  # noqa: F401
    DEFAULT_MASK_RADIUS,
    AhAOp,
    AhAPlan,
    Batch,
    CGSolver,
    aha_toeplitz,
    calc_mask,
    calc_toep,
    calc_toep_from_psf,
    create_op,
    make_config,
    num_tri,
    phi2_toep_shape,
    pinned_empty,
)

__version__ = "1.0.0"
