"""Helpers of the GPU parity tests (host <-> device transfers, seeded inputs)."""

import numpy as np


def dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    return t.detach().cpu().numpy()


def random_kernel(rng, shape):
    """Random packed kernel (not Gram-derived): only the block arithmetic and
    the triangle unpacking are under test, as in the reference's
    tests/check_bd_kernels.py."""
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)
