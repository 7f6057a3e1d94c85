"""Admission accounting of the serving backend, on the CPU (configuration
arithmetic only; the library's size functions need no GPU): the estimate
covers the kernel in the stored format (plus the complex64 build while a
16-bit one is converted), the capped plan buffers, the coil maps and the five
image-sized vectors of a solve, and the iteration cost orders requests by
size."""

import pytest

from mr_aha_b200 import serve


def _cfg(n=(64, 64, 8), L=4, C=4):
    import mr_aha_b200 as mr

    return mr.make_config("stack", n, L, n_coils=C)


def _req(cfg):
    return serve.Request(rid=0, arrival=0.0, cfg=cfg, SEs=None, phi2=None, traj=None, b=None,
                         n_iter=1)


def test_kernel_bytes_formats():
    cfg = _cfg()
    nloc = 128 * 128 * 8
    ntri = 10
    assert serve.kernel_bytes(cfg, "complex64") == nloc * ntri * 8
    assert serve.kernel_bytes(cfg, "int16") == nloc * ntri * 4 + nloc * 4
    assert serve.kernel_bytes(cfg, "bf16") == serve.kernel_bytes(cfg, "int16")


@pytest.mark.parametrize("fmt", ["complex64", "int16"])
def test_estimate_bytes(fmt):
    cfg = _cfg()
    be = serve.GPUBackend(kernel_format=fmt, plan_bytes=1e6)
    vimg = 64 * 64 * 8
    k = serve.kernel_bytes(cfg, fmt)
    if fmt != "complex64":
        k += serve.kernel_bytes(cfg, "complex64")
    assert be.estimate_bytes(_req(cfg)) == int(k + 1e6 + 8 * (vimg * 4 + 5 * vimg * 4))


def test_iteration_cost_orders_by_size():
    be = serve.GPUBackend()
    small = be.iteration_cost(_req(_cfg((64, 64, 8), 4, 4)))
    big_rank = be.iteration_cost(_req(_cfg((64, 64, 8), 16, 4)))
    big_grid = be.iteration_cost(_req(_cfg((128, 128, 8), 4, 4)))
    assert small < big_rank and small < big_grid
