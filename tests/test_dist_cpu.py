"""Multi-process (gloo, world size 2, CPU) test of the replica timing of
bench.py: every rank runs its own operator and the job is timed by the
slowest rank (max over ranks), throughput = ranks x steps / max time."""

import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, values, out):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    import bench

    m = bench.max_over_ranks(values[rank], dist, "cpu")
    out[rank] = (m, bench.replica_throughput(10, world, m))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_gloo():
    import torch.multiprocessing as mp

    world = 2
    values = [12.5, 20.0]
    mgr = mp.Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(world, _free_port(), values, out), nprocs=world,
                       join=True, start_method="spawn")
    for r in range(world):
        m, thr = out[r]
        assert m == 20.0
        assert thr == pytest.approx(2 * 10 / 0.020)


def test_single_process_helpers():
    import bench

    assert bench.max_over_ranks(3.0, None, None) == 3.0
    assert bench.replica_throughput(30, 1, 3000.0) == pytest.approx(10.0)
    wl = {"n_dim": (320, 320, 56), "phi2_dim": (640, 640, 56), "L": 16, "n_coils": 12}
    b = bench.alg_bytes(wl, 8, 0)
    assert b["apply"] == pytest.approx(97.99e9, rel=1e-3)
    assert bench.alg_bytes(wl, 4, 4)["apply"] == pytest.approx(85.60e9, rel=1e-3)


@pytest.mark.parametrize("workload", ["cg320", "batch48", "serve", "toep", "forms"])
def test_reference_arm_unavailable_line(workload):
    """The reference arm of the non-headline workloads prints one JSON line
    saying why it is unavailable and exits 0 (no GPU needed)."""
    import json
    import subprocess
    import sys
    from pathlib import Path

    root = Path(__file__).resolve().parents[1]
    r = subprocess.run([sys.executable, str(root / "bench.py"), "--impl", "reference",
                        "--workload", workload], capture_output=True, text=True, timeout=300,
                       cwd=root)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["unavailable"]
