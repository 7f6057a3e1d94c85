#!/usr/bin/env python
"""Headline benchmark: A^H A applies/s of the Toeplitz operator.

Workload (default ``stack320``): stack-of-stars golden-angle radial,
image 320 x 320 x 56, grid 640 x 640 x 56, L = 16, 12 coils, 1000 spokes x
640 readout points, Gram blocks from a random orthonormal 16 x 200 temporal
basis (spokes split evenly over 200 frames), smoothed coil maps with
sum |S_c|^2 = 1, x standard complex normal; all seeded synthetic data. One
step = one apply ``op(x)`` of the operator built by ``create_op`` (kernel
built on the GPU, complex64 unless ``--kernel-format`` says otherwise).

Arms:
* default: the CUDA library. ``value`` = applies/s with inputs resident on
  the GPU (CUDA events on the operator's stream, K timed steps between a
  barrier + synchronize on both sides, max over ranks); ``e2e`` = the same
  metric through ``op.apply_host`` (``mr_b200_op_execute_host``) with
  page-locked host buffers: every step copies x in and A^H A x out, the
  copies of consecutive steps overlapping the applies around them.
* ``--impl reference``: the reference has no CPU implementation of the path
  here (its CPU route, FINUFFT, is absent), so this times the FP32 CPU port of
  the reference's apply (``oracle/cpu_port.py``) on all host cores; one step
  is one coil's term of the apply (a bounded sample), scaled to applies/s.

Several GPUs (torchrun): independent replicas, one operator per GPU, no
collective on the data path (``scaling`` = weak).
"""

from __future__ import annotations

import argparse
import dataclasses
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "A^H A applies/s"
UNIT = "applies/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="stack320")
    ap.add_argument("--kernel-format", default="complex64",
                    choices=["complex64", "bf16", "int16"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-samples", type=int, default=2)
    ap.add_argument("--cg-size", default="stack320",
                    help="cg320: the operator's workload (stack320, or slab320 for profiling)")
    ap.add_argument("--tune", action="store_true",
                    help="autotune the kernels of each geometry before timing")
    ap.add_argument("--requests", type=int, default=12, help="serve: number of requests")
    ap.add_argument("--rate", type=float, default=2.0, help="serve: arrivals per second")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def max_over_ranks(x: float, dist, device) -> float:
    """Largest value of x over the ranks (x itself without a process group)."""
    if dist is None:
        return float(x)
    import torch

    t = torch.tensor([float(x)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(steps: int, world: int, ms_max: float) -> float:
    """Whole-job applies/s of `world` independent replicas that each ran
    `steps` applies, timed by the slowest rank."""
    return world * steps / (ms_max / 1e3)


def workload_config(name: str, wl: dict) -> dict:
    return {"workload": name, "traj_type": wl["traj_type"], "n_dim": list(wl["n_dim"]),
            "phi2_dim": list(wl["phi2_dim"]), "L": wl["L"], "n_coils": wl["n_coils"],
            "Ntrajs": int(wl["traj"].shape[2]), "Nkx": int(wl["traj"].shape[1])}


def alg_bytes(wl: dict, kbytes_per_elem: float, scale_bytes: int) -> dict:
    """Algorithmic bytes per apply (3-pass pruned design) and of pass 3.

    B_alg = 8 [Vimg L + Vimg C + 4 (Vpad/2) L C + Vimg C + Vimg L] + K,
    K = kernel bytes; pass 3 (x transform + block multiply) reads and writes
    the Mz*My*Nx intermediate of every plane and reads the kernel once.
    """
    n, m, L, C = wl["n_dim"], wl["phi2_dim"], wl["L"], wl["n_coils"]
    vimg = n[0] * n[1] * n[2]
    vpad = m[0] * m[1] * m[2]
    ntri = L * (L + 1) // 2
    K = vpad * ntri * kbytes_per_elem + (vpad * scale_bytes)
    b_apply = 8 * (vimg * L + vimg * C + 4 * (vpad // 2) * L * C + vimg * C + vimg * L) + K
    w1 = m[2] * m[1] * n[0] * L * C * 8
    b_pass3 = 2 * w1 + K
    return {"apply": float(b_apply), "x_blockdiag": float(b_pass3), "kernel": float(K)}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, dev_index: int):
        self.dev = dev_index
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak_hbm():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


def committed_traffic(kernel_format: str):
    """DRAM bytes per launch of pass 3 from the committed ncu summary, if any."""
    p = ROOT / "profiles" / "x_blockdiag_stack320.json"
    if not p.exists():
        return None
    try:
        d = json.loads(p.read_text())
        return d.get("dram_bytes_per_launch", {}).get(kernel_format)
    except Exception:
        return None


def cpu_baseline(wl: dict, samples: int) -> dict:
    from oracle import aha_oracle as O
    from oracle import cpu_port

    shape = (O.num_tri(wl["L"]),) + O.spatial_axes(wl["traj_type"], wl["phi2_dim"])
    cp = cpu_port.CpuToeplitz(wl["traj_type"], wl["n_dim"], wl["phi2_dim"], wl["L"],
                              wl["SEs"], cpu_port.timing_kernel(shape), natural=True)
    cp.apply_coil(wl["x"], 0)  # warm-up (FFT plans, page faults)
    ts = []
    for k in range(samples):
        t0 = time.perf_counter()
        cp.apply_coil(wl["x"], k % wl["n_coils"])
        ts.append(time.perf_counter() - t0)
    t = statistics.median(ts)
    return {"value": 1.0 / (t * wl["n_coils"]), "unit": UNIT, "cores": cpu_port.cores(),
            "kind": "port",
            "sample": f"one coil's term of the apply (1 of {wl['n_coils']}), median of "
                      f"{samples}, scaled x{wl['n_coils']}; FP32 scipy.fft + C/OpenMP block "
                      f"multiply with a timing kernel of the full size"}


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    from mr_aha_b200 import synth
    from oracle import aha_oracle as O
    from oracle import cpu_port

    wl = synth.workload(args.workload)
    ntri = O.num_tri(wl["L"])
    shape = (ntri,) + O.spatial_axes(wl["traj_type"], wl["phi2_dim"])
    cp = cpu_port.CpuToeplitz(wl["traj_type"], wl["n_dim"], wl["phi2_dim"], wl["L"],
                              wl["SEs"], cpu_port.timing_kernel(shape), natural=True)
    for k in range(args.warmup):
        cp.apply_coil(wl["x"], k % wl["n_coils"])
    ts = []
    for k in range(args.steps):
        t0 = time.perf_counter()
        cp.apply_coil(wl["x"], k % wl["n_coils"])
        ts.append(time.perf_counter() - t0)
    per_apply = sum(ts) / len(ts) * wl["n_coils"]
    v = 1.0 / per_apply
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * sum(ts) / len(ts),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c64",
            "data": "synthetic", "impl": "reference",
            "config": workload_config(args.workload, wl),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cpu_port.cores(), "kind": "port",
                             "sample": f"one coil's term per step (1 of {wl['n_coils']}), "
                                       f"scaled x{wl['n_coils']}"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    import torch

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist_mod

        dist_mod.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                    device_id=torch.device("cuda", local))
        dist = dist_mod
    import mr_aha_b200 as mr
    from mr_aha_b200 import synth

    wl = synth.workload(args.workload)
    dev = torch.device("cuda", local)
    t0 = time.perf_counter()
    x_h = torch.from_numpy(wl["x"]).pin_memory()
    x = x_h.to(dev)
    S = torch.from_numpy(wl["SEs"]).to(dev)
    phi2 = torch.from_numpy(wl["phi2"]).to(dev)
    traj = torch.from_numpy(wl["traj"]).to(dev)
    cfg = mr.make_config(wl["traj_type"], wl["n_dim"], wl["L"], phi2_dim=wl["phi2_dim"],
                         n_coils=wl["n_coils"], mem_fraction=0.9)
    op = mr.create_op(cfg, S, phi2, traj, kernel_format=args.kernel_format,
                      keep_complex64=args.kernel_format == "complex64")
    del phi2
    info = op.info
    tuned_ms = op.autotune(reps=2) if args.tune else None
    setup_s = time.perf_counter() - t0
    out = torch.empty_like(x)
    stream = torch.cuda.current_stream(dev)
    for _ in range(args.warmup):
        op(x, out=out)
    torch.cuda.synchronize(dev)
    prof = op.profile(x, out=out)
    launches = op.launches_per_apply

    # ---- device-resident timed region ----
    sampler = ClockSampler(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    sampler.start()
    time.sleep(0.3)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        op(x, out=out)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    clocks = sampler.stop()
    if dist:
        dist.barrier()
    ms = max_over_ranks(e0.elapsed_time(e1), dist, dev)
    value = replica_throughput(args.steps, world, ms)

    # ---- end-to-end from page-locked host buffers through op.apply_host ----
    # (mr_b200_op_execute_host): every step copies its input in and its
    # result out; the copies of consecutive steps overlap the applies around
    # them. Timed from an event recorded before the first call to one
    # recorded after the final host_sync (all results in host memory).
    y_h = torch.empty(x_h.shape, dtype=x_h.dtype).pin_memory()
    for _ in range(2):
        op.apply_host(x_h, y_h)
    op.host_sync()
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    e0.record(stream)
    for _ in range(args.steps):
        op.apply_host(x_h, y_h)
    op.host_sync()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    ms_e = max_over_ranks(e0.elapsed_time(e1), dist, dev)
    e2e_same = bool(torch.equal(y_h, out.cpu()))
    op.host_release()
    e2e = {"value": replica_throughput(args.steps, world, ms_e), "unit": UNIT,
           "h2d_bytes_per_step": int(x_h.numel() * 8), "d2h_bytes_per_step": int(y_h.numel() * 8),
           "api": "AhAOp.apply_host (mr_b200_op_execute_host), pinned host buffers, "
                  "copies pipelined with the applies", "equals_device_apply": e2e_same}

    # ---- roofline of the dominant kernel ----
    kb = {"complex64": 8, "bf16": 4, "int16": 4}[args.kernel_format]
    sb = 0 if args.kernel_format == "complex64" else 4
    ab = alg_bytes(wl, kb, sb)
    per_pass = {}
    for name, t in prof:
        per_pass[name] = per_pass.get(name, 0.0) + t
    total_prof = sum(per_pass.values())
    dom = max(per_pass, key=per_pass.get)
    n_dom = sum(1 for name, _ in prof if name == dom)
    dom_ms = per_pass[dom] / n_dom
    peak, peak_kind = measured_peak_hbm()
    dom_bytes = ab.get(dom)
    roof = None
    if dom_bytes is not None:
        ngroups = max(1, n_dom)
        achieved = (dom_bytes / ngroups) / (dom_ms / 1e3) / 1e9
        roof = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                "alg_bytes_per_launch": dom_bytes / ngroups,
                "launch_ms": dom_ms, "traffic": committed_traffic(args.kernel_format)}
    apply_ms = ms / args.steps
    apply_roof = {"alg_bytes": ab["apply"], "achieved_gbs": ab["apply"] / (apply_ms / 1e3) / 1e9,
                  "frac": ab["apply"] / (apply_ms / 1e3) / 1e9 / peak}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline(wl, args.cpu_samples)
        except Exception as exc:  # report, do not fail the bench line
            cpu = {"value": None, "error": f"{type(exc).__name__}: {exc}"}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": apply_ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "c64" if args.kernel_format == "complex64" else f"c64+{args.kernel_format}-kernel",
            "data": "synthetic",
            "config": dict(workload_config(args.workload, wl),
                           kernel_format=args.kernel_format,
                           parallelism=f"replicas{world}",
                           l2="inputs larger than L2 (25 GB kernel streamed per apply)"),
            "e2e": e2e,
            "roofline": roof,
            "apply_roofline": apply_roof,
            "passes_ms": {k: round(v, 4) for k, v in per_pass.items()},
            "profiled_apply_ms": total_prof,
            "gpu_launches": launches * args.steps,
            "clocks": clocks,
            "cpu_baseline": cpu,
            "setup_s": setup_s,
            "autotuned_ms": tuned_ms,
            "toep_ms": info["toep_ms"],
        }
        print(json.dumps(line), flush=True)
    op.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


# ---------------------------------------------------------------------------
# Further workloads (one JSON line each): CG at the headline size, the uneven
# batch and the serving loop
# ---------------------------------------------------------------------------

def _rel(a, b) -> float:
    import torch

    return float(torch.linalg.vector_norm((a - b).to(torch.complex128)) /
                 torch.linalg.vector_norm(b.to(torch.complex128)))


def run_cg(args):
    """CG on b = A^H A x_true + 1e-3 noise at the headline size, 30
    iterations from zero, with the kernel stored as complex64, int16 + scale
    and bf16 + scale; errors against the complex64 operator on the GPU (the
    FP64-oracle comparison runs at a reduced size in the GPU tests)."""
    import torch

    import mr_aha_b200 as mr
    from mr_aha_b200 import synth

    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    wl = synth.workload(args.cg_size)
    x = torch.from_numpy(wl["x"]).to(dev)
    S = torch.from_numpy(wl["SEs"]).to(dev)
    cfg = mr.make_config(wl["traj_type"], wl["n_dim"], wl["L"], phi2_dim=wl["phi2_dim"],
                         n_coils=wl["n_coils"], mem_fraction=0.6)
    op = mr.create_op(cfg, S, torch.from_numpy(wl["phi2"]).to(dev),
                      torch.from_numpy(wl["traj"]).to(dev))
    ax = op(x)
    g = torch.Generator(device=dev).manual_seed(7)
    sigma = 1e-3 * float(torch.linalg.vector_norm(ax)) / (ax.numel() ** 0.5)
    b = ax + sigma * torch.randn(ax.shape, dtype=ax.dtype, device=dev, generator=g)
    n_iter = 30
    # each solve (op.cg: solver vectors allocated, one iteration captured as
    # a graph and replayed) timed on its own; the median is reported, since
    # the multi-GB allocations of a solve occasionally stall after the kernel
    # copies of a format change were freed and allocated
    reps = max(5, args.steps // 6)
    res = {}
    x_c64 = None
    y_c64 = op(x)
    for fmt in ("complex64", "int16", "bf16"):
        op.set_kernel_format(fmt)
        y = op(x)
        xs, rr = op.cg(b, n_iter)               # warm-up (graph capture)
        torch.cuda.synchronize()
        times = []
        for _ in range(reps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            xs, rr = op.cg(b, n_iter)
            e1.record()
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
        ms = float(np.median(times))
        if fmt == "complex64":
            x_c64 = xs.clone()
        res[fmt] = {"solve_ms": ms, "solve_ms_all": times, "solves_per_s": 1e3 / ms,
                    "ms_per_iteration": ms / n_iter,
                    "apply_rel_l2_vs_complex64": _rel(y, y_c64),
                    "iterate_rel_l2_vs_complex64": _rel(xs, x_c64),
                    "rr_first_last": [float(rr[0]), float(rr[-1])]}
    op.close()
    line = {"metric": f"CG solves/s (30 iterations, {args.cg_size})",
            "value": res["int16"]["solves_per_s"], "unit": "solves/s", "n_gpus": 1,
            "higher_is_better": True, "data": "synthetic",
            "dtype": "c64 vectors, FP64 reductions, int16+scale kernel",
            "config": {"workload": f"{args.cg_size} CG", "n_iter": n_iter, "noise": 1e-3,
                       "reps": reps},
            "formats": res}
    print(json.dumps(line), flush=True)
    return 0


def _op_bytes(spec, fmt):
    n, _, nz = spec["n_dim"]
    vpad = (2 * n) * (2 * n) * nz
    ntri = spec["L"] * (spec["L"] + 1) // 2
    return vpad * ntri * (8 if fmt == "complex64" else 4) + (0 if fmt == "complex64" else 4 * vpad)


def _alg_bytes_spec(spec, fmt):
    n, _, nz = spec["n_dim"]
    wl = {"n_dim": spec["n_dim"], "phi2_dim": (2 * n, 2 * n, nz), "L": spec["L"],
          "n_coils": spec["n_coils"]}
    kb = 8 if fmt == "complex64" else 4
    return alg_bytes(wl, kb, 0 if fmt == "complex64" else 4)["apply"]


def run_batch(args):
    """48 uneven operators (random kernels of the right size), admitted in
    waves by device memory, each wave applied as one batch (worker streams,
    one captured CUDA graph), complex64 and int16 kernels."""
    import torch

    import mr_aha_b200 as mr
    from mr_aha_b200 import synth

    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    specs = synth.batch_specs(48, seed=3)
    budget = 150e9
    peak, peak_kind = measured_peak_hbm()
    steps = max(1, args.steps // 10)
    out = {}
    for fmt in ("complex64", "int16"):
        # waves: resident bytes of the wave plus, for 16-bit kernels, the
        # largest complex64 kernel alive while it is converted
        waves, cur, used, trans = [], [], 0.0, 0.0
        for sp in specs:
            img = sp["n_dim"][0] * sp["n_dim"][1] * sp["n_dim"][2]
            need = _op_bytes(sp, fmt) + 8 * img * (sp["n_coils"] + 2 * sp["L"]) + 6e9
            t = 0.0 if fmt == "complex64" else _op_bytes(sp, "complex64")
            if cur and used + need + max(trans, t) > budget:
                waves.append(cur)
                cur, used, trans = [], 0.0, 0.0
            cur.append(sp)
            used += need
            trans = max(trans, t)
        if cur:
            waves.append(cur)
        t_total, applies, bytes_total, tune_s = 0.0, 0, 0.0, 0.0
        for wave in waves:
            ops, keep = [], []
            for sp in wave:
                g = torch.Generator(device=dev).manual_seed(sp["seed"])
                cfg = mr.make_config("stack", sp["n_dim"], sp["L"], n_coils=sp["n_coils"],
                                     mem_fraction=0.03)
                img = tuple(reversed(sp["n_dim"]))
                S = torch.randn((sp["n_coils"],) + img, dtype=torch.complex64, device=dev,
                                generator=g)
                K = torch.randn(mr.phi2_toep_shape(cfg), dtype=torch.complex64, device=dev,
                                generator=g)
                x = torch.randn((sp["L"],) + img, dtype=torch.complex64, device=dev,
                                generator=g)
                # the operator borrows the kernel; after a 16-bit conversion
                # it lets go of it and the complex64 array is freed
                op = mr.create_op(cfg, S, None, None, _phi2_toep=K)
                if fmt != "complex64":
                    op.set_kernel_format(fmt, keep_complex64=False)
                    # waves are packed by the kernels' own bytes: no
                    # opportunistic blocked copy of the 16-bit codes
                    op.blocked_copy(False)
                del K
                torch.cuda.empty_cache()
                ops.append(op)
                keep.append((S, x))
            t0 = time.perf_counter()
            b = mr.Batch(ops, n_streams=4, graph=True, tune=args.tune)
            tune_s += time.perf_counter() - t0
            xs = [k[1] for k in keep]
            ys = [torch.empty_like(v) for v in xs]
            for _ in range(2):
                b(xs, ys)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(steps):
                b(xs, ys)
            e1.record()
            torch.cuda.synchronize()
            t_total += e0.elapsed_time(e1) / 1e3
            applies += steps * len(wave)
            bytes_total += steps * sum(_alg_bytes_spec(sp, fmt) for sp in wave)
            b.close()
            for op in ops:
                op.close()
            del keep, xs, ys
            torch.cuda.empty_cache()
        gbs = bytes_total / t_total / 1e9
        out[fmt] = {"applies_per_s": applies / t_total, "waves": len(waves),
                    "alg_gbs": gbs, "roofline_frac": gbs / peak, "timed_s": t_total,
                    "tune_s": tune_s if args.tune else 0.0}
    line = {"metric": "batched A^H A applies/s (48 uneven operators)",
            "value": out["int16"]["applies_per_s"], "unit": "applies/s", "n_gpus": 1,
            "higher_is_better": True, "data": "synthetic (random kernels of the right size)",
            "dtype": "c64", "config": {"workload": "batch48", "seed": 3,
                                       "budget_gb": budget / 1e9, "steps_per_wave": steps,
                                       "autotune": bool(args.tune), "peak_gbs": peak,
                                       "peak_kind": peak_kind},
            "modes": out}
    print(json.dumps(line), flush=True)
    return 0


def run_serve(args):
    """Poisson arrivals of CG requests sized from the uneven-batch
    distribution; the serving loop (int16 + scale kernel, up to 8 resident
    solves, 160 GB admission) against the plain complex64 operator one solve
    at a time, on the same requests."""
    import torch

    import mr_aha_b200 as mr
    from mr_aha_b200 import serve, synth

    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    n_req = args.requests
    specs = synth.batch_specs(n_req, seed=11)
    arrivals = synth.poisson_arrivals(args.rate, n_req, seed=12)
    rng = np.random.default_rng(13)
    reqs = []
    for i, sp in enumerate(specs):
        p = synth.spec_inputs(sp, with_x=False)
        cfg = mr.make_config("stack", p["n_dim"], p["L"], n_coils=p["n_coils"])
        img = tuple(reversed(p["n_dim"]))
        b = torch.randn((p["L"],) + img, dtype=torch.complex64, device=dev,
                        generator=torch.Generator(device=dev).manual_seed(100 + i))
        reqs.append(serve.Request(rid=i, arrival=float(arrivals[i]), cfg=cfg,
                                  SEs=torch.from_numpy(p["SEs"]).to(dev),
                                  phi2=torch.from_numpy(p["phi2"]).to(dev),
                                  traj=torch.from_numpy(p["traj"]).to(dev), b=b,
                                  n_iter=int(rng.integers(10, 41))))
    # warm-up: the first request alone through both paths (kernel loading)
    first = [dataclasses.replace(reqs[0], arrival=0.0)]
    serve.Server(serve.GPUBackend("int16"), hbm_budget=160e9).run(first)
    serve.run_sequential(serve.GPUBackend("complex64", graph=False), first)
    served = {}
    for fmt in ("complex64", "int16"):
        srv = serve.Server(serve.GPUBackend(fmt), hbm_budget=160e9, max_active=8, chunk=2)
        t0 = time.perf_counter()
        res = srv.run(reqs)
        served[fmt] = dict(serve.latency_stats(res), wall_s=time.perf_counter() - t0,
                           peak_active=srv.peak_active, peak_gb=srv.peak_bytes / 1e9)
    t0 = time.perf_counter()
    seq = serve.run_sequential(serve.GPUBackend("complex64", graph=False), reqs)
    t_seq = time.perf_counter() - t0
    st_seq = serve.latency_stats(seq)
    line = {"metric": "served CG solves/s", "value": served["complex64"]["solves_per_s"],
            "unit": "solves/s", "n_gpus": 1, "higher_is_better": True, "data": "synthetic",
            "dtype": "c64 vectors, FP64 reductions",
            "config": {"workload": "serve", "requests": n_req, "rate_per_s": args.rate,
                       "iters": "U{10..40}", "sizes": "uneven-batch distribution, seed 11",
                       "hbm_budget_gb": 160, "max_active": 8},
            "served": served,
            "sequential_complex64": dict(st_seq, wall_s=t_seq)}
    print(json.dumps(line), flush=True)
    return 0


def run_toep(args):
    """Kernel build (mr_calc_toep) timed both ways: the closed form (FP64
    GEMMs) and the spreading build (ES-kernel type-1 NUFFT with FP64
    accumulation), on the headline stack and on a 3-D kooshball grid
    (128^3 image, 256^3 grid, L = 4, 10000 spokes of 256 samples), with the
    two results compared (relative L2)."""
    import os

    import torch

    import mr_aha_b200 as mr
    from mr_aha_b200 import synth

    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    cases = {
        "stack320": synth.workload("stack320", with_x=False),
        "kooshball128": synth.spec_inputs(dict(traj_type="3D", n_dim=(128, 128, 128), L=4,
                                               n_coils=1, n_traj=10000, n_kx=256,
                                               n_frames=200, frame_rule="div", seed=41),
                                          with_x=False),
    }
    out = {}
    for name, w in cases.items():
        cfg = mr.make_config(w["traj_type"], w["n_dim"], w["L"], n_coils=w["n_coils"],
                             mem_fraction=0.6)
        phi2 = torch.from_numpy(w["phi2"]).to(dev)
        traj = torch.from_numpy(w["traj"]).to(dev)
        res, Ks = {}, {}
        for method, code in (("spread", "1"), ("closed_form", "2")):
            os.environ["MR_AHA_B200_TOEP_METHOD"] = code
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            Ks[method] = mr.calc_toep(cfg, phi2, traj)
            torch.cuda.synchronize()
            res[method + "_s"] = time.perf_counter() - t0
        os.environ.pop("MR_AHA_B200_TOEP_METHOD")
        res["rel_l2_spread_vs_closed_form"] = _rel(Ks["spread"], Ks["closed_form"])
        res["kernel_gb"] = Ks["spread"].numel() * 8 / 1e9
        del Ks
        torch.cuda.empty_cache()
        out[name] = res
    line = {"metric": "Toeplitz kernel build time", "value": out["kooshball128"]["spread_s"],
            "unit": "s", "n_gpus": 1, "higher_is_better": False, "data": "synthetic",
            "dtype": "FP64 accumulation, complex64 result",
            "config": {"workload": "toep", "cases": list(cases)}, "builds": out}
    print(json.dumps(line), flush=True)
    return 0


def run_forms(args):
    """The operator's other forms timed beside the plain Toeplitz apply of the
    same inputs (CUDA events, after 3 warm-up applies): the masked Toeplitz
    operator (kernel kept only at the grid locations near samples,
    mr_calc_mask) at stack320, and the NUFFT-method operator (per coil a
    type-2 NUFFT, the Gram multiply per sample and a type-1 NUFFT; no kernel)
    at stack64 and on a 3-D 64^3 kooshball; each with its relative L2 against
    the plain operator (the masked form drops the kernel outside the mask, so
    that figure is its approximation error, not rounding)."""
    import torch

    import mr_aha_b200 as mr
    from mr_aha_b200 import synth

    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    steps = max(3, args.steps // 3)

    def timed(op, x, out):
        for _ in range(3):
            op(x, out=out)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            op(x, out=out)
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    cases = {
        "stack320": (synth.workload("stack320"), "masked"),
        "stack64": (synth.workload("stack64"), "nufft"),
        "kooshball64": (synth.spec_inputs(dict(traj_type="3D", n_dim=(64, 64, 64), L=4,
                                               n_coils=4, n_traj=2000, n_kx=128, n_frames=40,
                                               frame_rule="div", seed=31)), "nufft"),
    }
    res = {}
    for name, (w, form) in cases.items():
        kw = dict(phi2_dim=w["phi2_dim"], n_coils=w["n_coils"], mem_fraction=0.6)
        cfg = mr.make_config(w["traj_type"], w["n_dim"], w["L"], **kw)
        x = torch.from_numpy(w["x"]).to(dev)
        S = torch.from_numpy(w["SEs"]).to(dev)
        phi2 = torch.from_numpy(w["phi2"]).to(dev)
        traj = torch.from_numpy(w["traj"]).to(dev)
        out = torch.empty_like(x)
        r = {}
        with mr.create_op(cfg, S, phi2, traj) as op:
            r["toeplitz_ms"] = timed(op, x, out)
        y_plain = out.clone()
        if form == "masked":
            mask = mr.calc_mask(cfg, traj)
            mcfg = mr.make_config(w["traj_type"], w["n_dim"], w["L"], is_masked=True,
                                  num_masked=int(mask.numel()), **kw)
            with mr.create_op(mcfg, S, phi2, traj, mask=mask) as mop:
                r["masked_ms"] = timed(mop, x, out)
            r["num_masked"] = int(mask.numel())
            r["grid_locations"] = int(np.prod(w["phi2_dim"]))
            r["masked_vs_unmasked_rel_l2"] = _rel(out, y_plain)
        else:
            with mr.create_op(cfg, S, phi2, traj, method="nufft") as nop:
                r["nufft_ms"] = timed(nop, x, out)
            r["nufft_vs_toeplitz_rel_l2"] = _rel(out, y_plain)
        res[name] = r
        del x, S, phi2, traj, out, y_plain
        torch.cuda.empty_cache()
    line = {"metric": "masked Toeplitz A^H A applies/s (stack320)",
            "value": 1e3 / res["stack320"]["masked_ms"], "unit": "applies/s", "n_gpus": 1,
            "higher_is_better": True, "data": "synthetic", "dtype": "c64",
            "config": {"workload": "forms", "cases": list(cases), "steps": steps},
            "forms": res}
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        if args.workload in ("cg320", "batch48", "serve", "toep", "forms"):
            print(json.dumps({"impl": "reference", "unavailable":
                              "no reference CPU implementation of this workload here: the "
                              "reference has no solver, batch or serving loop, and its kernel "
                              "build and NUFFT method run on FINUFFT / cufinufft, absent"}))
            return 0
        return run_reference(args)
    if args.workload == "cg320":
        return run_cg(args)
    if args.workload == "batch48":
        return run_batch(args)
    if args.workload == "serve":
        return run_serve(args)
    if args.workload == "forms":
        return run_forms(args)
    if args.workload == "toep":
        return run_toep(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
