"""Continuous-batching server of CG reconstructions (no reference counterpart:
the reference provides the operator, not a request loop).

Requests (each with its own coil maps, Gram blocks, trajectory, right-hand
side and iteration count) arrive over time. The loop admits them first come,
first served while the device memory they will hold -- Toeplitz kernel,
plan work buffers, maps, CG vectors -- fits an HBM budget and a slot is
free; builds each admitted request's operator; and keeps every admitted
solve resident on the device (``CGSolver``: vectors, step scalars, residual
history), issuing a few iterations at a time on the solver's own stream
whenever that stream has drained. Iterations of different requests are
therefore in flight on the GPU together, and new requests join while others
run. Latency is measured from arrival to the host seeing the last iteration
complete. The CG arithmetic is deterministic, so a request's result does not
depend on what it shared the GPU with.

The scheduling logic is separate from the device work (``Backend``), so it
is tested on the CPU with a fake backend.
"""

from __future__ import annotations

import collections
import dataclasses
import time
from typing import Any, Callable, List, Optional

import numpy as np


@dataclasses.dataclass
class Request:
    rid: int
    arrival: float               # seconds after the start of the run
    cfg: Any                     # MRConfig
    SEs: Any                     # device [C, (Nz,) Ny, Nx]
    phi2: Any                    # device Gram blocks
    traj: Any                    # device trajectory
    b: Any                       # device right-hand side, shaped like x
    n_iter: int
    lam: float = 0.0


@dataclasses.dataclass
class Result:
    rid: int
    x: Any
    rr: np.ndarray
    arrival: float
    admitted: float
    finished: float
    setup_s: float = 0.0         # host time spent building the request's operator

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


class Backend:
    """Device work of the server: build a request's operator and solver,
    issue iterations, report whether they are done, and tear down."""

    def estimate_bytes(self, req: Request) -> int:
        raise NotImplementedError

    def iteration_cost(self, req: Request) -> float:
        """Relative device time of one iteration (for scheduling)."""
        return 1.0

    def admit(self, req: Request):
        """Build the operator and the resident solver; returns (state, bytes)."""
        raise NotImplementedError

    def step(self, state, n: int) -> None:
        raise NotImplementedError

    def busy(self, state) -> bool:
        raise NotImplementedError

    def finish(self, state):
        """Residual history and the solution; frees the request's device state."""
        raise NotImplementedError


def kernel_bytes(cfg, kernel_format: str) -> int:
    """Device bytes of the operator's Toeplitz kernel in ``kernel_format``."""
    from . import api

    shape = api.phi2_toep_shape(cfg)
    nloc = int(np.prod(shape[1:]))
    ntri = int(shape[0])
    if kernel_format == "complex64":
        return nloc * ntri * 8
    return nloc * ntri * 4 + nloc * 4


class GPUBackend(Backend):
    """Operators of this library with their Toeplitz kernel built from the
    request's Gram blocks (``create_op``), stored in ``kernel_format``, and a
    resident ``CGSolver``. ``plan_bytes`` caps each plan's work buffers (the
    coil group shrinks to fit)."""

    def __init__(self, kernel_format: str = "int16", plan_bytes: float = 4e9,
                 graph: bool = True):
        self.kernel_format = kernel_format
        self.plan_bytes = float(plan_bytes)
        self.graph = graph

    def estimate_bytes(self, req: Request) -> int:
        from . import api

        cfg = req.cfg
        x_elems = int(api.lib.mr_x_size(api.ctypes.byref(cfg)))
        se = int(api.lib.mr_se_size(api.ctypes.byref(cfg)))
        k = kernel_bytes(cfg, self.kernel_format)
        if self.kernel_format != "complex64":
            k += kernel_bytes(cfg, "complex64")  # the complex64 build, until converted
        # plan buffers (capped), maps, b, x and three CG vectors
        return int(k + self.plan_bytes + 8 * (se + 5 * x_elems))

    def iteration_cost(self, req: Request) -> float:
        from . import api

        cfg = req.cfg
        vpad = int(api.lib.mr_pad_size(api.ctypes.byref(cfg)))
        # FFT work ~ L C per grid point, block multiply ~ L^2 C / 4
        return float(vpad) * cfg.n_coils * cfg.L * (1.0 + cfg.L / 4.0)

    def admit(self, req: Request):
        import torch

        from . import api

        cfg = api.MRConfig.from_buffer_copy(req.cfg)
        free, _ = torch.cuda.mem_get_info()
        cfg.mem_fraction = float(min(0.9, max(1e-4, self.plan_bytes / max(free, 1))))
        op = api.create_op(cfg, req.SEs, req.phi2, req.traj)
        op.blocked_copy(False)
        if self.kernel_format != "complex64":
            op.set_kernel_format(self.kernel_format, keep_complex64=False)
        # the server budgets device memory itself: no opportunistic blocked
        # kernel copy of either format (it would take memory budgeted for
        # other requests)
        op.blocked_copy(False)
        x = torch.empty_like(req.b)
        solver = op.cg_solver(req.b, x, lam=req.lam, max_iters=req.n_iter, zero_x=True,
                              graph=self.graph)
        nbytes = op.device_bytes + 8 * 4 * x.numel()
        return dict(op=op, solver=solver, x=x, req=req), nbytes

    def step(self, state, n: int) -> None:
        state["solver"].step(n)

    def busy(self, state) -> bool:
        return state["solver"].busy

    def finish(self, state):
        rr = state["solver"].residuals()
        state["solver"].close()
        state["op"].close()
        return rr, state["x"]


@dataclasses.dataclass
class _Active:
    req: Request
    state: Any
    nbytes: int
    admitted: float
    setup_s: float = 0.0
    issued: int = 0
    cost: float = 1.0


class Server:
    """The request loop. ``hbm_budget``: device bytes the admitted requests
    may hold together; ``max_active``: concurrent solves; ``chunk``:
    iterations issued per request each time its stream drains;
    ``background``: build and tear down requests' operators on a worker
    thread, so that the loop keeps the running solves fed meanwhile (their
    GPU work overlaps the builds); ``run_slots``: how many resident solves
    have iterations in flight at once, chosen by least remaining work
    (shortest remaining work first, re-decided every ``chunk`` iterations;
    ``None``: all of them, round robin)."""

    def __init__(self, backend: Backend, hbm_budget: float = 160e9, max_active: int = 8,
                 chunk: int = 2, clock: Callable[[], float] = time.perf_counter,
                 idle_sleep: float = 2e-4, background: bool = True,
                 run_slots: Optional[int] = 2):
        self.run_slots = run_slots
        self.backend = backend
        self.hbm_budget = float(hbm_budget)
        self.max_active = int(max_active)
        self.chunk = max(1, int(chunk))
        self.clock = clock
        self.idle_sleep = idle_sleep
        self.background = background
        self.peak_bytes = 0
        self.peak_active = 0
        self.trace: List[tuple] = []   # (time, event, rid)

    def run(self, requests: List[Request]) -> List[Result]:
        import concurrent.futures as cf

        for r in requests:
            if self.backend.estimate_bytes(r) > self.hbm_budget:
                raise ValueError(f"request {r.rid} needs more than the HBM budget on its own")
        pending = collections.deque(sorted(requests, key=lambda r: r.arrival))
        queue: collections.deque = collections.deque()
        active: List[_Active] = []
        admitting: list = []     # (request, future, admission time, bytes reserved)
        finishing: list = []     # (active entry, future, finish time)
        results: List[Result] = []
        used = 0
        ex = cf.ThreadPoolExecutor(max_workers=1) if self.background else None
        t0 = self.clock()
        try:
            while pending or queue or active or admitting or finishing:
                now = self.clock() - t0
                while pending and pending[0].arrival <= now:
                    queue.append(pending.popleft())
                progressed = False
                # admission: first come, first served, within memory and slots
                while (queue and not admitting and
                       len(active) + len(admitting) < self.max_active and
                       used + self.backend.estimate_bytes(queue[0]) <= self.hbm_budget):
                    req = queue.popleft()
                    est = self.backend.estimate_bytes(req)
                    t_adm = self.clock() - t0
                    used += est
                    self.trace.append((t_adm, "admit", req.rid))
                    if ex:
                        admitting.append((req, ex.submit(self.backend.admit, req), t_adm, est))
                    else:
                        state, nbytes = self.backend.admit(req)
                        used += max(nbytes, 0) - est
                        active.append(_Active(req, state, max(nbytes, 0), t_adm,
                                              self.clock() - t0 - t_adm,
                                              cost=self.backend.iteration_cost(req)))
                    self.peak_bytes = max(self.peak_bytes, used)
                    progressed = True
                for item in list(admitting):
                    req, fut, t_adm, est = item
                    if fut.done():
                        state, nbytes = fut.result()
                        admitting.remove(item)
                        used += max(nbytes, 0) - est
                        active.append(_Active(req, state, max(nbytes, 0), t_adm,
                                              self.clock() - t0 - t_adm,
                                              cost=self.backend.iteration_cost(req)))
                        self.peak_bytes = max(self.peak_bytes, used)
                        progressed = True
                self.peak_active = max(self.peak_active, len(active))
                # issue work / retire finished solves: the run_slots solves
                # with the least remaining work get iterations
                if self.run_slots is not None:
                    order = sorted(active, key=lambda a: (a.req.n_iter - a.issued) * a.cost)
                    allowed = set(id(a) for a in order[: self.run_slots])
                else:
                    allowed = None
                for a in list(active):
                    if self.backend.busy(a.state):
                        continue
                    if (allowed is not None and id(a) not in allowed and
                            a.issued < a.req.n_iter):
                        continue
                    if a.issued < a.req.n_iter:
                        k = min(self.chunk, a.req.n_iter - a.issued)
                        self.backend.step(a.state, k)
                        a.issued += k
                    else:
                        t_fin = self.clock() - t0
                        active.remove(a)
                        self.trace.append((t_fin, "finish", a.req.rid))
                        if ex:
                            finishing.append((a, ex.submit(self.backend.finish, a.state), t_fin))
                        else:
                            rr, x = self.backend.finish(a.state)
                            used -= a.nbytes
                            results.append(Result(a.req.rid, x, rr, a.req.arrival, a.admitted,
                                                  t_fin, a.setup_s))
                    progressed = True
                for item in list(finishing):
                    a, fut, t_fin = item
                    if fut.done():
                        rr, x = fut.result()
                        finishing.remove(item)
                        used -= a.nbytes
                        results.append(Result(a.req.rid, x, rr, a.req.arrival, a.admitted,
                                              t_fin, a.setup_s))
                        progressed = True
                if not progressed:
                    if not (active or queue or admitting or finishing) and pending:
                        wait = pending[0].arrival - (self.clock() - t0)
                        if wait > 0:
                            time.sleep(min(wait, 0.05))
                    elif self.idle_sleep:
                        time.sleep(self.idle_sleep)
        finally:
            if ex:
                ex.shutdown(wait=True)
        return sorted(results, key=lambda r: r.rid)


def run_sequential(backend: Backend, requests: List[Request],
                   clock: Callable[[], float] = time.perf_counter) -> List[Result]:
    """The plain reference point: one request at a time in arrival order,
    each solved to completion before the next is admitted."""
    srv = Server(backend, hbm_budget=float("inf"), max_active=1, chunk=1 << 30, clock=clock,
                 background=False)
    return srv.run(requests)


def latency_stats(results: List[Result], t_total: Optional[float] = None) -> dict:
    lat = np.array([r.latency for r in results])
    end = max(r.finished for r in results) if results else 0.0
    start = min(r.arrival for r in results) if results else 0.0
    span = t_total if t_total is not None else max(end - start, 1e-9)
    return dict(n=len(results), solves_per_s=len(results) / span,
                setup_s_total=float(sum(r.setup_s for r in results)),
                p50_s=float(np.percentile(lat, 50)) if len(lat) else None,
                p99_s=float(np.percentile(lat, 99)) if len(lat) else None,
                mean_s=float(lat.mean()) if len(lat) else None)
