"""Continuous-batching solve server for the teal residual / time-integration path.

Requests (mesh, Mach number, equations, flux scheme, step count or residual tolerance) arrive at any
time. The server admits a waiting request as soon as its device-memory estimate fits the HBM budget
and a slot is free, keeps its state resident on the GPU in its own context and CUDA stream, and
advances all admitted requests concurrently (one host thread per request; the device overlaps their
kernels). A finished request releases its memory and slot, which admits the next one. Each result
is the same bits as the request solved alone: contexts share nothing and every kernel is
deterministic.

The scheduler (`Scheduler`) is independent of the GPU: it takes an `execute(request)` callable, so
its admission and failure handling are testable on the host with a fake executor.
"""

import dataclasses
import heapq
import math
import threading
import time

import numpy as np

from . import _lib


@dataclasses.dataclass
class Request:
    """One solve request. `steps` bounds the explicit RK steps; `tolerance` (> 0) stops earlier once
    the maximum residual has dropped by that factor from the first step's."""

    id: int
    cells: tuple                     # (nx, ny, nz) of the channel box
    mach: float = 0.5
    angle: float = 0.0               # flow angle in degrees
    physics: int = _lib.TG_EULER
    flux: str = "hllc"
    limiter: str = "minmod"
    viscosity: float = 1e-3          # Navier-Stokes only
    steps: int = 100
    tolerance: float = 0.0
    courant: float = 0.5
    arrival: float = 0.0             # seconds after the server's start
    precision: int = _lib.TG_PRECISION_FP64
    # filled by the server
    admitted: float = math.nan
    finished: float = math.nan
    iterations: int = 0
    residual: object = None
    state: object = None
    error: str = ""
    cancelled: bool = False          # set by Scheduler.cancel; a running solve stops at its next chunk

    @property
    def num_cells(self):
        return int(np.prod(self.cells))

    @property
    def latency(self):
        return self.finished - self.arrival


def memory_estimate(req):
    """Device bytes a request holds while resident (FP64 layout; peak of the upload included)."""
    nx, ny, nz = req.cells
    cells = nx * ny * nz
    faces = 3 * cells + nx * ny + ny * nz + nz * nx
    per_cell = 700 + (80 if req.physics == _lib.TG_NAVIERSTOKES else 0)
    return int(per_cell * cells + 450 * faces + (8 << 20))


def free_stream(mach, angle_deg, gamma=1.4):
    """Primitive free-stream state with unit density and pressure 1/gamma (sound speed 1)."""
    a = math.radians(angle_deg)
    return np.array([1.0, mach * math.cos(a), mach * math.sin(a), 0.0, 1.0 / gamma])


class Scheduler:
    """Admission by memory budget and slot count; one worker thread per admitted request."""

    def __init__(self, budget_bytes, max_active, execute, estimate=memory_estimate, clock=time.perf_counter):
        self.budget = int(budget_bytes)
        self.max_active = int(max_active)
        self.execute = execute
        self.estimate = estimate
        self.clock = clock
        self.lock = threading.Condition()
        self.waiting = []      # heap of (arrival, id, request)
        self.active = {}       # id -> (request, bytes, thread)
        self.done = []
        self.used = 0
        self.peak_used = 0
        self.peak_active = 0
        self.t0 = None
        self._cancel_pending = set()

    def cancel(self, rid):
        """Cancel request `rid`: a waiting or not yet arrived request never runs, a running one stops
        at its next chunk boundary (its memory and slot are released when its worker returns)."""
        with self.lock:
            for k, (arrival, wid, r) in enumerate(self.waiting):
                if wid == rid:
                    self.waiting.pop(k)
                    heapq.heapify(self.waiting)
                    r.cancelled = True
                    r.error = "cancelled"
                    r.finished = (self.clock() - self.t0) if self.t0 is not None else r.arrival
                    self.done.append(r)
                    self.lock.notify_all()
                    return True
            if rid in self.active:
                self.active[rid][0].cancelled = True
                return True
            self._cancel_pending.add(rid)
            return False

    def submit(self, req):
        if req.id in self._cancel_pending or req.cancelled:
            req.cancelled = True
            req.error = "cancelled"
            req.finished = req.arrival
            with self.lock:
                self.done.append(req)
                self.lock.notify_all()
            return
        if self.estimate(req) > self.budget:
            req.error = "request exceeds the device memory budget"
            req.finished = req.arrival
            with self.lock:
                self.done.append(req)
            return
        with self.lock:
            heapq.heappush(self.waiting, (req.arrival, req.id, req))
            self.lock.notify_all()

    def _worker(self, req, nbytes):
        try:
            self.execute(req)
            if req.cancelled and not req.error:
                req.error = "cancelled"
        except Exception as exc:  # a failing request is reported, never fatal to the server
            req.error = f"{type(exc).__name__}: {exc}"
        with self.lock:
            req.finished = self.clock() - self.t0
            del self.active[req.id]
            self.used -= nbytes
            self.done.append(req)
            self.lock.notify_all()

    def run(self, requests, timeout=None):
        """Serve `requests` (arrival times relative to now) to completion; returns them."""
        self.t0 = self.clock()
        pending = sorted(requests, key=lambda r: (r.arrival, r.id))
        total = len(pending)
        deadline = None if timeout is None else self.t0 + timeout
        with self.lock:
            while len(self.done) < total:
                now = self.clock() - self.t0
                while pending and pending[0].arrival <= now:
                    r = pending.pop(0)
                    self.lock.release()
                    try:
                        self.submit(r)
                    finally:
                        self.lock.acquire()
                # admit in arrival order while memory and slots allow (no overtaking)
                while self.waiting and len(self.active) < self.max_active:
                    arrival, rid, r = self.waiting[0]
                    nbytes = self.estimate(r)
                    if self.used + nbytes > self.budget:
                        break
                    heapq.heappop(self.waiting)
                    self.used += nbytes
                    self.peak_used = max(self.peak_used, self.used)
                    r.admitted = self.clock() - self.t0
                    th = threading.Thread(target=self._worker, args=(r, nbytes), daemon=True)
                    self.active[r.id] = (r, nbytes, th)
                    self.peak_active = max(self.peak_active, len(self.active))
                    th.start()
                if deadline is not None and self.clock() > deadline:
                    raise TimeoutError("serving did not finish in time")
                wait = 0.05
                if pending:
                    wait = max(0.0, min(wait, pending[0].arrival - (self.clock() - self.t0)))
                self.lock.wait(timeout=wait)
        return sorted(self.done, key=lambda r: r.id)


def solve(req, stream=None, chunk=25):
    """Solve one request on the current GPU (its own context; used alone or by the server)."""
    from .api import Equations, Mesh

    nx, ny, nz = req.cells
    mesh = Mesh.create((0, 0, 0), (nx / ny, 1.0, nz / ny), (nx, ny, nz), (0, 0, 1))
    eqns = Equations.navierstokes(mesh) if req.physics == _lib.TG_NAVIERSTOKES else Equations.euler(mesh)
    eqns.set_convective_flux(req.flux)
    eqns.set_limiter(req.limiter, 1.0)
    if req.physics == _lib.TG_NAVIERSTOKES:
        eqns.set_property("dynamic viscosity", req.viscosity)
    free = free_stream(req.mach, req.angle)
    for side in ("left", "right", "top"):
        eqns.set_boundary_condition(side, "farfield", free)
    eqns.set_boundary_condition("bottom", "slipwall")
    # a density bump on the free stream: the solve relaxes it out through the far field
    c = mesh.cell_center
    prim = np.tile(free, (mesh.num_cells, 1))
    r2 = ((c[:, 0] - 0.5 * nx / ny) ** 2 + (c[:, 1] - 0.5) ** 2) / 0.02
    prim[:, 0] *= 1 + 0.2 * np.exp(-r2)
    eqns.set_initial_condition("domain", initial=None, compute=lambda x: prim[: x.shape[0]])
    ctx = eqns.context(req.precision)
    if stream is not None:
        ctx.set_stream(stream)
    method = _lib.TG_ADVANCE_LSERK
    t, it, res = ctx.run(method, req.courant, 1, context=(3, 3))
    total = it
    threshold = req.tolerance * float(np.max(res)) if req.tolerance > 0 else 0.0
    # the remaining steps in chunks (the same steps, replayed from the same graph), so a cancelled
    # request stops at the next chunk boundary
    while total < req.steps and not req.cancelled:
        n = min(chunk, req.steps - total)
        t, it, res = ctx.run(method, req.courant, n, threshold=threshold, context=(3, 3), time=t)
        total += it
        if it < n:  # the residual fell below the threshold
            break
    req.iterations = total
    req.residual = res
    req.state = ctx.get_primitive()[: mesh.num_inner_cells]
    ctx.close()
    return req


class Server:
    """GPU solve server: `Scheduler` with `solve` as the executor, one CUDA stream per request."""

    def __init__(self, budget_bytes=None, max_active=8, device=0):
        import torch

        torch.cuda.set_device(device)
        if budget_bytes is None:
            free, _ = torch.cuda.mem_get_info()
            budget_bytes = int(0.8 * free)
        self.torch = torch
        self.scheduler = Scheduler(budget_bytes, max_active, self._execute)

    def _execute(self, req):
        stream = self.torch.cuda.Stream()
        solve(req, stream.cuda_stream)

    def serve(self, requests, timeout=None):
        return self.scheduler.run(requests, timeout=timeout)


def poisson_requests(num, rate, seed, min_cells=20_000, max_cells=2_000_000, steps=(50, 200)):
    """Seeded Poisson arrivals; mesh sizes log-uniform in [min_cells, max_cells]; Mach 0.2-3.0;
    flux scheme per request; tolerance 1e-6..1e-10."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(num):
        t += rng.exponential(1.0 / rate)
        cells = math.exp(rng.uniform(math.log(min_cells), math.log(max_cells)))
        nz = 2
        ny = max(4, int(round(math.sqrt(cells / (3 * nz)))))
        nx = max(4, int(round(cells / (ny * nz))))
        out.append(Request(
            id=i, cells=(nx, ny, nz), mach=float(rng.uniform(0.2, 3.0)), angle=float(rng.uniform(0, 10)),
            flux=str(rng.choice(["roe", "hllc", "ausmd"])), steps=int(rng.integers(steps[0], steps[1] + 1)),
            tolerance=float(10 ** rng.uniform(-10, -6)), arrival=t))
    return out


def percentile(values, q):
    v = sorted(values)
    if not v:
        return math.nan
    k = (len(v) - 1) * q / 100.0
    f, c = math.floor(k), math.ceil(k)
    return v[int(k)] if f == c else v[f] + (v[c] - v[f]) * (k - f)
