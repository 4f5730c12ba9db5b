"""Continuous-batching solve server for the teal residual / time-integration path.

Requests (mesh, Mach number, equations, flux scheme, integrator, step budget or residual tolerance)
arrive at any time. The server admits a waiting request as soon as its device-memory estimate fits
the HBM budget, keeps its state resident on the GPU and batches it continuously with the requests
already running (`Server`): requests that share a scheme (equations, flux, limiter, precision,
integrator, CFL number) form a lane, and each lane advances all of its requests in one arena (one
launch per kernel for all of them, the step replayed from a CUDA graph), in rounds of a few steps.
Between rounds, requests that finished leave and newly admitted ones join: the lane re-packs its
arena, carrying every running request's state (exact FP64 rows) and clock over. Lanes run on their
own host threads and CUDA streams, so different schemes overlap on the device. Every result is the
same bits as the request solved alone: an instance's step depends on its own state only, and every
kernel is deterministic.

`StreamServer` is the simpler design kept for comparison: one context, CUDA stream and host thread
per request, overlapping on the device but sharing no launches. Its admission (`Scheduler`) is
independent of the GPU: it takes an `execute(request)` callable, so admission and failure handling
are testable on the host with a fake executor.
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
    """One solve request. `steps` bounds its steps (explicit RK, or implicit Euler for a steady
    solve); `tolerance` (> 0) stops it earlier once the maximum residual has dropped by that factor
    from the first step's."""

    id: int
    cells: tuple                     # (nx, ny, nz) of the channel box; (n, n, n) grid of a ramp
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
    method: str = "lserk"            # teal's advance name: "lserk" or "implicit euler" (steady solves)
    mesh: str = "channel"            # "channel" box, or "ramp": the mixed-element ramp of the batch workload
    seed: int = 0                    # mesh seed of a ramp
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
        if self.mesh == "ramp":
            return int(round(4.64 * self.cells[0] ** 3))  # a ramp grid holds ~4.64 cells per hexahedron
        return int(np.prod(self.cells))

    @property
    def latency(self):
        return self.finished - self.arrival


def memory_estimate(req):
    """Device bytes a request holds while resident (FP64 layout; peak of the upload included; the
    Krylov workspace of implicit steps)."""
    cells = req.num_cells
    if req.mesh == "ramp":
        faces = int(2.2 * cells)
    else:
        nx, ny, nz = req.cells
        faces = 3 * cells + nx * ny + ny * nz + nz * nx
    per_cell = 700 + (80 if req.physics == _lib.TG_NAVIERSTOKES else 0)
    if req.method == "implicit euler":
        per_cell += 40 * (31 + 8)  # Krylov basis (dimension 30) and the Newton vectors
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


def build_problem(req):
    """Host mesh and equations of a request (teal_b200 Equations with its initial state)."""
    from .api import Equations, Mesh

    if req.mesh == "ramp":
        from . import meshes

        n = int(req.cells[0])
        mesh = Mesh.from_cells(meshes.ramp_mesh(n=(n, n, n), seed=req.seed))
    else:
        nx, ny, nz = req.cells
        mesh = Mesh.create((0, 0, 0), (nx / ny, 1.0, nz / ny), (nx, ny, nz), (0, 0, 1))
    eqns = Equations.navierstokes(mesh) if req.physics == _lib.TG_NAVIERSTOKES else Equations.euler(mesh)
    eqns.set_convective_flux(req.flux)
    eqns.set_limiter(req.limiter, 1.0)
    if req.physics == _lib.TG_NAVIERSTOKES:
        eqns.set_property("dynamic viscosity", req.viscosity)
    free = free_stream(req.mach, req.angle)
    if req.mesh == "ramp":  # the batch workload's boundaries: far field around, slip walls
        for side in ("left", "right", "top"):
            eqns.set_boundary_condition(side, "farfield", free)
        for side in ("bottom", "back", "front"):
            eqns.set_boundary_condition(side, "slipwall")
        eqns.primitive[:] = np.tile(free, (mesh.num_cells, 1))
        return eqns
    for side in ("left", "right", "top"):
        eqns.set_boundary_condition(side, "farfield", free)
    eqns.set_boundary_condition("bottom", "slipwall")
    # a density bump on the free stream: the solve relaxes it out through the far field
    c = mesh.cell_center
    prim = np.tile(free, (mesh.num_cells, 1))
    r2 = ((c[:, 0] - 0.5 * nx / ny) ** 2 + (c[:, 1] - 0.5) ** 2) / 0.02
    prim[:, 0] *= 1 + 0.2 * np.exp(-r2)
    eqns.set_initial_condition("domain", initial=None, compute=lambda x: prim[: x.shape[0]])
    return eqns


def method_of(req):
    """(TG_ADVANCE_*, context) of a request's integrator: lserk{3,3}, or implicit Euler with teal's
    Newton-Krylov settings of its steady airfoil run (run/airfoil/run.c: {0.1, 0.3, 30})."""
    if req.method == "implicit euler":
        return _lib.TG_ADVANCE_IMPLICIT_EULER, (0.1, 0.3, 30)
    if req.method != "lserk":
        raise ValueError(f"invalid advance method ({req.method})")
    return _lib.TG_ADVANCE_LSERK, (3, 3)


def lane_key(req):
    """Requests with equal keys can share one arena (the arena shares equations, schemes, properties,
    precision, integrator and CFL number)."""
    ns = req.physics == _lib.TG_NAVIERSTOKES
    return (req.physics, req.flux, req.limiter, req.precision, req.method, req.courant,
            req.viscosity if ns else None)


def solve(req, stream=None, chunk=25):
    """Solve one request alone on the current GPU (its own context): one step, whose residual sets the
    tolerance's threshold, then the remaining steps with the residual test on the device."""
    eqns = build_problem(req)
    mesh = eqns.mesh
    ctx = eqns.context(req.precision)
    if stream is not None:
        ctx.set_stream(stream)
    method, mctx = method_of(req)
    t, it, res = ctx.run(method, req.courant, 1, context=mctx)
    total = it
    threshold = req.tolerance * float(np.max(res)) if req.tolerance > 0 else 0.0
    # the remaining steps in chunks (the same steps, replayed from the same graph), so a cancelled
    # request stops at the next chunk boundary
    while total < req.steps and not req.cancelled:
        n = min(chunk, req.steps - total)
        t, it, res = ctx.run(method, req.courant, n, threshold=threshold, context=mctx, time=t)
        total += it
        if threshold > 0 and float(np.max(res)) < threshold:  # the device's stop test (run.c:80-82)
            break
    req.iterations = total
    req.residual = res
    req.state = ctx.get_primitive()[: mesh.num_inner_cells]
    ctx.close()
    return req


class _Entry:
    """A running request inside a lane."""

    def __init__(self, req, eqns):
        self.req = req
        self.eqns = eqns
        self.time = 0.0
        self.iterations = 0
        self.threshold = None  # set from the first step's residual
        self.residual = None


class Lane:
    """Requests of one scheme advancing together in one resident arena (continuous batching).

    `round()` advances every running request by up to `chunk` steps in one batched run (a request's
    first step alone, as `solve` takes it, since its residual sets the request's threshold), then
    removes the requests that finished (step budget, tolerance, a non-finite state, cancellation).
    Joining requests get a new arena: it is built (host merge and upload of every mesh) on a
    background thread while the current arena keeps stepping; at the next round boundary the running
    requests' states (all rows, exact FP64) move over and the lane switches, so a request's steps are
    the ones it takes alone. Finished requests stay in the arena without steps until a re-pack, which
    also starts when they hold more than half of its cells."""

    def __init__(self, key, chunk, stream=None, device=0):
        self.key = key
        self.chunk = int(chunk)
        self.stream = stream
        self.device = device
        self.entries = []
        self.arena = None
        self.arena_entries = []
        self.next = None  # (thread, result holder, entries) of an arena being built
        self.repacks = 0
        self.repack_s = 0.0

    def join(self, req, eqns):
        self.entries.append(_Entry(req, eqns))

    def _build(self, entries):
        from .api import Batch

        t0 = time.perf_counter()
        arena = Batch([e.eqns for e in entries], precision=entries[0].req.precision)
        if self.stream is not None:
            arena.set_stream(self.stream)
        return arena, time.perf_counter() - t0

    def _start_build(self):
        import torch

        entries = list(self.entries)
        holder = {}

        def work():
            try:
                torch.cuda.set_device(self.device)
                holder["arena"], holder["secs"] = self._build(entries)
            except Exception as exc:  # reported at the switch
                holder["error"] = exc

        th = threading.Thread(target=work, daemon=True)
        th.start()
        self.next = (th, holder, entries)

    def _switch(self):
        """Move the running requests' states from the current arena into the built one."""
        th, holder, entries = self.next
        th.join()
        self.next = None
        if "error" in holder:
            raise holder["error"]
        arena = holder["arena"]
        t0 = time.perf_counter()
        if self.arena is not None:
            where = {id(e): i for i, e in enumerate(self.arena_entries)}
            for j, e in enumerate(entries):
                if id(e) in where:
                    arena.set_primitive(j, self.arena.get_primitive(where[id(e)]))
            self.arena.close()
        self.arena = arena
        self.arena_entries = entries
        self.repacks += 1
        self.repack_s += holder["secs"] + (time.perf_counter() - t0)

    def _needs_repack(self):
        """A request joined (it has no row in the arena), or finished requests, which sit in the arena
        without steps, hold more than half of its cells."""
        if self.arena is None:
            return True
        inside = {id(e) for e in self.arena_entries}
        if any(id(e) not in inside for e in self.entries):
            return True
        live = {id(e) for e in self.entries}
        idle = sum(e.eqns.mesh.num_inner_cells for e in self.arena_entries if id(e) not in live)
        total = sum(e.eqns.mesh.num_inner_cells for e in self.arena_entries)
        return 2 * idle > total

    def round(self):
        """One round; returns the requests that finished in it."""
        finished = [e for e in self.entries if e.req.cancelled]
        self.entries = [e for e in self.entries if not e.req.cancelled]
        for e in finished:
            e.req.error = "cancelled"
            e.req.iterations = e.iterations
        if not self.entries:
            self.close()
            return [e.req for e in finished]
        if self.next is not None and not self.next[0].is_alive():
            self._switch()
        if self.next is None and self._needs_repack():
            self._start_build()
        live = {id(e) for e in self.entries}
        if self.arena is None or not any(id(e) in live for e in self.arena_entries):
            if self.next is None:
                self._start_build()
            self._switch()  # nothing to step meanwhile: wait for the new arena
        req0 = self.entries[0].req
        method, mctx = method_of(req0)
        # requests that finished, or joined after this arena was built, take no steps in it
        max_iter = [0 if id(e) not in live else
                    1 if e.threshold is None else max(0, min(self.chunk, e.req.steps - e.iterations))
                    for e in self.arena_entries]
        thr = [0.0 if e.threshold is None else e.threshold for e in self.arena_entries]
        t, it, res = self.arena.run(method, req0.courant, max_iter, variable=-1, threshold=thr, context=mctx,
                                    time=[e.time for e in self.arena_entries])
        status = self.arena.status()
        done_ids = set()
        for i, e in enumerate(self.arena_entries):
            if id(e) not in live:
                continue
            e.time = float(t[i])
            e.iterations += int(it[i])
            e.residual = res[i].copy()
            first = e.threshold is None
            if first:
                e.threshold = e.req.tolerance * float(np.max(res[i])) if e.req.tolerance > 0 else 0.0
            # the device's stop test (run.c:80-82), also when it fired on the round's last step
            converged = not first and e.threshold > 0 and float(np.max(res[i])) < e.threshold
            if status[i] != 0 or converged or e.iterations >= e.req.steps:
                r = e.req
                r.iterations = e.iterations
                r.residual = e.residual
                if status[i] != 0:
                    r.error = "non-finite time step or residual"
                else:
                    r.state = self.arena.get_primitive(i)[: e.eqns.mesh.num_inner_cells].copy()
                finished.append(e)
                done_ids.add(id(e))
        self.entries = [e for e in self.entries if id(e) not in done_ids]
        return [e.req for e in finished]

    def close(self):
        if self.next is not None:
            th, holder, _ = self.next
            th.join()
            self.next = None
            if "arena" in holder:
                holder["arena"].close()
        if self.arena is not None:
            self.arena.close()
            self.arena = None
        self.arena_entries = []


class Server:
    """Continuous-batching GPU solve server: admission by HBM budget in arrival order (no overtaking),
    host meshes built on a thread pool as requests arrive, one `Lane` per scheme on its own thread
    and CUDA stream, requests joining and leaving their lane's arena between rounds of `chunk`
    steps."""

    def __init__(self, budget_bytes=None, max_active=64, chunk=10, device=0, builders=4):
        import torch

        torch.cuda.set_device(device)
        if budget_bytes is None:
            free, _ = torch.cuda.mem_get_info()
            budget_bytes = int(0.8 * free)
        self.torch = torch
        self.device = device
        self.budget = int(budget_bytes)
        self.max_active = int(max_active)
        self.chunk = int(chunk)
        self.builders = int(builders)
        self.used = 0
        self.peak_used = 0
        self.peak_active = 0
        self.lanes = {}
        self.repacks = 0
        self.repack_s = 0.0
        self._requests = {}
        self._cancel_pending = set()
        self._cancel_lock = threading.Lock()

    def cancel(self, rid):
        """Cancel request `rid`: one not yet admitted never runs; a running one leaves its lane at the
        next round (its memory is released then)."""
        with self._cancel_lock:
            r = self._requests.get(rid)
            if r is None:
                self._cancel_pending.add(rid)
                return False
            r.cancelled = True
            return True

    def serve(self, requests, timeout=None):
        """Serve `requests` (arrival times relative to now) to completion; returns them by id."""
        import concurrent.futures
        import queue

        torch = self.torch
        clock = time.perf_counter
        t0 = clock()
        pending = sorted(requests, key=lambda r: (r.arrival, r.id))
        with self._cancel_lock:
            self._requests = {r.id: r for r in pending}
            for rid in self._cancel_pending:
                if rid in self._requests:
                    self._requests[rid].cancelled = True
        total = len(pending)
        done = []
        building = {}  # id -> (request, future)
        waiting = []   # arrival order, host problem built or being built
        active = {}    # id -> bytes
        finished_q = queue.Queue()
        lane_inbox = {}
        threads = {}
        stop = threading.Event()
        lock = threading.Lock()

        def lane_loop(key, inbox):
            torch.cuda.set_device(self.device)
            stream = torch.cuda.Stream()
            lane = Lane(key, self.chunk, stream.cuda_stream, self.device)
            try:
                while not stop.is_set():
                    try:
                        while True:
                            req, eqns = inbox.get_nowait()
                            lane.join(req, eqns)
                    except queue.Empty:
                        pass
                    if not lane.entries:
                        lane.close()
                        try:
                            req, eqns = inbox.get(timeout=0.02)
                            lane.join(req, eqns)
                        except queue.Empty:
                            continue
                    try:
                        for r in lane.round():
                            finished_q.put(r)
                    except Exception as exc:  # the lane's requests fail, the server goes on
                        for e in lane.entries:
                            e.req.error = f"{type(exc).__name__}: {exc}"
                            finished_q.put(e.req)
                        lane.entries = []
                        lane.close()
            finally:
                lane.close()
                with lock:
                    self.repacks += lane.repacks
                    self.repack_s += lane.repack_s

        pool = concurrent.futures.ThreadPoolExecutor(max_workers=self.builders)
        deadline = None if timeout is None else t0 + timeout
        try:
            while len(done) < total:
                now = clock() - t0
                while pending and pending[0].arrival <= now:
                    r = pending.pop(0)
                    if memory_estimate(r) > self.budget:
                        r.error = "request exceeds the device memory budget"
                        r.finished = now
                        done.append(r)
                        continue
                    building[r.id] = (r, pool.submit(build_problem, r))
                    waiting.append(r)
                # admit in arrival order while memory and slots allow (no overtaking)
                while waiting and len(active) < self.max_active:
                    r = waiting[0]
                    if r.cancelled:  # never admitted
                        waiting.pop(0)
                        building.pop(r.id)[1].cancel()
                        r.error = "cancelled"
                        r.finished = clock() - t0
                        done.append(r)
                        continue
                    nbytes = memory_estimate(r)
                    if self.used + nbytes > self.budget:
                        break
                    fut = building[r.id][1]
                    if not fut.done():
                        break
                    waiting.pop(0)
                    del building[r.id]
                    try:
                        eqns = fut.result()
                    except Exception as exc:
                        r.error = f"{type(exc).__name__}: {exc}"
                        r.finished = clock() - t0
                        done.append(r)
                        continue
                    self.used += nbytes
                    self.peak_used = max(self.peak_used, self.used)
                    active[r.id] = nbytes
                    self.peak_active = max(self.peak_active, len(active))
                    r.admitted = clock() - t0
                    key = lane_key(r)
                    if key not in lane_inbox:
                        lane_inbox[key] = queue.Queue()
                        threads[key] = threading.Thread(target=lane_loop, args=(key, lane_inbox[key]), daemon=True)
                        threads[key].start()
                    lane_inbox[key].put((r, eqns))
                try:
                    wait = 0.01
                    if pending:
                        wait = max(0.0, min(wait, pending[0].arrival - (clock() - t0)))
                    r = finished_q.get(timeout=wait)
                    while True:
                        r.finished = clock() - t0
                        self.used -= active.pop(r.id)
                        done.append(r)
                        r = finished_q.get_nowait()
                except queue.Empty:
                    pass
                if deadline is not None and clock() > deadline:
                    raise TimeoutError("serving did not finish in time")
        finally:
            stop.set()
            for th in threads.values():
                th.join(timeout=60)
            pool.shutdown(wait=False, cancel_futures=True)
        self.lanes = list(threads)
        return sorted(done, key=lambda r: r.id)


class StreamServer:
    """GPU solve server without shared launches: `Scheduler` with `solve` as the executor, one
    context, CUDA stream and host thread per request (their kernels overlap on the device)."""

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


def poisson_requests(num, rate, seed, min_cells=20_000, max_cells=2_000_000, steps=(50, 200), mesh="channel",
                     physics=(_lib.TG_EULER,), method="lserk", courant=None):
    """Seeded Poisson arrivals; mesh sizes log-uniform in [min_cells, max_cells]; Mach 0.2-3.0; flux
    scheme (roe / hllc / ausmd), equations (from `physics`) and tolerance 1e-6..1e-10 per request;
    channel boxes, or the batch workload's ramp meshes (`mesh="ramp"`)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(num):
        t += rng.exponential(1.0 / rate)
        cells = math.exp(rng.uniform(math.log(min_cells), math.log(max_cells)))
        if mesh == "ramp":
            n = max(8, int(round((cells / 4.64) ** (1.0 / 3.0))))
            dims = (n, n, n)
        else:
            nz = 2
            ny = max(4, int(round(math.sqrt(cells / (3 * nz)))))
            nx = max(4, int(round(cells / (ny * nz))))
            dims = (nx, ny, nz)
        phys = int(rng.choice(list(physics)))
        out.append(Request(
            id=i, cells=dims, mach=float(rng.uniform(0.2, 3.0)), angle=float(rng.uniform(0, 10)),
            flux=str(rng.choice(["roe", "hllc", "ausmd"])), steps=int(rng.integers(steps[0], steps[1] + 1)),
            tolerance=float(10 ** rng.uniform(-10, -6)), arrival=t, physics=phys, mesh=mesh, seed=1000 + i,
            method=method, courant=courant if courant else (0.5 if method == "lserk" else 30.0),
            limiter="venkatakrishnan" if method == "implicit euler" else "minmod"))
    return out


def percentile(values, q):
    v = sorted(values)
    if not v:
        return math.nan
    k = (len(v) - 1) * q / 100.0
    f, c = math.floor(k), math.ceil(k)
    return v[int(k)] if f == c else v[f] + (v[c] - v[f]) * (k - f)
