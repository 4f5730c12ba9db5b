#!/usr/bin/env python
"""Benchmark of the teal residual / time-integration path on B200.

Workload (one GPU): compressible Navier-Stokes Taylor-Green vortex on a periodic 128^3 hex mesh over
[0, 2pi]^3, Re 1600, Ma 0.1, Pr 0.71, gamma 1.4; Roe flux, least-squares gradients, Venkatakrishnan
limiter (K = 1), low-storage RK {time order 3, 3 stages}, CFL 0.99, FP64. A step is one RK step
(3 residual evaluations + update). Metric: cell-updates/s = inner cells x steps / device seconds.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference] [--n 128] [--precision fp64]
                  [--workload tgv|ramp]

--workload ramp measures the unstructured case instead: a compression ramp on an 80^3 jittered grid
split into tetrahedra, prisms, hexahedra and pyramid transitions (about 2.4 M cells), Euler, Mach 2.5,
ausmd flux, Barth-Jespersen limiter, supersonic inflow / outflow and slip walls, lserk {3,3}.

With --gpus N (launched by torchrun) every rank advances its own replica of the workload (the path is
one mesh per GPU; there is no exchange), timed on the device, max over ranks; `value` is the
whole-job throughput. `--impl reference` times the reference solver (compiled from its own C
sources) on the host cores: for tgv teal's own MPI domain decomposition of the full case, one rank
per core (oracle/_ref/teal_ref_mpi); for ramp, whose partitioner needs ParMETIS, one single-process
run per core on a sample mesh (an upper bound of the MPI run).
"""

import argparse
import json
import math
import os
import queue
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cell-updates/s"
WORKLOAD = "taylor-green vortex {n}^3 periodic hex, navier-stokes, roe + ls gradient + venkatakrishnan(1), lserk{{3,3}}, cfl 0.99"
RAMP_WORKLOAD = ("compression ramp {n}^3 jittered hex grid split into tetrahedra / prisms / hexahedra / pyramid "
                 "transitions, 15 deg ramp, Mach 2.5, euler, ausmd + ls gradient + barth-jespersen, "
                 "supersonic inflow / outflow + slip walls, lserk{{3,3}}, cfl 0.99")
M25 = (1.0, 2.5, 0.0, 0.0, 1.0 / 1.4)


def workload_name(workload, n):
    """Description of the tgv / ramp workload at n cells per axis (None: the default size)."""
    if workload == "tgv":
        return WORKLOAD.format(n=n or 128)
    return RAMP_WORKLOAD.format(n=n or 80)
RAMP_BCS = {"left": ("supersonic inflow", M25), "right": ("supersonic outflow", None),
            "bottom": ("slipwall", None), "top": ("slipwall", None), "back": ("slipwall", None),
            "front": ("slipwall", None)}


def tgv_state(center, gamma=1.4, mach=0.1):
    """Taylor-Green initial field (the reference's run/taylor_green_vortex/run.c:10-21)."""
    x, y, z = center[:, 0], center[:, 1], center[:, 2]
    p0 = 1 / (gamma * mach**2)
    out = np.zeros((center.shape[0], 5))
    out[:, 1] = np.sin(x) * np.cos(y) * np.cos(z)
    out[:, 2] = -np.cos(x) * np.sin(y) * np.cos(z)
    out[:, 4] = p0 + (np.cos(2 * x) + np.cos(2 * y)) * (np.cos(2 * z) + 2) / 16
    out[:, 0] = out[:, 4] / p0
    return out


def stage_bytes(C, F, ns=True, g=8):
    """Algorithmic HBM bytes of one residual stage (unique-footprint count): Euler 408 C + 184 F,
    Navier-Stokes + 88 C + 32 F with FP64 elements; with the FP32-flux form's 4-byte gradient and
    geometry elements (g = 4; the state, U0 and volumes stay FP64) 288 C + 96 F, + 48 C + 16 F."""
    # per cell: q read (gradient) 40 + gradient write 15 g + q read (face) 40 + gradient read 15 g +
    # U0 read 40 + q write 40 + V 8; per face: cells 8 + weights 6 g + area g + basis 9 g + offsets 6 g
    b = (168 + 30 * g) * C + (8 + 22 * g) * F
    if ns:
        # unlimited gradient kept via psi (5 g written, 5 g read), eps^2 8; correction 4 g
        b += (10 * g + 8) * C + 4 * g * F
    return b


def kernel_bytes(C, F, S, NB, ns=True, fold=False, g=8, basis=3):
    """Unique bytes each hot-path kernel of one stage must move in teal_b200's layout: g is the
    gradient / geometry / flux-record element size (8 in FP64, 4 in the FP32-flux form), basis the
    basis rows a face reads (3: the normal, the plain forms; 9 in the exact form)."""
    grad_state = (15 + (0 if fold else 5)) * g
    return {
        # q of cells and boundary ghosts, per slot: neighbour 4 + weight 3 g + offset 3 g; counts,
        # eps^2; writes gradient (+ limiter factors)
        "gradient": 40 * (C + NB) + (4 + 6 * g) * S + 9 * C + grad_state * C,
        # per face: cells 8, area, basis rows, offsets (+ correction), G write 5 g; per cell: q,
        # gradient (+ psi); ghost rows
        "face": (8 + (1 + basis + 6 + 5 + (4 if ns else 0)) * g) * F + (40 + grad_state) * C + 40 * NB,
        # slot face indices, G read once, U0, volume, q write (last stage adds R, U0, projection)
        "cell": 4 * S + 1 * C + 5 * g * F + (40 + 8 + 40) * C,
    }


def read_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    REASONS = {
        "sw_power_cap": "clocks_event_reasons.sw_power_cap",
        "hw_slowdown": "clocks_event_reasons.hw_slowdown",
        "hw_thermal_slowdown": "clocks_event_reasons.hw_thermal_slowdown",
        "sw_thermal_slowdown": "clocks_event_reasons.sw_thermal_slowdown",
    }

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []
        self.thread = None
        self.first = threading.Event()

    def start(self):
        """Start sampling every 100 ms and return once the first sample is in (at most 3 s), so the
        timed region that follows is covered from its start."""
        q = "clocks.sm,clocks.max.sm," + ",".join(self.REASONS.values())
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits", "-lms", "100",
                 "-i", str(self.index)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, ValueError):
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()
        self.first.wait(timeout=3.0)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())
            self.first.set()
        self.first.set()

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=5)
        sm, smax, reasons = [], [], set()
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 2 + len(self.REASONS):
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for name, val in zip(self.REASONS, parts[2:]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def max_over_ranks(x, pg):
    """The largest of every rank's x (each rank's device time): the whole job ends with its slowest
    replica. Tensors live on the GPU for NCCL and on the host for gloo."""
    if pg is None:
        return float(x)
    import torch

    dev = "cuda" if pg.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(cells_per_rank, steps, world, seconds):
    """Cell updates per second of all replicas together (weak scaling: each rank advances its own
    mesh of cells_per_rank cells for the same steps; the job takes the slowest rank's time)."""
    return cells_per_rank * steps * world / seconds


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def ramp_state(center):
    return np.tile(np.array(M25), (center.shape[0], 1))


def configure(eqns, workload):
    """The plugin settings of a workload on teal_b200 or reference equations (same setter names)."""
    if workload == "tgv":
        eqns.set_convective_flux("roe")
        eqns.set_limiter("venkatakrishnan", 1.0)
        eqns.set_property("dynamic viscosity", 1 / 1600)
    else:
        eqns.set_convective_flux("ausmd")
        eqns.set_limiter("minmod", 0.0)
        for entity, (name, ctx) in RAMP_BCS.items():
            eqns.set_boundary_condition(entity, name, ctx)


def reference_cpu(n, steps, warmup=0, workload="tgv"):
    """Time the reference solver's own lserk step (oracle/_ref, one core) on the workload at mesh size
    n (TGV n^3; ramp n^3 grid cells before splitting). Returns (cell-updates/s, seconds, steps)."""
    from oracle import ref

    if workload == "tgv":
        m = ref.RefMesh((0, 0, 0), (2 * math.pi,) * 3, (n, n, n), (1, 1, 1))
        e = ref.RefEquations(m, navierstokes=True)
        init = tgv_state
    else:
        from teal_b200 import meshes

        m = ref.RefMesh.from_cells(meshes.ramp_mesh(n=(n, n, n)))
        e = ref.RefEquations(m, navierstokes=False)
        init = ramp_state
    configure(e, workload)
    c = m.arrays()["cells.center"]
    e.set_primitive(init(c))
    sim = ref.RefSimulation(e, "lserk", 0.99, rk=(3, 3))
    t = 0.0
    for _ in range(warmup):
        t, _, _ = sim.advance(t)
    t0 = time.perf_counter()
    for _ in range(steps):
        t, _, _ = sim.advance(t)
    dt = time.perf_counter() - t0
    C = e.num_inner
    return C * steps / dt, dt, steps


def _reference_process(n, steps, workload, barrier, out):
    """One host core's share of the all-core reference sample: build, warm up, wait for the others,
    time `steps` lserk steps."""
    try:
        from oracle import ref

        if workload == "tgv":
            m = ref.RefMesh((0, 0, 0), (2 * math.pi,) * 3, (n, n, n), (1, 1, 1))
            e = ref.RefEquations(m, navierstokes=True)
            init = tgv_state
        else:
            from teal_b200 import meshes

            m = ref.RefMesh.from_cells(meshes.ramp_mesh(n=(n, n, n)))
            e = ref.RefEquations(m, navierstokes=False)
            init = ramp_state
        configure(e, workload)
        e.set_primitive(init(m.arrays()["cells.center"]))
        sim = ref.RefSimulation(e, "lserk", 0.99, rk=(3, 3))
        t, _, _ = sim.advance(0.0)
        barrier.wait(timeout=900)
        t0 = time.perf_counter()
        for _ in range(steps):
            t, _, _ = sim.advance(t)
        out.put((e.num_inner, steps, time.perf_counter() - t0))
    except Exception as exc:  # reported by the parent
        out.put(("error", str(exc), 0.0))


def reference_cpu_all(n, steps, workload="tgv", procs=None):
    """All host cores at once: one single-process reference run per core (spawned processes, each
    on its own n^3 mesh), timed together. Returns (aggregate cell-updates/s, wall seconds, steps,
    processes). Without halo exchange this bounds teal's MPI run on the same cores from above."""
    import multiprocessing as mp

    procs = procs or min(len(os.sched_getaffinity(0)), 128)
    ctx = mp.get_context("spawn")
    barrier = ctx.Barrier(procs)
    out = ctx.Queue()
    ps = [ctx.Process(target=_reference_process, args=(n, steps, workload, barrier, out)) for _ in range(procs)]
    for p in ps:
        p.start()
    res, deadline = [], time.perf_counter() + 1800
    while len(res) < procs:
        try:
            res.append(out.get(timeout=5))
        except queue.Empty:
            dead = any(p.exitcode not in (None, 0) for p in ps)
            if dead or time.perf_counter() > deadline:
                for p in ps:
                    p.terminate()
                raise RuntimeError("a reference process failed or did not finish")
    for p in ps:
        p.join(timeout=60)
    errors = [r[1] for r in res if r[0] == "error"]
    if errors:
        raise RuntimeError(errors[0])
    wall = max(r[2] for r in res)
    return sum(r[0] * r[1] for r in res) / wall, wall, steps, procs


MPI_RUN = os.path.join(ROOT, "oracle", "_ref", "teal_ref_mpi")


def reference_mpi(n, steps, warmup=2, ranks=None):
    """teal's own domain-decomposed Taylor-Green run on all host cores (oracle/_ref/teal_ref_mpi: the
    reference's mesh_create split, halo exchanges and reductions over a fork / shared-memory MPI
    subset), n^3 cells, `steps` timed lserk steps after `warmup`. Returns (cell-updates/s, seconds of
    the slowest rank, steps, ranks)."""
    ranks = ranks or min(len(os.sched_getaffinity(0)), 1024)
    env = dict(os.environ, TEAL_SHIM_RANKS=str(ranks), TEAL_SHIM_TIMEOUT="900")
    r = subprocess.run([MPI_RUN, "--n", str(n), "--steps", str(steps), "--warmup", str(warmup)],
                       capture_output=True, text=True, env=env, timeout=1800)
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    if r.returncode != 0 or not lines:
        raise RuntimeError(f"teal_ref_mpi failed ({r.returncode}): {r.stderr[-500:]}")
    out = json.loads(lines[-1])
    return out["cells"] * out["steps"] / out["seconds"], out["seconds"], out["steps"], out["ranks"]


def mpi_sample(steps, warmup, ranks, n=128):
    return (f"teal's own MPI run of the full {n}^3 case (mesh_create domain decomposition, halo "
            f"exchanges, global reductions) on {ranks} ranks, one per host core, over a fork / "
            f"shared-memory MPI subset: {steps} lserk steps after {warmup} warm-up steps, slowest rank")


def run_split(args, world, rank, pg):
    """The Taylor-Green 128^3 workload as ONE mesh over all ranks (strong scaling): teal's grid of
    ranks and block split (src/mesh/create.c:10-97), or with --workload ramp the unstructured ramp
    split by recursive coordinate bisection, each GPU a partition with a one-cell halo;
    per RK stage the states and then the gradient records of the halo cross between GPUs (NCCL
    grouped send / receive on the ranks' streams), the step minimum and the residual sums by
    all-reduce. The state after each step equals the single-mesh run's (tests/test_partition_gpu.py).
    value = cells of the whole mesh x steps / device time of the slowest rank."""
    import torch

    import teal_b200 as tb
    from teal_b200 import partition as pt

    ramp = args.workload == "ramp"
    n = args.n or (80 if ramp else 128)
    t0 = time.perf_counter()
    if ramp:
        # unstructured: split by recursive coordinate bisection (teal's ParMETIS split is not available)
        from teal_b200 import meshes

        mesh = tb.Mesh.from_cells(meshes.ramp_mesh(n=(n, n, n)))
        eqns = tb.Equations.euler(mesh)
        configure(eqns, "ramp")
        ranks = pt.bisection_ranks(mesh, world)
        dims = "recursive coordinate bisection"
        prim = ramp_state(mesh.cell_center[: mesh.num_inner_cells])
    else:
        lo, hi, nc = (0, 0, 0), (2 * math.pi,) * 3, (n, n, n)
        mesh = tb.Mesh.create(lo, hi, nc, (1, 1, 1))
        eqns = tb.Equations.navierstokes(mesh)
        configure(eqns, "tgv")
        ranks, dims = pt.cell_ranks(mesh, lo, hi, nc, world)
        prim = tgv_state(mesh.cell_center[: mesh.num_inner_cells])
    part = pt.partition(mesh, ranks)[rank]
    run = pt.DistributedRun(part, eqns, world)
    run.rank.set_state(prim)
    t_setup = time.perf_counter() - t0
    t = 0.0
    for _ in range(args.warmup):
        t, s0, res = run.step(t, 0.99)
    stream = run.rank.stream
    torch.cuda.synchronize()
    pg.barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        t, s0, res = run.step(t, 0.99)
    ev1.record(stream)
    torch.cuda.synchronize()
    pg.barrier()
    ms = max_over_ranks(ev0.elapsed_time(ev1), pg)
    C = mesh.num_inner_cells
    line = {
        "metric": METRIC, "value": C * args.steps / (ms / 1000.0), "unit": "cell-updates/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": workload_name("ramp" if ramp else "tgv", n), "cells": C, "mesh": f"{n}^3",
                   "global_batch": 1,
                   "parallelism": f"one mesh split over {world} gpus ({dims if ramp else f'rank grid {dims}'}, "
                                  "one-cell halo)",
                   "halo_cells_rank0": int(len(part.halo))},
        "residual": [float(x) for x in res], "setup_s": t_setup,
    }
    run.close()
    if rank == 0:
        print(json.dumps(line))
    pg.barrier()
    pg.destroy_process_group()


def run_serving(args, world, rank):
    """Serving benchmark (the continuous-batching solve server): seeded Poisson arrivals of steady solve requests on
    the batch workload's ramp meshes (20k-2M cells, log-uniform), Mach 0.2-3.0, Euler or
    Navier-Stokes, flux scheme (roe / hllc / ausmd) and tolerance 1e-6..1e-10 per request, implicit
    Euler with teal's steady Newton-Krylov settings; served with continuous batching (lanes of one
    scheme sharing an arena, requests joining and leaving between rounds, admission by HBM budget),
    against the same requests solved one at a time in arrival order (first in, first out). Each
    latency runs from arrival to result on the host (mesh generation, upload, solve, read-back)."""
    import dataclasses

    import torch

    import teal_b200 as tb
    from teal_b200 import serving

    if rank != 0:
        return
    torch.cuda.set_device(0)
    reqs = serving.poisson_requests(args.requests, rate=args.rate, seed=7, steps=(10, 40), mesh="ramp",
                                    physics=(tb.TG_EULER, tb.TG_NAVIERSTOKES), method="implicit euler",
                                    courant=10.0)
    # warm-up: one small solve (library load, graph capture paths)
    serving.solve(serving.Request(id=-1, cells=(64, 32, 2), steps=5))
    torch.cuda.synchronize()

    server = serving.Server(max_active=args.max_active, chunk=5)
    sampler = ClockSampler(0)
    sampler.start()
    t0 = time.perf_counter()
    done = server.serve([dataclasses.replace(r) for r in reqs], timeout=1800)
    served_s = time.perf_counter() - t0
    clocks = sampler.stop()
    errors = {r.id: r.error for r in done if r.error}
    lat = [r.latency for r in done if not r.error]
    work = sum(r.num_cells * r.iterations for r in done if not r.error)
    stopped_by_tolerance = sum(1 for r in done if not r.error and r.iterations < r.steps)

    # one at a time: solve durations measured alone, queued first in, first out at the same arrivals
    durations = []
    for r in reqs:
        solo = dataclasses.replace(r)
        a = time.perf_counter()
        try:
            serving.solve(solo)
        except Exception:  # a request that fails alone fails in the server too
            pass
        durations.append(time.perf_counter() - a)
    finish, fifo_lat = 0.0, []
    for r, d in zip(reqs, durations):
        start = max(r.arrival, finish)
        finish = start + d
        fifo_lat.append(finish - r.arrival)
    seq_s = finish - reqs[0].arrival
    ok = [i for i, r in enumerate(done) if not r.error]
    line = {
        "metric": "serving: p50/p99 solve latency and aggregate cell-updates/s", "value": work / served_s,
        "unit": "cell-updates/s", "n_gpus": 1, "steps": len(reqs), "warmup": 1,
        "ms_per_step": 1000 * served_s / len(reqs), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"{len(reqs)} poisson requests at {args.rate}/s, ramp meshes 20k-2M cells, "
                               "mach 0.2-3.0, euler or navier-stokes, roe/hllc/ausmd + venkatakrishnan(1), "
                               "tolerance 1e-6..1e-10, 10-40 implicit euler steps cfl 10, newton-krylov "
                               "{0.1, 0.3, 30}, continuous batching in lanes of one scheme",
                   "max_active": args.max_active, "budget_bytes": server.budget, "round_steps": server.chunk},
        "latency_p50_s": serving.percentile(lat, 50), "latency_p99_s": serving.percentile(lat, 99),
        "makespan_s": served_s, "peak_active": server.peak_active, "lanes": len(server.lanes),
        "arena_repacks": server.repacks, "arena_repack_s": server.repack_s,
        "stopped_by_tolerance": stopped_by_tolerance, "errors": errors,
        "one_at_a_time": {"value": work / sum(durations[i] for i in ok) if ok else None,
                          "latency_p50_s": serving.percentile(fifo_lat, 50),
                          "latency_p99_s": serving.percentile(fifo_lat, 99), "makespan_s": seq_s},
        "clocks": clocks,
    }
    print(json.dumps(line))


def batch_specs(count, seed=11, lo=8_000, hi=512_000):
    """Instances of the batched workload: ramp-mesh sizes log-uniform in [lo, hi] cells, Mach
    U(0.3, 3.0), flow angle U(0, 10) degrees, a mesh seed each."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        cells = math.exp(rng.uniform(math.log(lo), math.log(hi)))
        n = max(8, int(round((cells / 4.64) ** (1.0 / 3.0))))  # the ramp grid holds ~4.64 cells per hex
        out.append((n, float(rng.uniform(0.3, 3.0)), float(rng.uniform(0.0, 10.0)), 1000 * seed + i))
    return out


def batch_problem(spec, flux="ausmd", limiter=("minmod", 0.0)):
    """Euler on a mixed-element ramp mesh, far field around, slip walls at the ramp and the sides
    (valid for subsonic and supersonic free streams), starting from the free stream."""
    import teal_b200 as tb
    from teal_b200 import meshes, serving

    n, mach, angle, mseed = spec
    m = tb.Mesh.from_cells(meshes.ramp_mesh(n=(n, n, n), seed=mseed))
    e = tb.Equations.euler(m)
    e.set_convective_flux(flux)
    e.set_limiter(*limiter)
    free = serving.free_stream(mach, angle)
    for side in ("left", "right", "top"):
        e.set_boundary_condition(side, "farfield", free)
    for side in ("bottom", "back", "front"):
        e.set_boundary_condition(side, "slipwall")
    e.primitive[:] = np.tile(free, (m.num_cells, 1))
    return e


def run_batch_implicit(args, specs):
    """Batched steady solves on `--instances` ramp meshes of 8k-512k cells: every instance takes
    implicit Euler steps until its maximum residual has dropped by `--drop` (1e-8) from its first
    step's, or `--steps` steps, in FP64 and in the FP32-matvec form (FP64 Newton residuals and Arnoldi, FP32 fluxes in the
    finite-difference matvec); all instances in one arena, each step one CUDA-graph launch with
    device-driven Newton / Arnoldi / Gram-Schmidt loops. The scheme is teal's steady airfoil case's
    (run/airfoil/run.c: hllc, Venkatakrishnan(1), Newton-Krylov {0.1, 0.3, 30}) at CFL 30: from the
    uniform start CFL 100 ends in non-finite residuals in the first step on some instances, and with
    teal's global time step (the minimum over a mesh's cells) the drop per step is slow on these
    mixed meshes, so the run reports how far each instance got. cell-updates/s = sum over instances
    of cells x steps taken / device time."""
    import torch

    import teal_b200 as tb

    t0 = time.perf_counter()
    problems = [batch_problem(sp, flux="hllc", limiter=("venkatakrishnan", 1.0)) for sp in specs]
    t_setup = time.perf_counter() - t0
    method = tb.TG_ADVANCE_IMPLICIT_EULER
    courant = args.courant if args.courant else 30.0
    context = (0.1, 0.3, 30)
    n = len(problems)
    cells = np.array([e.mesh.num_inner_cells for e in problems], dtype=np.float64)
    stream = torch.cuda.Stream()
    out, states = {}, {}
    for name, prec in (("fp64", tb.TG_PRECISION_FP64), ("fp32_matvec", tb.TG_PRECISION_FP32_FLUX)):
        b = tb.Batch(problems, precision=prec)
        b.set_stream(stream.cuda_stream)
        torch.cuda.synchronize()
        # the first step sets each instance's reference residual (and captures the step graph)
        t, it, res = b.run(method, courant, 1, context=context)
        first = res.max(axis=1)
        thr = np.where(first > 0, args.drop * first, 0.0)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        ev0.record(stream)
        t, it, res = b.run(method, courant, args.steps, variable=-1, threshold=thr, context=context, time=t)
        ev1.record(stream)
        torch.cuda.synchronize()
        secs = ev0.elapsed_time(ev1) / 1000.0
        steps = it.astype(np.float64)
        failed = b.status() != 0  # instances that went non-finite stopped alone
        drop = np.where(failed, np.inf, res.max(axis=1) / np.maximum(first, 1e-300))
        out[name] = {"value": float((cells * steps).sum() / secs), "seconds": secs,
                     "converged": int((drop <= args.drop).sum()), "instances": n, "failed": int(failed.sum()),
                     "steps_taken_max": int(steps.max()),
                     "drop_p50": float(np.percentile(drop[~failed], 50)) if (~failed).any() else None,
                     "drop_max": float(drop[~failed].max()) if (~failed).any() else None,
                     "drop_min": float(drop[~failed].min()) if (~failed).any() else None}
        states[name] = [None if failed[i] else b.get_primitive(i)[: e.mesh.num_inner_cells].copy()
                        for i, e in enumerate(problems)]
        b.close()
    err_var = np.zeros(5)
    for a, f in zip(states["fp64"], states["fp32_matvec"]):
        if a is None or f is None:
            continue
        d = np.sqrt(((f - a) ** 2).sum(axis=0)) / np.maximum(np.sqrt((a ** 2).sum(axis=0)), 1e-300)
        err_var = np.maximum(err_var, d)
    steps_max = max(1, out["fp32_matvec"]["steps_taken_max"])
    line = {
        "metric": "cell-updates/s batched implicit steady solves (FP32-matvec / FP64 Newton-Arnoldi)",
        "value": out["fp32_matvec"]["value"], "unit": "cell-updates/s", "n_gpus": 1, "steps": args.steps,
        "warmup": 1, "ms_per_step": 1000 * out["fp32_matvec"]["seconds"] / steps_max,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32-matvec-flux/f64-newton-arnoldi", "data": "synthetic",
        "config": {"workload": f"{n} euler ramp meshes (tets/prisms/hexes/pyramids), 8k-512k cells log-uniform, "
                               f"mach 0.3-3.0, angle 0-10 deg, hllc + venkatakrishnan(1), farfield + slip walls, "
                               f"implicit euler cfl {courant:g}, newton-krylov {{0.1, 0.3, 30}}, until a "
                               f"{args.drop:g} relative residual drop or {args.steps} steps",
                   "cells": int(cells.sum()), "instances": n},
        "fp64": out["fp64"], "fp32_matvec": out["fp32_matvec"],
        "fp32_matvec_over_fp64": out["fp32_matvec"]["value"] / out["fp64"]["value"],
        "fp32_matvec_rel_l2_vs_fp64_per_primitive": err_var.tolist(),
        "setup_s": t_setup,
    }
    print(json.dumps(line))


def run_batch(args, world, rank):
    """Batched forms: many ramp meshes of uneven size in one arena, advanced together (lserk, or
    implicit Euler with Newton-GMRES), in FP64 and in the FP32-flux form, against the same meshes
    solved one at a time in FP64. Reports throughput of each and the FP32-flux error against FP64."""
    import torch

    import teal_b200 as tb

    if rank != 0:
        return
    torch.cuda.set_device(0)
    specs = batch_specs(args.instances)
    if args.method == "implicit" and args.drop > 0:
        return run_batch_implicit(args, specs)
    t0 = time.perf_counter()
    problems = [batch_problem(sp) for sp in specs]
    t_setup = time.perf_counter() - t0
    cells = sum(e.mesh.num_inner_cells for e in problems)
    implicit = args.method == "implicit"
    method = tb.TG_ADVANCE_IMPLICIT_EULER if implicit else tb.TG_ADVANCE_LSERK
    # implicit: CFL 10; from the uniform start at CFL 100 the reference's own first step already
    # ends in non-finite residuals on some instances of this draw
    courant = 10.0 if implicit else 0.9
    context = (0.1, 0.3, 30) if implicit else (3, 3)
    steps = args.steps
    stream = torch.cuda.Stream()

    def timed(run):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(stream)
        run()
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b) / 1000.0

    out, states = {}, {}
    for name, prec in (("fp64", tb.TG_PRECISION_FP64), ("fp32_flux", tb.TG_PRECISION_FP32_FLUX)):
        b = tb.Batch(problems, precision=prec)
        b.set_stream(stream.cuda_stream)
        b.run(method, courant, min(args.warmup, 3) if not implicit else 1, context=context)
        for i, e in enumerate(problems):
            b.set_primitive(i, e.primitive)
        secs = timed(lambda: b.run(method, courant, steps, context=context))
        out[name] = {"value": cells * steps / secs, "seconds": secs}
        states[name] = [b.get_primitive(i)[: e.mesh.num_inner_cells].copy() for i, e in enumerate(problems)]
        b.close()
    # error of the FP32-flux form against FP64: relative L2 per conserved variable (the max over
    # instances), and over all five together
    def conserved(p, gamma=1.4):
        rho, u, pr = p[:, 0], p[:, 1:4], p[:, 4]
        return np.column_stack([rho, rho[:, None] * u, pr / (gamma - 1) + 0.5 * rho * (u ** 2).sum(axis=1)])

    err_var = np.zeros(5)
    err_mom = np.zeros(3)
    err_all = 0.0
    for a, f in zip(states["fp64"], states["fp32_flux"]):
        ua, uf = conserved(a), conserved(f)
        d = np.sqrt(((uf - ua) ** 2).sum(axis=0)) / np.maximum(np.sqrt((ua ** 2).sum(axis=0)), 1e-300)
        err_var = np.maximum(err_var, d)
        # momentum components against the norm of the whole momentum vector: a component that is
        # nearly zero in these flows (rho w, no cross flow) is measured on the scale FP32 rounds at
        mom = np.sqrt((ua[:, 1:4] ** 2).sum())
        err_mom = np.maximum(err_mom, np.sqrt(((uf[:, 1:4] - ua[:, 1:4]) ** 2).sum(axis=0)) / max(mom, 1e-300))
        err_all = max(err_all, float(np.sqrt(((uf - ua) ** 2).sum()) / np.sqrt((ua ** 2).sum())))

    # the same meshes one at a time in FP64 (a sample of them, throughput summed)
    sample = problems[: min(len(problems), args.solo_sample)]
    solo_cells, solo_secs = 0, 0.0
    for e in sample:
        ctx = tb.Context(e.mesh, e)
        ctx.set_stream(stream.cuda_stream)
        ctx.set_primitive(e.primitive)
        ctx.run(method, courant, 1, context=context)
        ctx.set_primitive(e.primitive)
        solo_secs += timed(lambda: ctx.run(method, courant, steps, context=context))
        solo_cells += e.mesh.num_inner_cells * steps
        ctx.close()
    solo = solo_cells / solo_secs
    line = {
        "metric": "cell-updates/s batched FP32-flux/FP64-accumulate vs plain FP64", "value": out["fp32_flux"]["value"],
        "unit": "cell-updates/s", "n_gpus": 1, "steps": steps, "warmup": args.warmup,
        "ms_per_step": 1000 * out["fp32_flux"]["seconds"] / steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32-flux/f64-accumulate", "data": "synthetic",
        "config": {"workload": f"{len(problems)} euler ramp meshes (tets/prisms/hexes/pyramids), 8k-512k cells "
                               f"log-uniform, mach 0.3-3.0, angle 0-10 deg, ausmd + barth-jespersen, "
                               + ("implicit euler cfl 10, newton-krylov {0.1, 0.3, 30}" if implicit
                                  else "lserk{3,3} cfl 0.9"),
                   "cells": cells, "instances": len(problems)},
        "batched_fp64": out["fp64"]["value"], "batched_fp32_flux": out["fp32_flux"]["value"],
        "solo_fp64": solo, "solo_sample": len(sample),
        "fp32_flux_over_batched_fp64": out["fp32_flux"]["value"] / out["fp64"]["value"],
        "fp32_flux_over_solo_fp64": out["fp32_flux"]["value"] / solo,
        "fp32_flux_rel_l2_vs_fp64": err_all, "fp32_flux_rel_l2_per_conserved": err_var.tolist(),
        "fp32_flux_momentum_rel_l2_vs_momentum_norm": err_mom.tolist(),
        "setup_s": t_setup,
    }
    print(json.dumps(line))


def run_reference_arm(args, world, rank):
    if rank != 0:
        return
    from oracle import ref

    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "reference library oracle/_ref not built"}))
        return
    if args.workload == "tgv" and os.path.exists(MPI_RUN):
        value, secs, steps, procs = reference_mpi(args.n, args.steps, args.warmup)
        sample = mpi_sample(steps, args.warmup, procs, args.n)
        config_extra = {"mesh": f"{args.n}^3", "parallelism": f"{procs} MPI ranks"}
    else:
        n_sample = args.ref_n
        value, secs, steps, procs = reference_cpu_all(n_sample, args.steps, workload=args.workload)
        sample = (f"{procs} single-process reference runs at once (one per host core), each {steps} lserk "
                  f"steps of the same case on a {n_sample}^3 mesh; no halo exchange, so an upper bound of "
                  "the all-core MPI run")
        config_extra = {"sample_mesh": f"{n_sample}^3 per core", "parallelism": f"{procs} cores"}
    line = {
        "metric": METRIC, "value": value, "unit": "cell-updates/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000 * secs / steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": dict({"workload": workload_name(args.workload, None)}, **config_extra),
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": "cell-updates/s", "cores": procs, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": value, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="teal_b200")
    ap.add_argument("--workload", default="tgv", choices=["tgv", "ramp", "serve", "batch"],
                    help="tgv: Taylor-Green 128^3 (the headline); ramp: the unstructured compression ramp; "
                         "serve: the solve server under Poisson arrivals; batch: many meshes in one arena")
    ap.add_argument("--instances", type=int, default=64, help="batch: meshes in the arena")
    ap.add_argument("--method", default="lserk", choices=["lserk", "implicit"], help="batch: time integrator")
    ap.add_argument("--drop", type=float, default=1e-8,
                    help="batch implicit: run each instance to this relative residual drop (0: fixed --steps)")
    ap.add_argument("--courant", type=float, default=None, help="batch implicit: CFL number (default 30)")
    ap.add_argument("--solo-sample", type=int, default=16, help="batch: meshes timed one at a time")
    ap.add_argument("--requests", type=int, default=32, help="serve: number of requests")
    ap.add_argument("--rate", type=float, default=8.0, help="serve: arrivals per second")
    ap.add_argument("--max-active", type=int, default=64, help="serve: requests resident at once")
    ap.add_argument("--n", type=int, default=None, help="mesh cells per axis (tgv 128, ramp 80)")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32", "exact"],
                    help="fp64: plain FP64; fp32: FP32-flux form; exact: FP64 with teal's exact arithmetic")
    ap.add_argument("--ref-n", type=int, default=None, help="mesh size of the CPU reference sample (tgv 48, ramp 32)")
    ap.add_argument("--ref-steps", type=int, default=None,
                    help="steps of the CPU baseline sample (tgv: the all-core MPI run, 10; ramp: 20)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--split", action="store_true",
                    help="tgv with --gpus N: one mesh split over the N GPUs (teal's rank grid, one-cell halo, "
                         "strong scaling) instead of N independent replicas")
    args = ap.parse_args()
    if args.n is None:
        args.n = 128 if args.workload == "tgv" else 80
    if args.ref_n is None:
        args.ref_n = 48 if args.workload == "tgv" else 32
    if args.ref_steps is None:
        args.ref_steps = 10 if args.workload == "tgv" else 20
    args.warmup = max(args.warmup, 3)
    world, rank, local = dist_setup()

    if args.impl == "reference":
        run_reference_arm(args, world, rank)
        return
    if args.workload == "serve":
        run_serving(args, world, rank)
        return
    if args.workload == "batch":
        run_batch(args, world, rank)
        return

    import torch

    torch.cuda.set_device(local)
    pg = None
    if world > 1 or args.split:
        import datetime

        import torch.distributed as dist

        if not dist.is_initialized():
            os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
            os.environ.setdefault("MASTER_PORT", "29511")
            dist.init_process_group("nccl", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=300))
        pg = dist
    if args.split:
        run_split(args, world, rank, pg)
        return

    import teal_b200 as tb

    n = args.n
    ns = args.workload == "tgv"
    t0 = time.perf_counter()
    if ns:
        mesh = tb.Mesh.create((0, 0, 0), (2 * math.pi,) * 3, (n, n, n), (1, 1, 1))
        eqns = tb.Equations.navierstokes(mesh)
    else:
        from teal_b200 import meshes

        cells = meshes.ramp_mesh(n=(n, n, n))
        mesh = tb.Mesh.from_cells(cells)
        eqns = tb.Equations.euler(mesh)
    t_mesh = time.perf_counter() - t0
    configure(eqns, args.workload)
    eqns.set_initial_condition("domain", tgv_state if ns else ramp_state)
    precision = {"fp64": tb.TG_PRECISION_FP64, "fp32": tb.TG_PRECISION_FP32_FLUX,
                 "exact": tb.TG_PRECISION_FP64_EXACT}[args.precision]
    t0 = time.perf_counter()
    ctx = eqns.context(precision)
    t_upload = time.perf_counter() - t0
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    LSERK = tb.TG_ADVANCE_LSERK
    rk = (3, 3)
    C = mesh.num_inner_cells
    F = mesh.num_faces
    s = mesh.struct
    NB = s.off_boundary_cells - C
    S = 2 * s.num_inner_faces + (F - s.num_inner_faces)

    # warm-up (graph capture happens here)
    ctx.run(LSERK, 0.99, args.warmup, context=rk)
    torch.cuda.synchronize()

    # timed region: K steps replayed from the step's CUDA graph, state resident in HBM
    sampler = ClockSampler(local)
    sampler.start()
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    launches0 = ctx.launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    ctx.run(LSERK, 0.99, args.steps, context=rk)
    ev1.record(stream)
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    clocks = sampler.stop()
    launches = ctx.launch_count() - launches0
    ms = max_over_ranks(ev0.elapsed_time(ev1), pg)
    value = whole_job_rate(C, args.steps, world, ms / 1000.0)

    # per-kernel CUDA-event timing of the same steps (plain launches, events on the same stream)
    ksteps = min(args.steps, 5)
    ctx.profile(True)
    ctx.run(LSERK, 0.99, ksteps, context=rk)
    prof = ctx.profile_read()
    ctx.profile(False)

    # end to end through the public API: every step uploads the state from pinned host memory,
    # advances one step and reads the state and residual back, in one call whose download overlaps
    # the step's last stage (tg_advance_host, the work of the drop-in Advance); beside it the same
    # steps as three calls in sequence (tg_set_primitive, tg_advance, tg_get_primitive)
    e2e_steps = min(args.steps, 10)
    host_in = torch.empty((mesh.num_cells, 5), dtype=torch.float64, pin_memory=True).numpy()
    host_out = torch.empty((mesh.num_cells, 5), dtype=torch.float64, pin_memory=True).numpy()
    start_state = ctx.get_primitive()

    def e2e_run(overlap):
        nonlocal host_in, host_out
        # one untimed call first (the overlapped call builds its chunk plan on first use)
        host_in[:] = start_state
        if overlap:
            ctx.advance_host(LSERK, 0.99, 0.0, prim_in=host_in, prim_out=host_out, context=rk)
        else:
            ctx.set_primitive(host_in)
            ctx.advance(LSERK, 0.99, 0.0, context=rk)
            ctx.get_primitive(host_out)
        host_in[:] = start_state
        torch.cuda.synchronize()
        if pg:
            pg.barrier()
        t0 = time.perf_counter()
        tt = 0.0
        for _ in range(e2e_steps):
            if overlap:
                tt, _, _ = ctx.advance_host(LSERK, 0.99, tt, prim_in=host_in, prim_out=host_out, context=rk)
            else:
                ctx.set_primitive(host_in)
                tt, _, _ = ctx.advance(LSERK, 0.99, tt, context=rk)
                ctx.get_primitive(host_out)
            host_in, host_out = host_out, host_in
        return max_over_ranks(time.perf_counter() - t0, pg)

    e2e_seq_s = e2e_run(False)
    e2e_s = e2e_run(True)
    e2e_value = whole_job_rate(C, e2e_steps, world, e2e_s)
    e2e_seq_value = whole_job_rate(C, e2e_steps, world, e2e_seq_s)

    # the exact FP64 form (teal's arithmetic, bit-identical results) on the same workload: its rate
    # beside the plain form's, from the same state, timed the same way
    exact_form = None
    if args.precision == "fp64":
        xctx = eqns.context(tb.TG_PRECISION_FP64_EXACT)
        xctx.set_stream(stream.cuda_stream)
        xctx.set_primitive(ctx.get_primitive())
        xsteps = min(args.steps, 10)
        xctx.run(LSERK, 0.99, 2, context=rk)
        torch.cuda.synchronize()
        if pg:
            pg.barrier()
        ev0.record(stream)
        xctx.run(LSERK, 0.99, xsteps, context=rk)
        ev1.record(stream)
        torch.cuda.synchronize()
        xms = max_over_ranks(ev0.elapsed_time(ev1), pg)
        xval = whole_job_rate(C, xsteps, world, xms / 1000.0)
        exact_form = {"value": xval, "unit": "cell-updates/s", "ms_per_step": xms / xsteps, "steps": xsteps,
                      "plain_over_exact": value / xval,
                      "parity": "bit-identical to the reference's residual and explicit steps"}
        xctx.close()
        eqns._ctx.pop(tb.TG_PRECISION_FP64_EXACT, None)

    # roofline of one RK stage (boundary + gradient + face + cell kernels)
    peak, peak_kind = read_peaks()
    stages = ksteps * rk[1]
    stage_ms = sum(prof[k][0] for k in ("boundary", "gradient", "face", "cell")) / stages
    g = 4 if args.precision == "fp32" else 8  # gradient / geometry / flux-record element size
    b_stage = stage_bytes(C, F, ns=ns, g=g)
    achieved = b_stage / (stage_ms / 1000.0) / 1e9
    kb = kernel_bytes(C, F, S, NB, ns=ns, fold=not ns, g=g, basis=9 if args.precision == "exact" else 3)
    kernels = {}
    for k in ("gradient", "face", "cell"):
        kms, kn = prof[k]
        if kn:
            avg = kms / kn
            kernels[k] = {"avg_ms": avg, "launches": kn, "unique_bytes": kb[k],
                          "gbs": kb[k] / (avg / 1000.0) / 1e9, "share": kms / max(1e-9, sum(v[0] for v in prof.values()))}
    dominant = max(kernels, key=lambda k: kernels[k]["avg_ms"] * kernels[k]["launches"]) if kernels else None

    traffic = None
    tpath = os.path.join(ROOT, "profiles", "stage_traffic.json")
    if ns and args.precision == "fp64" and os.path.exists(tpath):  # measured for the plain FP64 form
        with open(tpath) as f:
            tr = json.load(f)
        if tr.get("n") and tr.get("bytes_per_stage"):
            traffic = tr["bytes_per_stage"] * (C / (tr["n"] ** 3))

    line = {
        "metric": METRIC, "value": value, "unit": "cell-updates/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32-flux/f64-accumulate" if args.precision == "fp32" else "f64",
        "data": "synthetic",
        "config": {"workload": workload_name("tgv" if ns else "ramp", n), "cells": C, "faces": F, "mesh": f"{n}^3",
                   "global_batch": world, "parallelism": f"replicas x{world}" if world > 1 else "1 gpu",
                   "l2": f"inputs larger than L2 (state + geometry ~{b_stage / 1e9:.1f} GB per stage)"},
        "roofline": {"bound": "hbm", "kernel": "rk stage (boundary+gradient+face+cell)", "achieved": achieved,
                     "peak": peak, "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                     "peak_kind": peak_kind, "algorithmic_bytes_per_launch": b_stage,
                     "avg_launch_ms": stage_ms},
        "kernels": kernels, "dominant_kernel": dominant,
        "clocks": clocks,
        "e2e": {"value": e2e_value, "unit": "cell-updates/s", "h2d_bytes_per_step": host_in[: C].nbytes,
                "d2h_bytes_per_step": host_out.nbytes + 5 * 8, "steps": e2e_steps,
                "api": "tg_advance_host (download overlapped with the last stage)",
                "sequential_calls_value": e2e_seq_value},
        "gpu_launches": launches,
        "setup_s": {"mesh": t_mesh, "upload": t_upload},
    }
    if exact_form:
        line["exact_form"] = exact_form

    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            from oracle import ref

            if args.workload == "tgv" and os.path.exists(MPI_RUN):
                v, secs, st, procs = reference_mpi(args.n, args.ref_steps, 2)
                line["cpu_baseline"] = {"value": v, "unit": "cell-updates/s", "cores": procs, "kind": "reference",
                                        "sample": mpi_sample(st, 2, procs, args.n) + f" ({secs:.1f} s)"}
            elif ref.available():
                v, secs, st, procs = reference_cpu_all(args.ref_n, args.ref_steps, workload=args.workload)
                line["cpu_baseline"] = {"value": v, "unit": "cell-updates/s", "cores": procs, "kind": "reference",
                                        "sample": f"{procs} single-process reference runs at once (one per host "
                                                  f"core), each {st} lserk steps of the same case on a "
                                                  f"{args.ref_n}^3 mesh ({secs:.1f} s); no halo exchange, so an "
                                                  "upper bound of the all-core MPI run"}
        except Exception as exc:  # the baseline is reported, never required
            line["cpu_baseline"] = {"error": str(exc)}
    if rank == 0:
        print(json.dumps(line))
    if pg:
        pg.barrier()
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
