"""Autotuner of the hot kernels' launch shapes.

Builds the library once per candidate of (face-flux block size, face-flux blocks resident per SM,
face geometry staged by bulk copies or loaded, cell-gather block size) into a scratch directory,
times a fixed number of RK steps of a workload on the current GPU with each build (a fresh process
per build, selected with TEAL_B200_LIBRARY), and writes the fastest shape to
teal_b200/csrc/tuned.h (and to --out when given). Shapes and the Navier-Stokes staging switch are
tuned on the Taylor-Green vortex, the Euler staging switch on the unstructured ramp.

    python -m teal_b200.autotune [--n 96] [--ramp-n 64] [--steps 10] [--precision fp64] [--out tuned_candidate.h]

Needs nvcc and a GPU. Every candidate computes the same results; only speed differs.
"""

import argparse
import concurrent.futures
import itertools
import json
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
ROOT = os.path.dirname(HERE)

# face-flux block size x resident face threads per SM (65536 registers / threads = the cap per
# thread: 512 -> 128, 640 -> 102, 768 -> 85) x geometry staged in shared memory by bulk copies or
# loaded by the threads x cell-gather block size. The Navier-Stokes workload tunes the shapes and
# its staging switch; the Euler staging switch is then tuned on the unstructured ramp with the
# chosen shapes.
FACE_BLOCKS = [32, 64, 128]
FACE_THREADS = [512, 640, 768]
STAGED = [0, 1]
CELL_BLOCKS = [256]
# then cell-gather block size x blocks resident per SM (1536 threads -> 42 registers per thread)
CELL_SHAPES = [(256, 1), (128, 8), (128, 12), (64, 24)]
# then gradient blocks (160 threads) resident per SM: 9 leaves the registers free, 12 caps them at 32
GRAD_MINB = [9, 12]
# last, on the ramp: resident face threads per SM of the Euler face kernel (fewer registers than the
# Navier-Stokes one needs)
EULER_FACE_THREADS = [640, 768, 896, 1024]

TIMER = r"""
import json, math, sys, time
import torch
import teal_b200 as tb
n, steps, prec, workload = int(sys.argv[1]), int(sys.argv[2]), sys.argv[3], sys.argv[4]
def tgv(c, gamma=1.4, mach=0.1):
    import numpy as np
    x, y, z = c[:, 0], c[:, 1], c[:, 2]
    p0 = 1 / (gamma * mach**2)
    out = np.zeros((c.shape[0], 5))
    out[:, 1] = np.sin(x) * np.cos(y) * np.cos(z)
    out[:, 2] = -np.cos(x) * np.sin(y) * np.cos(z)
    out[:, 4] = p0 + (np.cos(2 * x) + np.cos(2 * y)) * (np.cos(2 * z) + 2) / 16
    out[:, 0] = out[:, 4] / p0
    return out
if workload == "tgv":
    m = tb.Mesh.create((0, 0, 0), (2 * math.pi,) * 3, (n, n, n), (1, 1, 1))
    e = tb.Equations.navierstokes(m)
    e.set_convective_flux("roe"); e.set_limiter("venkatakrishnan", 1.0); e.set_property("dynamic viscosity", 1 / 1600)
    e.set_initial_condition("domain", tgv)
else:
    import numpy as np
    from teal_b200 import meshes
    m = tb.Mesh.from_cells(meshes.ramp_mesh(n=(n, n, n)))
    e = tb.Equations.euler(m)
    e.set_convective_flux("ausmd"); e.set_limiter("minmod", 0.0)
    free = (1.0, 2.5, 0.0, 0.0, 1.0 / 1.4)
    e.set_boundary_condition("left", "supersonic inflow", free)
    e.set_boundary_condition("right", "supersonic outflow")
    for side in ("bottom", "top", "back", "front"):
        e.set_boundary_condition(side, "slipwall")
    e.set_initial_condition("domain", lambda c: np.tile(np.array(free), (c.shape[0], 1)))
ctx = e.context(tb.TG_PRECISION_FP64 if prec == "fp64" else tb.TG_PRECISION_FP32_FLUX)
s = torch.cuda.Stream(); ctx.set_stream(s.cuda_stream)
ctx.run(tb.TG_ADVANCE_LSERK, 0.99, 3, context=(3, 3)); torch.cuda.synchronize()
best = float("inf")
for _ in range(3):
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(s); ctx.run(tb.TG_ADVANCE_LSERK, 0.99, steps, context=(3, 3)); b.record(s); torch.cuda.synchronize()
    best = min(best, a.elapsed_time(b) / steps)
print(json.dumps({"ms_per_step": best}))
"""


def build(variant, workdir, jobs):
    name = "_".join(f"{k[3:].lower()}{v}" for k, v in variant.items())
    out = os.path.join(workdir, f"lib_{name}.so")
    tune = " ".join(f"-D{k}={v}" for k, v in variant.items())
    cmd = ["make", "-C", CSRC, f"-j{jobs}", f"OUT={out}", f"BUILD={os.path.join(workdir, 'build_' + name)}",
           f"TUNE={tune}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build of {name} failed:\n{r.stderr[-2000:]}")
    return name, out


def time_variant(lib, n, steps, precision, workload="tgv"):
    env = dict(os.environ, TEAL_B200_LIBRARY=lib, PYTHONPATH=ROOT + os.pathsep + os.environ.get("PYTHONPATH", ""))
    r = subprocess.run([sys.executable, "-c", TIMER, str(n), str(steps), precision, workload], capture_output=True,
                       text=True, env=env, timeout=600)
    if r.returncode != 0:
        raise RuntimeError(r.stderr[-2000:])
    return json.loads(r.stdout.strip().splitlines()[-1])["ms_per_step"]


def write_header(path, best):
    lines = ["// Launch shapes of the hot kernels, chosen by teal_b200/autotune.py on a B200 (fastest measured",
             "// RK step: TGV for the face, cell and gradient shapes and the Navier-Stokes staging switch, the",
             "// ramp for the Euler staging switch; times within 0.5 % of the fastest count as ties, resolved to",
             "// fewer resident face blocks, i.e. more registers per thread). A value given with -D at build",
             "// time wins.",
             "#pragma once", ""]
    notes = {"TG_FACE_BLOCK": "threads per face-flux block",
             "TG_FACE_MINB": "Navier-Stokes face-flux blocks kept resident per SM (caps registers per thread)",
             "TG_FACE_MINB_EULER": "Euler face-flux blocks kept resident per SM (caps registers per thread)",
             "TG_FACE_MINB_FP32": "FP32-flux face-flux blocks kept resident per SM (caps registers per thread)",
             "TG_CELL_BLOCK": "threads per cell-gather block",
             "TG_CELL_MINB": "cell-gather blocks kept resident per SM (caps registers per thread)",
             "TG_FACE_STAGED_NS": "Navier-Stokes face kernel: geometry staged by bulk copies (1) or loaded (0)",
             "TG_FACE_STAGED_EULER": "Euler face kernel: geometry staged by bulk copies (1) or loaded (0)",
             "TG_GRAD_MINB": "gradient blocks (160 threads) kept resident per SM (caps registers per thread)"}
    for k, v in best.items():
        lines += [f"#ifndef {k}", f"#define {k} {v}  // {notes[k]}", "#endif"]
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=96)
    ap.add_argument("--ramp-n", type=int, default=64, help="grid of the unstructured ramp (Euler staging switch)")
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32"])
    ap.add_argument("--out", default=None, help="also write the chosen header here")
    ap.add_argument("--jobs", type=int, default=os.cpu_count() or 8)
    args = ap.parse_args()
    variants = [{"TG_FACE_BLOCK": fb, "TG_FACE_MINB": ft // fb, "TG_CELL_BLOCK": cb, "TG_FACE_STAGED_NS": st}
                for fb, ft, st, cb in itertools.product(FACE_BLOCKS, FACE_THREADS, STAGED, CELL_BLOCKS)]

    def sweep(variants, workload, n, work, per):
        with concurrent.futures.ThreadPoolExecutor(max_workers=4) as pool:
            built = list(pool.map(lambda v: (v,) + build(v, work, per), variants))
        results = []
        for v, name, lib in built:
            try:
                ms = time_variant(lib, n, args.steps, args.precision, workload)
            except Exception as exc:  # a variant that fails is reported and skipped
                print(json.dumps({"variant": v, "error": str(exc)[-300:]}), flush=True)
                continue
            results.append((ms, v))
            print(json.dumps({"variant": v, "workload": workload, "ms_per_step": ms}), flush=True)
        if not results:
            raise SystemExit("no variant ran")
        # times within 0.5 % of the fastest are ties: take the one with the fewest resident face
        # threads per SM (most registers per thread, fewest spills)
        fastest = min(r[0] for r in results)
        ties = [r for r in results if r[0] <= 1.005 * fastest]
        return min(ties, key=lambda r: (r[1]["TG_FACE_BLOCK"] * r[1]["TG_FACE_MINB"], r[0]))

    with tempfile.TemporaryDirectory() as work:
        per = max(2, args.jobs // 4)
        ms, best = sweep(variants, "tgv", args.n, work, per)
        cells = [dict(best, TG_CELL_BLOCK=cb, TG_CELL_MINB=cm) for cb, cm in CELL_SHAPES]
        ms, best = sweep(cells, "tgv", args.n, work, per)
        grads = [dict(best, TG_GRAD_MINB=gm) for gm in GRAD_MINB]
        ms, best = sweep(grads, "tgv", args.n, work, per)
        euler = [dict(best, TG_FACE_STAGED_EULER=st) for st in STAGED]
        ms_e, best = sweep(euler, "ramp", args.ramp_n, work, per)
        occ = [dict(best, TG_FACE_MINB_EULER=t // best["TG_FACE_BLOCK"]) for t in EULER_FACE_THREADS]
        ms_e, best = sweep(occ, "ramp", args.ramp_n, work, per)
    write_header(os.path.join(CSRC, "tuned.h"), best)
    if args.out:
        write_header(args.out, best)
    print(json.dumps({"best": best, "ms_per_step": ms, "workload": f"tgv {args.n}^3 {args.precision}",
                      "ramp_ms_per_step": ms_e}))


if __name__ == "__main__":
    main()
