"""The drop-in inside teal: teal's own simulation_run with the device Advance installed.

oracle/_ref/teal_dropin is the reference's sources compiled in place plus oracle/dropin_run.c, which
builds teal's run cases with teal's public API and, in `device` mode, binds the equations to a
device context through INTEGRATION.md's binding (tg_mesh_of, tg_equations_of, tg_create, tg_bind)
and installs tg_teal_lserk / tg_teal_implicit_euler into `Simulation.advance.method`. The same
program in `stock` mode is teal alone. Both runs go through teal's run loop (run.c:22-113), which
prints one line per output interval: iteration, time, step and maximum residual must agree, and the
final state must equal teal's bit for bit in the exact FP64 form and within 1e-12 in the plain one.
Implicit steps keep the implicit bar (tree-summed Krylov dot products; test_parity_gpu.py).
"""

import os
import subprocess

import numpy as np
import pytest

from tests.cases import rel_l2

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DROPIN = os.path.join(ROOT, "oracle", "_ref", "teal_dropin")

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not os.path.exists(DROPIN), reason="teal_dropin not built (needs the reference tree)")]


def run(case, mode, tmp_path, precision="exact", steps=None):
    out = tmp_path / f"{case}_{mode}_{precision}.bin"
    cmd = [DROPIN, case, mode, "--precision", precision, "--out", str(out)]
    if steps:
        cmd += ["--steps", str(steps)]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    raw = np.fromfile(out, dtype=np.float64)
    # teal's run-loop lines: iteration, time, step, maximum residual (the wall time differs)
    lines = []
    for line in r.stdout.splitlines():
        f = line.split()
        if len(f) == 5 and f[0].isdigit():
            lines.append(f[:4])
    return raw[0], raw[1:].reshape(-1, 5), lines


@pytest.mark.parametrize("case", ["vortex", "tgv"])
def test_teal_run_loop_with_device_lserk(case, tmp_path):
    t_ref, q_ref, lines_ref = run(case, "stock", tmp_path)
    t_dev, q_dev, lines_dev = run(case, "device", tmp_path)
    assert lines_ref and lines_dev == lines_ref
    assert t_dev == t_ref
    assert np.array_equal(q_dev, q_ref), rel_l2(q_dev, q_ref)
    t_fp, q_fp, lines_fp = run(case, "device", tmp_path, precision="fp64")
    assert abs(t_fp - t_ref) <= 1e-13 * t_ref
    assert rel_l2(q_fp, q_ref).max() <= 1e-12
    assert [l[0] for l in lines_fp] == [l[0] for l in lines_ref]


def test_teal_run_loop_with_device_implicit_euler(tmp_path):
    t_ref, q_ref, lines_ref = run("implicit", "stock", tmp_path)
    t_dev, q_dev, lines_dev = run("implicit", "device", tmp_path)
    assert len(lines_dev) == len(lines_ref) == 3
    assert abs(t_dev - t_ref) <= 1e-13 * t_ref
    # Barth-Jespersen limiter: the implicit bar (the reference's own sensitivity, times 10). The z
    # velocity of this two-dimensional flow is rounding noise (1e-13) on both sides, so it is
    # measured against the speed's norm instead of its own
    err = rel_l2(q_dev, q_ref)
    assert err[[0, 1, 2, 4]].max() <= 1e-4, err
    speed = np.linalg.norm(q_ref[:, 1:4])
    assert np.linalg.norm(q_dev[:, 3] - q_ref[:, 3]) <= 1e-4 * speed
    for a, b in zip(lines_dev, lines_ref):
        assert a[0] == b[0] and a[1] == b[1] and a[2] == b[2]
        assert abs(float(a[3]) - float(b[3])) <= 1e-3 * abs(float(b[3]))
