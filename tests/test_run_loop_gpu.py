"""simulation_run's loop on the device (src/simulation/run.c:22-113): output points by time and by
iteration against the reference's own run loop, raw state files and restart, and a clean stop at
the next output point (teal's SIGINT / SIGTERM handling)."""

import os

import numpy as np
import pytest

import teal_b200 as tb
from oracle import ref
from tests.cases import rel_l2, vortex

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not ref.available(), reason="reference oracle not built")]

BOX = ((0, 0, 0), (10, 10, 0.625), (16, 16, 4), (1, 1, 1))


def vortex_pair():
    rm = ref.RefMesh(*BOX)
    re = ref.RefEquations(rm, False)
    m = tb.Mesh.create(*BOX)
    e = tb.Equations.euler(m)
    prim = vortex(m.cell_center)
    re.set_primitive(prim)
    e.primitive[:] = prim
    return re, e


@pytest.mark.parametrize("out", [("time", 0.05), ("iter", 5)])
def test_output_points_match_reference_run(out):
    re, e = vortex_pair()
    rs = ref.RefSimulation(re, "lserk", 0.99, rk=(3, 3))
    ds = tb.Simulation(e)
    ds.set_advance("lserk", 0.99, (3, 3))
    for s in (rs, ds):
        if out[0] == "time":
            s.set_max_time(0.2)
            s.set_out_time(out[1])
        else:
            s.set_max_iter(12)
            s.set_out_iter(out[1])
    t_ref = rs.run()
    lines = []
    t_dev = ds.run(log=lines.append)
    C = e.mesh.num_inner_cells
    assert abs(t_dev - t_ref) <= 1e-13 * max(1.0, t_ref)
    assert rel_l2(e.primitive[:C], re.primitive[:C]).max() <= 1e-12
    outputs = 4 if out[0] == "time" else 3
    assert len(lines) == 1 + outputs + 1  # header, one line per output point, computation time


def test_state_files_and_restart_are_bit_identical(tmp_path):
    _, e1 = vortex_pair()
    straight = tb.Simulation(e1)
    straight.set_max_iter(10)
    t1 = straight.run()

    _, e2 = vortex_pair()
    first = tb.Simulation(e2)
    first.set_max_iter(4)
    first.set_out_iter(2)
    prefix = os.path.join(tmp_path, "vortex")
    first.run(prefix=prefix)
    files = sorted(os.listdir(tmp_path))
    assert files == [f"vortex_{i:05d}.tgstate" for i in range(3)]  # initial state and two outputs

    _, e3 = vortex_pair()
    e3.primitive[:] = 0.0
    resumed = tb.Simulation(e3)
    resumed.load_state(os.path.join(tmp_path, "vortex_00002.tgstate"))
    resumed.set_max_iter(6)
    t3 = resumed.run()
    C = e1.mesh.num_inner_cells
    assert t3 == t1
    assert np.array_equal(e3.primitive[:C], e1.primitive[:C])


def test_stop_request_ends_at_the_next_output_point():
    _, e = vortex_pair()
    sim = tb.Simulation(e)
    sim.set_max_iter(100)
    sim.set_out_iter(3)
    seen = []

    def on_output(s, it, t, index):
        seen.append(it)
        s.request_stop()

    sim.run(on_output=on_output)
    assert seen == [3] and sim.iterations == 3


def test_runs_are_deterministic():
    """No floating-point atomics: the same steps give the same bits on every run (a fresh context
    each time)."""
    out = []
    for _ in range(2):
        m = tb.Mesh.create((0, 0, 0), (2 * np.pi,) * 3, (12, 12, 12), (1, 1, 1))
        e = tb.Equations.navierstokes(m)
        e.set_convective_flux("roe")
        e.set_limiter("venkatakrishnan", 1.0)
        e.set_property("dynamic viscosity", 1 / 1600)
        from tests.cases import taylor_green

        e.set_initial_condition("domain", taylor_green)
        ctx = tb.Context(m, e)
        ctx.set_primitive(e.primitive)
        t, it, res = ctx.run(tb.TG_ADVANCE_LSERK, 0.99, 7, context=(3, 3))
        out.append((t, res.copy(), ctx.get_primitive().copy()))
        ctx.close()
    assert out[0][0] == out[1][0]
    assert np.array_equal(out[0][1], out[1][1]) and np.array_equal(out[0][2], out[1][2])


def test_run_writes_vtu_at_output_points(tmp_path):
    from teal_b200 import output

    _, e = vortex_pair()
    sim = tb.Simulation(e)
    sim.set_max_iter(4)
    sim.set_out_iter(2)
    prefix = os.path.join(tmp_path, "vortex")
    sim.run(prefix=prefix, vtu=True)
    names = sorted(f for f in os.listdir(tmp_path) if f.endswith(".vtu"))
    assert names == [f"vortex_{i:05d}.vtu" for i in range(3)]
    d = output.read_vtu(os.path.join(tmp_path, names[-1]))
    C = e.mesh.num_inner_cells
    np.testing.assert_array_equal(d["density"], e.primitive[:C, 0])
    np.testing.assert_array_equal(d["pressure"], e.primitive[:C, 4])
    assert d["time"][0] > 0
