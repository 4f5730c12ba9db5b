"""One mesh over several ranks on the device: every rank a partition (tg_create_partition) with its
halo, all ranks driven in one process on one GPU (teal_b200.partition.LocalRun: the halo moved by
device copies between the ranks' exchange buffers, the reductions on the host). The state after
every step must equal the single-mesh run's bit for bit (each rank's cells see the same inputs and
sum their faces in the same order), the time too; the residual norm, a sum over ranks, to rounding.
"""

import numpy as np
import pytest

import teal_b200 as tb
from teal_b200 import partition as pt
from tests.cases import random_state, taylor_green, vortex

pytestmark = pytest.mark.gpu


def single_steps(e, prim, steps, courant, precision):
    ctx = tb.Context(e.mesh, e, precision=precision)
    ctx.set_primitive(prim)
    out, t = [], 0.0
    for _ in range(steps):
        t, s0, res = ctx.advance(tb.TG_ADVANCE_LSERK, courant, t, context=(3, 3))
        out.append((t, res.copy(), ctx.get_primitive()[: e.mesh.num_inner_cells].copy()))
    ctx.close()
    return out


def check(case, e, prim, size, steps=4, courant=0.9, precision=tb.TG_PRECISION_FP64, ranks=None):
    ref = single_steps(e, prim, steps, courant, precision)
    if ranks is None:
        ranks, _ = pt.cell_ranks(e.mesh, case[0], case[1], case[2], size)
    run = pt.LocalRun(pt.partition(e.mesh, ranks), e, precision)
    try:
        run.set_state(prim)
        t = 0.0
        for k in range(steps):
            t, s0, res = run.step(t, courant)
            rt, rres, rstate = ref[k]
            assert t == rt
            np.testing.assert_allclose(res, rres, rtol=1e-13, atol=0)
            state = run.state(e.mesh.num_inner_cells)
            assert np.array_equal(state, rstate), (k, np.abs(state - rstate).max())
    finally:
        run.close()


@pytest.mark.parametrize("size", [2, 3, 4])
def test_partitioned_taylor_green_equals_the_single_mesh(size):
    case = ((0, 0, 0), (2 * np.pi,) * 3, (12, 12, 12), (1, 1, 1))
    m = tb.Mesh.create(*case)
    e = tb.Equations.navierstokes(m)
    e.set_convective_flux("roe")
    e.set_limiter("venkatakrishnan", 1.0)
    e.set_property("dynamic viscosity", 1 / 1600)
    check(case, e, taylor_green(m.cell_center), size, courant=0.99)


@pytest.mark.parametrize("size", [2, 3])
def test_partitioned_vortex_equals_the_single_mesh(size):
    case = ((0, 0, 0), (10, 10, 0.625), (24, 24, 4), (1, 1, 1))
    m = tb.Mesh.create(*case)
    e = tb.Equations.euler(m)
    check(case, e, vortex(m.cell_center), size, courant=0.5)


@pytest.mark.parametrize("flux", ["hllc", "ausmd"])
def test_partitioned_box_with_boundaries_equals_the_single_mesh(flux):
    case = ((0, 0, 0), (2, 1, 1), (9, 7, 3), (0, 1, 0))
    m = tb.Mesh.create(*case)
    e = tb.Equations.euler(m)
    e.set_convective_flux(flux)
    free = (1.0, 0.6, 0.1, -0.05, 1.0 / 1.4)
    for side in ("left", "right"):
        e.set_boundary_condition(side, "farfield", free)
    for side in ("back", "front"):
        e.set_boundary_condition(side, "slipwall")
    check(case, e, random_state(m.num_cells, seed=4, mach=0.6), 3)


def test_partitioned_exact_form_equals_the_single_mesh():
    case = ((0, 0, 0), (2 * np.pi,) * 3, (10, 10, 10), (1, 1, 1))
    m = tb.Mesh.create(*case)
    e = tb.Equations.navierstokes(m)
    e.set_convective_flux("roe")
    e.set_limiter("venkatakrishnan", 1.0)
    e.set_property("dynamic viscosity", 1 / 1600)
    check(case, e, taylor_green(m.cell_center), 2, courant=0.99, precision=tb.TG_PRECISION_FP64_EXACT)


@pytest.mark.parametrize("size", [2, 3, 4])
def test_bisected_compression_ramp_equals_the_single_mesh(size):
    # the unstructured ramp (mixed elements, supersonic inflow / outflow, slip walls, AUSMD +
    # Barth-Jespersen), split by recursive coordinate bisection
    from teal_b200 import meshes

    m = tb.Mesh.from_cells(meshes.ramp_mesh(n=(12, 12, 12), seed=2))
    e = tb.Equations.euler(m)
    e.set_convective_flux("ausmd")
    e.set_limiter("minmod", 0.0)
    inflow = (1.0, 2.5, 0.0, 0.0, 1.0 / 1.4)
    e.set_boundary_condition("left", "supersonic inflow", inflow)
    e.set_boundary_condition("right", "supersonic outflow")
    for side in ("bottom", "top", "back", "front"):
        e.set_boundary_condition(side, "slipwall")
    check(None, e, random_state(m.num_cells, seed=7, mach=1.5), size, courant=0.9,
          ranks=pt.bisection_ranks(m, size))
