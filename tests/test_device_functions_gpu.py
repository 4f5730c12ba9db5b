"""Device functions on the GPU against the reference with the same formulas as host Compute callbacks
(oracle/ref_harness.c): a custom boundary that reads the inner state (a moving wall), one that reads
the ghost centre and the time (an unsteady inflow), and a source that reads all of them. Bar: the
plain FP64 parity bar, relative L2 per conserved variable <= 1e-12, for the residual at a given time
and for the state after explicit steps (whose stages reach the functions at time + alpha_i step).
Implicit steps: the bar of the implicit parity tests (1e-7 without a limiter)."""

import ctypes

import numpy as np
import pytest

import teal_b200 as tb
from oracle import ref
from teal_b200 import _lib
from tests.cases import random_state, rel_l2
from tests.device_functions import (AVERAGE_PROBE, HILL_FORCING, MOVING_WALL, UNSTEADY_INFLOW, UNSTEADY_SOURCE,
                                   hill_forcing)

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not ref.available(), reason="reference oracle not built")]

TOL = 1e-12


@pytest.fixture(scope="module", autouse=True)
def registered():
    tb.register_function("lid_wall", "boundary", MOVING_WALL)
    tb.register_function("unsteady_inflow", "boundary", UNSTEADY_INFLOW)
    tb.register_function("unsteady_source", "source", UNSTEADY_SOURCE)
    tb.register_function("hill_forcing", "source", HILL_FORCING)
    tb.register_function("average_probe", "source", AVERAGE_PROBE)
    tb.register_function("hill_forcing_mild", "source", hill_forcing("hill_forcing_mild", "1.0"))


def run_both(re, de, prim, method, courant, steps, rk=None, nk=None):
    re.set_primitive(prim)
    de.primitive[:] = prim
    rsim = ref.RefSimulation(re, method, courant, rk=rk, nk=nk)
    dsim = tb.Simulation(de)
    dsim.set_advance(method, courant, rk if method == "lserk" else nk)
    t_ref = t_dev = 0.0
    for _ in range(steps):
        t_ref, _, res_ref = rsim.advance(t_ref)
        t_dev, _, res_dev = dsim.advance(t_dev)
    return (t_ref, res_ref, re.primitive[: re.num_inner].copy()), (t_dev, res_dev, de.primitive[: re.num_inner].copy())


def cavity():
    """Lid-driven cavity (run/lid_driven_cavity/run.c): walls, the top one moving, on a 3D box
    periodic in z."""
    lo, hi, n = (0, 0, 0), (1, 1, 0.125), (16, 16, 2)
    rm = ref.RefMesh(lo, hi, n, (0, 0, 1))
    re = ref.RefEquations(rm, True)
    dm = tb.Mesh.create(lo, hi, n, (0, 0, 1))
    de = tb.Equations.navierstokes(dm)
    for e in (re, de):
        e.set_convective_flux("roe")
        e.set_limiter("venkatakrishnan", 1.0)
        e.set_property("dynamic viscosity", 0.01)
        for side in ("left", "right", "bottom"):
            e.set_boundary_condition(side, "wall")
    re.set_boundary_custom("top", "moving wall", 1.0)
    de.set_boundary_condition("top", "custom", compute="lid_wall")
    return re, de


def inflow_channel(source=False):
    """Euler channel fed by an unsteady inflow; optionally with the unsteady source."""
    lo, hi, n = (0, 0, 0), (3, 1, 0.25), (24, 8, 2)
    rm = ref.RefMesh(lo, hi, n, (0, 0, 1))
    re = ref.RefEquations(rm, False)
    dm = tb.Mesh.create(lo, hi, n, (0, 0, 1))
    de = tb.Equations.euler(dm)
    for e in (re, de):
        e.set_convective_flux("hllc")
        e.set_limiter("minmod", 0.0)
        e.set_boundary_condition("right", "supersonic outflow")
        e.set_boundary_condition("bottom", "slipwall")
        e.set_boundary_condition("top", "slipwall")
    re.set_boundary_custom("left", "unsteady inflow")
    de.set_boundary_condition("left", "custom", compute="unsteady_inflow")
    if source:
        re.set_source("unsteady")
        de.set_source("device function", compute="unsteady_source")
    return re, de


def test_moving_wall_cavity():
    re, de = cavity()
    prim = random_state(de.mesh.num_cells, seed=61, mach=0.3)
    a = re.derivative(prim)
    b = de.derivative(prim)
    assert rel_l2(b, a).max() <= TOL
    (tr, rr, pr), (td, rd, pd) = run_both(re, de, prim, "lserk", 0.5, 10, rk=(3, 3))
    assert rel_l2(pd, pr).max() <= TOL
    assert abs(td - tr) <= 1e-13 * tr


@pytest.mark.parametrize("time", [0.0, 0.37, 2.5])
def test_unsteady_inflow_residual_at_time(time):
    re, de = inflow_channel()
    prim = random_state(de.mesh.num_cells, seed=62, mach=0.8)
    a = re.derivative(prim, time)
    b = de.derivative(prim, time)
    assert rel_l2(b, a).max() <= TOL


def test_unsteady_inflow_time_reaches_the_function():
    re, de = inflow_channel()
    prim = random_state(de.mesh.num_cells, seed=63, mach=0.8)
    assert not np.allclose(de.derivative(prim, 0.0), de.derivative(prim, 1.0))


@pytest.mark.parametrize("method,rk", [("lserk", (3, 3)), ("lserk", (2, 2)), ("euler", None)])
def test_unsteady_inflow_stages(method, rk):
    re, de = inflow_channel()
    prim = random_state(de.mesh.num_cells, seed=64, mach=0.8)
    (tr, rr, pr), (td, rd, pd) = run_both(re, de, prim, method, 0.5, 8, rk=rk)
    assert rel_l2(pd, pr).max() <= TOL
    np.testing.assert_allclose(rd, rr, rtol=1e-10)


@pytest.mark.parametrize("time", [0.0, 0.7])
def test_unsteady_source_residual(time):
    re, de = inflow_channel(source=True)
    prim = random_state(de.mesh.num_cells, seed=65, mach=0.8)
    assert rel_l2(de.derivative(prim, time), re.derivative(prim, time)).max() <= TOL


def test_unsteady_source_lserk():
    re, de = inflow_channel(source=True)
    prim = random_state(de.mesh.num_cells, seed=66, mach=0.8)
    (tr, rr, pr), (td, rd, pd) = run_both(re, de, prim, "lserk", 0.5, 8, rk=(3, 3))
    assert rel_l2(pd, pr).max() <= TOL


def test_unsteady_source_implicit():
    # implicit Euler evaluates every residual at time + step
    re, de = inflow_channel(source=True)
    for e in (re, de):
        e.set_limiter(None, 0.0)
    prim = random_state(de.mesh.num_cells, seed=67, mach=0.8)
    (tr, rr, pr), (td, rd, pd) = run_both(re, de, prim, "implicit euler", 5.0, 2, nk=(0.1, 0.3, 30))
    assert rel_l2(pd, pr).max() <= 1e-7


def test_run_loop_with_device_functions_is_deterministic():
    finals = []
    for _ in range(2):
        _, de = inflow_channel(source=True)
        de.set_initial_condition("domain", lambda c: random_state(c.shape[0], seed=68, mach=0.8))
        ctx = de.context()
        t, it, res = ctx.run(tb.TG_ADVANCE_LSERK, 0.5, 20, context=(3, 3))
        finals.append((t, ctx.get_primitive()))
    assert finals[0][0] == finals[1][0]
    assert np.array_equal(finals[0][1], finals[1][1])


def test_unbound_custom_boundary_is_an_error():
    m = tb.Mesh.create((0, 0, 0), (3, 1, 0.25), (12, 4, 2), (0, 0, 1))
    e = tb.Equations.euler(m)
    for side in ("right", "bottom", "top"):
        e.set_boundary_condition(side, "slipwall")
    e.set_boundary_condition("left", "custom", compute="unsteady_inflow")
    names = [n for n, _, _ in m.entities][m.struct.num_inner_entities:]
    left, right = names.index("left"), names.index("right")
    s = e.struct()
    h = ctypes.c_void_p()
    assert _lib.lib.tg_create(ctypes.byref(m.struct), ctypes.byref(s), 0, ctypes.byref(h)) == _lib.TG_OK
    try:
        out = np.zeros((m.num_inner_cells, 5))
        prim = np.ascontiguousarray(random_state(m.num_cells, seed=69))
        rc = _lib.lib.tg_derivative(h, prim.ctypes.data, out.ctypes.data, 0.0)
        assert rc == _lib.TG_ERR_INVALID
        assert b"no device function" in _lib.lib.tg_last_error()
        # a kind mismatch and a wrong boundary are refused at binding
        assert _lib.lib.tg_bind_boundary_function(h, left, b"unsteady_source") == _lib.TG_ERR_INVALID
        assert _lib.lib.tg_bind_boundary_function(h, right, b"unsteady_inflow") == _lib.TG_ERR_INVALID
        assert _lib.lib.tg_bind_boundary_function(h, left, b"no_such_function") == _lib.TG_ERR_INVALID
        assert _lib.lib.tg_bind_boundary_function(h, left, b"unsteady_inflow") == _lib.TG_OK
        assert _lib.lib.tg_derivative(h, prim.ctypes.data, out.ctypes.data, 0.0) == _lib.TG_OK
    finally:
        _lib.lib.tg_destroy(h)


def test_batches_refuse_device_functions():
    _, de = inflow_channel()
    with pytest.raises(tb.TealError):
        tb.Batch([de])


def test_reregistration_keeps_bound_code():
    """A context keeps the code it was bound to; later bindings take the replacement."""
    src = """
__device__ void swap_src(double *source, const double *property, const double *center, double time,
                         const double *state)
{{ source[1] = {value}; }}
"""
    tb.register_function("swap_src", "source", src.format(value="1.0"))
    _, de = inflow_channel()
    de.set_source("device function", compute="swap_src")
    prim = random_state(de.mesh.num_cells, seed=70, mach=0.8)
    old_ctx = tb.Context(de.mesh, de)
    d1 = old_ctx.derivative(prim)
    tb.register_function("swap_src", "source", src.format(value="3.0"))
    np.testing.assert_array_equal(old_ctx.derivative(prim), d1)
    new_ctx = tb.Context(de.mesh, de)
    d2 = new_ctx.derivative(prim)
    np.testing.assert_allclose(d2[:, 1] - d1[:, 1], 2.0, rtol=0, atol=1e-9)
    np.testing.assert_array_equal(d2[:, [0, 2, 3, 4]], d1[:, [0, 2, 3, 4]])


def hill_channel(tau=0.001):
    """The periodic hill's walled channel (run/periodic_hill/run.c, coarse and without the hill):
    teal's bulk forcing with its Prepare in the reference, the device function with the average
    Prepare here (time scale 0.001 as in the run case, or 1)."""
    lo, hi, n = (0, 0, 0), (9, 3, 0.3), (18, 10, 2)
    rm = ref.RefMesh(lo, hi, n, (1, 0, 1))
    re = ref.RefEquations(rm, True)
    dm = tb.Mesh.create(lo, hi, n, (1, 0, 1))
    de = tb.Equations.navierstokes(dm)
    for e in (re, de):
        e.set_convective_flux("roe")
        e.set_limiter("venkatakrishnan", 1.0)
        e.set_property("dynamic viscosity", 0.01)
        e.set_boundary_condition("bottom", "wall")
        e.set_boundary_condition("top", "wall")
    re.set_source("bulk forcing", (1.0, tau))
    de.set_source("device function", compute="hill_forcing" if tau == 0.001 else "hill_forcing_mild",
                  prepare="average")
    return re, de


def test_prepare_average_matches_teals_prepare():
    re, de = hill_channel()
    prim = random_state(de.mesh.num_cells, seed=71, mach=0.4)
    for time in (0.0, 0.5):
        assert rel_l2(de.derivative(prim, time), re.derivative(prim, time)).max() <= TOL
    (tr, rr, pr), (td, rd, pd) = run_both(re, de, prim, "lserk", 0.3, 5, rk=(3, 3))
    assert rel_l2(pd, pr).max() <= TOL


def test_prepare_average_implicit():
    # the run case's time scale 0.001 makes the Newton systems stiff enough that the loose Krylov
    # tolerance amplifies last-bit differences of the average (teal sums it serially, the device by
    # pieces) above the implicit bar; time scale 1 keeps the systems as well conditioned as the
    # other implicit parity cases
    re, de = hill_channel(tau=1.0)
    for e in (re, de):
        e.set_limiter(None, 0.0)
    prim = random_state(de.mesh.num_cells, seed=72, mach=0.4)
    (tr, rr, pr), (td, rd, pd) = run_both(re, de, prim, "implicit euler", 2.0, 2, nk=(0.1, 0.3, 30))
    assert rel_l2(pd, pr).max() <= 1e-7


def test_prepare_average_values_and_default_zeros():
    """context[5..9] holds the volume average of the primitive state with the average Prepare and
    zeros without it; the source's conserved-variable residual contribution is S itself."""
    _, de = inflow_channel()
    prim = random_state(de.mesh.num_cells, seed=73, mach=0.8)
    C = de.mesh.num_inner_cells
    vol = np.asarray(de.mesh.cell_volume[:C])
    want = (vol[:, None] * prim[:C]).sum(axis=0) / vol.sum()
    base = de.derivative(prim)
    de.set_source("device function", compute="average_probe")
    assert np.array_equal(de.derivative(prim), base)
    de.set_source("device function", compute="average_probe", prepare="average")
    got = de.derivative(prim) - base
    # got = (R + S) - R: exact up to the rounding of R + S
    np.testing.assert_allclose(got, np.broadcast_to(want, got.shape), rtol=0,
                               atol=1e-12 * (1 + np.abs(base).max()))


def test_prepare_needs_a_device_source():
    _, de = inflow_channel(source=True)
    ctx = de.context()
    assert _lib.lib.tg_bind_source_prepare(ctx.handle, 7) == _lib.TG_ERR_INVALID
    _, de2 = inflow_channel()
    ctx2 = de2.context()
    assert _lib.lib.tg_bind_source_prepare(ctx2.handle, _lib.TG_PREPARE_AVERAGE) == _lib.TG_ERR_INVALID
