"""The exact FP64 form (TG_PRECISION_FP64_EXACT) against the reference solver, bit for bit.

In this form every kernel evaluates teal's expressions with teal's operations in teal's order (each
quotient a division, no multiply-add contraction, a cell's viscous face terms summed before its
convective ones), and every per-cell sum runs in teal's face order. FP64 + - * / and sqrt are
correctly rounded on both sides, so residuals, gradients, time steps and explicit RK steps must be
*equal* to the reference's: np.array_equal, no tolerance. Exceptions, each stated where it applies:
the residual norm and the bulk-forcing average are tree sums on the device (sequential in teal), and
the implicit Newton-GMRES step's dot products likewise, so those keep the bars of the plain form.
"""

import numpy as np
import pytest

import teal_b200 as tb
from oracle import ref
from teal_b200 import diagnostics
from tests import golden_cases
from tests.cases import random_state, rel_l2, taylor_green, vortex

EXACT = tb.TG_PRECISION_FP64_EXACT
GOLDEN = golden_cases.load()
pytestmark = pytest.mark.gpu
needs_ref = pytest.mark.skipif(not ref.available(), reason="reference oracle not built")
GAMMA = 1.4


def equal(a, b):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape
    if not np.array_equal(a, b):
        diff = np.abs(a - b)
        i = np.unravel_index(np.argmax(diff), diff.shape)
        raise AssertionError(f"{np.count_nonzero(a != b)} of {a.size} values differ; largest at {i}: "
                             f"{a[i]!r} vs {b[i]!r}; rel L2 {rel_l2(a.reshape(len(a), -1), b.reshape(len(b), -1))}")


@pytest.mark.parametrize("name", sorted(GOLDEN))
def test_exact_form_reproduces_golden_bit_for_bit(name):
    g = GOLDEN[name]
    case = g["case"]
    m, e = golden_cases.equations(case)
    prim = g["primitive"]
    C = m.num_inner_cells
    averaged = "source" in case and case["source"][0] == "bulk forcing"
    d = e.derivative(prim, precision=EXACT)
    if averaged:  # the forcing's volume average is a tree sum on the device
        assert rel_l2(d, g["derivative"]).max() <= 1e-14
    else:
        equal(d, g["derivative"])
    ctx = e.context(EXACT)
    ctx.set_primitive(prim)
    assert ctx.timestep() == float(g["timestep"])
    if "gradient" in g:
        ctx.set_primitive(prim)
        equal(ctx.gradient().reshape(C, 15), g["gradient"].reshape(C, 15))
        if case["limiter"]:
            equal(ctx.gradient(limited=True).reshape(C, 15), g["gradient_limited"].reshape(C, 15))
    adv = case.get("advance")
    if adv:
        e.primitive[:] = prim
        sim = tb.Simulation(e, precision=EXACT)
        sim.set_advance(adv["method"], adv["courant"], adv.get("rk") or adv.get("nk"))
        t = 0.0
        for _ in range(adv["steps"]):
            t, s0, res = sim.advance(t)
        if adv["method"] == "implicit euler":  # Krylov dot products are tree sums
            tol = 1e-4 if case["limiter"] else 1e-7
            assert rel_l2(e.primitive[:C], g["advance_state"]).max() <= tol
            assert abs(t - float(g["advance_time"])) <= 1e-13 * float(g["advance_time"])
        elif averaged:
            assert rel_l2(e.primitive[:C], g["advance_state"]).max() <= 1e-14
        else:
            equal(e.primitive[:C], g["advance_state"])
            assert t == float(g["advance_time"])


def pair(n, lo, hi, periodic, ns=False, flux="hllc", limiter="minmod", coeff=0.0, order=2, mu=None, bcs=None):
    rm = ref.RefMesh(lo, hi, n, periodic)
    re = ref.RefEquations(rm, ns)
    dm = tb.Mesh.create(lo, hi, n, periodic)
    de = tb.Equations.navierstokes(dm) if ns else tb.Equations.euler(dm)
    for e in (re, de):
        e.set_space_order(order)
        e.set_convective_flux(flux)
        e.set_limiter(limiter, coeff)
        if ns and mu is not None:
            e.set_property("dynamic viscosity", mu)
        for entity, (name, ctx) in (bcs or {}).items():
            e.set_boundary_condition(entity, name, ctx)
    return rm, re, dm, de


@needs_ref
@pytest.mark.parametrize("flux", ["roe", "hll", "hllc", "hlle", "ausmd", "ausmdv", "lxf", "central"])
@pytest.mark.parametrize("limiter", [None, "minmod", "venkatakrishnan"])
def test_exact_euler_flux_limiter_matrix(flux, limiter):
    rm, re, dm, de = pair((8, 7, 6), (0, 0, 0), (1, 1, 1), (1, 1, 1), flux=flux, limiter=limiter, coeff=1.0)
    prim = random_state(dm.num_cells, seed=hash((flux, limiter)) % 1000)
    equal(de.derivative(prim, precision=EXACT), re.derivative(prim))


@needs_ref
@pytest.mark.parametrize("limiter", [None, "minmod", "venkatakrishnan"])
@pytest.mark.parametrize("flux", ["roe", "hllc", "ausmd"])
def test_exact_navierstokes_random_state(flux, limiter):
    rm, re, dm, de = pair((7, 6, 5), (0, 0, 0), (1, 1, 1), (1, 1, 1), ns=True, flux=flux, limiter=limiter,
                          coeff=0.5, mu=0.05)
    prim = random_state(dm.num_cells, seed=11, mach=0.6)
    equal(de.derivative(prim, precision=EXACT), re.derivative(prim))


SIDES = ["left", "right", "bottom", "top", "back", "front"]
FREE = (1.0, 0.6, 0.1, -0.05, 1.0 / GAMMA)


@needs_ref
@pytest.mark.parametrize("bc", ["slipwall", "supersonic inflow", "supersonic outflow", "subsonic inflow",
                                "subsonic outflow", "pressure outflow", "farfield"])
def test_exact_boundary_conditions(bc):
    bcs = {s: (bc, FREE) for s in SIDES}
    rm, re, dm, de = pair((6, 5, 4), (0, 0, 0), (1, 1, 1), (0, 0, 0), bcs=bcs)
    prim = random_state(dm.num_cells, seed=5, mach=0.8)
    equal(de.derivative(prim, precision=EXACT), re.derivative(prim))


@needs_ref
def test_exact_navierstokes_wall_and_mixed_boundaries():
    bcs = {"left": ("subsonic inflow", FREE), "right": ("subsonic outflow", FREE),
           "bottom": ("adiabatic wall", None), "top": ("farfield", FREE)}
    rm, re, dm, de = pair((8, 6, 3), (0, 0, 0), (2, 1, 0.5), (0, 0, 1), ns=True, flux="roe",
                          limiter="venkatakrishnan", coeff=1.0, mu=0.01, bcs=bcs)
    prim = random_state(dm.num_cells, seed=9, mach=0.5)
    equal(de.derivative(prim, precision=EXACT), re.derivative(prim))


def run_both(re, de, prim, courant, rk, steps, record=None):
    """`steps` lserk steps of the reference and of the device's exact and plain FP64 forms from the same
    state; returns their times and states (and, with `record`, its value after every step)."""
    C = de.mesh.num_inner_cells
    out = {}
    re.set_primitive(prim)
    rsim = ref.RefSimulation(re, "lserk", courant, rk=rk)
    t, hist = 0.0, []
    for _ in range(steps):
        t, _, _ = rsim.advance(t)
        if record:
            hist.append(record(re.primitive[:C], re))
    out["ref"] = (t, re.primitive[:C].copy(), hist)
    for name, precision in (("exact", EXACT), ("fp64", tb.TG_PRECISION_FP64)):
        de.primitive[:] = prim
        sim = tb.Simulation(de, precision=precision)
        sim.set_advance("lserk", courant, rk)
        t, hist = 0.0, []
        for _ in range(steps):
            t, _, _ = sim.advance(t)
            if record:
                hist.append(record(de.primitive[:C], de, precision))
        out[name] = (t, de.primitive[:C].copy(), hist)
    return out


@needs_ref
def test_exact_isentropic_vortex_200_steps():
    """The isentropic vortex workload (64 x 64 x 4, hllc, Barth-Jespersen, lserk{3,3}, CFL 0.5) for all
    of its 200 steps: the exact form equals the reference after every step's 3 stages; the plain FP64
    form stays within 1e-12."""
    lo, hi, n, per = (0, 0, 0), (10, 10, 0.625), (64, 64, 4), (1, 1, 1)
    rm, re, dm, de = pair(n, lo, hi, per)
    prim = vortex(dm.cell_center)
    out = run_both(re, de, prim, 0.5, (3, 3), 200)
    assert out["exact"][0] == out["ref"][0]
    equal(out["exact"][1], out["ref"][1])
    assert abs(out["fp64"][0] - out["ref"][0]) <= 1e-13 * out["ref"][0]
    assert rel_l2(out["fp64"][1], out["ref"][1]).max() <= 1e-12


@needs_ref
def test_exact_taylor_green_48_cubed_200_steps_with_histories():
    """Taylor-Green vortex 48^3 (Navier-Stokes, Roe, Venkatakrishnan(1), Re 1600, Ma 0.1, lserk{3,3},
    CFL 0.99), 200 steps: the exact form's state, kinetic energy and enstrophy histories equal the
    reference's; the plain FP64 form's histories stay within 1e-12 relative of them."""
    n = 48
    rm, re, dm, de = pair((n, n, n), (0, 0, 0), (2 * np.pi,) * 3, (1, 1, 1), ns=True, flux="roe",
                          limiter="venkatakrishnan", coeff=1.0, mu=1 / 1600)
    C = dm.num_inner_cells
    volume = np.asarray(dm.cell_volume[:C])

    def record(p, eq, precision=None):
        if precision is None:
            g = eq.gradient()  # the reference's unlimited least-squares gradient of its whole state
        else:
            ctx = eq.context(precision)
            ctx.set_primitive(eq.primitive)
            g = ctx.gradient()
        return diagnostics.kinetic_energy(p, volume), diagnostics.enstrophy(p, np.asarray(g)[:C], volume)

    prim = taylor_green(dm.cell_center)
    out = run_both(re, de, prim, 0.99, (3, 3), 200, record=record)
    assert out["exact"][0] == out["ref"][0]
    equal(out["exact"][1], out["ref"][1])
    ref_hist, ex_hist, fp_hist = (np.array(out[k][2]) for k in ("ref", "exact", "fp64"))
    equal(ex_hist, ref_hist)
    assert np.all(np.abs(fp_hist - ref_hist) <= 1e-12 * np.abs(ref_hist))
    assert rel_l2(out["fp64"][1], out["ref"][1]).max() <= 1e-12
