"""Parity of the device path (through the C ABI) with the reference solver compiled in place.

Bar: relative L2 per conserved variable <= 1e-12 for the FP64 residual and for the state after
explicit steps. Implicit Newton-GMRES steps: 1e-7 without a limiter and 1e-4 with one, about 10x
the reference's own change under a 1e-16 relative input perturbation (its finite-difference matvec
divides rounding-level differences by the relative perturbation 1e-6, src/simulation/advance.c:157;
test_implicit_euler_newton_gmres states the measurement).
"""

import ctypes

import numpy as np
import pytest

import teal_b200 as tb
from oracle import ref
from teal_b200 import meshes
from tests.cases import rel_l2, random_state, taylor_green, vortex

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not ref.available(), reason="reference oracle not built")]

TOL = 1e-12
GAMMA = 1.4


def pair(n, lo, hi, periodic, ns=False, flux="hllc", limiter="minmod", coeff=0.0, order=2, viscous=True,
         mu=None, bcs=None, host_mesh=True):
    """Reference equations and device equations with identical settings."""
    rm = ref.RefMesh(lo, hi, n, periodic)
    re = ref.RefEquations(rm, ns)
    dm = tb.Mesh.create(lo, hi, n, periodic) if host_mesh else tb.Mesh.from_arrays(rm.arrays(), rm.entities())
    de = tb.Equations.navierstokes(dm) if ns else tb.Equations.euler(dm)
    for e in (re, de):
        e.set_space_order(order)
        e.set_convective_flux(flux)
        e.set_limiter(limiter, coeff)
        if ns:
            if not viscous:
                e.set_viscous_flux(None)
            if mu is not None:
                e.set_property("dynamic viscosity", mu)
        for entity, (name, ctx) in (bcs or {}).items():
            e.set_boundary_condition(entity, name, ctx)
    return rm, re, dm, de


def check_derivative(re, de, prim, tol=TOL):
    a = re.derivative(prim)
    b = de.derivative(prim)
    err = rel_l2(b, a)
    assert np.all(np.isfinite(b))
    assert err.max() <= tol, err
    return err


def test_vortex_config1_derivative():
    rm, re, dm, de = pair((64, 64, 4), (0, 0, 0), (10, 10, 0.625), (1, 1, 1))
    prim = vortex(dm.cell_center)
    check_derivative(re, de, prim)


def test_drop_in_mesh_from_reference_arrays():
    rm, re, dm, de = pair((16, 12, 4), (0, 0, 0), (10, 10, 0.625), (1, 1, 1), host_mesh=False)
    prim = vortex(dm.cell_center)
    check_derivative(re, de, prim)


@pytest.mark.parametrize("flux", ["roe", "hll", "hllc", "hlle", "ausmd", "ausmdv", "lxf", "central"])
@pytest.mark.parametrize("limiter", [None, "minmod", "venkatakrishnan"])
def test_euler_flux_limiter_matrix(flux, limiter):
    rm, re, dm, de = pair((8, 7, 6), (0, 0, 0), (1, 1, 1), (1, 1, 1), flux=flux, limiter=limiter, coeff=1.0)
    prim = random_state(dm.num_cells, seed=hash((flux, limiter)) % 1000)
    check_derivative(re, de, prim)


@pytest.mark.parametrize("flux", ["roe", "hllc", "ausmd"])
def test_first_order(flux):
    rm, re, dm, de = pair((8, 8, 3), (0, 0, 0), (1, 1, 1), (1, 1, 1), flux=flux, order=1)
    prim = random_state(dm.num_cells, seed=3)
    check_derivative(re, de, prim)


def test_taylor_green_navierstokes_roe_venkatakrishnan():
    rm, re, dm, de = pair((12, 12, 12), (0, 0, 0), (2 * np.pi,) * 3, (1, 1, 1), ns=True, flux="roe",
                          limiter="venkatakrishnan", coeff=1.0, mu=1 / 1600)
    prim = taylor_green(dm.cell_center)
    check_derivative(re, de, prim)


@pytest.mark.parametrize("limiter", [None, "minmod", "venkatakrishnan"])
def test_navierstokes_random_state(limiter):
    rm, re, dm, de = pair((7, 6, 5), (0, 0, 0), (1, 1, 1), (1, 1, 1), ns=True, flux="hllc", limiter=limiter,
                          coeff=0.5, mu=0.05)
    prim = random_state(dm.num_cells, seed=11, mach=0.6)
    check_derivative(re, de, prim)


SIDES = ["left", "right", "bottom", "top", "back", "front"]
FREE = (1.0, 0.6, 0.1, -0.05, 1.0 / GAMMA)


@pytest.mark.parametrize("bc", ["slipwall", "supersonic inflow", "supersonic outflow", "subsonic inflow",
                                "subsonic outflow", "pressure outflow", "farfield"])
def test_euler_boundary_conditions(bc):
    bcs = {s: (bc, FREE) for s in SIDES}
    rm, re, dm, de = pair((6, 5, 4), (0, 0, 0), (1, 1, 1), (0, 0, 0), bcs=bcs)
    prim = random_state(dm.num_cells, seed=5, mach=0.8)
    check_derivative(re, de, prim)


def test_mixed_boundaries_navierstokes_wall():
    bcs = {"left": ("subsonic inflow", FREE), "right": ("subsonic outflow", FREE),
           "bottom": ("adiabatic wall", None), "top": ("farfield", FREE)}
    rm, re, dm, de = pair((8, 6, 3), (0, 0, 0), (2, 1, 0.5), (0, 0, 1), ns=True, flux="roe",
                          limiter="venkatakrishnan", coeff=1.0, mu=0.01, bcs=bcs)
    prim = random_state(dm.num_cells, seed=9, mach=0.5)
    check_derivative(re, de, prim)


def test_gradient_matches_reference():
    rm, re, dm, de = pair((9, 8, 7), (0, 0, 0), (1, 1, 1), (1, 1, 1), limiter="venkatakrishnan", coeff=1.0)
    prim = random_state(dm.num_cells, seed=21)
    ctx = de.context()
    ctx.set_primitive(prim)
    C = dm.num_inner_cells
    for limited in (False, True):
        g_ref = re.gradient(prim, limited=limited)[:C].reshape(C, 15)
        g_dev = ctx.gradient(limited=limited).reshape(C, 15)
        assert rel_l2(g_dev, g_ref).max() <= TOL


def test_timestep_and_residual_match_reference():
    rm, re, dm, de = pair((16, 16, 4), (0, 0, 0), (10, 10, 0.625), (1, 1, 1))
    prim = vortex(dm.cell_center)
    re.set_primitive(prim)
    de.primitive[:] = prim
    dt_ref = re.timestep(prim)
    dt_dev = de.timestep()
    assert abs(dt_dev - dt_ref) <= 1e-14 * dt_ref
    d = re.derivative(prim)
    r_ref = re.residual(d)
    r_dev = de.residual(d)
    assert np.allclose(r_dev, r_ref, rtol=1e-13, atol=0)


def run_both(re, de, prim, method, courant, steps, rk=None, nk=None):
    re.set_primitive(prim)
    de.primitive[:] = prim
    rsim = ref.RefSimulation(re, method, courant, rk=rk, nk=nk)
    dsim = tb.Simulation(de)
    dsim.set_advance(method, courant, rk if method == "lserk" else nk)
    t_ref = t_dev = 0.0
    for _ in range(steps):
        t_ref, s_ref, res_ref = rsim.advance(t_ref)
        t_dev, s_dev, res_dev = dsim.advance(t_dev)
    return (t_ref, s_ref, res_ref, re.primitive[: re.num_inner].copy()), \
        (t_dev, s_dev, res_dev, de.primitive[: re.num_inner].copy())


def test_lserk_vortex_steps():
    rm, re, dm, de = pair((32, 32, 4), (0, 0, 0), (10, 10, 0.625), (1, 1, 1))
    prim = vortex(dm.cell_center)
    (tr, sr, rr, pr), (td, sd, rd, pd) = run_both(re, de, prim, "lserk", 0.5, 20, rk=(3, 3))
    assert abs(td - tr) <= 1e-13 * tr
    assert abs(sd - sr) <= 1e-12 * sr
    assert rel_l2(pd, pr).max() <= TOL
    assert np.allclose(rd, rr, rtol=1e-9)


def test_lserk_taylor_green_steps():
    rm, re, dm, de = pair((10, 10, 10), (0, 0, 0), (2 * np.pi,) * 3, (1, 1, 1), ns=True, flux="roe",
                          limiter="venkatakrishnan", coeff=1.0, mu=1 / 1600)
    prim = taylor_green(dm.cell_center)
    (tr, sr, rr, pr), (td, sd, rd, pd) = run_both(re, de, prim, "lserk", 0.99, 10, rk=(3, 3))
    assert rel_l2(pd, pr).max() <= TOL
    assert abs(td - tr) <= 1e-13 * tr


@pytest.mark.parametrize("rk", [(1, 1), (2, 3), (3, 6)])
def test_lserk_tables(rk):
    rm, re, dm, de = pair((12, 10, 3), (0, 0, 0), (10, 10, 0.625), (1, 1, 1))
    prim = vortex(dm.cell_center)
    (tr, sr, rr, pr), (td, sd, rd, pd) = run_both(re, de, prim, "lserk", 0.4, 3, rk=rk)
    assert rel_l2(pd, pr).max() <= TOL


def test_forward_euler_first_order():
    rm, re, dm, de = pair((12, 10, 3), (0, 0, 0), (10, 10, 0.625), (1, 1, 1), order=1)
    prim = vortex(dm.cell_center)
    (tr, sr, rr, pr), (td, sd, rd, pd) = run_both(re, de, prim, "euler", 0.5, 5)
    assert rel_l2(pd, pr).max() <= TOL


@pytest.mark.parametrize("limiter,tol", [(None, 1e-7), ("minmod", 1e-4)])
def test_implicit_euler_newton_gmres(limiter, tol):
    """The finite-difference Jacobian (relative perturbation 1e-6) makes the implicit step sensitive
    to rounding: the reference's own step moves by 3e-9..9e-9 (smooth, no limiter) and by
    5e-6..1.3e-5 (Barth-Jespersen limiter, whose is_close(delta2, 0) switch sits at the
    perturbation's scale) when its input is perturbed by 1e-16 relative. The bars are ~10x those."""
    bcs = {s: ("farfield", FREE) for s in SIDES[:4]}
    rm, re, dm, de = pair((10, 8, 2), (0, 0, 0), (1, 1, 0.2), (0, 0, 1), bcs=bcs, limiter=limiter)
    prim = np.tile(np.array(FREE), (dm.num_cells, 1))
    rng = np.random.default_rng(4)
    prim[:, 0] *= 1 + 0.05 * rng.random(dm.num_cells)
    # step 1 starts from the same state: same CFL step
    (tr, sr, rr, pr), (td, sd, rd, pd) = run_both(re, de, prim, "implicit euler", 20.0, 1, nk=(0.1, 0.3, 10))
    assert abs(td - tr) <= 1e-13 * tr
    assert rel_l2(pd, pr).max() <= tol
    assert np.allclose(rd, rr, rtol=100 * tol)
    # two steps: the reference's own two-step result moves by 6e-5..1e-4 under a 1e-16 input
    # perturbation even without a limiter (Newton / GMRES stopping decisions of step 2 flip)
    (tr, sr, rr, pr), (td, sd, rd, pd) = run_both(re, de, prim, "implicit euler", 20.0, 2, nk=(0.1, 0.3, 10))
    assert abs(td - tr) <= tol * tr
    assert rel_l2(pd, pr).max() <= 1e-3


def test_run_matches_repeated_advance():
    m = tb.Mesh.create((0, 0, 0), (10, 10, 0.625), (16, 16, 4), (1, 1, 1))
    e1 = tb.Equations.euler(m)
    e1.set_initial_condition("domain", vortex)
    e2 = tb.Equations.euler(m)
    e2.set_initial_condition("domain", vortex)
    s1 = tb.Simulation(e1)
    s1.set_max_iter(7)
    t1 = s1.run()
    s2 = tb.Simulation(e2)
    t2 = 0.0
    for _ in range(7):
        t2, _, _ = s2.advance(t2)
    assert t1 == t2
    assert np.array_equal(e1.primitive[: m.num_inner_cells], e2.primitive[: m.num_inner_cells])


def test_run_stops_at_max_time_like_reference():
    rm, re, dm, de = pair((16, 16, 4), (0, 0, 0), (10, 10, 0.625), (1, 1, 1))
    prim = vortex(dm.cell_center)
    re.set_primitive(prim)
    de.primitive[:] = prim
    rsim = ref.RefSimulation(re, "lserk", 0.99)
    rsim.set_max_time(0.05)
    t_ref = rsim.run()
    dsim = tb.Simulation(de)
    dsim.set_max_time(0.05)
    t_dev = dsim.run()
    assert abs(t_dev - t_ref) <= 1e-14
    assert rel_l2(de.primitive[: dm.num_inner_cells], re.primitive[: dm.num_inner_cells]).max() <= TOL


def test_drop_in_advance_signature():
    """tg_teal_lserk called with teal's Advance signature on a bound `Equations *` key."""
    m = tb.Mesh.create((0, 0, 0), (10, 10, 0.625), (16, 16, 4), (1, 1, 1))
    e = tb.Equations.euler(m)
    e.set_initial_condition("domain", vortex)
    ctx = e.context()
    host = np.ascontiguousarray(e.primitive.copy())
    key = ctypes.c_void_p(12345)
    L = tb.lib
    assert L.tg_bind(key, ctx.handle, ctypes.c_void_p(host.ctypes.data)) == 0
    t = ctypes.c_double(0.0)
    res = np.zeros(5)
    rk = tb._lib.TgRungeKutta(2, 3)
    step0 = L.tg_teal_lserk(key, ctypes.byref(t), ctypes.c_void_p(res.ctypes.data), 1e300, 0.99,
                           ctypes.cast(ctypes.byref(rk), ctypes.c_void_p))
    assert step0 > 0 and t.value == step0
    assert not np.array_equal(host, e.primitive)  # the host array was refreshed in place
    L.tg_unbind(key)


def test_gradient_convergence_rate_on_device():
    """The reference's only numerical hot-path test (test/2_equations/gradient.c:27-104), on the
    device: LS gradients of a trigonometric velocity field converge at rate > 1.99."""
    fac = 2 * np.pi
    errs = []
    for n in (16, 32, 64):
        m = tb.Mesh.create((0, 0, 0), (1, 1, 1), (n, n, n), (1, 1, 1))
        e = tb.Equations.euler(m)
        e.set_limiter(None)
        c = m.cell_center

        def field(x):
            out = np.ones((x.shape[0], 5))
            out[:, 1] = np.sin(fac * x[:, 0]) * np.cos(fac * x[:, 1]) * np.cos(fac * x[:, 2])
            out[:, 2] = np.cos(fac * x[:, 0]) * np.sin(fac * x[:, 1]) * np.cos(fac * x[:, 2])
            out[:, 3] = 0.0
            return out

        e.set_initial_condition("domain", field)
        g = e.context().gradient()
        C = m.num_inner_cells
        x, y, z = c[:C, 0], c[:C, 1], c[:C, 2]
        ex = np.zeros((C, 3, 3))
        ex[:, 0] = np.stack([fac * np.cos(fac * x) * np.cos(fac * y) * np.cos(fac * z),
                             -fac * np.sin(fac * x) * np.sin(fac * y) * np.cos(fac * z),
                             -fac * np.sin(fac * x) * np.cos(fac * y) * np.sin(fac * z)], 1)
        ex[:, 1] = np.stack([-fac * np.sin(fac * x) * np.sin(fac * y) * np.cos(fac * z),
                             fac * np.cos(fac * x) * np.cos(fac * y) * np.cos(fac * z),
                             -fac * np.cos(fac * x) * np.sin(fac * y) * np.sin(fac * z)], 1)
        vol = m.cell_volume[:C]
        err = [np.sqrt((vol * ((g[:, 1 + k] - ex[:, k]) ** 2).sum(1)).sum() / m.sum_volume) for k in range(3)]
        errs.append(max(err))
    rate1 = np.log(errs[0] / errs[1]) / np.log(2)
    rate2 = np.log(errs[1] / errs[2]) / np.log(2)
    assert rate1 > 1.99 and rate2 > 1.99


def test_nonfinite_state_is_reported():
    m = tb.Mesh.create((0, 0, 0), (1, 1, 1), (6, 6, 6), (1, 1, 1))
    e = tb.Equations.euler(m)
    prim = random_state(m.num_cells, seed=1)
    prim[17, 4] = np.nan
    e.primitive[:] = prim
    s = tb.Simulation(e)
    with pytest.raises(tb.TealError) as info:
        s.advance(0.0)
    assert info.value.code == tb._lib.TG_ERR_NONFINITE


# ---- unstructured compression ramp: tetrahedra, prisms, hexahedra, pyramid transitions --------

M25 = (1.0, 2.5, 0.0, 0.0, 1.0 / GAMMA)
RAMP_BCS = {"left": ("supersonic inflow", M25), "right": ("supersonic outflow", None),
            "bottom": ("slipwall", None), "top": ("slipwall", None), "back": ("slipwall", None),
            "front": ("slipwall", None)}


def ramp_pair(spec, ns=False, flux="ausmd", limiter="minmod", coeff=0.0, mu=None, bcs=RAMP_BCS):
    cells = meshes.ramp_mesh(**spec)
    rm = ref.RefMesh.from_cells(cells)
    re = ref.RefEquations(rm, ns)
    dm = tb.Mesh.from_cells(cells)
    de = tb.Equations.navierstokes(dm) if ns else tb.Equations.euler(dm)
    for e in (re, de):
        e.set_convective_flux(flux)
        e.set_limiter(limiter, coeff)
        if ns and mu is not None:
            e.set_property("dynamic viscosity", mu)
        for entity, (name, ctx) in bcs.items():
            e.set_boundary_condition(entity, name, ctx)
    return rm, re, dm, de


def ramp_state(num_cells, seed, amp=0.05):
    prim = np.tile(np.array(M25), (num_cells, 1))
    rng = np.random.default_rng(seed)
    prim[:, 0] *= 1 + amp * rng.random(num_cells)
    prim[:, 1:4] += amp * (rng.random((num_cells, 3)) - 0.5)
    prim[:, 4] *= 1 + amp * rng.random(num_cells)
    return prim


@pytest.mark.parametrize("flux,limiter", [("ausmd", "minmod"), ("ausmdv", "venkatakrishnan"), ("roe", "minmod"),
                                          ("hllc", None)])
def test_unstructured_ramp_derivative(flux, limiter):
    rm, re, dm, de = ramp_pair(dict(n=(24, 16, 16), block=4, seed=3), flux=flux, limiter=limiter, coeff=1.0)
    check_derivative(re, de, ramp_state(dm.num_cells, 21))


def test_unstructured_ramp_lserk_steps():
    """The ramp workload (Mach 2.5, ausmd, Barth-Jespersen, supersonic inflow / outflow, slip walls)."""
    rm, re, dm, de = ramp_pair(dict(n=(24, 16, 16), block=8, seed=4))
    prim = ramp_state(dm.num_cells, 22, amp=0.0)
    (tr, sr, rr, pr), (td, sd, rd, pd) = run_both(re, de, prim, "lserk", 0.99, 20, rk=(3, 3))
    assert abs(td - tr) <= 1e-13 * tr
    assert rel_l2(pd, pr).max() <= TOL
    assert np.allclose(rd, rr, rtol=1e-9)


def test_unstructured_ramp_navierstokes_wall():
    bcs = {**RAMP_BCS, "bottom": ("adiabatic wall", None)}
    rm, re, dm, de = ramp_pair(dict(n=(16, 12, 10), block=4, seed=5), ns=True, flux="roe",
                               limiter="venkatakrishnan", coeff=1.0, mu=0.01, bcs=bcs)
    prim = ramp_state(dm.num_cells, 23)
    check_derivative(re, de, prim)
    (tr, sr, rr, pr), (td, sd, rd, pd) = run_both(re, de, prim, "lserk", 0.8, 5, rk=(3, 3))
    assert rel_l2(pd, pr).max() <= TOL


def test_unstructured_ramp_implicit_step():
    rm, re, dm, de = ramp_pair(dict(n=(12, 8, 6), block=4, seed=6), flux="roe", limiter=None)
    prim = ramp_state(dm.num_cells, 24)
    (tr, sr, rr, pr), (td, sd, rd, pd) = run_both(re, de, prim, "implicit euler", 20.0, 1, nk=(0.1, 0.3, 10))
    assert abs(td - tr) <= 1e-13 * tr
    # the reference's own step on this case moves by 4.4e-8..4.6e-8 under a 1e-16 relative input
    # perturbation (measured, three seeds); the bar is ~10x that
    assert rel_l2(pd, pr).max() <= 5e-7


# ---- device source terms (in place of the run cases' host callbacks) ---------------------------

def rayleigh_taylor_state(center, gravity=0.1):
    """Heavy over light fluid in hydrostatic balance with a small velocity perturbation (the shape
    of run/rayleigh_taylor_instability/run.c's initial condition)."""
    x, y = center[:, 0], center[:, 1]
    rho = np.where(y > 0, 2.0, 1.0)
    out = np.zeros((center.shape[0], 5))
    out[:, 0] = rho
    out[:, 2] = 0.01 * (1 + np.cos(4 * np.pi * x)) * (1 + np.cos(3 * np.pi * y)) / 4
    out[:, 4] = 2.5 - gravity * rho * y
    return out


def test_source_body_force_rayleigh_taylor():
    bcs = {"bottom": ("slipwall", None), "top": ("slipwall", None)}
    rm, re, dm, de = pair((16, 48, 2), (-0.25, -0.75, 0), (0.25, 0.75, 0.05), (1, 0, 1), bcs=bcs)
    for e in (re, de):
        e.set_source("body force", (0.0, -0.1, 0.0))
    prim = rayleigh_taylor_state(dm.cell_center)
    check_derivative(re, de, prim)
    (tr, sr, rr, pr), (td, sd, rd, pd) = run_both(re, de, prim, "lserk", 0.5, 10, rk=(3, 3))
    assert rel_l2(pd, pr).max() <= TOL
    assert abs(td - tr) <= 1e-13 * tr


def test_source_bulk_forcing_channel():
    """Bulk forcing with the periodic hill's constants (target 1, time scale 0.001) on a walled
    channel: the prepare pass averages the state being differentiated, on the device."""
    bcs = {"bottom": ("wall", None), "top": ("wall", None)}
    rm, re, dm, de = pair((18, 10, 2), (0, 0, 0), (9, 3, 0.3), (1, 0, 1), ns=True, flux="roe",
                          limiter="venkatakrishnan", coeff=1.0, mu=0.01, bcs=bcs)
    for e in (re, de):
        e.set_source("bulk forcing", (1.0, 0.001))
    prim = random_state(dm.num_cells, seed=41, mach=0.4)
    check_derivative(re, de, prim)
    (tr, sr, rr, pr), (td, sd, rd, pd) = run_both(re, de, prim, "lserk", 0.3, 5, rk=(3, 3))
    assert rel_l2(pd, pr).max() <= TOL


def test_source_in_a_batch_is_bit_identical_to_solo():
    def problem(n):
        m = tb.Mesh.create((-0.25, -0.75, 0), (0.25, 0.75, 0.05), (n, 3 * n, 2), (1, 0, 1))
        e = tb.Equations.euler(m)
        for side in ("bottom", "top"):
            e.set_boundary_condition(side, "slipwall")
        e.set_source("body force", (0.0, -0.1, 0.0))
        e.set_initial_condition("domain", rayleigh_taylor_state)
        return e

    ps = [problem(8), problem(12)]
    b = tb.Batch(ps)
    t, it, res = b.run(tb.TG_ADVANCE_LSERK, 0.5, [4, 6], context=(3, 3))
    for i, e in enumerate(ps):
        ctx = tb.Context(e.mesh, e)
        ctx.set_primitive(e.primitive)
        t1, it1, res1 = ctx.run(tb.TG_ADVANCE_LSERK, 0.5, [4, 6][i], context=(3, 3))
        C = e.mesh.num_inner_cells
        assert t[i] == t1 and np.array_equal(res[i], res1)
        assert np.array_equal(b.get_primitive(i)[:C], ctx.get_primitive()[:C])


@pytest.mark.parametrize("n,periodic,ns", [((2, 2, 2), (1, 1, 1), True), ((2, 1, 1), (1, 1, 1), False),
                                           ((3, 1, 1), (0, 0, 0), False), ((4, 3, 1), (1, 0, 0), True),
                                           ((5, 2, 1), (0, 1, 0), False)])
def test_tiny_and_degenerate_meshes(n, periodic, ns):
    """Meshes of 2 to 12 cells: a cell whose neighbours across two faces are the same cell (periodic
    with 2 cells per axis), and one- and two-dimensional boxes (axes of one cell have no faces, so
    cells have 2 or 4 slots and the least-squares system is degenerate, teal's is_close tests
    skipping the empty directions)."""
    rm = ref.RefMesh((0, 0, 0), (1, 1, 1), n, periodic)
    a = rm.arrays()
    boundaries = [name for name, _, _ in rm.entities()][a["num_inner_entities"]:a["off_boundary_entities"]]
    bcs = {name: ("wall" if ns else "slipwall", None) for name in boundaries}
    rm, re, dm, de = pair(n, (0, 0, 0), (1, 1, 1), periodic, ns=ns, flux="hllc", limiter="venkatakrishnan",
                          coeff=1.0, mu=0.01 if ns else None, bcs=bcs)
    prim = random_state(dm.num_cells, seed=17, mach=0.5)
    check_derivative(re, de, prim)
    (tr, sr, rr, pr), (td, sd, rd, pd) = run_both(re, de, prim, "lserk", 0.5, 5, rk=(3, 3))
    assert abs(td - tr) <= 1e-13 * tr
    assert rel_l2(pd, pr).max() <= TOL


def test_mesh_without_faces_is_rejected():
    """A single non-periodic cell has no faces in teal's construction (its face cells pair with
    nothing); the device library refuses such a mesh instead of evaluating an empty residual."""
    m = tb.Mesh.create((0, 0, 0), (1, 1, 1), (1, 1, 1), (0, 0, 0))
    assert m.struct.num_faces == 0
    e = tb.Equations.euler(m)
    with pytest.raises(tb.TealError):
        e.context()
