"""The batched form: several meshes packed into one arena. Every instance must give the same bits
it gives alone (same face order inside each face class, reduction pieces aligned to instance
starts), stop on its own limits, and match the reference solver."""

import numpy as np
import pytest

import teal_b200 as tb
from oracle import ref
from tests.cases import rel_l2, vortex

pytestmark = pytest.mark.gpu

FREE = (1.0, 0.6, 0.1, -0.05, 1.0 / 1.4)


def vortex_problem(n):
    m = tb.Mesh.create((0, 0, 0), (10, 10, 0.625), (n, n, 4), (1, 1, 1))
    e = tb.Equations.euler(m)
    e.set_initial_condition("domain", vortex)
    return e


def channel_problem(nx, ny, mach, seed):
    m = tb.Mesh.create((0, 0, 0), (2, 1, 0.25), (nx, ny, 2), (0, 0, 1))
    e = tb.Equations.euler(m)
    free = np.array([1.0, mach * 1.183216, 0.1 * mach, 0.0, 1.0])
    for side in ("left", "right", "bottom", "top"):
        e.set_boundary_condition(side, "farfield", free)
    rng = np.random.default_rng(seed)
    prim = np.tile(free, (m.num_cells, 1))
    prim[:, 0] *= 1 + 0.05 * rng.random(m.num_cells)
    e.primitive[:] = prim
    return e


def problems():
    return [vortex_problem(16), channel_problem(12, 7, 0.5, 1), vortex_problem(24), channel_problem(9, 9, 2.0, 2)]


def alone(e, steps, courant=0.5):
    ctx = tb.Context(e.mesh, e)
    ctx.set_primitive(e.primitive)
    t, it, res = ctx.run(tb.TG_ADVANCE_LSERK, courant, steps, context=(3, 3))
    return t, it, res, ctx.get_primitive()


def test_batch_instances_are_bit_identical_to_solo_runs():
    ps = problems()
    steps = [7, 5, 9, 3]
    b = tb.Batch(ps)
    t, it, res = b.run(tb.TG_ADVANCE_LSERK, 0.5, steps, context=(3, 3))
    assert list(it) == steps
    for i, e in enumerate(ps):
        t1, it1, res1, p1 = alone(e, steps[i])
        C = e.mesh.num_inner_cells
        got = b.get_primitive(i)
        assert it1 == steps[i]
        assert t[i] == t1
        assert np.array_equal(res[i], res1)
        assert np.array_equal(got[:C], p1[:C])
        assert np.array_equal(got, p1)  # ghost rows too


def test_batch_fp32_flux_instances_are_bit_identical_to_solo_runs():
    """The FP32-flux form too: each instance's reference pressure is its own (its first cell), the
    same in the arena as alone."""
    fp32 = tb.TG_PRECISION_FP32_FLUX
    ps = problems()
    steps = [6, 4, 5, 3]
    b = tb.Batch(ps, precision=fp32)
    t, it, res = b.run(tb.TG_ADVANCE_LSERK, 0.5, steps, context=(3, 3))
    for i, e in enumerate(ps):
        ctx = tb.Context(e.mesh, e, precision=fp32)
        ctx.set_primitive(e.primitive)
        t1, it1, res1 = ctx.run(tb.TG_ADVANCE_LSERK, 0.5, steps[i], context=(3, 3))
        assert t[i] == t1
        assert np.array_equal(res[i], res1)
        assert np.array_equal(b.get_primitive(i), ctx.get_primitive())


def test_batch_stops_each_instance_on_its_own_limits():
    ps = problems()
    b = tb.Batch(ps)
    # instance 0: time limit; 1: residual threshold; 2, 3: iteration limits
    t, it, res = b.run(tb.TG_ADVANCE_LSERK, 0.5, [1000, 1000, 4, 6], max_time=[0.05, 1e300, 1e300, 1e300],
                       threshold=[0, 0.5 * 1e9, 0, 0], context=(3, 3))
    assert abs(t[0] - 0.05) <= 1e-12
    assert it[1] == 1  # the first residual is already below the (huge) threshold
    assert it[2] == 4 and it[3] == 6


def test_batch_matches_reference():
    sizes = [(12, 12, 4), (20, 14, 4)]
    ps, refs = [], []
    for n in sizes:
        m = tb.Mesh.create((0, 0, 0), (10, 10, 0.625), n, (1, 1, 1))
        e = tb.Equations.euler(m)
        e.set_initial_condition("domain", vortex)
        ps.append(e)
        rm = ref.RefMesh((0, 0, 0), (10, 10, 0.625), n, (1, 1, 1))
        re = ref.RefEquations(rm, False)
        re.set_primitive(e.primitive)
        refs.append(re)
    b = tb.Batch(ps)
    t, it, res = b.run(tb.TG_ADVANCE_LSERK, 0.5, 5, context=(3, 3))
    for i, re in enumerate(refs):
        rs = ref.RefSimulation(re, "lserk", 0.5, rk=(3, 3))
        tr = 0.0
        for _ in range(5):
            tr, _, rr = rs.advance(tr)
        C = ps[i].mesh.num_inner_cells
        assert rel_l2(b.get_primitive(i)[:C], re.primitive[:C]).max() <= 1e-12
        assert abs(t[i] - tr) <= 1e-13 * tr


def test_batch_rejects_mixed_lanes():
    a = vortex_problem(8)
    c = vortex_problem(8)
    c.set_convective_flux("roe")
    with pytest.raises(tb.TealError, match="differs"):
        tb.Batch([a, c])


@pytest.mark.parametrize("method", ["lserk", "implicit"])
def test_an_instance_that_goes_non_finite_stops_alone(method):
    """An instance whose state holds a non-finite value stops on its own; the others run to their
    limits with the same bits as alone, the batch call succeeds, and tg_batch_status names the failed
    one. A new state lets it run again."""
    ps = [channel_problem(12, 7, 0.5, 1), channel_problem(9, 9, 2.0, 2), channel_problem(10, 8, 0.8, 3)]
    bad = ps[1].primitive.copy()
    bad[5, 0] = np.nan
    b = tb.Batch(ps)
    b.set_primitive(1, bad)
    if method == "lserk":
        m, cfl, steps, ctx = tb.TG_ADVANCE_LSERK, 0.5, 6, (3, 3)
    else:
        m, cfl, steps, ctx = tb.TG_ADVANCE_IMPLICIT_EULER, 20.0, 3, NK
    t, it, res = b.run(m, cfl, steps, context=ctx)
    assert b.status().tolist() == [0, 4, 0]  # TG_OK, TG_ERR_NONFINITE, TG_OK
    for i in (0, 2):
        e = ps[i]
        one = tb.Context(e.mesh, e)
        one.set_primitive(e.primitive)
        t1, it1, res1 = one.run(m, cfl, steps, context=ctx)
        assert it[i] == it1 == steps
        assert t[i] == t1
        assert np.array_equal(b.get_primitive(i), one.get_primitive())
        one.close()
    assert it[1] < steps
    b.set_primitive(1, ps[1].primitive)
    t, it, res = b.run(m, cfl, 1, context=ctx)
    assert b.status().tolist() == [0, 0, 0]
    assert np.all(np.isfinite(res))
    # a single-mesh context reports the same condition as an error
    one = tb.Context(ps[1].mesh, ps[1])
    one.set_primitive(bad)
    with pytest.raises(tb.TealError) as err:
        one.run(m, cfl, 2, context=ctx)
    assert err.value.code == 4
    one.close()


# ---- batched implicit Euler (Jacobian-free Newton-GMRES per instance) ---------------------------

IMPLICIT_SPECS = [(10, 8, 0.5, 1), (14, 6, 1.5, 2), (7, 9, 0.8, 3)]  # nx, ny, Mach, seed
NK = (0.1, 0.3, 10)


def farfield_free(mach):
    return np.array([1.0, mach * 1.183216, 0.1 * mach, 0.0, 1.0 / 1.4])


def farfield_state(num_cells, mach, seed):
    rng = np.random.default_rng(seed)
    prim = np.tile(farfield_free(mach), (num_cells, 1))
    prim[:, 0] *= 1 + 0.05 * rng.random(num_cells)
    return prim


def farfield_problem(nx, ny, mach, seed):
    m = tb.Mesh.create((0, 0, 0), (1, 1, 0.2), (nx, ny, 2), (0, 0, 1))
    e = tb.Equations.euler(m)
    e.set_limiter(None, 0.0)
    for side in ("left", "right", "bottom", "top"):
        e.set_boundary_condition(side, "farfield", farfield_free(mach))
    e.primitive[:] = farfield_state(m.num_cells, mach, seed)
    return e


def farfield_reference(nx, ny, mach, seed):
    rm = ref.RefMesh((0, 0, 0), (1, 1, 0.2), (nx, ny, 2), (0, 0, 1))
    re = ref.RefEquations(rm, False)
    re.set_limiter(None, 0.0)
    for side in ("left", "right", "bottom", "top"):
        re.set_boundary_condition(side, "farfield", farfield_free(mach))
    re.set_primitive(farfield_state(rm.counts()["num_cells"], mach, seed))
    return re


def test_batch_implicit_instances_are_bit_identical_to_solo_runs():
    ps = [farfield_problem(*spec) for spec in IMPLICIT_SPECS]
    steps = [3, 1, 2]
    b = tb.Batch(ps)
    t, it, res = b.run(tb.TG_ADVANCE_IMPLICIT_EULER, 20.0, steps, context=NK)
    assert list(it) == steps
    for i, e in enumerate(ps):
        ctx = tb.Context(e.mesh, e)
        ctx.set_primitive(e.primitive)
        t1, it1, res1 = ctx.run(tb.TG_ADVANCE_IMPLICIT_EULER, 20.0, steps[i], context=NK)
        C = e.mesh.num_inner_cells
        assert it1 == steps[i]
        assert t[i] == t1
        assert np.array_equal(res[i], res1)
        assert np.array_equal(b.get_primitive(i)[:C], ctx.get_primitive()[:C])


def test_batch_implicit_matches_reference():
    """Two implicit steps of each instance against the reference. No limiter; the reference's own
    two-step result moves by up to 1e-4 under a 1e-16 relative input perturbation (Newton / GMRES
    stopping decisions of step 2 flip), so the bar is 1e-3, as for the single-mesh test."""
    specs = IMPLICIT_SPECS[:2]
    ps = [farfield_problem(*spec) for spec in specs]
    b = tb.Batch(ps)
    t, it, res = b.run(tb.TG_ADVANCE_IMPLICIT_EULER, 20.0, 2, context=NK)
    for i, spec in enumerate(specs):
        re = farfield_reference(*spec)
        rs = ref.RefSimulation(re, "implicit euler", 20.0, nk=NK)
        tr = 0.0
        for _ in range(2):
            tr, _, rr = rs.advance(tr)
        C = ps[i].mesh.num_inner_cells
        assert rel_l2(b.get_primitive(i)[:C], re.primitive[:C]).max() <= 1e-3
        assert abs(t[i] - tr) <= 1e-3 * tr
