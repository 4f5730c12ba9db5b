"""tg_advance_host: one step from a host state to a host state with the download overlapped with the
step's last stage (its face fluxes and cell updates in chunks of cells, each chunk copied down as
soon as it is final). Every element is computed by the same kernels as in tg_set_primitive +
tg_advance + tg_get_primitive, so states, times, steps and residuals must be the same bits: on
periodic boxes (Taylor-Green, Navier-Stokes), on the unstructured ramp with boundary ghosts (Euler),
in the FP32-flux and exact forms, for one-stage Euler and several Runge-Kutta tables, into pinned
(chunked) and pageable (one piece) host memory, and over several steps where each step's output is
the next one's input."""

import numpy as np
import pytest

import teal_b200 as tb
from teal_b200 import meshes
from tests.cases import taylor_green

pytestmark = pytest.mark.gpu

M25 = np.array([1.0, 2.5, 0.0, 0.0, 1.0 / 1.4])


def tgv(n=32):
    m = tb.Mesh.create((0, 0, 0), (2 * np.pi,) * 3, (n, n, n), (1, 1, 1))
    e = tb.Equations.navierstokes(m)
    e.set_convective_flux("roe")
    e.set_limiter("venkatakrishnan", 1.0)
    e.set_property("dynamic viscosity", 1 / 1600)
    e.primitive[:] = taylor_green(m.cell_center)
    return e


def ramp(n=(24, 20, 16)):
    m = tb.Mesh.from_cells(meshes.ramp_mesh(n=n, block=4, seed=3))
    e = tb.Equations.euler(m)
    e.set_convective_flux("ausmd")
    e.set_limiter("minmod")
    e.set_boundary_condition("left", "supersonic inflow", M25)
    e.set_boundary_condition("right", "supersonic outflow")
    for side in ("bottom", "top", "back", "front"):
        e.set_boundary_condition(side, "slipwall")
    e.primitive[:] = M25
    rng = np.random.default_rng(4)
    e.primitive[: m.num_inner_cells, 0] *= 1 + 0.05 * rng.random(m.num_inner_cells)
    return e


def host(shape, pinned):
    if not pinned:
        return np.zeros(shape)
    import torch

    return torch.zeros(shape, dtype=torch.float64, pin_memory=True).numpy()


def run_pair(e, precision, method, rk, steps, pinned):
    """The same steps through tg_advance_host and through the three calls, each step's output the
    next step's input; returns both histories of (time, step0, residual, state)."""
    ctx = e.context(precision)
    start = ctx.get_primitive()
    out = []
    for overlap in (False, True):
        state = host(start.shape, pinned)
        nxt = host(start.shape, pinned)
        state[:] = start
        t = 0.0
        hist = []
        for _ in range(steps):
            if overlap:
                t, s0, res = ctx.advance_host(method, 0.9, t, prim_in=state, prim_out=nxt, context=rk)
            else:
                ctx.set_primitive(state)
                t, s0, res = ctx.advance(method, 0.9, t, context=rk)
                ctx.get_primitive(nxt)
            hist.append((t, s0, res.copy(), nxt.copy()))
            state, nxt = nxt, state
        out.append(hist)
    return out


def assert_same(a, b):
    assert len(a) == len(b)
    for (ta, sa, ra, qa), (tb_, sb, rb, qb) in zip(a, b):
        assert ta == tb_ and sa == sb
        assert np.array_equal(ra, rb)
        assert np.array_equal(qa, qb)


@pytest.mark.parametrize("precision", [tb.TG_PRECISION_FP64, tb.TG_PRECISION_FP32_FLUX, tb.TG_PRECISION_FP64_EXACT],
                         ids=["fp64", "fp32-flux", "exact"])
def test_taylor_green_overlapped_step_equals_the_three_calls(precision):
    seq, ovl = run_pair(tgv(), precision, tb.TG_ADVANCE_LSERK, (3, 3), 3, pinned=True)
    assert_same(seq, ovl)


@pytest.mark.parametrize("method,rk", [(tb.TG_ADVANCE_LSERK, (3, 3)), (tb.TG_ADVANCE_LSERK, (3, 5)),
                                       (tb.TG_ADVANCE_EULER, None)], ids=["rk33", "rk35", "euler"])
@pytest.mark.parametrize("pinned", [True, False], ids=["pinned", "pageable"])
def test_ramp_overlapped_step_equals_the_three_calls(method, rk, pinned):
    seq, ovl = run_pair(ramp(), tb.TG_PRECISION_FP64, method, rk, 3, pinned)
    assert_same(seq, ovl)


def test_resident_state_and_no_readback():
    # prim_in None: the step starts from the resident state; prim_out None: nothing is read back
    e = tgv(24)
    ctx = e.context()
    start = ctx.get_primitive()
    t1, s1, r1 = ctx.advance(tb.TG_ADVANCE_LSERK, 0.9, 0.0, context=(3, 3))
    want = ctx.get_primitive()
    ctx.set_primitive(start)
    t2, s2, r2 = ctx.advance_host(tb.TG_ADVANCE_LSERK, 0.9, 0.0, context=(3, 3))
    assert (t1, s1) == (t2, s2) and np.array_equal(r1, r2)
    assert np.array_equal(ctx.get_primitive(), want)
    got = np.zeros_like(want)
    ctx.set_primitive(start)
    ctx.advance_host(tb.TG_ADVANCE_LSERK, 0.9, 0.0, prim_out=got, context=(3, 3))
    assert np.array_equal(got, want)


def test_implicit_method_and_shape_errors():
    e = ramp((12, 10, 8))
    ctx = e.context()
    start = ctx.get_primitive()
    nk = (0.1, 0.3, 10)
    ctx.set_primitive(start)
    t1, s1, r1 = ctx.advance(tb.TG_ADVANCE_IMPLICIT_EULER, 5.0, 0.0, context=nk)
    want = ctx.get_primitive()
    got = np.zeros_like(want)
    t2, s2, r2 = ctx.advance_host(tb.TG_ADVANCE_IMPLICIT_EULER, 5.0, 0.0, prim_in=start, prim_out=got, context=nk)
    assert (t1, s1) == (t2, s2) and np.array_equal(r1, r2) and np.array_equal(got, want)
    with pytest.raises(tb.TealError):
        ctx.advance_host(tb.TG_ADVANCE_LSERK, 0.9, 0.0, prim_in=start[:10])
    with pytest.raises(tb.TealError):
        ctx.advance_host(tb.TG_ADVANCE_LSERK, 0.9, 0.0, prim_out=np.zeros((want.shape[0], 5), np.float32))


def test_one_chunk_mesh_and_batch_rejection():
    # a mesh too small to split (one chunk) takes the same path with a single chunk
    seq, ovl = run_pair(tgv(8), tb.TG_PRECISION_FP64, tb.TG_ADVANCE_LSERK, (3, 3), 2, pinned=True)
    assert_same(seq, ovl)
    # a batch arena has no single host state
    import ctypes

    from teal_b200 import _lib

    b = tb.Batch([tgv(8), tgv(8)])
    t = ctypes.c_double(0.0)
    status = _lib.lib.tg_advance_host(b.handle, tb.TG_ADVANCE_LSERK, None, 0.9, ctypes.byref(t), 1e300, None, None,
                                      None, None)
    assert status == _lib.TG_ERR_INVALID
    b.close()
