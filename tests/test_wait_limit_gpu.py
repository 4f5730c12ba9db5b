"""Bounded device-side waits and loops, made to run out without a fault.

The staged kernels (the gradient kernel, whose tile of slot geometry arrives by bulk copies completing
on an mbarrier, and the Euler form's face-flux kernel, whose geometry tile does) poll the barrier a
bounded number of times. tg_set_wait_limit lowers that bound; at 0 every block gives up at once, sets
ERR_TIMEOUT in the context's error word, waits (with the full bound) for its own copies to land and
returns. The call must report TG_ERR_TIMEOUT, and the same context must then evaluate the residual
exactly as a fresh one does: no hang, no trap, no lost context.
"""

import numpy as np
import pytest

import teal_b200 as tb
from teal_b200 import _lib
from teal_b200 import TealError
from tests.cases import vortex

pytestmark = pytest.mark.gpu


def vortex_context(physics="euler"):
    m = tb.Mesh.create((0, 0, 0), (10, 10, 0.625), (16, 16, 4), (1, 1, 1))
    # Euler: the face kernel stages its geometry too (tuned.h); Navier-Stokes: only the gradient
    e = tb.Equations.euler(m) if physics == "euler" else tb.Equations.navierstokes(m)
    return m, e, tb.Context(m, e)


@pytest.mark.parametrize("physics", ["euler", "navierstokes"])
def test_wait_that_runs_out_reports_timeout_and_leaves_the_context_usable(physics):
    m, e, ctx = vortex_context(physics)
    try:
        prim = vortex(m.cell_center)
        expect = ctx.derivative(prim)
        ctx.set_wait_limit(0)
        with pytest.raises(TealError) as err:
            ctx.derivative(prim)
        assert err.value.code == _lib.TG_ERR_TIMEOUT
        assert b"gave up" in _lib.lib.tg_last_error()
        # again: the error word was cleared, so the next give-up is reported afresh
        with pytest.raises(TealError) as err:
            ctx.derivative(prim)
        assert err.value.code == _lib.TG_ERR_TIMEOUT
        ctx.set_wait_limit()  # back to the default bound
        assert np.array_equal(ctx.derivative(prim), expect)
        # whole steps replayed from the step graph after the limit changed back
        ctx.set_primitive(prim)
        t, it, res = ctx.run(tb.TG_ADVANCE_LSERK, 0.5, 3, context=(3, 3))
        assert it == 3 and np.all(np.isfinite(res))
    finally:
        ctx.close()


def test_wait_limit_rejects_negative_polls():
    m, e, ctx = vortex_context()
    try:
        with pytest.raises(TealError) as err:
            ctx.set_wait_limit(-1)
        assert err.value.code == _lib.TG_ERR_INVALID
    finally:
        ctx.close()


def test_newton_loop_of_the_step_graph_is_bounded():
    """The implicit step's Newton loop runs on the device (a conditional node of the step's graph).
    With a Newton tolerance no iteration can meet, teal's own bound (128 (cells + 1) iterations)
    would keep the device busy for a long time; the graph stops after 1000 iterations and the call
    reports TG_ERR_TIMEOUT. The context then takes a normal implicit step."""
    m, e, ctx = vortex_context()
    try:
        prim = vortex(m.cell_center)
        ctx.set_primitive(prim)
        with pytest.raises(TealError) as err:
            ctx.advance(tb.TG_ADVANCE_IMPLICIT_EULER, 5.0, 0.0, context=(1e-300, 0.3, 2))
        assert err.value.code == _lib.TG_ERR_TIMEOUT
        assert b"Newton iterations" in _lib.lib.tg_last_error()
        ctx.set_primitive(prim)
        t, s0, res = ctx.advance(tb.TG_ADVANCE_IMPLICIT_EULER, 5.0, 0.0, context=(0.1, 0.3, 10))
        assert t > 0 and np.all(np.isfinite(res))
    finally:
        ctx.close()
