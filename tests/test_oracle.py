"""The CPU restatement (oracle/liboracle.so) pinned against the reference: bit for bit against the
golden vectors written by the reference solver, and live against oracle/_ref when it is built."""

import numpy as np
import pytest

from oracle import port, ref
from tests import golden_cases
from tests.cases import random_state, rel_l2

GOLDEN = golden_cases.load()
pytestmark = pytest.mark.skipif(not port.available(), reason="oracle/liboracle.so not built")


@pytest.mark.parametrize("name", sorted(GOLDEN))
def test_port_reproduces_golden_bit_for_bit(name):
    g = GOLDEN[name]
    case = g["case"]
    m, e = golden_cases.equations(case)
    P = port.Port(m, e)
    prim = g["primitive"]
    assert np.array_equal(P.derivative(prim), g["derivative"])
    assert P.timestep(prim) == float(g["timestep"])
    assert np.array_equal(P.residual(g["derivative"]), g["residual"])
    C = m.num_inner_cells
    if "gradient" in g:
        assert np.array_equal(P.gradient(prim)[:C], g["gradient"])
        if case["limiter"]:
            assert np.array_equal(P.gradient(prim, limited=True)[:C], g["gradient_limited"])
    adv = case.get("advance")
    if adv:
        method = {"lserk": "lserk", "euler": "euler", "implicit euler": "implicit"}[adv["method"]]
        s, t, s0, r = P.advance(prim, method, adv["courant"], adv["steps"], rk=adv.get("rk"), nk=adv.get("nk"))
        assert np.array_equal(s[:C], g["advance_state"])
        assert t == float(g["advance_time"])
        assert np.array_equal(r, g["advance_residual"])


@pytest.mark.skipif(not ref.available(), reason="reference oracle not built")
@pytest.mark.parametrize("flux", ["roe", "hllc", "ausmdv"])
def test_port_matches_live_reference(flux):
    import teal_b200 as tb

    lo, hi, n, per = (0, 0, 0), (1, 2, 1), (9, 7, 5), (1, 0, 1)
    rm = ref.RefMesh(lo, hi, n, per)
    re = ref.RefEquations(rm, True)
    m = tb.Mesh.create(lo, hi, n, per)
    e = tb.Equations.navierstokes(m)
    for q in (re, e):
        q.set_convective_flux(flux)
        q.set_limiter("venkatakrishnan", 2.0)
        q.set_property("dynamic viscosity", 0.02)
        q.set_boundary_condition("bottom", "wall")
        q.set_boundary_condition("top", "farfield", (1.0, 0.3, 0.0, 0.0, 0.7))
    prim = random_state(m.num_cells, seed=31, mach=0.7)
    assert np.array_equal(port.Port(m, e).derivative(prim), re.derivative(prim))


def test_rel_l2_helper():
    a = np.ones((4, 5))
    b = a.copy()
    b[0, 0] += 1e-3
    err = rel_l2(b, a)
    assert err[0] == pytest.approx(1e-3 / 2)
    assert (err[1:] == 0).all()
