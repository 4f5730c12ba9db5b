"""C ABI: the library loads, exports every declared entry point, and selects teal's plugin names."""

import os
import re

import pytest

import teal_b200 as tb
from teal_b200 import _lib

HEADER = os.path.join(os.path.dirname(os.path.dirname(__file__)), "include", "teal_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z_0-9]*\s*\**\s*(tg_[a-z_0-9]+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_every_declared_symbol_is_exported():
    names = declared_functions()
    assert len(names) >= 25
    for n in names:
        assert hasattr(_lib.lib, n), n


def test_every_declared_symbol_has_a_binding():
    bound = {n for n, _, _ in _lib.SIGNATURES}
    assert set(declared_functions()) <= bound


@pytest.mark.parametrize("name,kind", [
    ("roe", 1), ("hll", 2), ("hllc", 3), ("hlle", 4), ("ausmd", 5), ("ausmdv", 6), ("lxf", 7), ("central", 8),
    ("godunov", -1), ("AUSM", -1), ("", -1)])
def test_convective_select(name, kind):
    assert _lib.lib.tg_convective_select(name.encode()) == kind


def test_limiter_and_viscous_select():
    L = _lib.lib
    assert L.tg_limiter_select(b"minmod") == 1
    assert L.tg_limiter_select(b"barth jespersen") == 1
    assert L.tg_limiter_select(b"venkatakrishnan") == 2
    assert L.tg_limiter_select(b"superbee") == -1
    assert L.tg_viscous_select(b"central") == 1
    assert L.tg_viscous_select(b"upwind") == -1


def test_boundary_select_follows_the_plugin():
    L = _lib.lib
    assert L.tg_boundary_select(b"slipwall", 0) == L.tg_boundary_select(b"symmetry", 0) == 1
    assert L.tg_boundary_select(b"farfield", 0) == 7
    assert L.tg_boundary_select(b"wall", 0) == -1          # Euler has no wall
    assert L.tg_boundary_select(b"wall", 1) == 8           # Navier-Stokes adiabatic wall
    assert L.tg_boundary_select(b"adiabatic wall", 1) == 8
    assert L.tg_boundary_select(b"supersonic inflow", 1) == 2  # falls back to the Euler BCs


def test_advance_select():
    L = _lib.lib
    assert L.tg_advance_select(b"euler") == 0
    assert L.tg_advance_select(b"lserk") == 1
    assert L.tg_advance_select(b"implicit euler") == 2
    assert L.tg_advance_select(b"rk4") == -1


def test_api_errors_mirror_teal_messages():
    m = tb.Mesh.create((0, 0, 0), (1, 1, 1), (4, 4, 4), (1, 1, 1))
    e = tb.Equations.euler(m)
    with pytest.raises(tb.TealError, match="invalid convective flux"):
        e.set_convective_flux("godunov")
    with pytest.raises(tb.TealError, match="invalid limiter"):
        e.set_limiter("superbee")
    with pytest.raises(tb.TealError, match="invalid property"):
        e.set_property("dynamic viscosity", 1.0)  # Euler has no viscosity
    with pytest.raises(tb.TealError, match="invalid viscous flux"):
        e.set_viscous_flux("central")
    s = tb.Simulation(e)
    with pytest.raises(tb.TealError, match="invalid number of stages"):
        s.set_advance("lserk", 0.5, (3, 7))
    with pytest.raises(tb.TealError, match="invalid advance method"):
        s.set_advance("rk4", 0.5)
    s.set_termination("momentum-y", 1e-6)
    assert s.variable == 2
    s.set_termination("energy", 1e-6)
    assert s.variable == 4


def test_create_rejects_invalid_input_before_touching_a_device():
    m = tb.Mesh.create((0, 0, 0), (1, 1, 1), (4, 4, 4), (1, 1, 1))
    e = tb.Equations.euler(m)
    s = e.struct()
    s.space_order = 3
    h = _lib.ctypes.c_void_p()
    st = _lib.lib.tg_create(_lib.ctypes.byref(m.struct), _lib.ctypes.byref(s), 0, _lib.ctypes.byref(h))
    assert st == _lib.TG_ERR_INVALID
    assert b"space order" in _lib.lib.tg_last_error()


def test_source_select():
    assert _lib.lib.tg_source_select(b"body force") == _lib.TG_SOURCE_BODY_FORCE
    assert _lib.lib.tg_source_select(b"bulk forcing") == _lib.TG_SOURCE_BULK_FORCING
    assert _lib.lib.tg_source_select(b"gravity") == -1
