"""Device functions (teal's Compute callbacks as CUDA C, compiled with NVRTC): registration and the
host-side API. Compiling needs no GPU; binding and running are in test_device_functions_gpu.py."""

import ctypes

import numpy as np
import pytest

import teal_b200 as tb
from teal_b200 import _lib
from tests.device_functions import AVERAGE_PROBE, HILL_FORCING, MOVING_WALL, UNSTEADY_INFLOW, UNSTEADY_SOURCE


def test_register_compiles():
    tb.register_function("lid_wall", "boundary", MOVING_WALL)
    tb.register_function("unsteady_inflow", "boundary", UNSTEADY_INFLOW)
    tb.register_function("unsteady_source", "source", UNSTEADY_SOURCE)
    tb.register_function("hill_forcing", "source", HILL_FORCING)
    tb.register_function("average_probe", "source", AVERAGE_PROBE)


def test_compile_error_carries_the_log():
    with pytest.raises(tb.TealError) as err:
        tb.register_function("broken", "boundary", "__device__ void broken(double *o) { o[0] = undefined_name; }")
    assert err.value.code == _lib.TG_ERR_INVALID
    assert "does not compile" in str(err.value) and "undefined_name" in str(err.value)


def test_signature_mismatch_is_a_compile_error():
    # the wrapper calls the function with teal's five Compute arguments
    with pytest.raises(tb.TealError):
        tb.register_function("short_args", "source", "__device__ void short_args(double *o) { o[0] = 0; }")


@pytest.mark.parametrize("name", ["tg_mine", "1abc", "a-b", "", "x" * 65])
def test_invalid_names(name):
    with pytest.raises(tb.TealError):
        tb.register_function(name, "boundary", MOVING_WALL)


def test_invalid_kind():
    with pytest.raises(tb.TealError):
        tb.register_function("lid_wall", "flux", MOVING_WALL)
    log = ctypes.create_string_buffer(64)
    assert _lib.lib.tg_function_register(b"lid_wall", 7, MOVING_WALL.encode(), log, 64) == _lib.TG_ERR_INVALID


def test_select_names():
    assert _lib.lib.tg_boundary_select(b"custom", _lib.TG_EULER) == _lib.TG_BC_CUSTOM
    assert _lib.lib.tg_source_select(b"device function") == _lib.TG_SOURCE_DEVICE


def test_equations_api_requires_a_function_for_custom_kinds():
    m = tb.Mesh.create((0, 0, 0), (1, 1, 0.25), (4, 4, 2), (0, 0, 1))
    e = tb.Equations.euler(m)
    with pytest.raises(tb.TealError):
        e.set_boundary_condition("top", "custom")
    with pytest.raises(tb.TealError):
        e.set_boundary_condition("top", "slipwall", compute="lid_wall")
    e.set_boundary_condition("top", "custom", compute="lid_wall")
    i = [n for n, _, _ in m.entities].index("top") - m.struct.num_inner_entities
    assert e.boundary_kind[i] == _lib.TG_BC_CUSTOM and e.boundary_function[i] == "lid_wall"
    with pytest.raises(tb.TealError):
        e.set_source("device function")
    with pytest.raises(tb.TealError):
        e.set_source("body force", (0, -1, 0), compute="unsteady_source")
    e.set_source("device function", compute="unsteady_source")
    assert e.source_function == "unsteady_source"
    e.set_source(None)
    assert e.source is None and e.source_function is None

    with pytest.raises(tb.TealError):
        e.set_source("device function", compute="hill_forcing", prepare="sum")
    with pytest.raises(tb.TealError):
        e.set_source("bulk forcing", (1.0, 0.001), prepare="average")
    e.set_source("device function", compute="hill_forcing", prepare="average")
    assert e.source_prepare == "average"
    e.set_source(None)
    assert e.source_prepare is None
