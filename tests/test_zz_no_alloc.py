"""tg_residual_noalloc (the residual norm that allocates no device memory) through the C ABI against
tg_residual on the same derivative, two calls in a row, bit for bit; that its calls leave the device's
free memory unchanged; and the inputs it refuses."""

import ctypes

import numpy as np
import pytest
import torch

import teal_b200 as tb
from teal_b200 import _lib
from tests.cases import taylor_green, vortex

pytestmark = pytest.mark.gpu

# Both paths sum the same products in the same order (pieces of 4096 cells, the same block shapes),
# so the results are compared bit for bit.


def noalloc(deriv, volume, num_cells, sum_volume, out, stream):
    return _lib.lib.tg_residual_noalloc(deriv.data_ptr(), volume.data_ptr(), num_cells, sum_volume,
                                        out.data_ptr(), stream)


def check_against_context(m, e, prim):
    C = m.num_inner_cells
    deriv = e.derivative(prim)[:C]
    expect = e.residual(deriv)  # tg_residual through a context
    d = torch.from_numpy(np.ascontiguousarray(deriv)).cuda()
    v = torch.from_numpy(np.ascontiguousarray(m.cell_volume[:C])).cuda()
    out = torch.empty(5, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):
        out.fill_(float("nan"))
        _lib.check(noalloc(d, v, C, m.sum_volume, out, stream))
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert np.all(np.isfinite(got))
        assert np.array_equal(got, expect), (got, expect)
    # what the entry point exists for: after the first call's set-up, calls allocate nothing
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    held0 = torch.cuda.memory_allocated()
    for _ in range(20):
        _lib.check(noalloc(d, v, C, m.sum_volume, out, stream))
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, f"device free memory changed by {free0 - free1} bytes across calls"
    assert torch.cuda.memory_allocated() == held0
    assert np.array_equal(out.cpu().numpy(), expect)


def test_noalloc_residual_vortex_one_piece():
    m = tb.Mesh.create((0, 0, 0), (10, 10, 0.625), (32, 32, 4), (1, 1, 1))
    e = tb.Equations.euler(m)
    check_against_context(m, e, vortex(m.cell_center))


def test_noalloc_residual_taylor_green_ragged_pieces():
    # 30^3 = 27000 cells: six full pieces of 4096 cells and a ragged seventh
    m = tb.Mesh.create((0, 0, 0), (2 * np.pi,) * 3, (30, 30, 30), (1, 1, 1))
    e = tb.Equations.navierstokes(m)
    e.set_convective_flux("roe")
    e.set_limiter("venkatakrishnan", 1.0)
    e.set_property("dynamic viscosity", 1 / 1600)
    check_against_context(m, e, taylor_green(m.cell_center))


def test_noalloc_rejects_sizes_beyond_the_limit():
    d = torch.zeros(5, dtype=torch.float64, device="cuda")
    out = torch.zeros(5, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    too_many = _lib.TG_NOALLOC_MAX_CELLS + 1
    assert noalloc(d, d, too_many, 1.0, out, stream) == _lib.TG_ERR_INVALID
    assert b"TG_NOALLOC_MAX_CELLS" in _lib.lib.tg_last_error()
    host = np.zeros(5)
    status = _lib.lib.tg_residual_noalloc(host.ctypes.data_as(ctypes.c_void_p), host.ctypes.data_as(ctypes.c_void_p),
                                          1, 1.0, out.data_ptr(), stream)
    assert status == _lib.TG_ERR_INVALID  # host memory is refused before any launch
    # the divisor must be finite and positive
    for bad in (0.0, -1.0, float("nan"), float("inf")):
        assert noalloc(d, d, 1, bad, out, stream) == _lib.TG_ERR_INVALID
        assert b"sum_volume" in _lib.lib.tg_last_error()
    # no cells: the norm of nothing is zero
    out.fill_(float("nan"))
    _lib.check(noalloc(d, d, 0, 1.0, out, stream))
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), np.zeros(5))
