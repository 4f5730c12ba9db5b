"""Device mesh upload: the integer layout the device builds (periodic ghost -> owner redirection,
per-cell face slots sorted by face index, neighbour rows) is bit-identical to a host recompute."""

import ctypes

import numpy as np
import pytest

import teal_b200 as tb

pytestmark = pytest.mark.gpu


def layout(ctx, name, dtype, count):
    out = np.zeros(count, dtype=dtype)
    tb._lib.check(tb.lib.tg_layout(ctx.handle, name.encode(), ctypes.c_void_p(out.ctypes.data), count))
    return out


def host_layout(m):
    s = m.struct
    C, F = s.num_inner_cells, s.num_faces
    lr = m.array("faces.cell_idx").astype(np.int64).copy()
    # owner of each periodic ghost: receive tag matched with the send posted under it
    tags = m.array("neighbors.tag")
    roff = m.array("neighbors.recv_off")
    soff = m.array("neighbors.send.off")
    sidx = m.array("neighbors.send.idx")
    owner = np.full(s.num_cells - s.off_boundary_cells, -1)
    used = set()
    for k in range(s.num_neighbors):
        j = next(j for j in range(s.num_neighbors) if j not in used and tags[j, 1] == tags[k, 0])
        used.add(j)
        cnt = roff[k + 1] - roff[k]
        owner[roff[k] - s.off_boundary_cells: roff[k + 1] - s.off_boundary_cells] = sidx[soff[j]:soff[j] + cnt]
    per = np.arange(F) >= s.off_boundary_faces
    lr[per, 1] = owner[lr[per, 1] - s.off_boundary_cells]
    # slots: faces of each inner cell in face order, ~f on the right side of two-sided faces
    slots = [[] for _ in range(C)]
    for f in range(F):
        slots[lr[f, 0]].append((f, f, lr[f, 1]))
        if f < s.num_inner_faces:
            slots[lr[f, 1]].append((f, ~f, lr[f, 0]))
    cnt = np.array([len(x) for x in slots], dtype=np.uint8)
    sf = np.zeros((6, C), dtype=np.int32)
    sn = np.zeros((6, C), dtype=np.int32)
    for c in range(C):
        for j in range(6):
            if j < len(slots[c]):
                _, code, nbr = sorted(slots[c])[j]
                sf[j, c], sn[j, c] = code, nbr
            else:
                sf[j, c], sn[j, c] = 0, c
    return lr.astype(np.int32), owner.astype(np.int32), cnt, sf, sn


@pytest.mark.parametrize("case", [
    ((0, 0, 0), (10, 10, 0.625), (16, 16, 4), (1, 1, 1)),
    ((0, 0, 0), (1, 1, 1), (7, 6, 5), (1, 0, 1)),
    ((0, 0, 0), (1, 1, 1), (5, 4, 3), (0, 0, 0)),
])
def test_device_layout_matches_host_recompute(case):
    m = tb.Mesh.create(*case)
    e = tb.Equations.euler(m)
    for i in range(len(e.boundary_name)):
        e.set_boundary_condition(m.entities[m.struct.num_inner_entities + i][0], "slipwall")
    ctx = e.context()
    s = m.struct
    C, F = s.num_inner_cells, s.num_faces
    lr, owner, cnt, sf, sn = host_layout(m)
    assert np.array_equal(layout(ctx, "face_lr", np.int32, 2 * F).reshape(F, 2), lr)
    assert np.array_equal(layout(ctx, "owner", np.int32, owner.size), owner)
    assert np.array_equal(layout(ctx, "slot_cnt", np.uint8, C), cnt)
    assert np.array_equal(layout(ctx, "slot_face", np.int32, 6 * C).reshape(6, C), sf)
    assert np.array_equal(layout(ctx, "slot_nbr", np.int32, 6 * C).reshape(6, C), sn)


def test_layout_rejects_wrong_count():
    m = tb.Mesh.create((0, 0, 0), (1, 1, 1), (4, 4, 4), (1, 1, 1))
    ctx = tb.Equations.euler(m).context()
    out = np.zeros(3, dtype=np.int32)
    st = tb.lib.tg_layout(ctx.handle, b"slot_face", ctypes.c_void_p(out.ctypes.data), 3)
    assert st == tb._lib.TG_ERR_INVALID


def test_gradient_tiles_carry_each_tiles_largest_slot_count():
    # the gradient kernel stages the slot geometry of 32 cells as one tile holding as many slots as
    # the tile's cell with the most faces: no padding slots beyond that on a mixed-element mesh
    from teal_b200 import meshes

    m = tb.Mesh.from_cells(meshes.ramp_mesh(n=(10, 10, 10), seed=3))
    e = tb.Equations.euler(m)
    for i in range(len(e.boundary_name)):
        e.set_boundary_condition(m.entities[m.struct.num_inner_entities + i][0], "slipwall")
    ctx = e.context()
    C = m.num_inner_cells
    cnt = layout(ctx, "slot_cnt", np.uint8, C).astype(np.int32)
    nt = (C + 31) // 32
    tiles = layout(ctx, "tile_slots", np.int32, nt)
    assert np.array_equal(tiles, [cnt[32 * t: 32 * t + 32].max() for t in range(nt)])
    assert tiles.min() < 6
    # hexahedra only: every tile has 6 slots
    h = tb.Mesh.create((0, 0, 0), (1, 1, 1), (7, 6, 5), (1, 1, 1))
    hctx = tb.Equations.euler(h).context()
    assert np.all(layout(hctx, "tile_slots", np.int32, (h.num_inner_cells + 31) // 32) == 6)
