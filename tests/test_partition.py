"""Partitions of one mesh over several ranks (teal_b200.partition), on the host: teal's grid of ranks,
coverage of the mesh, every rank's cells seeing all of their faces in the global order, and the halo
maps, checked in one process and over two gloo processes that exchange global cell numbers through
the same send / receive segments the GPUs use."""

import os

import numpy as np
import pytest

import teal_b200 as tb
from teal_b200 import partition as pt

CASES = [
    ((0, 0, 0), (2 * np.pi,) * 3, (8, 8, 8), (1, 1, 1)),   # Taylor-Green box, periodic
    ((0, 0, 0), (10, 10, 0.625), (16, 12, 4), (1, 1, 1)),  # vortex box
    ((0, 0, 0), (2, 1, 1), (9, 7, 3), (0, 1, 0)),          # walls and one periodic axis
]


def test_rank_grid_follows_teals_split():
    assert pt.rank_grid((128, 128, 128), 8) == [2, 2, 2]
    assert pt.rank_grid((128, 128, 128), 2) == [2, 1, 1]
    assert pt.rank_grid((64, 64, 4), 4) == [2, 2, 1]
    assert pt.rank_grid((100, 10, 1), 6) == [6, 1, 1]
    assert pt.rank_grid((9, 7, 3), 3) == [3, 1, 1]
    assert np.prod(pt.rank_grid((10, 20, 30), 12)) == 12
    with pytest.raises(ValueError):
        pt.rank_grid((2, 1, 1), 3)


def faces_of_cells(fc, num_inner_faces, C):
    """face indices of every inner cell (as left, or as right of an inner face), ascending"""
    out = [[] for _ in range(C)]
    for f, (l, r) in enumerate(fc):
        if l < C:
            out[l].append(f)
        if f < num_inner_faces and r < C:
            out[r].append(f)
    return out


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("size", [2, 3, 4])
def test_partitions_cover_the_mesh_in_global_face_order(case, size):
    mesh = tb.Mesh.create(*case)
    ranks, dims = pt.cell_ranks(mesh, case[0], case[1], case[2], size)
    assert int(np.prod(dims)) == size and set(ranks.tolist()) == set(range(size))
    check_partitions(mesh, ranks, size)


@pytest.mark.parametrize("size", [2, 3, 5])
def test_bisection_splits_an_unstructured_mesh(size):
    # the mixed-element compression ramp (tetrahedra, prisms, pyramids, hexahedra; walls, inflow,
    # outflow): recursive coordinate bisection, ranks within one cell of each other
    from teal_b200 import meshes

    mesh = tb.Mesh.from_cells(meshes.ramp_mesh(n=(8, 8, 8), seed=5))
    ranks = pt.bisection_ranks(mesh, size)
    count = np.bincount(ranks, minlength=size)
    assert count.sum() == mesh.num_inner_cells and count.max() - count.min() <= 1
    check_partitions(mesh, ranks, size)
    with pytest.raises(ValueError):
        pt.bisection_ranks(mesh, mesh.num_inner_cells + 1)


def check_partitions(mesh, ranks, size):
    s = mesh.struct
    C = s.num_inner_cells
    parts = pt.partition(mesh, ranks)
    owned = np.concatenate([p.cells for p in parts])
    assert np.array_equal(np.sort(owned), np.arange(C))
    gfc = mesh.array("faces.cell_idx")
    gfaces = faces_of_cells(gfc, s.num_inner_faces, C)
    owner_g = pt.periodic_owners(mesh)
    for p in parts:
        a = p.arrays
        Cl, OBl = a["num_inner_cells"], a["off_boundary_cells"]
        lfc = a["faces.cell_idx"]
        lfaces = faces_of_cells(lfc, a["num_inner_faces"], Cl)
        for i, g in enumerate(p.cells):
            # the same faces, in the same (global) order
            assert [int(p.faces[f]) for f in lfaces[i]] == gfaces[g]
        # every row a face references is an own cell, a boundary ghost, a periodic ghost or a halo row
        rows_of = np.concatenate([p.cells, -1 - np.arange(OBl - Cl)])
        for f, (l, r) in enumerate(lfc):
            gf = p.faces[f]
            gl, gr = gfc[gf]
            assert (p.cells[l] if l < Cl else p.halo[l - OBl]) == gl
            if f < a["num_inner_faces"]:
                assert (p.cells[r] if r < Cl else p.halo[r - OBl]) == gr
            elif f >= a["off_boundary_faces"]:
                row = p.owner[r - OBl]
                assert (p.cells[row] if row < Cl else p.halo[row - OBl]) == owner_g[gr - s.off_boundary_cells]
        assert len(rows_of) == OBl
        # geometry is the global faces'
        assert np.array_equal(a["faces.basis"], mesh.array("faces.basis")[p.faces])
        assert np.array_equal(a["cells.volume"][:Cl], mesh.array("cells.volume")[p.cells])
    # halo maps: what rank s sends to rank r is r's halo segment from s, in order
    for r in parts:
        for src, beg, n in r.recv_segments(size):
            s_ = parts[src]
            seg = {d: (b, k) for d, b, k in s_.send_segments(size)}[r.rank]
            assert seg[1] == n
            sent = s_.cells[s_.send_rows[seg[0]: seg[0] + n]]
            assert np.array_equal(sent, r.halo[beg: beg + n])


def _exchange_worker(rank, size, port, case, out):
    import torch
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=size)
    try:
        mesh = tb.Mesh.create(*case)
        ranks, _ = pt.cell_ranks(mesh, case[0], case[1], case[2], size)
        p = pt.partition(mesh, ranks)[rank]
        send = torch.from_numpy(p.cells[p.send_rows].astype(np.int64))
        recv = torch.full((len(p.halo),), -1, dtype=torch.int64)
        ops = [dist.P2POp(dist.isend, send[b: b + n], d) for d, b, n in p.send_segments(size)]
        ops += [dist.P2POp(dist.irecv, recv[b: b + n], s) for s, b, n in p.recv_segments(size)]
        for w in dist.batch_isend_irecv(ops):
            w.wait()
        ok = bool(np.array_equal(recv.numpy(), p.halo))
        # the reductions of a step: minimum and sum over ranks
        t = torch.tensor([float(rank + 1)], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MIN)
        u = torch.tensor([float(len(p.cells))], dtype=torch.float64)
        dist.all_reduce(u, op=dist.ReduceOp.SUM)
        out.put((rank, ok, float(t.item()), int(u.item())))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("case", CASES[:2])
def test_two_gloo_ranks_exchange_their_halo(case):
    import multiprocessing as mp
    import socket

    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    procs = [ctx.Process(target=_exchange_worker, args=(r, 2, port, case, out)) for r in range(2)]
    for p in procs:
        p.start()
    res = [out.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    C = tb.Mesh.create(*case).num_inner_cells
    for rank, ok, tmin, total in res:
        assert ok, f"rank {rank} received the wrong halo"
        assert tmin == 1.0 and total == C
