"""Raw state files of the run loop on the host (no GPU): round trip and rejection of a file written
for another mesh."""

import os

import numpy as np
import pytest

import teal_b200 as tb


def test_state_file_round_trip(tmp_path):
    m = tb.Mesh.create((0, 0, 0), (1, 1, 1), (6, 5, 4), (1, 1, 1))
    e = tb.Equations.euler(m)
    e.primitive[:] = np.random.default_rng(3).random(e.primitive.shape)
    saved = e.primitive.copy()
    sim = tb.Simulation(e)
    path = os.path.join(tmp_path, "s.tgstate")
    sim.save_state(path, 0.125, 7)
    e.primitive[:] = 0.0
    sim.load_state(path)
    assert np.array_equal(e.primitive, saved)
    assert sim.start_time == 0.125 and sim.start_index == 7


def test_restart_onto_another_mesh_takes_the_nearest_cells(tmp_path):
    """teal's restart onto a different mesh (src/equations/read.c:101-144): every inner cell takes the
    state of the file's nearest cell centre. The choice is compared with the reference's own kd-tree
    search (src/core/kdtree.c) on meshes without exactly equidistant centres; with exact ties this
    library takes the lowest index, where teal takes the first its tree traversal meets."""
    from oracle import ref

    a = tb.Equations.euler(tb.Mesh.create((0, 0, 0), (1, 1, 1), (8, 6, 4), (1, 1, 1)))
    a.primitive[:] = np.random.default_rng(4).random(a.primitive.shape)
    path = os.path.join(tmp_path, "s_00003.tgstate")
    tb.Simulation(a).save_state(path, 0.5, 3)
    for n, disp in (((16, 12, 8), None), ((5, 5, 5), None), ((7, 6, 5), 0.03)):
        d = None
        if disp:
            nodes = (n[0] + 1) * (n[1] + 1) * (n[2] + 1)
            d = disp * (2 * np.random.default_rng(9).random((nodes, 3)) - 1) / max(n)
        mb = tb.Mesh.create((0, 0, 0), (1, 1, 1), n, (0, 0, 0), displacement=d)
        b = tb.Equations.euler(mb)
        sim = tb.Simulation(b)
        sim.load_state(path)
        C = mb.num_inner_cells
        if ref.available():
            old = a.mesh.cell_center[: a.mesh.num_inner_cells]
            idx = ref.kdtree_nearest(old, mb.cell_center[:C])
            d = old[:, None, :] - mb.cell_center[None, :C, :]
            d2 = (d[..., 0] * d[..., 0] + d[..., 1] * d[..., 1]) + d[..., 2] * d[..., 2]
            unique = (d2 == d2.min(axis=0)).sum(axis=0) == 1
            assert unique.mean() > 0.5
            assert np.array_equal(b.primitive[:C][unique], a.primitive[idx][unique])
        assert sim.start_time == 0.5 and sim.start_index == 3


def test_nearest_cells_ties_take_the_lowest_index():
    from teal_b200.api import nearest_cells

    centers = np.array([[0.0, 0, 0], [2.0, 0, 0], [1.0, 1, 0], [1.0, -1, 0]])
    q = np.array([[1.0, 0, 0], [1.9, 0, 0], [1.0, 0.6, 0]])
    assert nearest_cells(centers, q).tolist() == [0, 1, 2]


def test_corrupt_state_file_is_rejected(tmp_path):
    a = tb.Equations.euler(tb.Mesh.create((0, 0, 0), (1, 1, 1), (6, 5, 4), (1, 1, 1)))
    path = os.path.join(tmp_path, "s.tgstate")
    tb.Simulation(a).save_state(path, 0.0, 0)
    with open(path, "r+b") as f:
        f.write(b"X")
    with pytest.raises(tb.TealError):
        tb.Simulation(a).load_state(path)
    with open(path, "wb") as f:
        f.write(b"TEALB200STATE2\n" + np.array([10, 8], dtype=np.int64).tobytes())
    with pytest.raises(tb.TealError):
        tb.Simulation(a).load_state(path)
