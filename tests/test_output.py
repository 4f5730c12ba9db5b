"""Visualisation output (teal_b200.output): teal's VTKHDF content written as a VTK XML unstructured
grid. Host-only: meshes come from the library's mesh builder, no GPU is needed."""

import numpy as np

import teal_b200 as tb
from teal_b200 import meshes, output


def tet6(p, a, b, c, d):
    return np.einsum("ij,ij->i", np.cross(p[:, b] - p[:, a], p[:, c] - p[:, a]), p[:, d] - p[:, a])


# VTK node order -> tetrahedra whose signed volumes sum to the cell's (positive when oriented)
DECOMPOSE = {4: [(0, 1, 2, 3)], 5: [(0, 1, 2, 4), (0, 2, 3, 4)], 6: [(0, 1, 2, 3), (1, 2, 3, 4), (2, 3, 4, 5)],
             8: [(0, 1, 3, 4), (1, 2, 3, 6), (1, 3, 4, 6), (1, 4, 5, 6), (3, 4, 6, 7)]}


def test_cartesian_round_trip(tmp_path):
    m = tb.Mesh.create((0, 0, 0), (1, 2, 3), (3, 4, 5), (0, 0, 0))
    prim = np.random.default_rng(1).random((m.num_cells, 5))
    path = str(tmp_path / "box.vtu")
    output.write_vtu(path, m, prim, time=0.25, properties={"heat capacity ratio": 1.4})
    d = output.read_vtu(path)
    c = m.num_inner_cells
    assert d["types"].shape == (c,) and np.all(d["types"] == 12)
    assert d["offsets"][-1] == d["connectivity"].size == 8 * c
    assert d["Points"].shape == ((3 + 1) * (4 + 1) * (5 + 1), 3)
    np.testing.assert_array_equal(d["density"], prim[:c, 0])
    np.testing.assert_array_equal(d["velocity"], prim[:c, 1:4])
    np.testing.assert_array_equal(d["pressure"], prim[:c, 4])
    np.testing.assert_array_equal(d["volume"], m.cell_volume[:c])
    assert d["time"][0] == 0.25 and d["heat capacity ratio"][0] == 1.4


def test_mixed_cells_are_positively_oriented(tmp_path):
    # planar cells (no jitter, no ramp): the tetrahedron decompositions give the exact volumes
    m = tb.Mesh.from_cells(meshes.ramp_mesh(n=(16, 16, 16), jitter=0.0, ramp_angle=0.0))
    path = str(tmp_path / "ramp.vtu")
    output.write_vtu(path, m, np.ones((m.num_cells, 5)))
    d = output.read_vtu(path)
    types = d["types"]
    assert set(np.unique(types).tolist()) == {10, 12, 13, 14}
    offsets = np.concatenate([[0], d["offsets"]])
    conn, xyz = d["connectivity"], d["Points"]
    vol = np.asarray(m.cell_volume[: m.num_inner_cells])
    for k in (4, 5, 6, 8):
        cells = np.where(np.diff(offsets) == k)[0]
        p = xyz[conn[offsets[cells][:, None] + np.arange(k)[None, :]]]
        v = sum(tet6(p, *t) for t in DECOMPOSE[k]) / 6
        np.testing.assert_allclose(v, vol[cells], rtol=1e-12)
    # the entity of every inner cell is the domain (entity 0)
    assert np.all(d["entity"] == 0)
