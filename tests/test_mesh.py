"""Host mesh generation: bit-identical to the reference's mesh_create + mesh_generate, and the
integer invariants of the reference's mesh_validate (src/mesh/validate.c:100-255) recomputed here."""

import numpy as np
import pytest

import teal_b200 as tb
from oracle import ref
from teal_b200 import meshes

ARRAYS = ["cells.cell.off", "cells.cell.idx", "cells.volume", "cells.center", "cells.projection",
          "cells.offset", "faces.cell_idx", "faces.area", "faces.basis", "faces.weight", "faces.offset",
          "faces.correction", "entities.face_off", "neighbors.tag", "neighbors.recv_off",
          "neighbors.send.off", "neighbors.send.idx"]

CASES = [
    ((0, 0, 0), (10, 10, 0.625), (64, 64, 4), (1, 1, 1)),        # isentropic vortex box
    ((0, 0, 0), (2 * np.pi,) * 3, (12, 12, 12), (1, 1, 1)),      # Taylor-Green box
    ((0, 0, 0), (1, 1, 1), (8, 6, 5), (1, 0, 1)),                # walls in y
    ((0, 0, 0), (2, 1, 1), (12, 7, 1), (0, 0, 0)),               # 2D, all boundary
    ((-1, -2, 0), (3, 1, 0.5), (5, 4, 3), (0, 0, 0)),            # 3D, all boundary
    ((0, 0, 0), (2 * np.pi,) * 3, (48, 48, 48), (1, 1, 1)),      # large enough for threaded geometry
]

needs_ref = pytest.mark.skipif(not ref.available(), reason="reference oracle not built")


@needs_ref
@pytest.mark.parametrize("case", CASES)
def test_host_mesh_matches_reference_bit_for_bit(case):
    r = ref.RefMesh(*case)
    a = r.arrays()
    m = tb.Mesh.create(*case)
    for k in ARRAYS:
        assert np.array_equal(a[k], m.array(k)), k
    assert a["sum_volume"] == m.sum_volume
    assert r.entities() == m.entities


@needs_ref
def test_jittered_mesh_matches_reference():
    n = (6, 5, 4)
    rng = np.random.default_rng(7)
    nodes = (n[0] + 1) * (n[1] + 1) * (n[2] + 1)
    disp = 0.2 * 0.1 * (2 * rng.random((nodes, 3)) - 1)
    case = ((0, 0, 0), (0.6, 0.5, 0.4), n, (0, 0, 0))
    r = ref.RefMesh(*case, displacement=disp)
    a = r.arrays()
    m = tb.Mesh.create(*case, displacement=disp)
    for k in ARRAYS:
        assert np.array_equal(a[k], m.array(k)), k


@pytest.mark.parametrize("case", CASES)
def test_mesh_invariants(case):
    check_invariants(tb.Mesh.create(*case))


RAMPS = [dict(n=(10, 8, 6), block=4, seed=1), dict(n=(16, 12, 10), block=4, seed=2),
         dict(n=(20, 16, 12), block=8, seed=5),
         dict(n=(48, 40, 32), block=8, seed=9)]  # threaded geometry (more than 32768 cells per thread)


@needs_ref
@pytest.mark.parametrize("spec", RAMPS)
def test_unstructured_ramp_matches_reference_bit_for_bit(spec):
    cells = meshes.ramp_mesh(**spec)
    r = ref.RefMesh.from_cells(cells)
    r.validate()  # teal_error would exit the process
    a = r.arrays()
    m = tb.Mesh.from_cells(cells)
    for k in ARRAYS:
        assert np.array_equal(a[k], m.array(k)), k
    assert a["sum_volume"] == m.sum_volume
    assert r.entities() == m.entities


@pytest.mark.parametrize("spec", RAMPS)
def test_unstructured_ramp_invariants(spec):
    cells = meshes.ramp_mesh(**spec)
    c = cells["counts"]
    assert min(c["tetrahedra"], c["pyramids"], c["prisms"], c["hexahedra"]) > 0
    assert c["tetrahedra"] + c["pyramids"] + c["prisms"] + c["hexahedra"] == cells["num_inner"]
    m = tb.Mesh.from_cells(cells)
    check_invariants(m)
    # the ramp: the bottom wall is flat, then rises at 15 degrees
    assert [e[0] for e in m.entities] == ["domain", "left", "right", "bottom", "top", "back", "front"]


def test_nonconforming_cells_are_rejected():
    cells = meshes.ramp_mesh(n=(6, 5, 4), block=2, seed=0)
    cells["node_idx"] = cells["node_idx"].copy()
    cells["node_idx"][:4] = cells["node_idx"][0]  # a degenerate tetrahedron
    with pytest.raises(tb.TealError):
        tb.Mesh.from_cells(cells)


def check_invariants(m):
    """Integer and geometric invariants of mesh_validate, recomputed in numpy."""
    s = m.struct
    C, N, F = s.num_inner_cells, s.num_cells, s.num_faces
    lr = m.array("faces.cell_idx")
    off = m.array("cells.cell.off")
    idx = m.array("cells.cell.idx")
    assert (lr[:, 0] < lr[:, 1]).all()
    assert (lr[:, 0] < C).all()
    assert (lr[: s.num_inner_faces, 1] < C).all()
    assert ((lr[s.num_inner_faces:s.off_boundary_faces, 1] >= C)
            & (lr[s.num_inner_faces:s.off_boundary_faces, 1] < s.off_boundary_cells)).all()
    assert (lr[s.off_boundary_faces:, 1] >= s.off_boundary_cells).all()
    # adjacency symmetric, at most 6 neighbours, no self loops
    deg = np.diff(off)
    assert deg.max() <= 6 and deg[:C].min() >= 1
    pairs = set()
    for c in range(N):
        for j in idx[off[c]:off[c + 1]]:
            assert j != c
            pairs.add((c, int(j)))
    assert all((b, a) in pairs for a, b in pairs)
    # every face appears in the adjacency, faces sorted as teal sorts them
    assert all((int(a), int(b)) in pairs for a, b in lr)
    assert (np.diff(lr[: s.num_inner_faces, 0]) >= 0).all()
    assert (np.diff(lr[s.num_inner_faces:, 1]) > 0).all()
    # geometry
    basis = m.array("faces.basis")
    assert np.allclose(np.einsum("fij,fkj->fik", basis, basis), np.eye(3)[None], atol=1e-12)
    center = m.cell_center
    delta = center[lr[:, 1]] - center[lr[:, 0]]
    assert (np.einsum("fi,fi->f", basis[:, 0], delta) > 1e-12).all()
    assert (m.array("faces.area") > 0).all()
    assert (m.cell_volume[:C] > 0).all()
    assert np.isclose(m.cell_volume[:C].sum(), m.sum_volume)
    # entity face ranges cover the one-sided faces
    fo = m.array("entities.face_off")
    assert fo[0] == s.num_inner_faces and fo[s.off_boundary_entities] == s.off_boundary_faces
    assert fo[-1] == F


@needs_ref
def test_reference_mesh_validates():
    r = ref.RefMesh(*CASES[0])
    r.validate()  # teal_error would exit the process
