"""Gmsh 4.1 files: teal_b200.gmsh's reader against teal's own mesh_read (src/mesh/read.c, gmsh.c,
core/parse.c compiled in place, one rank) on the same files, written here from the unstructured
compression ramp (tetrahedra, prisms, pyramids, hexahedra; six boundary surfaces) and from boxes of
hexahedra or tetrahedra with periodic links (teal's test/1_mesh/mesh.geo pattern: x and z periodic
by translation): ASCII, binary and byte-swapped binary. The meshes must agree bit for bit after
mesh_generate, periodic ghosts and their exchange tables included."""

import os

import numpy as np
import pytest

import teal_b200 as tb
from oracle import ref
from teal_b200 import gmsh, meshes
from tests.test_mesh import ARRAYS

needs_ref = pytest.mark.skipif(not ref.available(), reason="reference oracle not built")

RAMPS = [dict(n=(6, 6, 6), seed=1), dict(n=(12, 10, 8), block=4, seed=3), dict(n=(10, 8, 6), jitter=0.0, seed=2)]
KINDS = [dict(binary=False), dict(binary=True), dict(binary=True, byteorder=">")]


def cells_of(d, beg, end):
    """The cells [beg, end) of a mesh dict as sorted tuples of their node coordinates."""
    off, idx, c = d["node_off"], d["node_idx"], d["coord"]
    return sorted(tuple(c[idx[off[i]: off[i + 1]]].ravel().tolist()) for i in range(beg, end))


@needs_ref
@pytest.mark.parametrize("kind", KINDS, ids=["ascii", "binary", "binary-big-endian"])
@pytest.mark.parametrize("spec", RAMPS)
def test_reader_matches_the_reference_mesh_read(tmp_path, spec, kind):
    path = str(tmp_path / "ramp.msh")
    gmsh.write_msh(path, meshes.ramp_mesh(**spec), **kind)
    r = ref.RefMesh.read(path)
    r.validate()
    a = r.arrays()
    m = tb.Mesh.read(path)
    for k in ARRAYS:
        assert np.array_equal(a[k], m.array(k)), k
    assert a["sum_volume"] == m.sum_volume
    assert r.entities() == m.entities


@pytest.mark.parametrize("kind", KINDS, ids=["ascii", "binary", "binary-big-endian"])
def test_written_mesh_reads_back(tmp_path, kind):
    cells = meshes.ramp_mesh(n=(8, 6, 5), seed=4)
    path = str(tmp_path / "ramp.msh")
    gmsh.write_msh(path, cells, **kind)
    back = gmsh.read_msh(path)
    assert back["num_inner"] == cells["num_inner"]
    assert [e for e in back["entities"]] == [tuple(e) for e in cells["entities"]]
    assert np.array_equal(back["coord"], cells["coord"])  # every node is used, tags in order
    for (_, beg, end) in cells["entities"]:
        assert cells_of(back, beg, end) == cells_of(cells, beg, end)
    # each entity's cells come back grouped by element type (one Gmsh block per type)
    counts = np.diff(back["node_off"][: back["num_inner"] + 1])
    assert np.all(np.diff([{4: 0, 8: 1, 6: 2, 5: 3}[int(k)] for k in counts]) >= 0)


def test_unused_nodes_are_dropped_and_tags_looked_up(tmp_path):
    # a node no cell uses is dropped (read.c keeps the nodes of its cells only), and the cells'
    # node tags are looked up across node blocks
    cells = meshes.ramp_mesh(n=(4, 4, 4), seed=5)
    extra = dict(cells)
    extra["coord"] = np.vstack([cells["coord"], [[9.0, 9.0, 9.0]]])
    path = str(tmp_path / "extra.msh")
    gmsh.write_msh(path, extra)
    back = gmsh.read_msh(path)
    assert len(back["coord"]) == len(cells["coord"])
    assert not np.any(np.all(back["coord"] == 9.0, axis=1))


def box_mesh(n=(6, 3, 3), length=(9.0, 3.0, 3.0), jitter=0.2, seed=3, tets=False):
    """A box of hexahedra (or of 6 tetrahedra per hexahedron, the same split in every one, so that
    opposite sides are triangulated alike), interior nodes jittered; entities domain, left, right,
    bottom, top, back, front, as the mesh dicts of teal_b200.meshes."""
    nx, ny, nz = n
    h = np.array(length) / np.array(n)
    i, j, k = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), np.arange(nz + 1), indexing="ij")
    i, j, k = (a.transpose(2, 1, 0).ravel() for a in (i, j, k))
    coord = np.stack([i * h[0], j * h[1], k * h[2]], axis=1).astype(float)
    inner = (i > 0) & (i < nx) & (j > 0) & (j < ny) & (k > 0) & (k < nz)
    coord[inner] += np.random.default_rng(seed).uniform(-jitter, jitter, (int(inner.sum()), 3)) * h

    def nid(a, b, c):
        return (c * (ny + 1) + b) * (nx + 1) + a

    cells = []
    for c in range(nz):
        for b in range(ny):
            for a in range(nx):
                v = [nid(a, b, c), nid(a + 1, b, c), nid(a + 1, b + 1, c), nid(a, b + 1, c),
                     nid(a, b, c + 1), nid(a + 1, b, c + 1), nid(a + 1, b + 1, c + 1), nid(a, b + 1, c + 1)]
                if not tets:
                    cells.append(v)
                    continue
                for t in ((0, 1, 2, 6), (0, 1, 5, 6), (0, 3, 2, 6), (0, 3, 7, 6), (0, 4, 5, 6), (0, 4, 7, 6)):
                    q = [v[x] for x in t]
                    d = np.linalg.det(coord[q[1:]] - coord[q[0]])
                    cells.append(q if d > 0 else [q[0], q[2], q[1], q[3]])
    num_inner = len(cells)
    # boundary faces: faces of one cell only, by side
    count = {}
    for cell in cells:
        faces = ([cell[x] for x in f] for f in ((0, 1, 2), (0, 1, 3), (0, 2, 3), (1, 2, 3))) if tets else \
                ([cell[x] for x in f] for f in ((0, 3, 2, 1), (4, 5, 6, 7), (0, 1, 5, 4), (3, 7, 6, 2),
                                                 (0, 4, 7, 3), (1, 2, 6, 5)))
        for f in faces:
            key = tuple(sorted(f))
            count[key] = (count.get(key, (0, f))[0] + 1, f)
    sides = {"left": (0, 0.0), "right": (0, length[0]), "bottom": (1, 0.0), "top": (1, length[1]),
             "back": (2, 0.0), "front": (2, length[2])}
    ents = [("domain", 0, num_inner)]
    for name, (axis, val) in sides.items():
        beg = len(cells)
        cells.extend(f for n_, f in count.values() if n_ == 1 and np.allclose(coord[f, axis], val))
        ents.append((name, beg, len(cells)))
    off = np.zeros(len(cells) + 1, np.int64)
    off[1:] = np.cumsum([len(c) for c in cells])
    return {"coord": coord, "node_off": off.astype(np.int32), "node_idx": np.concatenate(cells).astype(np.int32),
            "num_inner": num_inner, "entities": ents}


PERIODIC = [("right", "left", (9.0, 0.0, 0.0)), ("front", "back", (0.0, 0.0, 3.0))]


@needs_ref
@pytest.mark.parametrize("kind", KINDS, ids=["ascii", "binary", "binary-big-endian"])
@pytest.mark.parametrize("tets", [False, True], ids=["hexahedra", "tetrahedra"])
def test_periodic_links_match_the_reference_mesh_read(tmp_path, kind, tets):
    cells = box_mesh(tets=tets)
    path = str(tmp_path / "box.msh")
    gmsh.write_msh(path, cells, periodic=PERIODIC, **kind)
    r = ref.RefMesh.read(path)
    r.validate()
    a = r.arrays()
    m = tb.Mesh.read(path)
    for k in ARRAYS:
        assert np.array_equal(a[k], m.array(k)), k
    assert a["sum_volume"] == m.sum_volume
    assert r.entities() == m.entities
    s = m.struct
    assert s.num_neighbors == 4 and s.off_periodic_cells > s.off_boundary_cells


def test_unsupported_files_are_rejected(tmp_path):
    cells = meshes.ramp_mesh(n=(4, 4, 4), seed=6)
    good = str(tmp_path / "good.msh")
    gmsh.write_msh(good, cells)
    text = open(good).read()
    cases = {
        "version": text.replace("4.1 0 8", "2.2 0 8", 1),
        "data-size": text.replace("4.1 0 8", "4.1 0 4", 1),
        "periodic": text + "$Periodic\n1\n2 1 999\n16 1 0 0 0 0 1 0 0 0 0 1 0 0 0 0 1\n0\n$EndPeriodic\n",
        "section": text + "$NodeData\n$EndNodeData\n",
        "physical": text.replace('3 1 "domain"', '3 7 "domain"', 1),
    }
    for name, body in cases.items():
        p = str(tmp_path / f"{name}.msh")
        with open(p, "w") as f:
            f.write(body)
        with pytest.raises(gmsh.MshError):
            gmsh.read_msh(p)


@needs_ref
@pytest.mark.gpu
@pytest.mark.parametrize("tets", [False, True], ids=["hexahedra", "tetrahedra"])
def test_residual_on_a_read_periodic_mesh_equals_the_reference(tmp_path, tets):
    # the device's exact FP64 form on the mesh read from a periodic file against teal's own
    # residual on its mesh_read of the same file: bit for bit (periodic ghosts through the read
    # path's exchange tables, walls at the bottom and top)
    from tests.cases import random_state

    path = str(tmp_path / "box.msh")
    gmsh.write_msh(path, box_mesh(tets=tets), periodic=PERIODIC, binary=True)
    rm = ref.RefMesh.read(path)
    re = ref.RefEquations(rm, False)
    m = tb.Mesh.read(path)
    e = tb.Equations.euler(m)
    for q in (re, e):
        q.set_convective_flux("hllc")
        q.set_limiter("minmod")
        q.set_boundary_condition("bottom", "slipwall")
        q.set_boundary_condition("top", "slipwall")
    prim = random_state(m.num_cells, seed=9, mach=0.7)
    expect = re.derivative(prim)
    got = e.derivative(prim, precision=tb.TG_PRECISION_FP64_EXACT)
    assert np.array_equal(got, expect)
