"""Gmsh 4.1 files: teal_b200.gmsh's reader against teal's own mesh_read (src/mesh/read.c, gmsh.c,
core/parse.c compiled in place, one rank) on the same files, written here from the unstructured
compression ramp (tetrahedra, prisms, pyramids, hexahedra; six boundary surfaces): ASCII, binary
and byte-swapped binary. The meshes must agree bit for bit after mesh_generate."""

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


def test_unsupported_files_are_rejected(tmp_path):
    cells = meshes.ramp_mesh(n=(4, 4, 4), seed=6)
    good = str(tmp_path / "good.msh")
    gmsh.write_msh(good, cells)
    text = open(good).read()
    cases = {
        "version": text.replace("4.1 0 8", "2.2 0 8", 1),
        "data-size": text.replace("4.1 0 8", "4.1 0 4", 1),
        "periodic": text + "$Periodic\n0\n$EndPeriodic\n",
        "section": text + "$NodeData\n$EndNodeData\n",
        "physical": text.replace('3 1 "domain"', '3 7 "domain"', 1),
    }
    for name, body in cases.items():
        p = str(tmp_path / f"{name}.msh")
        with open(p, "w") as f:
            f.write(body)
        with pytest.raises(gmsh.MshError):
            gmsh.read_msh(p)
