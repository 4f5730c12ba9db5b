"""mesh_split (src/mesh/split.c): an entity's cells cut by a plane into "<name>-a" and "<name>-b"
before generation. The host mesh builder against teal's own mesh_split + mesh_generate on the same
meshes: teal's test/1_mesh/create.c configuration (a periodic channel whose bottom is split at x = 3,
nodes displaced by its tanh bump), several splits in a row, an inner entity split on a periodic box
(the periodic exchange's sent cells move with it) and a split of a mesh read from a Gmsh file. The
meshes must agree bit for bit after mesh_generate; the GPU test runs the exact FP64 residual on a
split mesh with different boundary conditions on the two halves."""

import ctypes

import numpy as np
import pytest

import teal_b200 as tb
from oracle import ref
from teal_b200 import gmsh
from tests.test_gmsh import PERIODIC, box_mesh
from tests.test_mesh import ARRAYS

needs_ref = pytest.mark.skipif(not ref.available(), reason="reference oracle not built")

CHANNEL = ((0, 0, 0), (9, 3, 3), (30, 10, 10), (1, 0, 1))


def bump(case):
    """teal's test/1_mesh/create.c node modification as displacements of the Cartesian nodes
    (x fastest): y += (3 - y) (1 + tanh(3.5 (|x - 4.5| - 3.5))) / 6."""
    lo, hi, n, _ = case
    i, j, k = np.meshgrid(*(np.arange(c + 1) for c in n), indexing="ij")
    i, j = (a.transpose(2, 1, 0).ravel() for a in (i, j))
    x = lo[0] + i * ((hi[0] - lo[0]) / n[0])
    y = lo[1] + j * ((hi[1] - lo[1]) / n[1])
    disp = np.zeros((x.size, 3))
    disp[:, 1] = (3 - y) * (1 + np.tanh(3.5 * (np.abs(x - 4.5) - 3.5))) / 6.0
    return disp


def ref_split(r, splits):
    for name, root, normal in splits:
        ref.lib().ref_mesh_split(r.ptr, name.encode(), (ctypes.c_double * 3)(*root),
                                 (ctypes.c_double * 3)(*normal))
    ref.lib().ref_mesh_generate(r.ptr)
    r.validate()
    return r


def assert_same(r, m):
    a = r.arrays()
    for k in ARRAYS:
        assert np.array_equal(a[k], m.array(k)), k
    assert a["sum_volume"] == m.sum_volume
    assert r.entities() == m.entities


SPLITS = {
    "bottom": [("bottom", (3, 0, 0), (1, 0, 0))],
    "bottom-twice": [("bottom", (3, 0, 0), (1, 0, 0)), ("bottom-b", (6, 0, 0), (1, 0, 0))],
    "top-oblique": [("top", (4.5, 3, 1.5), (1, 0.2, -0.7)), ("top-a", (2, 3, 1.5), (0, 0, 1))],
    "domain": [("domain", (4.5, 1.5, 1.5), (1, 1, 0))],
}


@needs_ref
@pytest.mark.parametrize("name", list(SPLITS))
def test_split_channel_matches_the_reference(name):
    disp = bump(CHANNEL)
    r = ref_split(ref.RefMesh(*CHANNEL, displacement=disp, generate=False), SPLITS[name])
    m = tb.Mesh.create(*CHANNEL, displacement=disp, splits=SPLITS[name])
    assert_same(r, m)
    assert len(m.entities) == 7 + len(SPLITS[name])


@needs_ref
def test_split_inner_entity_of_a_periodic_box_matches_the_reference():
    # the inner entity split in two: its cells are reordered, and with them the cells the periodic
    # self-exchange sends (reorder.c:125-131)
    case = ((0, 0, 0), (1, 1, 1), (8, 6, 5), (1, 1, 1))
    splits = [("domain", (0.5, 0.5, 0.5), (1, -1, 0.5)), ("domain-a", (0.3, 0.5, 0.5), (1, 0, 0))]
    r = ref_split(ref.RefMesh(*case, generate=False), splits)
    m = tb.Mesh.create(*case, splits=splits)
    assert_same(r, m)
    assert [e[0] for e in m.entities[:3]] == ["domain-a-a", "domain-a-b", "domain-b"]
    assert m.struct.num_inner_entities == 3


@needs_ref
@pytest.mark.parametrize("periodic", [False, True], ids=["walls", "periodic"])
def test_split_of_a_read_mesh_matches_the_reference(tmp_path, periodic):
    path = str(tmp_path / "box.msh")
    gmsh.write_msh(path, box_mesh(tets=True), periodic=PERIODIC if periodic else (), binary=True)
    splits = [("bottom", (3, 0, 0), (1, 0, 0)), ("domain", (4.5, 1.5, 1.5), (0, 1, 1))]
    r = ref_split(ref.RefMesh.read(path, generate=False), splits)
    m = tb.Mesh.read(path, splits=splits)
    assert_same(r, m)


def test_split_of_a_missing_or_periodic_entity_is_rejected(tmp_path):
    with pytest.raises(tb.TealError):
        tb.Mesh.create(*CHANNEL, splits=[("floor", (3, 0, 0), (1, 0, 0))])
    with pytest.raises(tb.TealError):  # the first split renamed "bottom"
        tb.Mesh.create(*CHANNEL, splits=[("bottom", (3, 0, 0), (1, 0, 0)), ("bottom", (6, 0, 0), (1, 0, 0))])
    # periodic entities are not splittable (split.c:10-18 searches inner and boundary entities)
    with pytest.raises(tb.TealError):
        tb.Mesh.create(*CHANNEL, splits=[("left", (0, 1.5, 1.5), (0, 1, 0))])
    path = str(tmp_path / "box.msh")
    gmsh.write_msh(path, box_mesh(), periodic=PERIODIC)
    periodic = [e[0] for e in tb.Mesh.read(path).entities][-1]
    with pytest.raises(tb.TealError):
        tb.Mesh.read(path, splits=[(periodic, (3, 0, 0), (1, 0, 0))])


def test_empty_half_keeps_an_empty_entity():
    # every cell on one side: "-a" holds them all and "-b" is empty, as in teal
    m = tb.Mesh.create(*CHANNEL, splits=[("bottom", (100, 0, 0), (1, 0, 0))])
    names = {e[0]: (e[1], e[2]) for e in m.entities}
    beg, end = names["bottom-b"]
    assert beg == end and names["bottom-a"][1] - names["bottom-a"][0] == 30 * 10


@needs_ref
@pytest.mark.gpu
def test_residual_on_a_split_channel_equals_the_reference():
    # supersonic inflow on bottom-a and a slip wall on bottom-b (teal's double Mach reflection
    # pattern), the exact FP64 form against teal's residual on its own split mesh: bit for bit
    from tests.cases import random_state

    disp = bump(CHANNEL)
    splits = SPLITS["bottom"]
    rm = ref_split(ref.RefMesh(*CHANNEL, displacement=disp, generate=False), splits)
    re = ref.RefEquations(rm, False)
    m = tb.Mesh.create(*CHANNEL, displacement=disp, splits=splits)
    e = tb.Equations.euler(m)
    post = np.array([8.0, 7.1, -4.1, 0.0, 116.5])
    for q in (re, e):
        q.set_convective_flux("hllc")
        q.set_limiter("venkatakrishnan", 1.0)
        q.set_boundary_condition("bottom-a", "supersonic inflow", post)
        q.set_boundary_condition("bottom-b", "slipwall")
        q.set_boundary_condition("top", "supersonic outflow")
    prim = random_state(m.num_cells, seed=11, mach=1.5)
    expect = re.derivative(prim)
    got = e.derivative(prim, precision=tb.TG_PRECISION_FP64_EXACT)
    assert np.array_equal(got, expect)
