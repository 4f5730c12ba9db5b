"""Synthetic unstructured meshes, built as teal holds a mesh before generation (nodes, cells as node
lists, entities as cell ranges) and handed to the library's mesh generation.

ramp_mesh: a 3-D compression ramp on a jittered structured grid, with tetrahedra, prisms, hexahedra
and pyramid/tetrahedron transition cells. Every quadrilateral of the grid is either kept whole or
cut along its diagonal from its lowest to its highest corner (the same diagonal from both sides), so
the cells meet face to face, as teal's face construction requires (src/mesh/generate.c:227-321):

* a tetrahedron block splits each hexahedron into the 6 tetrahedra around its main diagonal
  (all six faces cut);
* a prism block splits each hexahedron into 2 prisms along z (the two z faces cut);
* a hexahedron block keeps the hexahedron (no face cut);
* a hexahedron whose faces, as cut by its neighbours, match none of these gets a centre node and
  one pyramid per whole face plus two tetrahedra per cut face.

Block types are drawn per block of `block` cells per axis with fixed shares (1/2 tetrahedron,
1/4 prism, 1/4 hexahedron), seeded.
"""

import math

import numpy as np

TET, PRISM, HEX = 0, 1, 2

# corner (dx, dy, dz) -> local index in teal's / Gmsh's hexahedron order
_HEX = [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)]
_CORNER = {c: i for i, c in enumerate(_HEX)}


def _kuhn_tets():
    """The 6 tetrahedra around the (0,0,0)-(1,1,1) diagonal, as local corner indices."""
    out = []
    for perm in ((0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)):
        p = [0, 0, 0]
        tet = [_CORNER[tuple(p)]]
        for ax in perm:
            p[ax] = 1
            tet.append(_CORNER[tuple(p)])
        out.append(tet)
    return out


KUHN = _kuhn_tets()
# two prisms along z: triangles (0,0)-(1,0)-(1,1) and (0,0)-(1,1)-(0,1), bottom then top
PRISMS = [[0, 1, 2, 4, 5, 6], [0, 2, 3, 4, 6, 7]]
# the six faces of a hexahedron as (axis, side) with their corners in cyclic order, the first and the
# third corner being the face's lowest and highest corner (the cut diagonal)
FACES = {
    (0, 0): [0, 3, 7, 4], (0, 1): [1, 2, 6, 5],
    (1, 0): [0, 1, 5, 4], (1, 1): [3, 2, 6, 7],
    (2, 0): [0, 1, 2, 3], (2, 1): [4, 5, 6, 7],
}


def ramp_mesh(n=(80, 80, 80), length=None, ramp_start=0.25, ramp_angle=15.0, jitter=0.2, block=8, seed=0):
    """Compression ramp: x in [0, Lx], the bottom wall flat up to x = ramp_start, then rising at
    `ramp_angle` degrees; the grid is compressed above it. Interior nodes jittered by up to
    `jitter` cell sizes per axis (seeded uniform) before the ramp mapping. `length` defaults to
    cubic cells of size 1 / n[1] (a unit-high box); strongly anisotropic cells with jitter give
    warped quadrilaterals that teal's face construction rejects.

    Returns a dict: coord [num_nodes, 3], node_off [num_cells + 1], node_idx, num_inner,
    entities [(name, cell_beg, cell_end)] (domain; left, right, bottom, top, back, front) and
    counts of the cell kinds.
    """
    nx, ny, nz = n
    if length is None:
        length = (nx / ny, 1.0, nz / ny)
    lx, ly, lz = length
    rng = np.random.default_rng(seed)
    hx, hy, hz = lx / nx, ly / ny, lz / nz

    # nodes: structured, x fastest; jitter inside, then the ramp mapping
    i, j, k = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), np.arange(nz + 1), indexing="ij")
    i, j, k = (a.transpose(2, 1, 0).ravel() for a in (i, j, k))
    x, y, z = i * hx, j * hy, k * hz
    inner = (i > 0) & (i < nx) & (j > 0) & (j < ny) & (k > 0) & (k < nz)
    d = rng.uniform(-jitter, jitter, size=(x.size, 3))
    x = np.where(inner, x + d[:, 0] * hx, x)
    y = np.where(inner, y + d[:, 1] * hy, y)
    z = np.where(inner, z + d[:, 2] * hz, z)
    ramp_start = round(ramp_start / hx) * hx  # the corner lies on a grid line
    yb = np.tan(math.radians(ramp_angle)) * np.maximum(0.0, x - ramp_start)
    y = yb + y * (ly - yb) / ly
    coord = np.stack([x, y, z], axis=1)

    def nid(a, b, c):
        return a + (nx + 1) * (b + (ny + 1) * c)

    # wanted type per cell from its block
    nb = [-(-m // block) for m in n]
    kinds = np.full(int(np.prod(nb)), HEX)
    kinds[: kinds.size // 2] = TET
    kinds[kinds.size // 2: kinds.size // 2 + kinds.size // 4] = PRISM
    kinds = rng.permutation(kinds).reshape(nb[2], nb[1], nb[0])
    ci, cj, ck = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    want = kinds[ck // block, cj // block, ci // block]  # [nx, ny, nz]

    # cut state of every grid face: cut when a cell on either side wants it cut
    cut_xy = want == TET
    cut_z = (want == TET) | (want == PRISM)
    cx = np.zeros((nx + 1, ny, nz), bool)
    cx[:-1] |= cut_xy
    cx[1:] |= cut_xy
    cy = np.zeros((nx, ny + 1, nz), bool)
    cy[:, :-1] |= cut_xy
    cy[:, 1:] |= cut_xy
    cz = np.zeros((nx, ny, nz + 1), bool)
    cz[:, :, :-1] |= cut_z
    cz[:, :, 1:] |= cut_z
    pattern = np.stack([cx[:-1], cx[1:], cy[:, :-1], cy[:, 1:], cz[:, :, :-1], cz[:, :, 1:]], axis=-1)

    all_cut = pattern.all(-1)
    none_cut = ~pattern.any(-1)
    prism = (~pattern[..., :4].any(-1)) & pattern[..., 4:].all(-1)
    trans = ~(all_cut | none_cut | prism)

    # corner node ids of every cell, [nx, ny, nz, 8]
    corners = np.stack([nid(ci + dx, cj + dy, ck + dz) for dx, dy, dz in _HEX], axis=-1)
    cell_id = ci + nx * (cj + ny * ck)

    rows, parent, sub = [], [], []

    def emit(mask, local_lists):
        cs = corners[mask]
        pid = cell_id[mask]
        for s, loc in enumerate(local_lists):
            rows.append(cs[:, loc])
            parent.append(pid)
            sub.append(np.full(pid.size, s))

    emit(all_cut, KUHN)
    emit(prism, PRISMS)
    emit(none_cut, [list(range(8))])

    # transition cells: a centre node each, a pyramid per whole face, two tetrahedra per cut face
    tcells = np.argwhere(trans)
    num_struct = coord.shape[0]
    centres = coord[corners[trans]].mean(axis=1)
    centre_id = num_struct + np.arange(tcells.shape[0])
    coord = np.concatenate([coord, centres]) if tcells.size else coord
    tcorn = corners[trans]
    tpat = pattern[trans]
    tpid = cell_id[trans]
    for f, (axis, side) in enumerate(FACES):
        q = np.array(FACES[(axis, side)])
        whole = ~tpat[:, f]
        if whole.any():
            rows.append(np.concatenate([tcorn[whole][:, q], centre_id[whole, None]], axis=1))
            parent.append(tpid[whole])
            sub.append(np.full(int(whole.sum()), 10 + 3 * f))
        cutf = tpat[:, f]
        if cutf.any():
            for s, tri in enumerate(([0, 1, 2], [0, 2, 3])):
                rows.append(np.concatenate([tcorn[cutf][:, q[tri]], centre_id[cutf, None]], axis=1))
                parent.append(tpid[cutf])
                sub.append(np.full(int(cutf.sum()), 11 + 3 * f + s))

    # inner cells ordered by their grid cell, then by piece
    par = np.concatenate(parent)
    sb = np.concatenate(sub)
    order = np.lexsort((sb, par))
    lens = np.concatenate([np.full(r.shape[0], r.shape[1]) for r in rows])[order]
    pad = np.full((lens.size, 8), -1, np.int64)
    pos = 0
    for r in rows:
        pad[pos:pos + r.shape[0], : r.shape[1]] = r
        pos += r.shape[0]
    pad = pad[order]
    num_inner = lens.size
    counts = {
        "tetrahedra": int(np.sum(lens == 4)), "pyramids": int(np.sum(lens == 5)),
        "prisms": int(np.sum(lens == 6)), "hexahedra": int(np.sum(lens == 8)),
        "transition_hexahedra": int(trans.sum()),
    }

    # boundary face cells by entity: whole faces as quads, cut faces as two triangles
    def side_faces(axis, side):
        if axis == 0:
            a = 0 if side == 0 else nx
            b, c = np.meshgrid(np.arange(ny), np.arange(nz), indexing="ij")
            quad = np.stack([nid(a, b, c), nid(a, b + 1, c), nid(a, b + 1, c + 1), nid(a, b, c + 1)], -1)
            cut = cx[a][b, c]
        elif axis == 1:
            a = 0 if side == 0 else ny
            b, c = np.meshgrid(np.arange(nx), np.arange(nz), indexing="ij")
            quad = np.stack([nid(b, a, c), nid(b + 1, a, c), nid(b + 1, a, c + 1), nid(b, a, c + 1)], -1)
            cut = cy[:, a][b, c]
        else:
            a = 0 if side == 0 else nz
            b, c = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
            quad = np.stack([nid(b, c, a), nid(b + 1, c, a), nid(b + 1, c + 1, a), nid(b, c + 1, a)], -1)
            cut = cz[:, :, a][b, c]
        quad = quad.reshape(-1, 4)
        cut = cut.reshape(-1)
        out = np.full((quad.shape[0], 2, 4), -1, np.int64)
        out[:, 0] = quad
        out[cut, 0, 3] = -1
        out[cut, 1, :3] = quad[cut][:, [0, 2, 3]]
        out = out.reshape(-1, 4)
        return out[out[:, 0] >= 0]

    names = ["domain", "left", "right", "bottom", "top", "back", "front"]
    bfaces = [side_faces(axis, side) for axis in range(3) for side in range(2)]
    entities = [("domain", 0, num_inner)]
    beg = num_inner
    for name, bf in zip(names[1:], bfaces):
        entities.append((name, beg, beg + bf.shape[0]))
        beg += bf.shape[0]
    allc = np.concatenate([pad] + [np.pad(bf, ((0, 0), (0, 4)), constant_values=-1) for bf in bfaces])
    clen = (allc >= 0).sum(axis=1)
    node_off = np.zeros(allc.shape[0] + 1, np.int64)
    np.cumsum(clen, out=node_off[1:])
    node_idx = allc[allc >= 0]
    return {
        "coord": np.ascontiguousarray(coord, np.float64),
        "node_off": node_off.astype(np.int32),
        "node_idx": node_idx.astype(np.int32),
        "num_inner": int(num_inner),
        "entities": entities,
        "counts": counts,
    }
