"""Gmsh 4.1 mesh files (.msh, ASCII or binary): a reader that gives the one-process mesh teal's
`mesh_read` builds from a file, and a writer for meshes made here.

teal reads a mesh with `mesh_read` (src/mesh/read.c:901-917): `grid_gmsh` parses the file
(src/mesh/gmsh.c, through src/core/parse.c) into nodes, cells and entities, the cells are
partitioned over the ranks (ParMETIS) and the nodes renumbered per rank, and `mesh_generate` then
builds faces and geometry. On one process that comes down to:

* element blocks ordered as gmsh.c's `compare_entity` orders them (gmsh.c:619-636): blocks of
  entities without a periodic link first, then higher physical dimension first, lower physical
  tag first, lower entity tag first, and otherwise the file's order (the C library's merge sort is
  stable); every element block belongs to an entity with exactly one physical group;
* cells: the elements of the ordered blocks, in file order within a block, their node tags mapped
  to the position of the node in the file's node blocks (grid.c:65-110);
* entities: consecutive blocks of one physical group form one entity named after the group
  (gmsh.c:837-889); the first must be a volume (dimension 3), the rest volumes or surfaces;
* nodes: only the nodes that some cell uses, in file order (read.c:762-846 on one rank), the cells'
  node indices renumbered to match.

* periodic links ($Periodic): every element block with a link is an entity of its own, after all
  others, with its partner entity, rotation and translation (gmsh.c:762-817); its faces become
  periodic ghost cells, and the self-exchange tables send each ghost the inner cell across the
  link (read.c:294-372, dual.c:162-313).

The result is the dict `Mesh.from_cells` takes (coord, node_off, node_idx, num_inner, entities,
and for periodic files off_boundary, off_boundary_entities, rotation, translation, neighbors), so
`Mesh.read(path)` equals teal's `mesh_read` + `mesh_generate` of the same file bit for bit
(tests/test_gmsh.py runs both).
"""

import re
import struct

import numpy as np

# nodes of the element types teal accepts (gmsh.c:369-380)
NODES_OF_TYPE = {2: 3, 3: 4, 4: 4, 5: 8, 6: 6, 7: 5}
TYPE_OF_NODES_3D = {4: 4, 8: 5, 6: 6, 5: 7}  # cell node count -> element type
TYPE_OF_NODES_2D = {3: 2, 4: 3}


class MshError(ValueError):
    pass


class _Reader:
    """Tokens of the ASCII parts and raw reads of the binary parts of a .msh file."""

    def __init__(self, data):
        self.data = data
        self.pos = 0

    def token(self):
        d, n = self.data, len(self.data)
        p = self.pos
        while p < n and d[p : p + 1].isspace():
            p += 1
        if p >= n:
            self.pos = n
            return None
        if d[p : p + 1] in (b'"', b"'", b"`"):
            q = d.find(d[p : p + 1], p + 1)
            if q < 0:
                raise MshError("unterminated quoted string")
            self.pos = q + 1  # after the closing quote (parse.c:75-101)
            return d[p + 1 : q].decode()
        q = p
        while q < n and not d[q : q + 1].isspace():
            q += 1
        self.pos = q + 1 if q < n else q  # the delimiter is consumed, as parse.c does
        return d[p:q].decode()

    def ascii(self, count, kind):
        out = []
        for _ in range(count):
            t = self.token()
            if t is None:
                raise MshError("unexpected end of file")
            out.append(float(t) if kind == "d" else int(t))
        return out

    def binary(self, count, fmt, swap):
        size = struct.calcsize(fmt)
        raw = self.data[self.pos : self.pos + count * size]
        if len(raw) != count * size:
            raise MshError(f"short read ({len(raw) // size} / {count})")
        self.pos += count * size
        dtype = np.dtype(fmt).newbyteorder(">" if swap else "<")
        return np.frombuffer(raw, dtype=dtype).astype(np.dtype(fmt).newbyteorder("="))


def _parse(data):
    r = _Reader(data)
    binary, swap = False, False
    physical, ents, node_blocks, elem_blocks, links = {}, {2: {}, 3: {}}, [], [], []

    def val(count, fmt):
        if binary:
            return r.binary(count, fmt, swap).tolist()
        return r.ascii(count, "d" if fmt == "d" else "i")

    while True:
        section = r.token()
        if section is None:
            break
        if section == "$MeshFormat":
            version = float(r.token())
            if abs(version - 4.1) > 1e-8 * 4.1 + 1e-12:
                raise MshError(f"unsupported version ({version:g})")
            binary = int(r.token()) == 1
            size = int(r.token())
            if size != 8:
                raise MshError(f"unsupported data-size ({size})")
            if binary:
                one = struct.unpack("<i", data[r.pos : r.pos + 4])[0]
                swap = one != 1
                r.pos += 4
        elif section == "$PhysicalNames":  # ASCII in both kinds of file
            for _ in range(int(r.token())):
                dim, tag = int(r.token()), int(r.token())
                physical[(dim, tag)] = r.token()
        elif section == "$Entities":
            counts = val(4, "Q")
            for dim in range(4):
                for _ in range(counts[dim]):
                    tag = val(1, "i")[0]
                    val(3 if dim == 0 else 6, "d")
                    tags = val(val(1, "Q")[0], "i")
                    if dim > 0:
                        val(val(1, "Q")[0], "i")
                    if dim >= 2:
                        ents[dim][tag] = tags
        elif section == "$Nodes":
            num_blocks = val(4, "Q")[0]
            for _ in range(num_blocks):
                dim, tag, para = val(3, "i")
                num = val(1, "Q")[0]
                tags = val(num, "Q")
                ncoord = 3 + (dim if para else 0)
                coord = np.asarray(val(num * ncoord, "d"), np.float64).reshape(num, ncoord)[:, :3]
                node_blocks.append((np.asarray(tags, np.int64), coord))
        elif section == "$Elements":
            num_blocks = val(4, "Q")[0]
            for _ in range(num_blocks):
                dim, tag, etype = val(3, "i")
                num = val(1, "Q")[0]
                if etype not in NODES_OF_TYPE:
                    raise MshError(f"unsupported element type ({etype})")
                n = NODES_OF_TYPE[etype]
                rows = np.asarray(val(num * (1 + n), "Q"), np.int64).reshape(num, 1 + n)
                elem_blocks.append((dim, tag, etype, rows[:, 1:]))
        elif section == "$Periodic":
            for _ in range(val(1, "Q")[0]):
                dim, tag, master = val(3, "i")
                affine = val(val(1, "Q")[0], "d")
                num = val(1, "Q")[0]
                pairs = np.asarray(val(2 * num, "Q"), np.int64).reshape(num, 2)
                links.append((dim, tag, master, affine, pairs[:, 0], pairs[:, 1]))
        elif section.startswith("$End"):
            continue
        else:
            raise MshError(f"unsupported mesh section ({section})")
    return physical, ents, node_blocks, elem_blocks, links


def _cross(a, b):
    return ((a[1] * b[2]) - (a[2] * b[1]), (a[2] * b[0]) - (a[0] * b[2]), (a[0] * b[1]) - (a[1] * b[0]))


def _dot(a, b):
    return ((a[0] * b[0]) + (a[1] * b[1])) + (a[2] * b[2])


def _affine(affine, master_side):
    """Rotation rows and translation of a periodic entity (gmsh.c:784-817): the link's 4 x 4 affine
    map, inverted for the master side with teal's matrix_inverse (rows = cross products of the
    rows / determinant, core/matrix.c:40-54) and translation -(R t)."""
    if len(affine) != 16:
        raise MshError(f"unsupported affine transformation size ({len(affine)})")
    rows = [tuple(affine[4 * r: 4 * r + 3]) for r in range(3)]
    t = (affine[3], affine[7], affine[11])
    det = _dot(rows[0], _cross(rows[1], rows[2]))
    if not abs(det - 1) <= max(1e-8, 1e-5 * max(abs(det), 1.0)):
        raise MshError(f"invalid affine transformation determinant ({det:g})")
    if master_side:
        adj = (_cross(rows[1], rows[2]), _cross(rows[2], rows[0]), _cross(rows[0], rows[1]))
        d = _dot(rows[0], adj[0])
        rows = [tuple(x / d for x in a) for a in adj]
        t = tuple(-1.0 * _dot(r, t) for r in rows)
    return [x for r in rows for x in r], list(t)


def read_msh(path):
    """The one-process mesh of a Gmsh 4.1 file as teal's mesh_read leaves it, as the dict
    `Mesh.from_cells` takes: coord, node_off, node_idx, num_inner, entities."""
    with open(path, "rb") as f:
        data = f.read()
    physical, ents, node_blocks, elem_blocks, links = _parse(data)
    if not node_blocks or sum(len(t) for t, _ in node_blocks) == 0:
        raise MshError("mesh does not contain any nodes")
    if not elem_blocks or sum(len(b[3]) for b in elem_blocks) == 0:
        raise MshError("mesh does not contain any elements")

    # each element block's physical group (gmsh.c:557-595), then teal's block order
    keyed = []
    for i, (dim, tag, etype, nodes) in enumerate(elem_blocks):
        if dim not in (2, 3):
            raise MshError(f"unsupported element block dimension ({dim})")
        if tag not in ents[dim]:
            raise MshError(f"could not find {'surface' if dim == 2 else 'volume'} entity ({tag})")
        ptags = ents[dim][tag]
        if len(ptags) != 1:
            raise MshError(f"unsupported number of physical tags ({len(ptags)})")
        if (dim, ptags[0]) not in physical:
            raise MshError(f"could not find physical name ({dim}, {ptags[0]})")
        link = next((k for k in links if k[0] == dim and (k[1] == tag or k[2] == tag)), None)
        keyed.append(((link is not None, -dim, ptags[0], tag, i), (dim, ptags[0]), nodes, tag, link))
    keyed.sort(key=lambda k: k[0])
    if keyed[0][1][0] != 3:
        raise MshError("mesh does not contain any volumes")

    # nodes in file order; node tags -> positions
    tags = np.concatenate([t for t, _ in node_blocks])
    coord = np.concatenate([c for _, c in node_blocks])
    order = np.argsort(tags, kind="stable")
    sorted_tags = tags[order]

    def to_index(t):
        pos = np.searchsorted(sorted_tags, t)
        pos = np.minimum(pos, len(sorted_tags) - 1)
        if not np.array_equal(sorted_tags[pos], t):
            bad = t[sorted_tags[pos] != t]
            raise MshError(f"node tag ({int(bad.flat[0])}) was not converted to index")
        return order[pos]

    # cells and entities: consecutive blocks of one physical group form one entity; a block with a
    # periodic link is an entity of its own, after all others (gmsh.c:722-889)
    counts, cell_nodes, entities, num_inner = [], [], [], None
    for (key, phys, nodes, tag, link) in keyed:
        if link is not None and link[0] != 2:
            raise MshError(f"unsupported periodic dimension ({link[0]})")
        if phys[0] not in (2, 3):
            raise MshError(f"unsupported physical dimension ({phys[0]})")
        if link is None and entities and entities[-1][0] == phys and entities[-1][3] is None:
            entities[-1][2] += len(nodes)
        else:
            start = entities[-1][2] if entities else 0
            if phys[0] == 2 and num_inner is None:
                num_inner = start
            entities.append([phys, start, start + len(nodes), link, tag])
        counts.append(np.full(len(nodes), nodes.shape[1], np.int64))
        cell_nodes.append(to_index(nodes).reshape(-1))
    if num_inner is None:
        num_inner = entities[-1][2]
    off_boundary_entities = next((i for i, e in enumerate(entities) if e[3] is not None), len(entities))
    count = np.concatenate(counts)
    node_off = np.zeros(len(count) + 1, np.int64)
    np.cumsum(count, out=node_off[1:])
    idx = np.concatenate(cell_nodes)

    # only the nodes some cell uses, in file order (read.c:762-846 on one rank)
    used = np.unique(idx)
    new = np.full(len(tags), -1, np.int64)
    new[used] = np.arange(len(used))
    out = {
        "coord": np.ascontiguousarray(coord[used]),
        "node_off": node_off.astype(np.int32),
        "node_idx": new[idx].astype(np.int32),
        "num_inner": int(num_inner),
        "entities": [(physical[e[0]], int(e[1]), int(e[2])) for e in entities],
    }
    if off_boundary_entities < len(entities):
        out.update(_periodic(entities, off_boundary_entities, int(num_inner), to_index, used, new, out))
    return out


def _periodic(entities, off_bnd, num_inner, to_index, used, new, mesh):
    """Periodic entities as read.c leaves them on one process: each periodic entity's partner
    (gmsh.c:762-782), rotation and translation, and the self-exchange of its ghost cells
    (read.c:294-372), whose sent cells are found as dual.c:162-313 finds them: a periodic face's
    inner cell is the one holding all of its nodes (ParMETIS' dual graph with three common nodes),
    and the inner cell across is that of the partner's face whose nodes the link maps this face's
    nodes to. `used` maps mesh nodes to file nodes, `new` file nodes to mesh nodes."""
    num = len(entities)
    off = mesh["node_off"].astype(np.int64)
    idx = mesh["node_idx"].astype(np.int64)
    base = entities[off_bnd][1]

    partner, rotation, translation, node_map = [0] * num, np.zeros((num, 9)), np.zeros((num, 3)), {}
    for i in range(off_bnd, num):
        _, _, _, link, tag = entities[i]
        _, slave, master, affine, snodes, mnodes = link
        other = master if slave == tag else slave
        j = next((k for k in range(off_bnd, num) if entities[k][4] == other), None)
        if j is None:
            raise MshError(f"could not find periodic link ({other})")
        partner[i] = j
        rot, tr = _affine(affine, master_side=(tag == master))
        rotation[i], translation[i] = rot, tr
        node_map[i] = to_index(snodes if slave == tag else mnodes)  # file node indices

    # inner cells by node, for the inner cell of a face
    node_cells = {}
    for c in range(num_inner):
        for n in idx[off[c]: off[c + 1]].tolist():
            node_cells.setdefault(n, []).append(c)

    def inner_of(c):
        cand = None
        for n in idx[off[c]: off[c + 1]].tolist():
            cells = set(node_cells.get(n, ()))
            cand = cells if cand is None else cand & cells
        if not cand or len(cand) != 1:
            raise MshError(f"face cell ({c}) does not bound exactly one inner cell")
        return cand.pop()

    # the periodic faces of each entity by their sorted mesh node lists
    faces = {}
    for i in range(off_bnd, num):
        for c in range(entities[i][1], entities[i][2]):
            faces[(i, tuple(sorted(idx[off[c]: off[c + 1]].tolist())))] = c

    recv_idx = np.zeros(entities[-1][2] - base, np.int64)
    for i in range(off_bnd, num):
        j = partner[i]
        if len(node_map[i]) != len(node_map[j]):
            raise MshError("periodic node lists of unequal length")
        peer_of = dict(zip(node_map[i].tolist(), node_map[j].tolist()))
        for c in range(entities[i][1], entities[i][2]):
            peer = []
            for n in idx[off[c]: off[c + 1]].tolist():
                f = peer_of.get(int(used[n]))
                if f is None or new[f] < 0:
                    raise MshError(f"missing periodic peer node ({i}, {n})")
                peer.append(int(new[f]))
            pc = faces.get((j, tuple(sorted(peer))))
            if pc is None:
                raise MshError(f"missing periodic peer cell ({j}, {c})")
            recv_idx[c - base] = inner_of(pc)

    # one neighbour per periodic entity with faces: receive tag the entity, send tag its partner;
    # an entity sends the cells whose indices its partner computed (matched by tag, one rank)
    ents = [i for i in range(off_bnd, num) if entities[i][2] > entities[i][1]]
    tag = np.array([[i, partner[i]] for i in ents], np.int32).reshape(-1, 2)
    recv_off = np.array([entities[i][1] for i in ents] + [entities[-1][2]], np.int32)
    send_off = (recv_off - base).astype(np.int32)
    send_idx = np.zeros(int(send_off[-1]), np.int32)
    for k, i in enumerate(ents):
        j = next((q for q in range(len(ents)) if tag[q][1] == i), None)
        if j is None:
            raise MshError(f"periodic entity ({i}) receives from no partner")
        seg = recv_idx[send_off[j]: send_off[j + 1]]
        if len(seg) != send_off[k + 1] - send_off[k]:
            raise MshError("periodic surfaces with different numbers of faces")
        send_idx[send_off[k]: send_off[k + 1]] = seg
    return {
        "off_boundary": int(base),
        "off_boundary_entities": int(off_bnd),
        "rotation": rotation,
        "translation": translation,
        "neighbors": {"tag": tag, "recv_off": recv_off, "send_off": send_off, "send_idx": send_idx},
    }


def write_msh(path, mesh, binary=False, byteorder="<", periodic=()):
    """Write a mesh given as the dict of teal_b200.meshes / `read_msh` (coord, node_off, node_idx,
    num_inner, entities) as a Gmsh 4.1 file. Every entity becomes one physical group (volumes for
    the entities of inner cells, surfaces for the boundary ones, in entity order) with one Gmsh
    entity per element type, so that teal's reader (and `read_msh`) gives back the same entities,
    each entity's cells grouped by element type. Node tags start at 1 in the given order. A binary
    file is written little-endian unless `byteorder` is ">" (readers detect and swap it).
    `periodic` lists (slave entity, master entity, translation) links between boundary entities of
    one element type each: the slave surface is the master moved by the translation, and the link
    pairs every slave node with the master node at its position minus the translation."""
    if byteorder not in ("<", ">"):
        raise MshError(f"byte order ({byteorder})")
    bo = byteorder
    coord = np.asarray(mesh["coord"], np.float64)
    off = np.asarray(mesh["node_off"], np.int64)
    idx = np.asarray(mesh["node_idx"], np.int64)
    num_inner = int(mesh["num_inner"])
    ents = mesh["entities"]
    nn = off[1:] - off[:-1]

    groups = []  # (dim, physical tag, name, [(entity tag, element type, node tags rows)])
    next_tag = {2: 1, 3: 1}
    next_entity = {2: 1, 3: 1}
    elem_tag = 1
    for name, beg, end in ents:
        dim = 3 if end <= num_inner else 2
        if re.search(r'["\s]', name):
            raise MshError(f"entity name ({name}) with spaces or quotes")
        ptag = next_tag[dim]
        next_tag[dim] += 1
        blocks = []
        types = TYPE_OF_NODES_3D if dim == 3 else TYPE_OF_NODES_2D
        for k, etype in types.items():
            cells = np.arange(beg, end)[nn[beg:end] == k]
            if len(cells) == 0:
                continue
            rows = idx[off[cells][:, None] + np.arange(k)[None, :]] + 1
            etags = np.arange(elem_tag, elem_tag + len(cells))
            elem_tag += len(cells)
            blocks.append((next_entity[dim], etype, np.column_stack([etags, rows])))
            next_entity[dim] += 1
        groups.append((dim, ptag, name, blocks))

    tag_of = {}  # entity name -> its Gmsh surface entity tag (one element type)
    for dim, ptag, name, bl in groups:
        if dim == 2 and len(bl) == 1:
            tag_of[name] = bl[0][0]
    ent_cells = {name: (beg, end) for name, beg, end in ents}
    scale = float(np.abs(coord).max()) if len(coord) else 1.0
    link_rows = []
    for slave, master, shift in periodic:
        if slave not in tag_of or master not in tag_of:
            raise MshError(f"periodic link ({slave}, {master}) needs two boundary entities of one element type")
        shift = np.asarray(shift, np.float64)

        def side_nodes(name):
            b, e = ent_cells[name]
            return np.unique(np.concatenate([idx[off[c]: off[c + 1]] for c in range(b, e)]))

        sn, mn = side_nodes(slave), side_nodes(master)
        grid = scale * 1e-9  # positions compared on a grid far below any cell size

        def key(x):
            return tuple(np.round(x / grid).astype(np.int64).tolist())

        at = {key(coord[n]): n for n in mn.tolist()}
        peer = [at.get(key(coord[n] - shift)) for n in sn.tolist()]
        if any(p is None for p in peer):
            raise MshError(f"periodic link ({slave}, {master}): a slave node has no master node")
        affine = [1.0, 0.0, 0.0, shift[0], 0.0, 1.0, 0.0, shift[1], 0.0, 0.0, 1.0, shift[2], 0.0, 0.0, 0.0, 1.0]
        link_rows.append((tag_of[slave], tag_of[master], [float(a) for a in affine],
                          np.column_stack([sn + 1, np.asarray(peer) + 1])))

    lo, hi = coord.min(axis=0), coord.max(axis=0)
    box = [lo[0], lo[1], lo[2], hi[0], hi[1], hi[2]]
    surfaces = [(t, ptag) for dim, ptag, _, bl in groups if dim == 2 for (t, _, _) in bl]
    volumes = [(t, ptag) for dim, ptag, _, bl in groups if dim == 3 for (t, _, _) in bl]
    blocks = [(dim, t, et, rows) for dim, _, _, bl in sorted(groups, key=lambda g: -g[0]) for (t, et, rows) in bl]
    num_nodes = len(coord)
    num_elems = sum(len(rows) for *_, rows in blocks)

    out = bytearray()

    def text(s):
        out.extend(s.encode())

    text(f"$MeshFormat\n4.1 {1 if binary else 0} 8\n")
    if binary:
        out.extend(struct.pack(bo + "i", 1))
        text("\n")
    text("$EndMeshFormat\n$PhysicalNames\n")
    text(f"{len(groups)}\n")
    for dim, ptag, name, _ in groups:
        text(f'{dim} {ptag} "{name}"\n')
    text("$EndPhysicalNames\n$Entities\n")
    if binary:
        out.extend(struct.pack(bo + "4Q", 0, 0, len(surfaces), len(volumes)))
        for t, ptag in surfaces + volumes:
            out.extend(struct.pack(bo + "i6dQiQ", t, *box, 1, ptag, 0))
        text("\n")
    else:
        text(f"0 0 {len(surfaces)} {len(volumes)}\n")
        for t, ptag in surfaces + volumes:
            text(f"{t} " + " ".join(repr(float(x)) for x in box) + f" 1 {ptag} 0\n")
    text("$EndEntities\n$Nodes\n")
    # two node blocks, so that node tags are looked up across blocks
    half = num_nodes // 2
    node_parts = [(0, half), (half, num_nodes)]
    node_parts = [(b, e) for b, e in node_parts if e > b]
    if binary:
        out.extend(struct.pack(bo + "4Q", len(node_parts), num_nodes, 1, num_nodes))
        for b, e in node_parts:
            out.extend(struct.pack(bo + "3iQ", 3, 1, 0, e - b))
            out.extend(np.arange(b + 1, e + 1, dtype=bo + "u8").tobytes())
            out.extend(np.ascontiguousarray(coord[b:e], dtype=bo + "f8").tobytes())
        text("\n")
    else:
        text(f"{len(node_parts)} {num_nodes} 1 {num_nodes}\n")
        for b, e in node_parts:
            text(f"3 1 0 {e - b}\n")
            text("".join(f"{t}\n" for t in range(b + 1, e + 1)))
            text("".join(f"{x!r} {y!r} {z!r}\n" for x, y, z in coord[b:e].tolist()))
    text("$EndNodes\n$Elements\n")
    if binary:
        out.extend(struct.pack(bo + "4Q", len(blocks), num_elems, 1, num_elems))
        for dim, t, et, rows in blocks:
            out.extend(struct.pack(bo + "3iQ", dim, t, et, len(rows)))
            out.extend(np.ascontiguousarray(rows, dtype=bo + "u8").tobytes())
        text("\n")
    else:
        text(f"{len(blocks)} {num_elems} 1 {num_elems}\n")
        for dim, t, et, rows in blocks:
            text(f"{dim} {t} {et} {len(rows)}\n")
            text("".join(" ".join(str(v) for v in row) + "\n" for row in rows.tolist()))
    text("$EndElements\n")
    if link_rows:
        text("$Periodic\n")
        if binary:
            out.extend(struct.pack(bo + "Q", len(link_rows)))
            for t, m, affine, pairs in link_rows:
                out.extend(struct.pack(bo + "3iQ", 2, t, m, 16))
                out.extend(struct.pack(bo + "16d", *affine))
                out.extend(struct.pack(bo + "Q", len(pairs)))
                out.extend(np.ascontiguousarray(pairs, dtype=bo + "u8").tobytes())
            text("\n")
        else:
            text(f"{len(link_rows)}\n")
            for t, m, affine, pairs in link_rows:
                text(f"2 {t} {m}\n16 " + " ".join(repr(float(a)) for a in affine) + f"\n{len(pairs)}\n")
                text("".join(f"{a} {b}\n" for a, b in pairs.tolist()))
        text("$EndPeriodic\n")
    with open(path, "wb") as f:
        f.write(bytes(out))
