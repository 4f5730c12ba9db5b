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

The result is the dict `Mesh.from_cells` takes (coord, node_off, node_idx, num_inner, entities),
so `Mesh.read(path)` equals teal's `mesh_read` + `mesh_generate` of the same file bit for bit
(tests/test_gmsh.py runs both). Files with periodic links ($Periodic) are refused: teal turns them
into periodic ghost cells and a neighbour graph (read.c:294-500), which this reader does not
restate.
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
    physical, ents, node_blocks, elem_blocks = {}, {2: {}, 3: {}}, [], []

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
            raise MshError("periodic links are not supported by this reader")
        elif section.startswith("$End"):
            continue
        else:
            raise MshError(f"unsupported mesh section ({section})")
    return physical, ents, node_blocks, elem_blocks


def read_msh(path):
    """The one-process mesh of a Gmsh 4.1 file as teal's mesh_read leaves it, as the dict
    `Mesh.from_cells` takes: coord, node_off, node_idx, num_inner, entities."""
    with open(path, "rb") as f:
        data = f.read()
    physical, ents, node_blocks, elem_blocks = _parse(data)
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
        keyed.append(((-dim, ptags[0], tag, i), (dim, ptags[0]), nodes))
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

    # cells and entities: consecutive blocks of one physical group form one entity
    counts, cell_nodes, entities, num_inner = [], [], [], None
    for (key, phys, nodes) in keyed:
        if entities and entities[-1][0] == phys:
            entities[-1][2] += len(nodes)
        else:
            start = entities[-1][2] if entities else 0
            if phys[0] == 2 and num_inner is None:
                num_inner = start
            entities.append([phys, start, start + len(nodes)])
        counts.append(np.full(len(nodes), nodes.shape[1], np.int64))
        cell_nodes.append(to_index(nodes).reshape(-1))
    if num_inner is None:
        num_inner = entities[-1][2]
    count = np.concatenate(counts)
    node_off = np.zeros(len(count) + 1, np.int64)
    np.cumsum(count, out=node_off[1:])
    idx = np.concatenate(cell_nodes)

    # only the nodes some cell uses, in file order (read.c:762-846 on one rank)
    used = np.unique(idx)
    new = np.full(len(tags), -1, np.int64)
    new[used] = np.arange(len(used))
    return {
        "coord": np.ascontiguousarray(coord[used]),
        "node_off": node_off.astype(np.int32),
        "node_idx": new[idx].astype(np.int32),
        "num_inner": int(num_inner),
        "entities": [(physical[p], int(b), int(e)) for p, b, e in entities],
    }


def write_msh(path, mesh, binary=False, byteorder="<"):
    """Write a mesh given as the dict of teal_b200.meshes / `read_msh` (coord, node_off, node_idx,
    num_inner, entities) as a Gmsh 4.1 file. Every entity becomes one physical group (volumes for
    the entities of inner cells, surfaces for the boundary ones, in entity order) with one Gmsh
    entity per element type, so that teal's reader (and `read_msh`) gives back the same entities,
    each entity's cells grouped by element type. Node tags start at 1 in the given order. A binary
    file is written little-endian unless `byteorder` is ">" (readers detect and swap it)."""
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
    with open(path, "wb") as f:
        f.write(bytes(out))
