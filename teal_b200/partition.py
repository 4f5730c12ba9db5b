"""One mesh over several GPUs: teal's domain decomposition with a one-cell halo.

teal splits a Cartesian mesh over MPI ranks on a grid of ranks (src/mesh/create.c:10-97) and, three
times per residual, exchanges the states and gradients of one layer of ghost cells
(src/equations/exchange.c:8-51); the time step and the residual norm are global reductions
(src/equations/timestep.c:28, residual.c:28). Here every rank is one GPU holding a partition
(tg_create_partition): its inner cells, the global mesh's faces that touch them (in global order and
orientation) and halo rows for the inner cells of other ranks on those faces. A step is

    local minimum of the cells' steps -> minimum over ranks -> CFL step
    per RK stage: boundary states, exchange states, gradient + limiter, exchange gradient records,
                  face fluxes and the stage update
    sums of V R^2 -> sum over ranks -> residual norm

so each rank's cells see exactly the inputs they see in the single-mesh run, and the state after
every step equals it bit for bit (the residual norm, a sum over ranks, agrees to rounding).

`cell_ranks` splits a Cartesian mesh as teal does, `bisection_ranks` any mesh by recursive
coordinate bisection; `partition` builds the ranks' partitions and halo maps on the host from the
single-process mesh;
`LocalRun` drives all ranks in one process on one GPU (the halo moved by device copies; for tests);
`DistributedRun` drives one rank per process and GPU over torch.distributed (the halo by
send/receive, the reductions by all-reduce).
"""

import ctypes
import dataclasses

import numpy as np

from . import _lib
from ._lib import check, lib


def rank_grid(num_cells, size):
    """Ranks per axis for `size` ranks on an (nx, ny, nz) grid, as teal's mesh_create splits it
    (src/mesh/create.c:10-73): the prime factors of `size`, largest first, each multiply the axis
    (among the axes with more than one cell, in the order of their cell counts, largest first, ties
    by axis) that keeps the most cells per rank."""
    count = [max(1, int(n)) for n in num_cells]
    if size > count[0] * count[1] * count[2]:
        raise ValueError(f"using more ranks ({size}) than cells is not supported")
    perm = [0, 1, 2]
    if count[perm[1]] > count[perm[0]]:
        perm[0], perm[1] = perm[1], perm[0]
    if count[perm[2]] > count[perm[1]]:
        perm[1], perm[2] = perm[2], perm[1]
    if count[perm[1]] > count[perm[0]]:
        perm[0], perm[1] = perm[1], perm[0]
    dims = [1, 1, 1]
    ndims = sum(1 for n in num_cells if n > 1)
    prime = size
    while prime > 1:
        factor = 2
        while factor <= prime // factor and prime % factor != 0:
            factor += 1
        if factor > prime // factor:
            factor = prime
        best, score = -1, -1
        for i in range(ndims):
            axis = perm[i]
            if dims[axis] > count[axis] // factor:
                continue
            s = count[axis] // dims[axis]
            if s > score:
                best, score = axis, s
        if best < 0:
            raise ValueError(f"cannot split {num_cells} over {size} ranks")
        dims[best] *= factor
        prime //= factor
    return dims


def _block(index, n, d):
    """The rank coordinate of cell `index` along an axis of n cells split into d blocks, the first
    n % d blocks one cell longer (src/mesh/create.c:75-97)."""
    base, extra = n // d, n % d
    head = (base + 1) * extra
    return np.where(index < head, index // (base + 1), extra + (index - head) // max(base, 1))


def cell_ranks(mesh, min_coord, max_coord, num_cells, size):
    """Rank of every inner cell of a Cartesian mesh: its block on teal's grid of ranks, ranks
    numbered row-major over the grid (MPI's Cartesian numbering)."""
    dims = rank_grid(num_cells, size)
    C = mesh.num_inner_cells
    lo, hi, n = np.asarray(min_coord, float), np.asarray(max_coord, float), np.asarray(num_cells)
    width = np.where(n > 0, (hi - lo) / np.maximum(n, 1), 1.0)
    ijk = np.floor((mesh.cell_center[:C] - lo) / width).astype(np.int64)
    ijk = np.clip(ijk, 0, np.maximum(n - 1, 0))
    coord = [_block(ijk[:, a], max(int(n[a]), 1), dims[a]) for a in range(3)]
    return ((coord[0] * dims[1] + coord[1]) * dims[2] + coord[2]).astype(np.int64), dims


def bisection_ranks(mesh, size):
    """Rank of every inner cell of any mesh, by recursive coordinate bisection of the cell centres:
    a group of cells going to n ranks is split across the longest extent of its bounding box, the
    first n // 2 ranks taking that share of its cells (cells ordered by the coordinate, ties by
    index). For unstructured meshes, whose split in teal is ParMETIS's (src/mesh/read.c:275-292 over
    the dual graph of src/mesh/dual.c), a library that is not available here: any split gives the
    same results (each rank's cells sum their faces in the global order); only the balance and the
    halo sizes differ."""
    C = mesh.num_inner_cells
    if not 1 <= size <= C:
        raise ValueError(f"cannot split {C} cells over {size} ranks")
    center = np.asarray(mesh.cell_center[:C])
    ranks = np.empty(C, dtype=np.int64)
    stack = [(np.arange(C), 0, size)]
    while stack:
        idx, r0, n = stack.pop()
        if n == 1:
            ranks[idx] = r0
            continue
        pts = center[idx]
        axis = int(np.argmax(pts.max(axis=0) - pts.min(axis=0)))
        nl = n // 2
        k = len(idx) * nl // n
        order = np.lexsort((idx, pts[:, axis]))
        stack.append((idx[order[:k]], r0, nl))
        stack.append((idx[order[k:]], r0 + nl, n - nl))
    return ranks


def periodic_owners(mesh):
    """Owner (inner cell) of every periodic ghost of a one-process mesh: each receive matched with
    the send posted under its tag, as the one-process exchange does (exchange.c:8-36)."""
    s = mesh.struct
    off, num = s.off_boundary_cells, s.num_cells - s.off_boundary_cells
    owner = np.full(num, -1, dtype=np.int64)
    if num == 0:
        return owner
    tag = mesh.array("neighbors.tag")
    recv_off = mesh.array("neighbors.recv_off")
    send_off = mesh.array("neighbors.send.off")
    send_idx = mesh.array("neighbors.send.idx")
    used = np.zeros(len(tag), dtype=bool)
    for k in range(len(tag)):
        j = next(j for j in range(len(tag)) if not used[j] and tag[j][1] == tag[k][0])
        used[j] = True
        n = recv_off[k + 1] - recv_off[k]
        owner[recv_off[k] - off: recv_off[k] - off + n] = send_idx[send_off[j]: send_off[j] + n]
    if (owner < 0).any():
        raise ValueError("a periodic ghost receives no state")
    return owner


@dataclasses.dataclass
class Part:
    """One rank's partition: the arrays of its local mesh (teal's layout, tg_mesh keys), the halo and
    send maps, and its place in the global mesh."""

    rank: int
    arrays: dict
    entities: list
    owner: np.ndarray          # periodic ghost -> state row
    cells: np.ndarray          # global index of each inner cell (local order)
    halo: np.ndarray           # global inner cell of each halo row (grouped by source rank)
    halo_src: np.ndarray       # source rank of each halo row
    send_rows: np.ndarray      # local inner rows sent, grouped by destination rank
    send_dst: np.ndarray       # destination rank of each sent row
    faces: np.ndarray          # global index of each local face

    def recv_segments(self, size):
        """[(source rank, first halo row, count)] in halo order."""
        return _segments(self.halo_src, size)

    def send_segments(self, size):
        return _segments(self.send_dst, size)


def _segments(ranks, size):
    out, beg = [], 0
    for r in range(size):
        n = int((ranks == r).sum())
        if n:
            out.append((r, beg, n))
        beg += n
    return out


def partition(mesh, ranks):
    """Partitions of a one-process mesh for the given rank of every inner cell (`cell_ranks`)."""
    s = mesh.struct
    C, OB, N = s.num_inner_cells, s.off_boundary_cells, s.num_cells
    F, F_in, F_bd = s.num_faces, s.num_inner_faces, s.off_boundary_faces
    size = int(ranks.max()) + 1
    fc = mesh.array("faces.cell_idx").astype(np.int64)
    owner_g = periodic_owners(mesh)
    cls = np.where(np.arange(F) < F_in, 0, np.where(np.arange(F) < F_bd, 1, 2))
    left, right = fc[:, 0], fc[:, 1]
    right_owner = np.where(cls == 2, owner_g[np.clip(right - OB, 0, max(len(owner_g) - 1, 0))] if len(owner_g) else 0,
                           right)
    rank_l = ranks[left]
    rank_r = np.where(cls == 0, ranks[np.clip(right, 0, C - 1)], -1)
    ent_off = mesh.array("entities.face_off")
    volume, center = mesh.array("cells.volume"), mesh.array("cells.center")
    proj = mesh.array("cells.projection")
    area, basis = mesh.array("faces.area"), mesh.array("faces.basis")
    weight, offset = mesh.array("faces.weight"), mesh.array("faces.offset")
    corr = mesh.array("faces.correction")
    parts = []
    halos = []
    for r in range(size):
        own = ranks == r
        fmask = (rank_l == r) | ((cls == 0) & (rank_r == r))
        faces = np.nonzero(fmask)[0]
        cells = np.nonzero(own)[0]
        local = np.full(C, -1, dtype=np.int64)
        local[cells] = np.arange(len(cells))
        fl, fr, fk = left[faces], right[faces], cls[faces]
        ext = np.concatenate([fl[~own[fl]], fr[(fk == 0) & ~own[np.clip(fr, 0, C - 1)]]])
        per = right_owner[faces][fk == 2]
        ext = np.unique(np.concatenate([ext, per[~own[per]]]))
        order = np.lexsort((ext, ranks[ext]))
        halo = ext[order]
        halos.append(halo)
        bfaces, pfaces = faces[fk == 1], faces[fk == 2]
        NB, P = len(bfaces), len(pfaces)
        OBl = len(cells) + NB
        row = local.copy()
        row[halo] = OBl + np.arange(len(halo))
        lc = np.zeros((len(faces), 2), dtype=np.int64)
        lc[:, 0] = row[fl]
        inner = fk == 0
        lc[inner, 1] = row[fr[inner]]
        lc[fk == 1, 1] = len(cells) + np.arange(NB)
        lc[fk == 2, 1] = OBl + np.arange(P)
        owner = row[right_owner[pfaces]]
        gcells = np.concatenate([cells, right[bfaces], right[pfaces]])  # global cell of each local cell
        ncell = len(gcells)
        # entities: inner entities keep the inner cells, boundary and periodic ones their ghosts
        ents, eoff = [], []
        for i, (name, beg, end) in enumerate(mesh.entities):
            fb, fe = ent_off[i], ent_off[i + 1]
            eoff.append(int(np.searchsorted(faces, fb)))
            if i < s.num_inner_entities:
                ents.append((name, 0, len(cells)))
            else:
                sel = (faces >= fb) & (faces < fe)
                first = int(np.searchsorted(faces, fb))
                n_in = int(sel.sum())
                # local ghosts of this entity's faces, in face order
                base = len(cells) if i < s.off_boundary_entities else OBl
                start = first - (int(np.searchsorted(faces, F_in)) if i < s.off_boundary_entities
                                 else int(np.searchsorted(faces, F_bd)))
                ents.append((name, base + start, base + start + n_in))
        eoff.append(len(faces))
        arrays = {
            "num_cells": ncell, "num_inner_cells": len(cells), "off_boundary_cells": OBl,
            "off_periodic_cells": ncell,
            "cells.cell.off": np.zeros(ncell + 1, np.int32), "cells.cell.idx": np.zeros(1, np.int32),
            "cells.volume": volume[gcells], "cells.center": center[gcells], "cells.projection": proj[gcells],
            "cells.offset": np.zeros((1, 3)),
            "sum_volume": s.sum_volume,
            "num_faces": len(faces), "num_inner_faces": int(inner.sum()),
            "off_boundary_faces": int(inner.sum()) + NB,
            "faces.cell_idx": lc.astype(np.int32), "faces.area": area[faces], "faces.basis": basis[faces],
            "faces.weight": weight[faces], "faces.offset": offset[faces], "faces.correction": corr[faces],
            "num_entities": s.num_entities, "num_inner_entities": s.num_inner_entities,
            "off_boundary_entities": s.off_boundary_entities,
            "entities.face_off": np.array(eoff, np.int32),
            "num_neighbors": 0, "neighbors.tag": np.zeros((1, 2), np.int32),
            "neighbors.recv_off": np.zeros(1, np.int32), "neighbors.send.off": np.zeros(1, np.int32),
            "neighbors.send.idx": np.zeros(1, np.int32),
        }
        parts.append(Part(rank=r, arrays=arrays, entities=ents, owner=owner.astype(np.int32), cells=cells,
                          halo=halo, halo_src=ranks[halo], send_rows=None, send_dst=None, faces=faces))
    # sends: rank r sends, to each rank d in order, the cells of d's halo it owns, in d's halo order
    for p in parts:
        rows, dst = [], []
        local = np.full(C, -1, dtype=np.int64)
        local[p.cells] = np.arange(len(p.cells))
        for d, h in enumerate(halos):
            mine = h[ranks[h] == p.rank]
            rows.append(local[mine])
            dst.append(np.full(len(mine), d))
        p.send_rows = np.concatenate(rows).astype(np.int32) if rows else np.zeros(0, np.int32)
        p.send_dst = np.concatenate(dst) if dst else np.zeros(0, np.int64)
    return parts


class _DeviceBytes:
    """A device buffer of `n` bytes at `ptr` for torch.as_tensor (no copy)."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": "|u1", "data": (int(ptr), False),
                                         "version": 3}


def _configure(eqns, like):
    """The same plugin settings as `like` (a teal_b200 Equations of the whole mesh)."""
    eqns.set_space_order(like.space_order)
    eqns.convective, eqns.viscous = like.convective, like.viscous
    eqns.limiter, eqns.limiter_coefficient = like.limiter, like.limiter_coefficient
    eqns.property = list(like.property)
    eqns.boundary_name = list(like.boundary_name)
    eqns.boundary_kind = like.boundary_kind.copy()
    eqns.boundary_context = like.boundary_context.copy()


class Rank:
    """One rank's device context (tg_create_partition) and its exchange buffers as torch tensors."""

    def __init__(self, part, eqns, precision=_lib.TG_PRECISION_FP64):
        import torch

        from .api import Equations, Mesh

        self.part = part
        self.mesh = Mesh.from_arrays(part.arrays, part.entities)
        self.eqns = Equations(self.mesh, eqns.physics)
        _configure(self.eqns, eqns)
        self.struct = self.eqns.struct()
        self.handle = ctypes.c_void_p()
        send = np.ascontiguousarray(part.send_rows, dtype=np.int32)
        owner = np.ascontiguousarray(part.owner, dtype=np.int32)
        check(lib.tg_create_partition(ctypes.byref(self.mesh.struct), ctypes.byref(self.struct), precision,
                                      owner.ctypes.data_as(ctypes.c_void_p), len(part.halo),
                                      send.ctypes.data_as(ctypes.c_void_p), len(send), ctypes.byref(self.handle)))
        p = [ctypes.c_void_p() for _ in range(4)]
        rb = ctypes.c_long()
        check(lib.tg_part_buffers(self.handle, *[ctypes.byref(x) for x in p], ctypes.byref(rb)))
        self.record_bytes = rb.value
        ns, nh = len(send), len(part.halo)
        dev = torch.device("cuda", torch.cuda.current_device())

        def view(ptr, n):  # a rank without neighbours has no exchange buffers (NULL, zero bytes)
            if not ptr or n == 0:
                return torch.empty(0, dtype=torch.uint8, device=dev)
            return torch.as_tensor(_DeviceBytes(ptr, n), device=dev)

        self.send_q = view(p[0].value, 40 * ns)
        self.recv_q = view(p[1].value, 40 * nh)
        self.send_rec = view(p[2].value, rb.value * ns)
        self.recv_rec = view(p[3].value, rb.value * nh)
        st = ctypes.c_void_p()
        check(lib.tg_stream_of(self.handle, ctypes.byref(st)))
        self.stream = torch.cuda.ExternalStream(st.value)

    def set_state(self, primitive_global):
        """The partition's rows of a state of the whole mesh (teal rows: inner cells first)."""
        C = len(self.part.cells)
        rows = np.zeros((self.mesh.num_cells, 5))
        rows[:C] = primitive_global[self.part.cells]
        check(lib.tg_set_primitive(self.handle, rows.ctypes.data_as(ctypes.c_void_p)))

    def state(self):
        out = np.empty((self.mesh.num_cells, 5))
        check(lib.tg_get_primitive(self.handle, out.ctypes.data_as(ctypes.c_void_p)))
        return out[: len(self.part.cells)]

    def step_begin(self):
        m = ctypes.c_double()
        check(lib.tg_part_step_begin(self.handle, ctypes.byref(m)))
        return m.value

    def set_step(self, step, time):
        check(lib.tg_part_set_step(self.handle, float(step), float(time)))

    def phase(self, k, alpha=0.0, last=0):
        check(lib.tg_part_phase(self.handle, int(k), float(alpha), int(last)))

    def residual_sums(self):
        out = np.zeros(5)
        check(lib.tg_part_residual_sums(self.handle, out.ctypes.data_as(ctypes.c_void_p)))
        return out

    def close(self):
        if self.handle:
            lib.tg_destroy(self.handle)
            self.handle = ctypes.c_void_p()


def lserk_alpha(order, stages):
    a = np.zeros(stages + 1)
    check(lib.tg_lserk_alpha(int(order), int(stages), a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
    return a


class LocalRun:
    """All ranks of a partitioned mesh in one process on the current GPU: one context per rank, the
    halo moved between their buffers by device copies, the reductions on the host. For tests of the
    partitioned path (one GPU; nothing waits on another rank's kernels: the host orders the phases)."""

    def __init__(self, parts, eqns, precision=_lib.TG_PRECISION_FP64):
        self.size = len(parts)
        self.ranks = [Rank(p, eqns, precision) for p in parts]
        self.sum_volume = eqns.mesh.sum_volume

    def set_state(self, primitive_global):
        for r in self.ranks:
            r.set_state(primitive_global)

    def _exchange(self, what):
        import torch

        torch.cuda.synchronize()
        for r in self.ranks:
            for src, beg, n in r.part.recv_segments(self.size):
                s = self.ranks[src]
                seg = dict((d, (b, k)) for d, b, k in s.part.send_segments(self.size))[r.part.rank]
                assert seg[1] == n
                if what == "q":
                    r.recv_q[40 * beg: 40 * (beg + n)].copy_(s.send_q[40 * seg[0]: 40 * (seg[0] + n)])
                else:
                    b = r.record_bytes
                    r.recv_rec[b * beg: b * (beg + n)].copy_(s.send_rec[b * seg[0]: b * (seg[0] + n)])
        torch.cuda.synchronize()

    def step(self, time, courant, rk=(3, 3), max_step=np.inf):
        """One lserk step of the whole mesh; returns (time, step0, residual[5])."""
        alpha = lserk_alpha(*rk)
        m = min(r.step_begin() for r in self.ranks)
        step0 = courant * m
        step = min(step0, max_step)
        for r in self.ranks:
            r.set_step(step, time)
        stages = rk[1]
        for i in range(stages):
            for r in self.ranks:
                r.phase(0)
            self._exchange("q")
            for r in self.ranks:
                r.phase(1)
            self._exchange("rec")
            for r in self.ranks:
                r.phase(2, alpha[i + 1], int(i == stages - 1))
        sums = np.zeros(5)
        for r in self.ranks:
            sums += r.residual_sums()
        return time + step, step0, np.sqrt(sums / self.sum_volume)

    def state(self, num_inner):
        out = np.zeros((num_inner, 5))
        for r in self.ranks:
            out[r.part.cells] = r.state()
        return out

    def close(self):
        for r in self.ranks:
            r.close()


class DistributedRun:
    """This process's rank of a partitioned mesh, one GPU per process over torch.distributed (NCCL):
    the halo by grouped send / receive between the ranks' exchange buffers, ordered on the
    context's stream, the step minimum and the residual sums by all-reduce."""

    def __init__(self, part, eqns, size, precision=_lib.TG_PRECISION_FP64):
        import torch

        self.torch = torch
        self.size = size
        self.rank = Rank(part, eqns, precision)
        self.sum_volume = eqns.mesh.sum_volume

    def _exchange(self, what):
        import torch.distributed as dist

        r = self.rank
        send, recv, row = (r.send_q, r.recv_q, 40) if what == "q" else (r.send_rec, r.recv_rec, r.record_bytes)
        ops = []
        with self.torch.cuda.stream(r.stream):
            for d, beg, n in r.part.send_segments(self.size):
                ops.append(dist.P2POp(dist.isend, send[row * beg: row * (beg + n)], d))
            for s, beg, n in r.part.recv_segments(self.size):
                ops.append(dist.P2POp(dist.irecv, recv[row * beg: row * (beg + n)], s))
            if ops:
                for w in dist.batch_isend_irecv(ops):
                    w.wait()

    def step(self, time, courant, rk=(3, 3), max_step=np.inf):
        import torch.distributed as dist

        torch = self.torch
        r = self.rank
        alpha = lserk_alpha(*rk)
        m = torch.tensor([r.step_begin()], dtype=torch.float64, device="cuda")
        dist.all_reduce(m, op=dist.ReduceOp.MIN)
        step0 = courant * float(m.item())
        step = min(step0, max_step)
        r.set_step(step, time)
        stages = rk[1]
        for i in range(stages):
            r.phase(0)
            self._exchange("q")
            r.phase(1)
            self._exchange("rec")
            r.phase(2, alpha[i + 1], int(i == stages - 1))
        sums = torch.tensor(r.residual_sums(), dtype=torch.float64, device="cuda")
        dist.all_reduce(sums, op=dist.ReduceOp.SUM)
        return time + step, step0, np.sqrt(sums.cpu().numpy() / self.sum_volume)

    def close(self):
        self.rank.close()
