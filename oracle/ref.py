"""Python handle on the reference solver compiled in place (oracle/_ref/libteal_ref.so).

TEST INFRASTRUCTURE ONLY: the oracle. Used by tests/, __graft_entry__.smoke() and bench.py's CPU
baseline to obtain teal's own results; never by the product path. The library is built from the
reference's own C sources by oracle/Makefile (`make -C oracle ref`), with single-rank MPI / METIS
stand-ins that carry no arithmetic of the hot path.
"""

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libteal_ref.so")

_lib = None


def available():
    return os.path.exists(REF_LIB)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError(f"{REF_LIB} not built (make -C oracle ref needs the reference tree)")
        L = ctypes.CDLL(REF_LIB)
        vp, dp, ip = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)
        sig = {
            "ref_init": (ctypes.c_int, []),
            "ref_set_quiet": (None, [ctypes.c_int]),
            "ref_mesh_cartesian": (vp, [dp, dp, ip, ip]),
            "ref_mesh_displace": (None, [vp, dp, ctypes.c_int]),
            "ref_mesh_read": (vp, [ctypes.c_char_p]),
            "ref_mesh_cells": (vp, [ctypes.c_int, dp, ctypes.c_int, ctypes.c_int, ip, ip, ctypes.c_int,
                                    ctypes.POINTER(ctypes.c_char_p), ip]),
            "ref_mesh_split": (None, [vp, ctypes.c_char_p, dp, dp]),
            "ref_mesh_generate": (None, [vp]),
            "ref_mesh_validate": (None, [vp]),
            "ref_mesh_destroy": (None, [vp]),
            "ref_mesh_counts": (None, [vp, ctypes.POINTER(ctypes.c_long)]),
            "ref_kdtree_nearest": (None, [dp, ctypes.c_int, dp, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]),
            "ref_mesh_sum_volume": (ctypes.c_double, [vp]),
            "ref_mesh_array": (vp, [vp, ctypes.c_char_p]),
            "ref_mesh_entity_name": (ctypes.c_char_p, [vp, ctypes.c_int]),
            "ref_equations": (vp, [vp, ctypes.c_int]),
            "ref_set_space_order": (None, [vp, ctypes.c_int]),
            "ref_set_convective": (None, [vp, ctypes.c_char_p]),
            "ref_set_viscous": (None, [vp, ctypes.c_char_p]),
            "ref_set_limiter": (None, [vp, ctypes.c_char_p, ctypes.c_double]),
            "ref_set_property": (None, [vp, ctypes.c_char_p, ctypes.c_double]),
            "ref_set_source": (None, [vp, ctypes.c_int, dp]),
            "ref_set_boundary": (None, [vp, ctypes.c_char_p, ctypes.c_char_p, dp]),
            "ref_set_boundary_custom": (None, [vp, ctypes.c_char_p, ctypes.c_int, ctypes.c_double]),
            "ref_primitive": (dp, [vp]),
            "ref_limiter_parameter": (dp, [vp]),
            "ref_derivative": (None, [vp, dp, dp, ctypes.c_double]),
            "ref_boundary": (None, [vp, dp, ctypes.c_double]),
            "ref_gradient": (None, [vp, dp, dp]),
            "ref_limiter": (None, [vp, dp, dp]),
            "ref_timestep": (ctypes.c_double, [vp, dp]),
            "ref_residual": (None, [vp, dp, dp]),
            "ref_equations_destroy": (None, [vp]),
            "ref_simulation": (vp, [vp, ctypes.c_char_p, ctypes.c_double, ip, dp]),
            "ref_simulation_set_max_iter": (None, [vp, ctypes.c_int]),
            "ref_simulation_set_max_time": (None, [vp, ctypes.c_double]),
            "ref_simulation_set_termination": (None, [vp, ctypes.c_char_p, ctypes.c_double]),
            "ref_simulation_set_out_time": (None, [vp, ctypes.c_double]),
            "ref_simulation_set_out_iter": (None, [vp, ctypes.c_int]),
            "ref_simulation_run": (ctypes.c_double, [vp]),
            "ref_advance": (ctypes.c_double, [vp, dp, dp, ctypes.c_double]),
            "ref_simulation_destroy": (None, [vp]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype, f.argtypes = res, args
        L.ref_init()
        _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


COUNT_NAMES = ["num_nodes", "num_inner_nodes", "num_cells", "num_inner_cells", "off_boundary_cells",
               "off_periodic_cells", "num_faces", "num_inner_faces", "off_boundary_faces", "cell_nnz",
               "num_entities", "num_inner_entities", "off_boundary_entities", "num_neighbors", "send_nnz",
               "node_nnz"]


class RefMesh:
    """A teal Mesh built by the reference's mesh_create / mesh_generate."""

    def __init__(self, min_coord, max_coord, num_cells, periodic, displacement=None, generate=True):
        L = lib()
        lo = (ctypes.c_double * 3)(*min_coord)
        hi = (ctypes.c_double * 3)(*max_coord)
        n = (ctypes.c_int * 3)(*num_cells)
        p = (ctypes.c_int * 3)(*[int(bool(x)) for x in periodic])
        self.ptr = ctypes.c_void_p(L.ref_mesh_cartesian(lo, hi, n, p))
        if displacement is not None:
            self._disp = np.ascontiguousarray(displacement, dtype=np.float64)
            L.ref_mesh_displace(self.ptr, _d(self._disp), self._disp.shape[0])
        if generate:
            L.ref_mesh_generate(self.ptr)

    @classmethod
    def from_cells(cls, mesh, generate=True):
        """A one-rank mesh from nodes / cells / entities (the dict of teal_b200.meshes), then
        mesh_generate."""
        L = lib()
        self = cls.__new__(cls)
        coord = np.ascontiguousarray(mesh["coord"], np.float64)
        off = np.ascontiguousarray(mesh["node_off"], np.int32)
        idx = np.ascontiguousarray(mesh["node_idx"], np.int32)
        ents = mesh["entities"]
        names = (ctypes.c_char_p * len(ents))(*[e[0].encode() for e in ents])
        eoff = np.array([e[1] for e in ents] + [ents[-1][2]], np.int32)
        ip = ctypes.POINTER(ctypes.c_int)
        self.ptr = ctypes.c_void_p(L.ref_mesh_cells(coord.shape[0], _d(coord), off.size - 1, mesh["num_inner"],
                                                    off.ctypes.data_as(ip), idx.ctypes.data_as(ip), len(ents),
                                                    names, eoff.ctypes.data_as(ip)))
        if generate:
            L.ref_mesh_generate(self.ptr)
        return self

    @classmethod
    def read(cls, path, generate=True):
        """teal's mesh_read of a Gmsh 4.1 file (one rank), then mesh_generate."""
        L = lib()
        self = cls.__new__(cls)
        self.ptr = ctypes.c_void_p(L.ref_mesh_read(str(path).encode()))
        if generate:
            L.ref_mesh_generate(self.ptr)
        return self

    def validate(self):
        lib().ref_mesh_validate(self.ptr)

    def counts(self):
        c = (ctypes.c_long * 16)()
        lib().ref_mesh_counts(self.ptr, c)
        return dict(zip(COUNT_NAMES, list(c)))

    def _view(self, name, dtype, shape):
        addr = lib().ref_mesh_array(self.ptr, name.encode())
        n = int(np.prod(shape))
        if n == 0 or not addr:
            return np.zeros(shape, dtype=dtype)
        buf = (ctypes.c_char * (n * np.dtype(dtype).itemsize)).from_address(addr)
        return np.frombuffer(buf, dtype=dtype).reshape(shape).copy()

    def arrays(self):
        """teal's Mesh arrays (copies) in the key layout of teal_b200.api.Mesh.from_arrays."""
        c = self.counts()
        N, F = c["num_cells"], c["num_faces"]
        a = {
            "num_cells": N, "num_inner_cells": c["num_inner_cells"],
            "off_boundary_cells": c["off_boundary_cells"], "off_periodic_cells": c["off_periodic_cells"],
            "num_faces": F, "num_inner_faces": c["num_inner_faces"],
            "off_boundary_faces": c["off_boundary_faces"],
            "num_entities": c["num_entities"], "num_inner_entities": c["num_inner_entities"],
            "off_boundary_entities": c["off_boundary_entities"], "num_neighbors": c["num_neighbors"],
            "sum_volume": lib().ref_mesh_sum_volume(self.ptr),
        }
        cell_off = self._view("cells.cell.off", np.int32, (N + 1,))
        a["cells.cell.off"] = cell_off
        a["cells.cell.idx"] = self._view("cells.cell.idx", np.int32, (c["cell_nnz"],))
        a["cells.node.off"] = self._view("cells.node.off", np.int32, (N + 1,))
        a["cells.node.idx"] = self._view("cells.node.idx", np.int32, (c["node_nnz"],))
        a["nodes.coord"] = self._view("nodes.coord", np.float64, (c["num_nodes"], 3))
        a["cells.volume"] = self._view("cells.volume", np.float64, (N,))
        a["cells.center"] = self._view("cells.center", np.float64, (N, 3))
        a["cells.projection"] = self._view("cells.projection", np.float64, (N, 3))
        a["cells.offset"] = self._view("cells.offset", np.float64, (int(cell_off[c["num_inner_cells"]]), 3))
        a["faces.cell_idx"] = self._view("faces.cell_idx", np.int32, (F, 2))
        a["faces.area"] = self._view("faces.area", np.float64, (F,))
        a["faces.center"] = self._view("faces.center", np.float64, (F, 3))
        a["faces.basis"] = self._view("faces.basis", np.float64, (F, 3, 3))
        a["faces.weight"] = self._view("faces.weight", np.float64, (F, 2, 3))
        a["faces.offset"] = self._view("faces.offset", np.float64, (F, 2, 3))
        a["faces.correction"] = self._view("faces.correction", np.float64, (F, 4))
        a["entities.cell_off"] = self._view("entities.cell_off", np.int32, (c["num_entities"] + 1,))
        a["entities.face_off"] = self._view("entities.face_off", np.int32, (c["num_entities"] + 1,))
        nn = c["num_neighbors"]
        a["neighbors.tag"] = self._view("neighbors.tag", np.int32, (nn, 2))
        a["neighbors.recv_off"] = self._view("neighbors.recv_off", np.int32, (nn + 1,))
        a["neighbors.send.off"] = self._view("neighbors.send.off", np.int32, (nn + 1,))
        a["neighbors.send.idx"] = self._view("neighbors.send.idx", np.int32, (c["send_nnz"],))
        return a

    def entities(self):
        c = self.counts()
        off = self._view("entities.cell_off", np.int32, (c["num_entities"] + 1,))
        return [(lib().ref_mesh_entity_name(self.ptr, i).decode(), int(off[i]), int(off[i + 1]))
                for i in range(c["num_entities"])]


class RefEquations:
    """teal Equations created by euler_create / navierstokes_create on a RefMesh."""

    def __init__(self, mesh, navierstokes=False):
        self.mesh = mesh
        self.ptr = ctypes.c_void_p(lib().ref_equations(mesh.ptr, int(bool(navierstokes))))
        c = mesh.counts()
        self.num_cells, self.num_inner = c["num_cells"], c["num_inner_cells"]

    def set_space_order(self, order):
        lib().ref_set_space_order(self.ptr, order)

    def set_convective_flux(self, name):
        lib().ref_set_convective(self.ptr, (name or "").encode())

    def set_viscous_flux(self, name):
        lib().ref_set_viscous(self.ptr, (name or "").encode())

    def set_limiter(self, name, coefficient=0.0):
        self.limiter = name
        lib().ref_set_limiter(self.ptr, (name or "").encode(), coefficient)

    def set_property(self, name, value):
        lib().ref_set_property(self.ptr, name.encode(), value)

    def set_source(self, name, parameters=()):
        """The run cases' source callbacks: "body force" (gx, gy, gz) or "bulk forcing" (U, tau), or
        "unsteady" (the harness's time- and position-dependent forcing)."""
        kind = {None: 0, "body force": 1, "bulk forcing": 2, "unsteady": 3}[name]
        p = [float(x) for x in parameters][:4]
        self._src = np.array(p + [0.0] * (4 - len(p)))
        lib().ref_set_source(self.ptr, kind, _d(self._src))

    def set_boundary_custom(self, entity, kind, speed=1.0):
        """teal's "custom" boundary with the harness's Compute callback: "moving wall" (speed along x)
        or "unsteady inflow"."""
        k = {"moving wall": 1, "unsteady inflow": 2}[kind]
        lib().ref_set_boundary_custom(self.ptr, entity.encode(), k, float(speed))

    def set_boundary_condition(self, entity, name, context=None):
        ctx = None
        if context is not None:
            # teal keeps the pointer (equations/set.c:92): one live array per entity
            keep = self.__dict__.setdefault("_ctx_keep", {})
            keep[entity] = np.ascontiguousarray(context, dtype=np.float64)
            ctx = _d(keep[entity])
        lib().ref_set_boundary(self.ptr, entity.encode(), name.encode(), ctx)

    @property
    def primitive(self):
        p = lib().ref_primitive(self.ptr)
        return np.ctypeslib.as_array(p, shape=(self.num_cells * 5,)).reshape(self.num_cells, 5)

    def set_primitive(self, prim):
        self.primitive[:] = prim

    def limiter_parameter(self):
        p = lib().ref_limiter_parameter(self.ptr)
        if not p:
            return None
        return np.ctypeslib.as_array(p, shape=(self.num_inner,)).copy()

    def derivative(self, prim=None, time=0.0):
        """equations_derivative on a copy of `prim` (default: the current state)."""
        work = np.array(self.primitive if prim is None else prim, dtype=np.float64, copy=True)
        out = np.zeros((self.num_inner, 5))
        lib().ref_derivative(self.ptr, _d(work), _d(out), time)
        return out

    def gradient(self, prim=None, limited=False, time=0.0):
        work = np.array(self.primitive if prim is None else prim, dtype=np.float64, copy=True)
        lib().ref_boundary(self.ptr, _d(work), time)
        grad = np.zeros((self.num_cells, 5, 3))
        lib().ref_gradient(self.ptr, _d(work), _d(grad))
        if limited and getattr(self, "limiter", "minmod"):  # teal's limiter pass needs a limiter kind
            lib().ref_limiter(self.ptr, _d(work), _d(grad))
        return grad

    def timestep(self, prim=None):
        work = np.array(self.primitive if prim is None else prim, dtype=np.float64, copy=True)
        return lib().ref_timestep(self.ptr, _d(work))

    def residual(self, deriv):
        d = np.ascontiguousarray(deriv, dtype=np.float64)
        out = np.zeros(5)
        lib().ref_residual(self.ptr, _d(d), _d(out))
        return out


class RefSimulation:
    def __init__(self, eqns, method="lserk", courant=0.99, rk=None, nk=None):
        self.eqns = eqns
        ip = (ctypes.c_int * 2)(*rk) if rk else None
        dp = (ctypes.c_double * 3)(*nk) if nk else None
        self.ptr = ctypes.c_void_p(lib().ref_simulation(eqns.ptr, method.encode(), courant, ip, dp))

    def set_max_iter(self, n):
        lib().ref_simulation_set_max_iter(self.ptr, n)

    def set_max_time(self, t):
        lib().ref_simulation_set_max_time(self.ptr, t)

    def set_termination(self, condition, threshold):
        lib().ref_simulation_set_termination(self.ptr, condition.encode(), threshold)

    def set_out_time(self, t):
        lib().ref_simulation_set_out_time(self.ptr, t)

    def set_out_iter(self, n):
        lib().ref_simulation_set_out_iter(self.ptr, n)

    def run(self):
        return lib().ref_simulation_run(self.ptr)

    def advance(self, time, max_step=1.7976931348623157e308):
        t = ctypes.c_double(time)
        res = np.zeros(5)
        step0 = lib().ref_advance(self.ptr, ctypes.byref(t), _d(res), max_step)
        return t.value, step0, res


def kdtree_nearest(points, queries):
    """The reference's kd-tree nearest-point search (src/core/kdtree.c) for every query point."""
    p = np.ascontiguousarray(points, dtype=np.float64)
    q = np.ascontiguousarray(queries, dtype=np.float64)
    out = np.zeros(len(q), dtype=np.int32)
    lib().ref_kdtree_nearest(_d(p), len(p), _d(q), len(q), out.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
    return out
