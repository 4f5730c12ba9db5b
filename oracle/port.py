"""Python handle on the CPU restatement (oracle/liboracle.so). TEST INFRASTRUCTURE ONLY.

Takes meshes and equations in the C ABI's descriptions (teal_b200.api.Mesh / Equations structs) and
teal's AoS state arrays; see oracle/teal_oracle.h.
"""

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_LIB = os.path.join(HERE, "liboracle.so")
_lib = None


def available():
    return os.path.exists(PORT_LIB)


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(PORT_LIB)
        vp, d = ctypes.c_void_p, ctypes.c_double
        dp = ctypes.POINTER(ctypes.c_double)
        sig = {
            "oracle_derivative": (ctypes.c_int, [vp, vp, vp, vp, d]),
            "oracle_gradient": (ctypes.c_int, [vp, vp, vp, ctypes.c_int, vp]),
            "oracle_timestep": (d, [vp, vp, vp]),
            "oracle_residual": (None, [vp, vp, vp]),
            "oracle_euler": (d, [vp, vp, vp, dp, vp, d, d]),
            "oracle_lserk": (d, [vp, vp, vp, dp, vp, d, d, ctypes.c_int, ctypes.c_int]),
            "oracle_implicit_euler": (d, [vp, vp, vp, dp, vp, d, d, d, d, ctypes.c_int]),
        }
        for n, (r, a) in sig.items():
            f = getattr(L, n)
            f.restype, f.argtypes = r, a
        _lib = L
    return _lib


def _v(a):
    return ctypes.c_void_p(a.ctypes.data)


class Port:
    """The restated solver bound to one mesh + equations (teal_b200.api objects)."""

    def __init__(self, mesh, eqns):
        self.mesh = mesh
        self.es = eqns.struct()
        self._keep = (eqns.boundary_kind, eqns.boundary_context)
        self.mp = ctypes.cast(ctypes.byref(mesh.struct), ctypes.c_void_p)
        self.ep = ctypes.cast(ctypes.byref(self.es), ctypes.c_void_p)
        self.N, self.C = mesh.num_cells, mesh.num_inner_cells

    def _state(self, prim):
        s = np.zeros((self.N, 5))
        s[: prim.shape[0]] = prim
        return s

    def derivative(self, prim):
        s = self._state(prim)
        d = np.zeros((self.C, 5))
        lib().oracle_derivative(self.mp, self.ep, _v(s), _v(d), 0.0)
        return d

    def gradient(self, prim, limited=False):
        s = self._state(prim)
        g = np.zeros((self.N, 5, 3))
        lib().oracle_gradient(self.mp, self.ep, _v(s), int(bool(limited)), _v(g))
        return g

    def timestep(self, prim):
        s = self._state(prim)
        return lib().oracle_timestep(self.mp, self.ep, _v(s))

    def residual(self, d):
        d = np.ascontiguousarray(d, dtype=np.float64)
        r = np.zeros(5)
        lib().oracle_residual(self.mp, _v(d), _v(r))
        return r

    def advance(self, prim, method, courant, steps=1, rk=(2, 3), nk=(0.1, 0.3, 32), max_step=1.7976931348623157e308):
        """Advance `steps` steps; returns (state [num_cells][5], time, last step0, residual)."""
        s = self._state(prim)
        t = ctypes.c_double(0.0)
        r = np.zeros(5)
        step0 = 0.0
        for _ in range(steps):
            if method == "lserk":
                step0 = lib().oracle_lserk(self.mp, self.ep, _v(s), ctypes.byref(t), _v(r), max_step, courant, *rk)
            elif method == "euler":
                step0 = lib().oracle_euler(self.mp, self.ep, _v(s), ctypes.byref(t), _v(r), max_step, courant)
            else:
                step0 = lib().oracle_implicit_euler(self.mp, self.ep, _v(s), ctypes.byref(t), _v(r), max_step,
                                                    courant, nk[0], nk[1], int(nk[2]))
        return s, t.value, step0, r
