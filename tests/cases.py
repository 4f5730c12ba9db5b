"""Shared test cases: initial conditions of the reference's run cases and seeded synthetic states.

The initial conditions restate the reference run programs' formulas in numpy; both the device path
and the oracle receive the same arrays, so the comparison never depends on libm differences.
"""

import numpy as np

from oracle import ref


def vortex(center, gamma=1.4, strength=5.0, position=(5.0, 5.0), velocity=(1.0, 1.0), time=0.0,
           domain=10.0):
    """Isentropic vortex (run/isentropic_vortex/run.c:10-27)."""
    def wrap(x, lo, hi):
        return np.where(x >= 0, lo, hi) + np.fmod(x, hi - lo)

    x, y = center[:, 0], center[:, 1]
    dx = wrap(x - velocity[0] * time, 0, domain) - position[0]
    dy = wrap(y - velocity[1] * time, 0, domain) - position[1]
    r2 = dx * dx + dy * dy
    rho = (1 - (gamma - 1) * strength**2 / (8 * gamma * np.pi**2) * np.exp(1 - r2)) ** (1 / (gamma - 1))
    e = strength / (2 * np.pi) * np.exp((1 - r2) / 2)
    out = np.zeros((center.shape[0], 5))
    out[:, 0] = rho
    out[:, 1] = velocity[0] - e * dy
    out[:, 2] = velocity[1] + e * dx
    out[:, 3] = 0.0
    out[:, 4] = rho**gamma
    return out


def taylor_green(center, gamma=1.4, mach=0.1):
    """Taylor-Green vortex (run/taylor_green_vortex/run.c:10-21)."""
    x, y, z = center[:, 0], center[:, 1], center[:, 2]
    p0 = 1 / (gamma * mach**2)
    out = np.zeros((center.shape[0], 5))
    out[:, 1] = np.sin(x) * np.cos(y) * np.cos(z)
    out[:, 2] = -np.cos(x) * np.sin(y) * np.cos(z)
    out[:, 4] = p0 + (np.cos(2 * x) + np.cos(2 * y)) * (np.cos(2 * z) + 2) / 16
    out[:, 0] = out[:, 4] / p0
    return out


def random_state(n, seed, mach=1.2, gamma=1.4):
    """Seeded smooth-plus-noise state with sub- and supersonic regions (every flux branch)."""
    rng = np.random.default_rng(seed)
    out = np.zeros((n, 5))
    out[:, 0] = 1.0 + 0.3 * rng.random(n)
    out[:, 4] = 1.0 + 0.3 * rng.random(n)
    c = np.sqrt(gamma * out[:, 4] / out[:, 0])
    out[:, 1:4] = mach * c[:, None] * (2 * rng.random((n, 3)) - 1)
    return out


def rel_l2(a, b):
    """Relative L2 error per variable (column); a variable whose reference norm is negligible against
    the whole field is measured against the whole field's norm."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    total = np.linalg.norm(b)
    out = []
    for v in range(b.shape[1]):
        den = np.linalg.norm(b[:, v])
        if den < 1e-12 * total:
            den = total
        out.append(np.linalg.norm(a[:, v] - b[:, v]) / (den if den > 0 else 1.0))
    return np.array(out)


def ref_case(n, lo, hi, periodic, navierstokes=False):
    m = ref.RefMesh(lo, hi, n, periodic)
    e = ref.RefEquations(m, navierstokes)
    return m, e


def device_mesh_from_ref(refmesh):
    import teal_b200 as tb

    return tb.Mesh.from_arrays(refmesh.arrays(), refmesh.entities())
