"""Generate the golden vectors in tests/golden/golden.npz from the reference solver compiled in place
(oracle/_ref/libteal_ref.so, built by `make -C oracle ref` from the reference's own sources).

    python tests/golden/make_golden.py

Every case stores its settings (JSON), the input primitive state and the reference's outputs:
residual, unlimited and limited gradients, time step, residual norm, and the state, time and
residual after a few Advance steps. Meshes are rebuilt from the settings (the host mesh generator
reproduces the reference's mesh arrays bit for bit, tests/test_mesh.py).
"""

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import ref  # noqa: E402
from tests.cases import random_state, taylor_green, vortex  # noqa: E402

FREE = [1.0, 0.6, 0.1, -0.05, 1.0 / 1.4]
FREE_M25 = [1.0, 2.5, 0.0, 0.0, 1.0 / 1.4]  # Mach 2.5 (sound speed 1)
RAMP_BCS = {"left": ["supersonic inflow", FREE_M25], "right": ["supersonic outflow", None],
            "bottom": ["slipwall", None], "top": ["slipwall", None], "back": ["slipwall", None],
            "front": ["slipwall", None]}
SIDES = ["left", "right", "bottom", "top", "back", "front"]


def cases():
    out = []
    out.append(dict(name="vortex_euler_hllc_bj", n=[16, 16, 4], lo=[0, 0, 0], hi=[10, 10, 0.625], periodic=[1, 1, 1],
                    ns=False, flux="hllc", limiter="minmod", coeff=0.0, state="vortex",
                    advance=dict(method="lserk", courant=0.5, rk=[3, 3], steps=3)))
    out.append(dict(name="tgv_ns_roe_venkat", n=[8, 8, 8], lo=[0, 0, 0], hi=[2 * np.pi] * 3, periodic=[1, 1, 1],
                    ns=True, flux="roe", limiter="venkatakrishnan", coeff=1.0, mu=1 / 1600, state="tgv",
                    advance=dict(method="lserk", courant=0.99, rk=[3, 3], steps=3)))
    for flux in ["roe", "hll", "hllc", "hlle", "ausmd", "ausmdv", "lxf", "central"]:
        for lim in [None, "minmod", "venkatakrishnan"]:
            out.append(dict(name=f"flux_{flux}_{lim}", n=[6, 5, 4], lo=[0, 0, 0], hi=[1, 1, 1], periodic=[1, 1, 1],
                            ns=False, flux=flux, limiter=lim, coeff=1.0, state="random", seed=17, mach=1.2))
    for bc in ["slipwall", "supersonic inflow", "supersonic outflow", "subsonic inflow", "subsonic outflow",
               "pressure outflow", "farfield"]:
        out.append(dict(name=f"bc_{bc.replace(' ', '_')}", n=[5, 4, 3], lo=[0, 0, 0], hi=[1, 1, 1], periodic=[0, 0, 0],
                        ns=False, flux="hllc", limiter="minmod", coeff=0.0, state="random", seed=5, mach=0.8,
                        bcs={s: [bc, FREE] for s in SIDES}))
    out.append(dict(name="ns_walls", n=[8, 6, 3], lo=[0, 0, 0], hi=[2, 1, 0.5], periodic=[0, 0, 1], ns=True,
                    flux="roe", limiter="venkatakrishnan", coeff=1.0, mu=0.01, state="random", seed=9, mach=0.5,
                    bcs={"left": ["subsonic inflow", FREE], "right": ["subsonic outflow", FREE],
                         "bottom": ["adiabatic wall", None], "top": ["farfield", FREE]},
                    advance=dict(method="lserk", courant=0.8, rk=[2, 3], steps=2)))
    out.append(dict(name="order1_euler", n=[12, 10, 3], lo=[0, 0, 0], hi=[10, 10, 0.625], periodic=[1, 1, 1],
                    ns=False, flux="roe", limiter="minmod", coeff=0.0, order=1, state="vortex",
                    advance=dict(method="euler", courant=0.5, steps=3)))
    out.append(dict(name="implicit_farfield", n=[10, 8, 2], lo=[0, 0, 0], hi=[1, 1, 0.2], periodic=[0, 0, 1],
                    ns=False, flux="hllc", limiter="minmod", coeff=0.0, state="freestream", seed=4,
                    bcs={s: ["farfield", FREE] for s in SIDES[:4]},
                    advance=dict(method="implicit euler", courant=20.0, nk=[0.1, 0.3, 10], steps=1)))
    out.append(dict(name="implicit_farfield_smooth", n=[10, 8, 2], lo=[0, 0, 0], hi=[1, 1, 0.2], periodic=[0, 0, 1],
                    ns=False, flux="roe", limiter=None, coeff=0.0, state="freestream", seed=6,
                    bcs={s: ["farfield", FREE] for s in SIDES[:4]},
                    advance=dict(method="implicit euler", courant=20.0, nk=[0.1, 0.3, 10], steps=1)))
    # device source terms in place of the run cases' callbacks: a body force (Rayleigh-Taylor-like
    # stratification between slip walls) and bulk forcing of the x velocity (channel between walls)
    out.append(dict(name="source_body_force", n=[10, 12, 2], lo=[-0.25, -0.75, 0], hi=[0.25, 0.75, 0.1],
                    periodic=[1, 0, 1], ns=False, flux="hllc", limiter="minmod", coeff=0.0, state="random",
                    seed=21, mach=0.3, bcs={"bottom": ["slipwall", None], "top": ["slipwall", None]},
                    source=["body force", [0.0, -0.1, 0.0]],
                    advance=dict(method="lserk", courant=0.5, rk=[3, 3], steps=3)))
    out.append(dict(name="source_bulk_forcing", n=[12, 8, 2], lo=[0, 0, 0], hi=[3, 1, 0.25], periodic=[1, 0, 1],
                    ns=True, flux="roe", limiter="venkatakrishnan", coeff=1.0, mu=0.01, state="random",
                    seed=22, mach=0.3, bcs={"bottom": ["adiabatic wall", None], "top": ["adiabatic wall", None]},
                    source=["bulk forcing", [1.0, 0.5]],
                    advance=dict(method="lserk", courant=0.5, rk=[3, 3], steps=3)))
    # the unstructured compression ramp (tetrahedra, prisms, hexahedra, pyramid transitions)
    ramp = dict(kind="ramp", n=[10, 8, 6], block=4, seed=1)
    out.append(dict(name="ramp_euler_ausmd_bj", mesh=ramp, ns=False, flux="ausmd", limiter="minmod", coeff=0.0,
                    state="freestream", free=FREE_M25, seed=12, bcs=RAMP_BCS,
                    advance=dict(method="lserk", courant=0.5, rk=[3, 3], steps=3)))
    out.append(dict(name="ramp_ns_roe_venkat", mesh=ramp, ns=True, flux="roe", limiter="venkatakrishnan",
                    coeff=1.0, mu=0.01, state="random", seed=13, mach=0.6,
                    bcs={**RAMP_BCS, "bottom": ["adiabatic wall", None]},
                    advance=dict(method="lserk", courant=0.8, rk=[3, 3], steps=2)))
    return out


def ramp_cells(spec):
    from teal_b200 import meshes

    return meshes.ramp_mesh(n=tuple(spec["n"]), block=spec["block"], seed=spec["seed"])


def make_state(case, center, num_cells):
    if case["state"] == "vortex":
        return vortex(center)
    if case["state"] == "tgv":
        return taylor_green(center)
    if case["state"] == "freestream":
        p = np.tile(np.array(case.get("free", FREE)), (num_cells, 1))
        p[:, 0] *= 1 + 0.05 * np.random.default_rng(case["seed"]).random(num_cells)
        return p
    return random_state(num_cells, case["seed"], mach=case["mach"])


def ref_equations(case):
    if "mesh" in case:
        m = ref.RefMesh.from_cells(ramp_cells(case["mesh"]))
    else:
        m = ref.RefMesh(case["lo"], case["hi"], case["n"], case["periodic"])
    e = ref.RefEquations(m, case["ns"])
    e.set_space_order(case.get("order", 2))
    e.set_convective_flux(case["flux"])
    e.set_limiter(case["limiter"], case["coeff"])
    if case["ns"] and "mu" in case:
        e.set_property("dynamic viscosity", case["mu"])
    for ent, (name, ctx) in case.get("bcs", {}).items():
        e.set_boundary_condition(ent, name, ctx)
    if "source" in case:
        e.set_source(*case["source"])
    return m, e


def main():
    data = {}
    for case in cases():
        m, e = ref_equations(case)
        a = m.arrays()
        C = a["num_inner_cells"]
        prim = make_state(case, a["cells.center"], a["num_cells"])
        k = case["name"]
        data[f"{k}/case"] = np.array(json.dumps(case))
        data[f"{k}/primitive"] = prim
        data[f"{k}/derivative"] = e.derivative(prim)
        if case.get("order", 2) == 2:
            data[f"{k}/gradient"] = e.gradient(prim)[:C]
            data[f"{k}/gradient_limited"] = e.gradient(prim, limited=True)[:C]
        data[f"{k}/timestep"] = np.array(e.timestep(prim))
        data[f"{k}/residual"] = e.residual(data[f"{k}/derivative"])
        adv = case.get("advance")
        if adv:
            e.set_primitive(prim)
            sim = ref.RefSimulation(e, adv["method"], adv["courant"], rk=adv.get("rk"), nk=adv.get("nk"))
            t = 0.0
            for _ in range(adv["steps"]):
                t, s0, res = sim.advance(t)
            data[f"{k}/advance_state"] = e.primitive[:C].copy()
            data[f"{k}/advance_time"] = np.array(t)
            data[f"{k}/advance_step0"] = np.array(s0)
            data[f"{k}/advance_residual"] = res
    np.savez_compressed(os.path.join(HERE, "golden.npz"), **data)
    print(f"{len([k for k in data if k.endswith('/case')])} cases written")


if __name__ == "__main__":
    main()
