"""Golden vectors (tests/golden/golden.npz, written by tests/golden/make_golden.py from the reference
solver compiled from its own sources) and builders of the same cases for the device path and the
CPU restatement."""

import json
import os

import numpy as np

import teal_b200 as tb

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden.npz")


def load():
    z = np.load(GOLDEN)
    names = sorted({k.split("/")[0] for k in z.files})
    out = {}
    for n in names:
        d = {k.split("/", 1)[1]: z[k] for k in z.files if k.startswith(n + "/")}
        d["case"] = json.loads(str(d["case"]))
        out[n] = d
    return out


def equations(case):
    """Host mesh + teal_b200 Equations configured as the case."""
    if "mesh" in case:
        from teal_b200 import meshes

        spec = case["mesh"]
        m = tb.Mesh.from_cells(meshes.ramp_mesh(n=tuple(spec["n"]), block=spec["block"], seed=spec["seed"]))
    else:
        m = tb.Mesh.create(case["lo"], case["hi"], case["n"], case["periodic"])
    e = tb.Equations.navierstokes(m) if case["ns"] else tb.Equations.euler(m)
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
