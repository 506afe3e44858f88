"""Rebuilds a cases.Case (inputs, configuration) and the reference outputs
from a committed ref_<case>.npz fixture."""

import json

import numpy as np

from tests.golden import cases as C


def load_fixture(path, sf):
    z = np.load(path, allow_pickle=False)
    meta = json.loads(str(z["meta"]))
    cfg = C.obj_to_struct(sf.SimulationConfig, meta["config"])
    scalars = [C.obj_to_struct(sf.ScalarFieldDesc, s) for s in meta["scalars"]]
    vectors = [C.obj_to_struct(sf.VectorFieldDesc, v) for v in meta["vectors"]]
    init = {int(k[len("in_init_scalar"):]): z[k] for k in z.files if k.startswith("in_init_scalar")}
    sources = {int(k[len("in_source"):]): z[k] for k in z.files if k.startswith("in_source")}
    forces = {}
    for k in z.files:
        if k.startswith("in_force") and k.endswith("_x"):
            h = int(k[len("in_force"):-2])
            forces[h] = tuple(z[f"in_force{h}_{c}"] for c in "xyz")
    impulse = tuple(z[f"in_impulse_{c}"] for c in "xyz") if "in_impulse_x" in z.files else None
    case = C.Case(meta["name"], cfg, scalars, vectors, meta["steps"], init, sources, forces, impulse, meta["force_ramp"])
    outputs = {k[len("out_"):]: z[k] for k in z.files if k.startswith("out_")}
    return case, outputs
