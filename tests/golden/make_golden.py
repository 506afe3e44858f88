"""Generates tests/golden/ref_<case>.npz: the outputs of the REFERENCE
library (oracle/_ref/libstable-fluids-ref.so, compiled unmodified from the
reference's backend-cuda.cu) on the seeded cases of cases.py, together with
every input and the configuration, so the CPU tests can pin the oracle
without a GPU.

Run on a machine with a CUDA device, from the repository root:
    python tests/golden/make_golden.py
"""

import importlib
import json
import pathlib
import sys

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import oracle as orc  # noqa: E402
from tests.golden import cases as C  # noqa: E402


def main():
    sf = importlib.import_module("stable-fluids_b200")
    ref = sf.load_library(orc.REF_LIB_PATH)
    out_dir = pathlib.Path(__file__).resolve().parent
    for case in C.build_cases():
        sim = sf.Simulation(case.config, case.scalars, case.vectors, lib=ref)
        case.drive(sim)
        outs = C.collect_outputs(sim, sf, case)
        sim.close()
        arrays = {f"out_{k}": v.astype(np.float32) for k, v in outs.items()}
        for h, a in case.init_scalars.items():
            arrays[f"in_init_scalar{h}"] = a
        for h, a in case.sources.items():
            arrays[f"in_source{h}"] = a
        for h, f in case.forces.items():
            for k in range(3):
                arrays[f"in_force{h}_{'xyz'[k]}"] = f[k]
        if case.impulse is not None:
            for k in range(3):
                arrays[f"in_impulse_{'xyz'[k]}"] = case.impulse[k]
        arrays["meta"] = np.array(case.to_json(sf))
        np.savez_compressed(out_dir / f"ref_{case.name}.npz", **arrays)
        print(case.name, {k: float(np.abs(v).max()) for k, v in outs.items()})


if __name__ == "__main__":
    main()
