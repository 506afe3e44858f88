"""Parity at the sizes the benchmarked configurations name.

- config 1 as configured (256^3 plume, 20 diffusion / 80 red-black pressure
  iterations, 50 steps): every output field against the reference library
  (backend-cuda.cu:612-671), bit for bit and so within the required 1e-5;
- config 3's mixed precision (BF16 storage of velocity and density, FP32
  arithmetic and pressure) on the config-1 scene generator for 50 steps,
  against the FP64 oracle, next to the FP32 library's own error;
- the reference's unchanged benchmark.cu, linked once against the reference
  library and once against this one, prints the same density checksums
  (benchmark.cu:232-254).
"""

import pathlib
import re
import subprocess

import numpy as np
import pytest

from tests.golden import cases as C

ROOT = pathlib.Path(__file__).resolve().parent.parent
REF_BENCH = ROOT / "oracle" / "_ref" / "stable-fluids-benchmark-ref"
B200_BENCH = ROOT / "oracle" / "_ref" / "stable-fluids-benchmark-b200"


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.mark.gpu
def test_config1_256_50_steps_matches_reference_library(sf, lib, ref_lib, cuda):
    """256^3, 20/80 iterations, 50 steps: bit-equal to the reference library
    on velocity, pressure, divergence, |u| and density."""
    scene = sf.scenes.config1()
    assert (scene.config.nx, scene.config.diffuse_iterations, scene.config.pressure_iterations, scene.steps) == (256, 20, 80, 50)
    case = C.Case("config1", scene.config, scene.scalars, scene.vectors, scene.steps)
    outs = []
    for L in (lib, ref_lib):
        sim = sf.Simulation(scene.config, scene.scalars, scene.vectors, lib=L)
        sf.scenes.run(sim, scene)
        outs.append(C.collect_outputs(sim, sf, case))
        sim.close()
    err = {k: C.max_rel_err(outs[0][k], outs[1][k], 1e-3) for k in outs[1]}
    assert max(err.values()) <= 1e-5, err
    diff = {k: int(np.sum(np.asarray(outs[0][k], np.float32) != np.asarray(outs[1][k], np.float32))) for k in outs[1]}
    assert not any(diff.values()), diff


@pytest.mark.gpu
@pytest.mark.parametrize("n", [96])
def test_config3_bf16_50_steps_against_fp64_oracle(n, sf, lib, orc, cuda):
    """The config-1 scene generator at n^3 with config 3's storage (BF16
    velocity and density), 20/80 red-black iterations, 50 steps, against the
    FP64 oracle running the same iterations; the FP32 library beside it.
    Prints the relative L2 error per field."""
    scene = sf.scenes.config1(n=n, steps=50)
    outs = {}
    for storage in (sf.STORAGE_FP32, sf.STORAGE_BF16):
        opts = sf.default_options(lib)
        opts.storage = storage
        sim = sf.Simulation(scene.config, scene.scalars, scene.vectors, lib=lib, options=opts)
        sf.scenes.run(sim, scene)
        outs[storage] = {"density": sim.fetch(sf.VIEW_SCALAR_FIELD_DATA, sim.scalar_handles[0]), "velocity": np.stack(sim.fetch(sf.VIEW_FLOW_VELOCITY)), "pressure": sim.fetch(sf.VIEW_FLOW_PRESSURE)}
        sim.close()
    o = orc.Oracle(scene.config, scene.scalars, scene.vectors, precision=64, scheme=orc.RBGS)
    sf.scenes.run(o, scene)
    ref = {"density": o.get(orc.SCALAR, 1), "velocity": np.stack(o.velocity()), "pressure": o.get(orc.PRESSURE)}
    errs = {k: {"fp32": rel_l2(outs[sf.STORAGE_FP32][k], ref[k]), "bf16": rel_l2(outs[sf.STORAGE_BF16][k], ref[k]), "bf16_vs_fp32": rel_l2(outs[sf.STORAGE_BF16][k], outs[sf.STORAGE_FP32][k])} for k in ref}
    print(f"config 3 storage at {n}^3, 50 steps, relative L2 error vs the FP64 oracle:", errs)
    for k, e in errs.items():
        assert e["fp32"] <= 1e-4, (k, errs)
        assert np.isfinite(e["bf16"]) and e["bf16"] <= 1e-1, (k, errs)


def _checksums(binary, args):
    out = subprocess.run([str(binary), *args], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr
    m = re.search(r"total_density=(\S+) peak_density=(\S+)", out.stdout)
    assert m, out.stdout
    return m.group(1), m.group(2)


@pytest.mark.gpu
@pytest.mark.parametrize("args", [
    ["--warmup", "4", "--steps", "16"],  # the benchmark's own default grid and iterations (128x160x128, 24/96)
    ["--nx", "256", "--ny", "256", "--nz", "256", "--diffuse-iters", "20", "--pressure-iters", "80", "--warmup", "2", "--steps", "8"],
], ids=["default_grid", "256_cubed_20_80"])
def test_unchanged_benchmark_prints_reference_checksums(args, cuda):
    """The reference's benchmark.cu, compiled unchanged and linked against
    each library (oracle/Makefile), prints the same total and peak density."""
    if not (REF_BENCH.exists() and B200_BENCH.exists()):
        pytest.skip("benchmark binaries not built (oracle/_ref)")
    assert _checksums(B200_BENCH, args) == _checksums(REF_BENCH, args)
