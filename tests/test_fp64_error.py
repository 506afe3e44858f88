"""Error of each benchmarked configuration against the FP64 oracle, on the
benchmark's scene at 32^3 (the config-1 plume: two seeded sources, 20
diffusion iterations, Stam walls), after 8 steps:

  - the reference configuration (80 red-black Gauss-Seidel iterations per
    step) against the FP64 oracle running the same iterations: the FP32
    rounding error alone;
  - every variant of the residual-driven benchmark (learned warm start,
    plain Jacobi from zero, Jacobi from the previous pressure, red-black
    Gauss-Seidel from zero; rel_res <= 1e-3 checked every 16 sweeps) and
    the reference configuration against the FP64 oracle with its pressure
    solved to rel_res <= 1e-9 in every step: what stopping the solve early
    costs, next to the rounding error.

The pressure is compared with its mean removed (all-wall boundaries fix it
only up to a constant). The errors are printed (pytest -s) and bounded.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

STEPS = 8
TOL = 1e-3
CHECK_INTERVAL = 16
CAP = 20000


def scene(sf, seed=1):
    return sf.scenes.config1(steps=STEPS, seed=seed, n=32)


def rel_l2(a, ref):
    a = np.asarray(a, np.float64)
    ref = np.asarray(ref, np.float64)
    return float(np.linalg.norm(a - ref) / max(np.linalg.norm(ref), 1e-300))


def fields_of(sim, sf):
    p = np.asarray(sim.fetch(sf.VIEW_FLOW_PRESSURE), np.float64)
    return {"velocity": np.stack(sim.fetch(sf.VIEW_FLOW_VELOCITY)), "density": sim.fetch(sf.VIEW_SCALAR_FIELD_DATA, sim.scalar_handles[0]), "pressure": p - p.mean()}


def oracle_fields(o, orc):
    p = np.asarray(o.get(orc.PRESSURE), np.float64)
    return {"velocity": np.stack(o.velocity()), "density": o.get(orc.SCALAR, 1), "pressure": p - p.mean()}


def variant_options(sf, lib, variant):
    o = sf.default_options(lib)
    o.scheme = sf.SCHEME_RBGS if variant in ("rbgs", "reference_80") else sf.SCHEME_JACOBI
    o.compute_residual = 1
    if variant == "reference_80":
        return o
    o.warm_start = {"learned": sf.WARM_START_LEARNED, "plain": sf.WARM_START_ZERO, "previous": sf.WARM_START_PREVIOUS, "rbgs": sf.WARM_START_ZERO}[variant]
    o.residual_tolerance = TOL
    o.residual_check_interval = CHECK_INTERVAL
    o.max_pressure_iterations = CAP
    o.warm_start_trial_iterations = CHECK_INTERVAL
    return o


def trained_network(sf, lib):
    """A network trained briefly on pairs from another seed of the scene."""
    other = scene(sf, seed=5)

    def make():
        o = sf.default_options(lib)
        o.scheme = sf.SCHEME_JACOBI
        o.warm_start = sf.WARM_START_PREVIOUS
        o.compute_residual = 0
        s = sf.Simulation(other.config, other.scalars, other.vectors, lib=lib, options=o)
        for k in range(2):
            sf.scenes.apply_inputs(s, other, k)
        return s

    pairs = list(sf.warmstart.training_pairs(make, steps=16, skip=2))
    net = sf.WarmStartNetwork(seed=11, lib=lib)
    for _ in range(20):
        for b, p, t in pairs:
            net.train_step(b, p, t, other.config.cell_size, 2e-3)
    return net


def test_benchmark_variants_against_fp64_oracle(sf, lib, orc, cuda):
    sc = scene(sf)
    # FP64 references: the same 80 RBGS iterations, and a converged solve
    ref80 = orc.Oracle(sc.config, sc.scalars, sc.vectors, precision=64, scheme=orc.RBGS)
    sf.scenes.run(ref80, sc)
    fields80 = oracle_fields(ref80, orc)
    ref80.close()
    conv = orc.Oracle(sc.config, sc.scalars, sc.vectors, precision=64, scheme=orc.JACOBI)
    conv.set_solver(tolerance=1e-9, max_iterations=200000, check_interval=CHECK_INTERVAL, warm_previous=True, compute_residual=True)
    sf.scenes.run(conv, sc)
    assert conv.stats()["rel_residual"] <= 1e-9
    converged = oracle_fields(conv, orc)
    conv.close()

    net = trained_network(sf, lib)
    errors, iterations = {}, {}
    try:
        for variant in ("reference_80", "learned", "plain", "previous", "rbgs"):
            sim = sf.Simulation(sc.config, sc.scalars, sc.vectors, lib=lib, options=variant_options(sf, lib, variant))
            if variant == "learned":
                net.attach(sim)
            its = []
            for k in range(STEPS):
                sf.scenes.apply_inputs(sim, sc, k)
                sim.step(1)
                st = sim.stats()
                its.append(st.pressure_iterations)
                if variant != "reference_80":
                    assert st.rel_residual <= TOL and not st.hit_cap, (variant, k, st.rel_residual)
            got = fields_of(sim, sf)
            if variant == "learned":
                sf.WarmStartNetwork.detach(sim)
            sim.close()
            iterations[variant] = its
            errors[variant] = {k: rel_l2(got[k], converged[k]) for k in got}
            if variant == "reference_80":
                errors["reference_80 vs FP64 same iterations"] = {k: rel_l2(got[k], fields80[k]) for k in got}
    finally:
        net.close()

    for name, e in errors.items():
        print(f"{name:40s} " + "  ".join(f"{k} {v:.2e}" for k, v in e.items()), iterations.get(name, ""))
    # rounding alone: FP32 against FP64 with the same arithmetic (measured
    # 1-3e-7 per field)
    for k, v in errors["reference_80 vs FP64 same iterations"].items():
        assert v <= 1e-5, (k, v)
    # stopping at rel_res <= 1e-3: every variant within 5e-3 of the converged
    # FP64 step in every field (measured 4e-4 - 1.2e-3); the reference's own
    # 80 iterations are far from converged (measured 0.17 - 0.25)
    for variant in ("learned", "plain", "previous", "rbgs"):
        for k, v in errors[variant].items():
            assert np.isfinite(v) and v <= 5e-3, (variant, k, errors[variant])
    assert min(errors["reference_80"].values()) > 10 * max(errors["plain"].values())
