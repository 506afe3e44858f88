"""Small seeded cases that cover every boundary kind of the ABI, used for the
golden fixtures (outputs of the reference library itself) and for the GPU
parity tests.

Coverage: all four flow boundary kinds (no-slip with a moving wall,
free-slip, outflow with a non-zero pressure, periodic), all three scalar
kinds (fixed value, zero flux, periodic), odd grid sizes, two scalars, two
force fields, a time-varying force, dissipation, and the alpha <= 0 path
(zero viscosity / diffusion). Periodic axes have even sizes: with an odd
periodic size the reference's red-black sweep updates two neighbouring
cells of the same colour concurrently, so its result is not deterministic.
"""

from __future__ import annotations

import ctypes
import json
from dataclasses import dataclass, field

import numpy as np


def struct_to_obj(s):
    if isinstance(s, ctypes.Structure):
        return {name: struct_to_obj(getattr(s, name)) for name, _ in s._fields_}
    if isinstance(s, ctypes.Array):
        return [struct_to_obj(v) for v in s]
    return s


def obj_to_struct(cls, obj):
    s = cls()
    for name, ftype in cls._fields_:
        v = obj[name]
        if isinstance(ftype, type) and issubclass(ftype, ctypes.Structure):
            setattr(s, name, obj_to_struct(ftype, v))
        elif isinstance(ftype, type) and issubclass(ftype, ctypes.Array):
            arr = getattr(s, name)
            for i, x in enumerate(v):
                arr[i] = x
        else:
            setattr(s, name, v)
    return s


@dataclass
class Case:
    name: str
    config: object
    scalars: list
    vectors: list
    steps: int
    init_scalars: dict = field(default_factory=dict)   # handle -> (nz, ny, nx)
    sources: dict = field(default_factory=dict)        # handle -> (nz, ny, nx)
    forces: dict = field(default_factory=dict)         # handle -> (fx, fy, fz)
    impulse: tuple | None = None                       # added to vector 1 on step 0
    force_ramp: float = 0.0                            # vector 1 scaled by (1 + ramp * step)

    @property
    def shape(self):
        return (self.config.nz, self.config.ny, self.config.nx)

    def force_at(self, handle, k):
        f = self.forces[handle]
        if handle == 1 and self.force_ramp:
            f = tuple((c * np.float32(1.0 + self.force_ramp * k)).astype(np.float32) for c in f)
        if handle == 1 and k == 0 and self.impulse is not None:
            f = tuple((f[i] + self.impulse[i]).astype(np.float32) for i in range(3))
        return f

    def drive(self, sim, steps=None, start=0):
        steps = self.steps if steps is None else steps
        if start == 0:
            for h, a in self.init_scalars.items():
                sim.set_scalar(h, a)
            for h, a in self.sources.items():
                sim.set_scalar_source(h, a)
        for k in range(start, start + steps):
            for h in self.forces:
                if k == 0 or (h == 1 and (self.force_ramp or (self.impulse is not None and k == 1))):
                    sim.set_vector(h, *self.force_at(h, k))
            sim.step(1)

    def to_json(self, sf):
        return json.dumps({
            "name": self.name, "steps": self.steps, "force_ramp": self.force_ramp,
            "config": struct_to_obj(self.config),
            "scalars": [struct_to_obj(s) for s in self.scalars],
            "vectors": [struct_to_obj(v) for v in self.vectors],
        })


def _sf():
    import importlib
    return importlib.import_module("stable-fluids_b200")


def build_cases():
    sf = _sf()
    sc = sf.scenes
    cases = []

    # 1. Stam walls, plume source, initial velocity impulse.
    s = sc.plume("walls", (16, 12, 10), sources=[(8, 4, 5, 3.0, 10.0, 5.0)], velocity_seed=0, diffuse_iterations=4, pressure_iterations=8)
    cases.append(Case("walls_16x12x10", s.config, s.scalars, s.vectors, 4, sources={1: s.sources[0]}, forces={1: s.force}, impulse=s.impulse))

    # 2. The reference benchmark's boundaries with a moving floor and a
    #    non-zero outflow pressure; two scalars (one with fixed values), two
    #    force fields, time-varying force, dissipation.
    n = (16, 12, 16)
    shape = (n[2], n[1], n[0])
    vel = [(0, 0, 0), (0, 0, 0), (0.2, 0.0, -0.1), (0, 0, 0), (0, 0, 0), (0, 0, 0)]
    prs = [0, 0, 0, 0.25, 0, 0]
    flow = sc.flow_boundary([sf.FLOW_PERIODIC, sf.FLOW_PERIODIC, sf.FLOW_NO_SLIP_WALL, sf.FLOW_OUTFLOW, sf.FLOW_PERIODIC, sf.FLOW_PERIODIC], vel, prs)
    s1 = sf.ScalarFieldDesc(diffusion=5e-5, dissipation=0.35, initial_value=0.0, boundary=sc.scalar_boundary([sf.SCALAR_PERIODIC, sf.SCALAR_PERIODIC, sf.SCALAR_ZERO_FLUX, sf.SCALAR_ZERO_FLUX, sf.SCALAR_PERIODIC, sf.SCALAR_PERIODIC]))
    s2 = sf.ScalarFieldDesc(diffusion=2e-4, dissipation=0.0, initial_value=0.3, boundary=sc.scalar_boundary([sf.SCALAR_PERIODIC, sf.SCALAR_PERIODIC, sf.SCALAR_FIXED_VALUE, sf.SCALAR_FIXED_VALUE, sf.SCALAR_PERIODIC, sf.SCALAR_PERIODIC], [0, 0, 1.0, 0.5, 0, 0]))
    cfg = sc.make_config(n, 0.01, 1.0 / 90.0, 1.2e-4, 5, 10, flow)
    g = sc.gaussian(shape, (8, 3, 8), 3.0).astype(np.float32)
    rng = np.random.default_rng(3)
    swirl = tuple(rng.uniform(-0.5, 0.5, size=shape).astype(np.float32) for _ in range(3))
    vecs = [sf.VectorFieldDesc(sf.VECTOR_FIELD_FORCE, 0, 0, 0), sf.VectorFieldDesc(sf.VECTOR_FIELD_FORCE, 0.05, 0, 0)]
    cases.append(Case("benchmark_walls_16x12x16", cfg, [s1, s2], vecs, 4, sources={1: (28 * g).astype(np.float32), 2: (3 * g).astype(np.float32)}, forces={1: (np.zeros(shape, np.float32), (7.5 * g).astype(np.float32), np.zeros(shape, np.float32)), 2: swirl}, force_ramp=0.1))

    # 3. alpha <= 0: no viscosity, no diffusion (advection results dropped).
    s = sc.plume("quirk", (12, 10, 8), viscosity=0.0, diffusion=0.0, dissipation=0.2, sources=[(6, 3, 4, 2.5, 10.0, 4.0)], velocity_seed=1, diffuse_iterations=3, pressure_iterations=6)
    cases.append(Case("alpha_zero_12x10x8", s.config, s.scalars, s.vectors, 3, sources={1: s.sources[0]}, forces={1: s.force}, impulse=s.impulse))

    # 4. Odd sizes, every non-periodic kind mixed, moving walls, outflow
    #    pressures, random initial scalar and force.
    n = (17, 9, 13)
    shape = (n[2], n[1], n[0])
    types = [sf.FLOW_NO_SLIP_WALL, sf.FLOW_OUTFLOW, sf.FLOW_FREE_SLIP_WALL, sf.FLOW_NO_SLIP_WALL, sf.FLOW_OUTFLOW, sf.FLOW_FREE_SLIP_WALL]
    vel = [(0, 0.3, 0), (0, 0, 0), (0.1, 0.2, 0.3), (-0.2, 0, 0.1), (0, 0, 0), (0.05, 0.05, 0.05)]
    prs = [0, 0.1, 0, 0, -0.05, 0]
    flow = sc.flow_boundary(types, vel, prs)
    sbc = sc.scalar_boundary([sf.SCALAR_FIXED_VALUE, sf.SCALAR_ZERO_FLUX, sf.SCALAR_ZERO_FLUX, sf.SCALAR_FIXED_VALUE, sf.SCALAR_ZERO_FLUX, sf.SCALAR_ZERO_FLUX], [2.0, 0, 0, 0.0, 0, 0])
    cfg = sc.make_config(n, float(np.float32(1 / 17)), 0.05, 5e-4, 4, 9, flow)
    rng = np.random.default_rng(5)
    rho0 = rng.uniform(0, 1, size=shape).astype(np.float32)
    frc = tuple(rng.uniform(-2, 2, size=shape).astype(np.float32) for _ in range(3))
    cases.append(Case("mixed_odd_17x9x13", cfg, [sf.ScalarFieldDesc(1e-3, 0.0, 0.0, sbc)], [sf.VectorFieldDesc(sf.VECTOR_FIELD_FORCE, 0, 0, 0)], 3, init_scalars={1: rho0}, forces={1: frc}))

    # 5. Fully periodic (singular pressure system), random force.
    n = (16, 8, 12)
    shape = (n[2], n[1], n[0])
    flow = sc.flow_boundary([sf.FLOW_PERIODIC] * 6)
    sbc = sc.scalar_boundary([sf.SCALAR_PERIODIC] * 6)
    cfg = sc.make_config(n, 0.0625, 0.1, 2e-4, 4, 8, flow)
    rng = np.random.default_rng(7)
    frc = tuple(rng.uniform(-1, 1, size=shape).astype(np.float32) for _ in range(3))
    rho0 = rng.uniform(0, 2, size=shape).astype(np.float32)
    cases.append(Case("periodic_16x8x12", cfg, [sf.ScalarFieldDesc(1e-3, 0.0, 0.0, sbc)], [sf.VectorFieldDesc(sf.VECTOR_FIELD_FORCE, 0, 0, 0)], 3, init_scalars={1: rho0}, forces={1: frc}))
    return cases


OUTPUTS = ("velocity_x", "velocity_y", "velocity_z", "pressure", "divergence", "magnitude")


def collect_outputs(sim, sf, case):
    """Final fields of a library-backed simulation, by name."""
    out = {}
    u = sim.fetch(sf.VIEW_FLOW_VELOCITY)
    for k in range(3):
        out[OUTPUTS[k]] = u[k]
    out["pressure"] = sim.fetch(sf.VIEW_FLOW_PRESSURE)
    out["divergence"] = sim.fetch(sf.VIEW_FLOW_DIVERGENCE)
    out["magnitude"] = sim.fetch(sf.VIEW_FLOW_VELOCITY_MAGNITUDE)
    for i, h in enumerate(sim.scalar_handles):
        out[f"scalar{i + 1}"] = sim.fetch(sf.VIEW_SCALAR_FIELD_DATA, h)
    return out


def collect_oracle(o, orc, case):
    out = {}
    for k in range(3):
        out[OUTPUTS[k]] = o.get(orc.VELOCITY, 0, k)
    out["pressure"] = o.get(orc.PRESSURE)
    out["divergence"] = o.get(orc.DIVERGENCE)
    out["magnitude"] = o.get(orc.MAGNITUDE)
    for i in range(len(case.scalars)):
        out[f"scalar{i + 1}"] = o.get(orc.SCALAR, i + 1)
    return out


def max_rel_err(a, b, floor=1e-6):
    """max |a - b| / max(|b|, floor * max|b|) -- relative error with a floor so
    that values near zero are judged against the field's scale."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    scale = float(np.abs(b).max())
    if scale == 0.0:
        return float(np.abs(a).max())
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), floor * scale)))
