"""Seeded synthetic scenes (buoyant plumes) for the tests and the benchmark.

No dataset is involved: every input is generated on the host from a seed and
fed identically to every backend (this library, the reference library, the
CPU oracle).

Recorded choices the workload descriptions leave open:
  - cell size h = 1 / nx (unit-width domain);
  - a Gaussian source of radius R cells has profile exp(-r^2 / (2 sigma^2))
    with sigma = R / 2, cut to zero for r > R (r in cells, measured from cell
    centres);
  - the initial velocity perturbation u0 ~ U[-0.01, 0.01]^3 cannot be set
    through the ABI (there is no velocity update entry point), so it enters as
    a one-step impulse: on step 0 the force field is f + u0 / dt.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import (
    FLOW_FREE_SLIP_WALL,
    FLOW_NO_SLIP_WALL,
    FLOW_OUTFLOW,
    FLOW_PERIODIC,
    SCALAR_PERIODIC,
    SCALAR_ZERO_FLUX,
    VECTOR_FIELD_FORCE,
    FlowBoundary,
    FlowFace,
    ScalarBoundary,
    ScalarFace,
    ScalarFieldDesc,
    SimulationConfig,
    VectorFieldDesc,
)

FACES = ("x_minus", "x_plus", "y_minus", "y_plus", "z_minus", "z_plus")


def flow_boundary(types, velocities=None, pressures=None) -> FlowBoundary:
    b = FlowBoundary()
    for k, name in enumerate(FACES):
        v = velocities[k] if velocities is not None else (0.0, 0.0, 0.0)
        p = pressures[k] if pressures is not None else 0.0
        setattr(b, name, FlowFace(types[k], v[0], v[1], v[2], p))
    return b


def scalar_boundary(types, values=None) -> ScalarBoundary:
    b = ScalarBoundary()
    for k, name in enumerate(FACES):
        setattr(b, name, ScalarFace(types[k], values[k] if values is not None else 0.0))
    return b


def stam_walls():
    """All six faces free-slip walls (normal velocity reflected, tangential
    copied, Neumann pressure) and zero-flux scalars."""
    return flow_boundary([FLOW_FREE_SLIP_WALL] * 6), scalar_boundary([SCALAR_ZERO_FLUX] * 6)


def benchmark_walls():
    """The reference benchmark's boundaries (benchmark.cu:93-98, 109-114):
    periodic x and z, no-slip floor, outflow top; scalar periodic x/z,
    zero-flux y."""
    f = flow_boundary([FLOW_PERIODIC, FLOW_PERIODIC, FLOW_NO_SLIP_WALL, FLOW_OUTFLOW, FLOW_PERIODIC, FLOW_PERIODIC])
    s = scalar_boundary([SCALAR_PERIODIC, SCALAR_PERIODIC, SCALAR_ZERO_FLUX, SCALAR_ZERO_FLUX, SCALAR_PERIODIC, SCALAR_PERIODIC])
    return f, s


def gaussian(shape, centre, radius):
    """Profile on cell centres, shape (nz, ny, nx), centre (cx, cy, cz) in
    cells."""
    nz, ny, nx = shape
    cx, cy, cz = centre
    z, y, x = np.meshgrid(np.arange(nz) + 0.5, np.arange(ny) + 0.5, np.arange(nx) + 0.5, indexing="ij")
    r2 = (x - cx) ** 2 + (y - cy) ** 2 + (z - cz) ** 2
    sigma = radius / 2.0
    g = np.exp(-r2 / (2.0 * sigma * sigma))
    g[r2 > radius * radius] = 0.0
    return g


@dataclass
class Scene:
    name: str
    config: SimulationConfig
    scalars: list
    vectors: list
    sources: list  # per scalar: (nz, ny, nx) float32 source, or None
    force: tuple  # (fx, fy, fz) for vector field 0
    impulse: tuple | None = None  # added to the force on step 0 only
    steps: int = 1
    meta: dict = field(default_factory=dict)

    @property
    def shape(self):
        return (self.config.nz, self.config.ny, self.config.nx)


def make_config(n, h, dt, viscosity, diffuse_iterations, pressure_iterations, flow) -> SimulationConfig:
    nx, ny, nz = n
    return SimulationConfig(nx=nx, ny=ny, nz=nz, cell_size=h, dt=dt, viscosity=viscosity, diffuse_iterations=diffuse_iterations, pressure_iterations=pressure_iterations, flow_boundary=flow)


def plume(name, n, *, h=None, dt=0.1, viscosity=1e-4, diffusion=1e-5, dissipation=0.0, diffuse_iterations=20, pressure_iterations=40, sources=(), walls=None, velocity_seed=None, steps=1) -> Scene:
    """A plume scene: `sources` is a list of (cx, cy, cz, radius, density
    strength, upward force) in cells."""
    nx, ny, nz = n
    h = float(np.float32(1.0 / nx)) if h is None else h
    flow, sbc = walls if walls is not None else stam_walls()
    cfg = make_config(n, h, dt, viscosity, diffuse_iterations, pressure_iterations, flow)
    shape = (nz, ny, nx)
    src = np.zeros(shape, np.float64)
    fy = np.zeros(shape, np.float64)
    for cx, cy, cz, radius, strength, up in sources:
        g = gaussian(shape, (cx, cy, cz), radius)
        src += strength * g
        fy += up * g
    zero = np.zeros(shape, np.float32)
    force = (zero, fy.astype(np.float32), zero.copy())
    impulse = None
    if velocity_seed is not None:
        rng = np.random.default_rng(velocity_seed)
        u0 = rng.uniform(-0.01, 0.01, size=(3,) + shape)
        impulse = tuple((u0[k] / dt).astype(np.float32) for k in range(3))
    scalar = ScalarFieldDesc(diffusion=diffusion, dissipation=dissipation, initial_value=0.0, boundary=sbc)
    vector = VectorFieldDesc(usage=VECTOR_FIELD_FORCE, initial_value_x=0.0, initial_value_y=0.0, initial_value_z=0.0)
    return Scene(name, cfg, [scalar], [vector], [src.astype(np.float32)], force, impulse, steps, {"sources": list(sources), "h": h})


def config0(steps=100) -> Scene:
    """Plain method, small: 64^3, dt 0.1, viscosity 1e-4, density diffusion
    1e-5, 20 diffusion / 40 pressure iterations, Stam walls, u0 ~ U[-0.01,
    0.01]^3 from seed 0, one Gaussian source (radius 4 cells, strength 10) at
    bottom centre with an upward force of 5, 100 steps."""
    n = 64
    r = 4.0
    return plume("config0-64^3", (n, n, n), dt=0.1, viscosity=1e-4, diffusion=1e-5, diffuse_iterations=20, pressure_iterations=40, sources=[(n / 2, 4 + r, n / 2, r, 10.0, 5.0)], velocity_seed=0, steps=steps)


def config1(steps=50, seed=1, n=256) -> Scene:
    """Plain method, GPU scale: 256^3 buoyant plume, config-0 coefficients,
    20 diffusion / 80 pressure iterations, two Gaussian sources (radius 8) at
    seeded floor positions with upward forces U[1, 10], 50 steps."""
    r = 8.0
    rng = np.random.default_rng(seed)
    sources = []
    for _ in range(2):
        cx, cz = rng.uniform(r + 2, n - r - 2, size=2)
        sources.append((float(cx), 4 + r, float(cz), r, 10.0, float(rng.uniform(1.0, 10.0))))
    return plume(f"config1-{n}^3", (n, n, n), dt=0.1, viscosity=1e-4, diffusion=1e-5, diffuse_iterations=20, pressure_iterations=80, sources=sources, steps=steps)


def training_scene(seed: int, n: int = 128, pressure_iterations: int = 1000) -> Scene:
    """Learned warm start, training scenes: an n^3 plume (config-0
    coefficients) with 1-4 Gaussian sources of radius U[4, 12] cells at
    seeded floor positions, each with an upward force U[1, 10]; the pressure
    solve is the target generator (`pressure_iterations` sweeps)."""
    rng = np.random.default_rng(1000 + seed)
    sources = []
    for _ in range(int(rng.integers(1, 5))):
        r = float(rng.uniform(4.0, 12.0))
        cx, cz = rng.uniform(r + 2, n - r - 2, size=2)
        sources.append((float(cx), 4 + r, float(cz), r, 10.0, float(rng.uniform(1.0, 10.0))))
    return plume(f"train-{seed}-{n}^3", (n, n, n), dt=0.1, viscosity=1e-4, diffusion=1e-5, diffuse_iterations=20, pressure_iterations=pressure_iterations, sources=sources, steps=1)


def batch_scenes(count: int = 64, seed: int = 4, steps: int = 100) -> list[Scene]:
    """Batched workload: `count` plumes with sizes drawn from the seed over
    {32, 48, 64, 96, 128}^3, each with its own seeded Gaussian source
    (radius 2-6 cells, strength 10) and upward force U[1, 10], config-0
    coefficients (dt 0.1, viscosity 1e-4, diffusion 1e-5, 20 diffusion and 40
    pressure iterations, Stam walls), `steps` steps."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        n = int(rng.choice([32, 48, 64, 96, 128]))
        r = float(rng.uniform(2.0, 6.0))
        cx, cz = rng.uniform(r + 2, n - r - 2, size=2)
        src = [(float(cx), 2 + r, float(cz), r, 10.0, float(rng.uniform(1.0, 10.0)))]
        out.append(plume(f"batch-{k}-{n}^3", (n, n, n), dt=0.1, viscosity=1e-4, diffusion=1e-5, diffuse_iterations=20, pressure_iterations=40, sources=src, steps=steps))
    return out


def apply_inputs(sim, scene: Scene, step_index: int):
    """Uploads the scene's source and force for step `step_index` (the
    impulse only on step 0). `sim` is anything with set_scalar_source and
    set_vector (the library binding or the oracle binding)."""
    if step_index == 0:
        for k, src in enumerate(scene.sources):
            if src is not None:
                sim.set_scalar_source(k + 1, src)
    if scene.impulse is not None and step_index == 0:
        f = tuple((scene.force[k].astype(np.float32) + scene.impulse[k]).astype(np.float32) for k in range(3))
        sim.set_vector(1, *f)
    elif step_index == 0 or (scene.impulse is not None and step_index == 1):
        sim.set_vector(1, *scene.force)


def run(sim, scene: Scene, steps: int | None = None, start: int = 0):
    steps = scene.steps if steps is None else steps
    for k in range(start, start + steps):
        apply_inputs(sim, scene, k)
        sim.step(1)
