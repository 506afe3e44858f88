"""The reference viewer's plume scene generated on the device
(stable_fluids_b200_plume_scene_setup / _forces) against the CPU
restatement of vulkan-app/scene_plume.cpp:229-335 (oracle/scene_plume.py)."""

import numpy as np
import pytest

from oracle import scene_plume as sp


def test_oracle_masks_are_the_viewers_shapes():
    """Weights in [0, 1] and zero outside their spheres; the swirl mask is
    tangential (perpendicular to the horizontal radius) and zero on the axis."""
    nx, ny, nz, h = 40, 56, 32, np.float32(1.0 / 40)
    m = sp.masks(nx, ny, nz, h)
    g = sp.geometry(nx, ny, nz, h)
    for k in ("source", "drift"):
        assert m[k].min() >= 0.0 and m[k].max() <= 1.0 and m[k].max() > 0.5
    z, y, x = np.meshgrid(*[(np.arange(n) + 0.5) * float(h) for n in (nz, ny, nx)], indexing="ij")
    far = (x - g["source_x"]) ** 2 + (y - g["source_y"]) ** 2 + (z - g["source_z"]) ** 2 >= float(g["source_r"]) ** 2 * 1.0001
    assert np.all(m["source"][far] == 0.0)
    dx, dz = x - g["source_x"], z - g["source_z"]
    dot = dx * m["swirl_x"] + dz * m["swirl_z"]
    assert np.max(np.abs(dot)) <= 1e-6 * max(float(np.max(np.abs(m["swirl_x"]))), 1e-30)
    fx, fz = sp.step_forces(nx, ny, nz, h, 0, m)
    assert fx.dtype == np.float32 and np.array_equal(fx, np.float32(0.0) * m["drift"] + np.float32(1.65) * m["swirl_x"])
    assert sp.animation_scalars(0) == (np.float32(0.0), np.float32(0.85), np.float32(1.65))


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(40, 56, 32), (33, 20, 17)])
def test_device_scene_equals_the_viewers_host_fields(shape, sf, lib, cuda):
    """Density source, force y (setup) and force x / z for three animation
    steps equal the host restatement bit for bit, and a step runs on them."""
    nx, ny, nz = shape
    scene = sf.scenes.plume("viewer", (nx, ny, nz), diffuse_iterations=4, pressure_iterations=8)
    h = scene.config.cell_size
    sim = sf.Simulation(scene.config, scene.scalars, scene.vectors, lib=lib)
    sim.plume_scene_setup()
    ref = sp.setup_fields(nx, ny, nz, h)
    src = sim.fetch(sf.VIEW_SCALAR_FIELD_SOURCE, sim.scalar_handles[0])
    fx, fy, fz = sim.fetch(sf.VIEW_VECTOR_FIELD, sim.vector_handles[0])
    assert np.array_equal(src, ref["density_source"]) and np.array_equal(fy, ref["force_y"])
    assert not fx.any() and not fz.any()
    m = sp.masks(nx, ny, nz, h)
    for step in (0, 7, 123):
        sim.plume_scene_forces(step)
        gx, gy, gz = sim.fetch(sf.VIEW_VECTOR_FIELD, sim.vector_handles[0])
        rx, rz = sp.step_forces(nx, ny, nz, h, step, m)
        assert np.array_equal(gx, rx), (step, int(np.sum(gx != rx)))
        assert np.array_equal(gz, rz), (step, int(np.sum(gz != rz)))
        assert np.array_equal(gy, ref["force_y"])
        sim.step(1)
    rho = sim.fetch(sf.VIEW_SCALAR_FIELD_DATA, sim.scalar_handles[0])
    assert np.isfinite(rho).all() and rho.max() > 0.0
    sim.close()
