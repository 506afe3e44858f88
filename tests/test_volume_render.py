"""Headless volume rendering (stable_fluids_b200_render_volume): the CUDA
restatement of the viewer's volume shader against the NumPy restatement
(oracle/volume.py), for a positive and a signed field, perspective and
orthographic cameras."""

import numpy as np
import pytest

from oracle import volume


def _camera(projection, nx, ny, nz, h, width=64, height=48):
    ext = np.array([nx * h, ny * h, nz * h], np.float32)
    centre = ext / 2
    eye = centre + np.array([0.35, 0.25, -1.6], np.float32) * ext.max()
    fwd = centre - eye
    fwd /= np.linalg.norm(fwd)
    right = np.cross(np.array([0, 1, 0], np.float32), fwd)
    right /= np.linalg.norm(right)
    up = np.cross(fwd, right)
    return {"eye": eye, "right": right, "up": up, "forward": fwd, "volume_min": np.zeros(3, np.float32), "volume_max": ext,
            "color_a": np.array([0.1, 0.2, 0.9], np.float32), "color_b": np.array([1.0, 0.6, 0.1], np.float32),
            "aspect": width / height, "tan_half_fov": 0.55, "value_scale": 1.0, "density": 18.0, "value_min": 0.0, "value_max": 1.0,
            "ortho_height": float(ext.max()) * 1.4, "steps": 48, "projection": projection, "width": width, "height": height}


def test_oracle_render_basics():
    """Empty field renders transparent; a dense blob renders an opaque-ish
    centre and transparent corners; alpha stays in [0, 1]."""
    nx, ny, nz, h = 24, 20, 16, 1.0 / 24
    cam = _camera(0, nx, ny, nz, h)
    img = volume.render(np.zeros((nz, ny, nx), np.float32), cam)
    assert not img.any()
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    blob = np.exp(-((x - nx / 2) ** 2 + (y - ny / 2) ** 2 + (z - nz / 2) ** 2) / 18.0).astype(np.float32)
    img = volume.render(blob, cam)
    a = img[..., 3]
    assert a.min() >= 0.0 and a.max() <= 1.0 and a[24, 32] > 0.3 and a[0, 0] == 0.0


@pytest.mark.gpu
@pytest.mark.parametrize("projection,signed", [(0, False), (1, False), (0, True)])
def test_device_render_matches_restated_shader(projection, signed, sf, lib, cuda):
    nx, ny, nz = 24, 20, 16
    scene = sf.scenes.plume("render", (nx, ny, nz), diffuse_iterations=2, pressure_iterations=4)
    h = scene.config.cell_size
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    blob = np.exp(-((x - nx / 2) ** 2 + (y - ny / 2.5) ** 2 + (z - nz / 2) ** 2) / 18.0).astype(np.float32)
    if signed:
        blob = (blob * np.sin(x / 3.0)).astype(np.float32)
    sim = sf.Simulation(scene.config, scene.scalars, scene.vectors, lib=lib)
    sim.set_scalar(sim.scalar_handles[0], blob)
    cam = _camera(projection, nx, ny, nz, h)
    if signed:
        cam["value_min"], cam["value_max"] = -1.0, 1.0
    p = sf.B200VolumeRender()
    for k, val in cam.items():
        if isinstance(val, np.ndarray):
            getattr(p, k)[:] = [float(t) for t in val]
        else:
            setattr(p, k, val)
    got = sim.render_volume(sf.VIEW_SCALAR_FIELD_DATA, p, sim.scalar_handles[0]).cpu().numpy()
    sim.close()
    ref = volume.render(blob, cam)
    err = np.abs(got - ref)
    assert np.isfinite(got).all()
    assert err.max() <= 2e-2, float(err.max())
    assert np.mean(err <= 1e-4) >= 0.995, float(np.mean(err <= 1e-4))
    assert ref[..., 3].max() > 0.2
