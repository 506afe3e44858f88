"""CPU restatement of the reference viewer's plume scene inputs (test
infrastructure only: the library never imports this module).

vulkan-app/scene_plume.cpp:229-300 builds, once, the density source and the
force's y component of a source sphere and two host masks (a swirl field
around the plume axis, a drift sphere above the source); :323-330 then
recomputes the force's x and z components on the host every animation step.
The arithmetic here is the viewer's float32 arithmetic, one rounding per
operation (NumPy float32 elementwise operations and np.sqrt are correctly
rounded and never contracted), and the three animated scalars come from the C
library's sinf / cosf, as the viewer's std::sin / std::cos on float do.

Parity unpinned against the viewer itself: its code is a C++ module built
against Vulkan and cannot run here; the restatement follows the source line
by line instead.
"""

from __future__ import annotations

import ctypes
import ctypes.util

import numpy as np

_libm = ctypes.CDLL(ctypes.util.find_library("m") or "libm.so.6")
_libm.sinf.argtypes = [ctypes.c_float]
_libm.sinf.restype = ctypes.c_float
_libm.cosf.argtypes = [ctypes.c_float]
_libm.cosf.restype = ctypes.c_float

F = np.float32


def geometry(nx: int, ny: int, nz: int, h: float) -> dict:
    """scene_plume.cpp:229-246 (world units)."""
    h = F(h)
    ex, ey, ez = F(nx) * h, F(ny) * h, F(nz) * h
    g = {"h": h, "source_x": ex * F(0.50), "source_y": ey * F(0.13), "source_z": ez * F(0.50), "source_r": h * F(6.0)}
    g["swirl_y"] = g["source_y"] + g["source_r"] * F(0.90)
    g["drift_y"] = g["source_y"] + g["source_r"] * F(1.35)
    g["swirl_r"] = g["source_r"] * F(1.65)
    g["drift_r"] = g["source_r"] * F(2.10)
    return g


def _radial_weight(px, py, pz, cx, cy, cz, radius):
    """scene_plume.cpp:257-265: 1 - |p - c|^2 / r^2 inside the sphere, else 0."""
    dx, dy, dz = px - cx, py - cy, pz - cz
    r2 = F(radius) * F(radius)
    d2 = (dx * dx + dy * dy) + dz * dz
    w = F(1.0) - d2 / r2
    return np.where((d2 >= r2) | (r2 <= F(0.0)), F(0.0), w).astype(F)


def _centres(nx, ny, nz, h):
    x = (np.arange(nx, dtype=F) + F(0.5)) * F(h)
    y = (np.arange(ny, dtype=F) + F(0.5)) * F(h)
    z = (np.arange(nz, dtype=F) + F(0.5)) * F(h)
    return x[None, None, :], y[None, :, None], z[:, None, None]


def masks(nx: int, ny: int, nz: int, h: float) -> dict:
    """Arrays (nz, ny, nx), float32: source weight, swirl x/z masks, drift mask
    (scene_plume.cpp:267-287)."""
    g = geometry(nx, ny, nz, h)
    px, py, pz = _centres(nx, ny, nz, g["h"])
    shape = (nz, ny, nx)
    px, py, pz = np.broadcast_to(px, shape), np.broadcast_to(py, shape), np.broadcast_to(pz, shape)
    source_w = _radial_weight(px, py, pz, g["source_x"], g["source_y"], g["source_z"], g["source_r"])
    swirl_w = _radial_weight(px, py, pz, g["source_x"], g["swirl_y"], g["source_z"], g["swirl_r"])
    drift_w = _radial_weight(px, py, pz, g["source_x"], g["drift_y"], g["source_z"], g["drift_r"])
    dx = px - g["source_x"]
    dz = pz - g["source_z"]
    radial = np.sqrt(dx * dx + dz * dz)
    with np.errstate(divide="ignore"):
        inv = np.where(radial > F(1.0e-5), F(1.0) / radial, F(0.0)).astype(F)
    return {"source": source_w, "swirl_x": (-dz * inv) * swirl_w, "swirl_z": (dx * inv) * swirl_w, "drift": drift_w}


def setup_fields(nx: int, ny: int, nz: int, h: float) -> dict:
    """The constant inputs: density source 32 w, force y 7.6 w (:285-286)."""
    m = masks(nx, ny, nz, h)
    return {"density_source": F(32.0) * m["source"], "force_y": F(7.6) * m["source"]}


def animation_scalars(step: int) -> tuple[float, float, float]:
    """drift_x, drift_z, swirl of one animation step (scene_plume.cpp:323-326)."""
    phase = F(step) * F(0.045)
    drift_x = F(1.15) * F(_libm.sinf(phase))
    drift_z = F(0.85) * F(_libm.cosf(phase * F(0.71)))
    swirl = F(1.65) * F(_libm.cosf(phase * F(0.53)))
    return drift_x, drift_z, swirl


def step_forces(nx: int, ny: int, nz: int, h: float, step: int, m: dict | None = None) -> tuple[np.ndarray, np.ndarray]:
    """Force x and z of one animation step (scene_plume.cpp:327-330)."""
    m = masks(nx, ny, nz, h) if m is None else m
    drift_x, drift_z, swirl = animation_scalars(step)
    fx = drift_x * m["drift"] + swirl * m["swirl_x"]
    fz = drift_z * m["drift"] + swirl * m["swirl_z"]
    return fx.astype(F), fz.astype(F)
