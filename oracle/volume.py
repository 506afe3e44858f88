"""CPU restatement of the reference viewer's volume shader
(vulkan-app/shaders/field_volume.slang:37-175) in NumPy float32, vectorised
over pixels -- test infrastructure only: the library never imports this
module. Parity unpinned against the shader itself (no graphics stack on this
machine); it follows the shader's expressions line by line."""

from __future__ import annotations

import numpy as np

F = np.float32


def _normalize(v):
    n = np.sqrt(v[..., 0] * v[..., 0] + v[..., 1] * v[..., 1] + v[..., 2] * v[..., 2])
    return v / n[..., None]


def _sample_field(field, uvw):
    """sample_field (:37-59); field is (nz, ny, nx)."""
    nz, ny, nx = field.shape
    uvw = np.clip(uvw, F(0.0), F(1.0))
    p = uvw * np.array([nx - 1, ny - 1, nz - 1], dtype=F)
    fl = np.floor(p)
    lo = fl.astype(np.int64)
    hi = np.minimum(lo + 1, np.array([nx - 1, ny - 1, nz - 1]))
    t = (p - fl).astype(F)

    def at(x, y, z):
        return field[z, y, x]

    def lerp(a, b, s):
        return a + s * (b - a)

    lx, ly, lz = lo[..., 0], lo[..., 1], lo[..., 2]
    hx, hy, hz = hi[..., 0], hi[..., 1], hi[..., 2]
    c00 = lerp(at(lx, ly, lz), at(hx, ly, lz), t[..., 0])
    c10 = lerp(at(lx, hy, lz), at(hx, hy, lz), t[..., 0])
    c01 = lerp(at(lx, ly, hz), at(hx, ly, hz), t[..., 0])
    c11 = lerp(at(lx, hy, hz), at(hx, hy, hz), t[..., 0])
    return lerp(lerp(c00, c10, t[..., 1]), lerp(c01, c11, t[..., 1]), t[..., 2])


def render(field: np.ndarray, p: dict) -> np.ndarray:
    """RGBA image (height, width, 4), premultiplied colour; `p` holds the
    keys of StableFluidsB200VolumeRender."""
    field = np.asarray(field, F)
    W, H = int(p["width"]), int(p["height"])
    v3 = {k: np.asarray(p[k], F) for k in ("eye", "right", "up", "forward", "volume_min", "volume_max", "color_a", "color_b")}
    px, py = np.meshgrid(np.arange(W, dtype=F), np.arange(H, dtype=F))
    u = (px + F(0.5)) / F(W) * F(2.0) - F(1.0)
    v = -((py + F(0.5)) / F(H) * F(2.0) - F(1.0))
    if int(p["projection"]) != 0:
        hh = F(p["ortho_height"]) * F(0.5)
        hw = hh * F(p["aspect"])
        origin = v3["eye"] + v3["right"] * (u * hw)[..., None] + v3["up"] * (v * hh)[..., None]
        d = _normalize(v3["forward"][None, None, :].repeat(H, 0).repeat(W, 1))
    else:
        origin = np.broadcast_to(v3["eye"], (H, W, 3)).astype(F)
        d = _normalize(v3["forward"] + v3["right"] * (u * F(p["aspect"]) * F(p["tan_half_fov"]))[..., None] + v3["up"] * (v * F(p["tan_half_fov"]))[..., None])
    safe = np.where(np.abs(d) < F(1e-6), np.where(d < 0, F(-1e-6), F(1e-6)), d).astype(F)
    inv = F(1.0) / safe
    t0v = (v3["volume_min"] - origin) * inv
    t1v = (v3["volume_max"] - origin) * inv
    entry = np.max(np.minimum(t0v, t1v), axis=-1)
    exit_ = np.min(np.maximum(t0v, t1v), axis=-1)
    t0 = np.maximum(entry, F(0.0))
    t1 = exit_
    hit = t1 > t0
    steps = max(int(p["steps"]), 1)
    step_len = ((t1 - t0) / F(steps)).astype(F)
    extent = np.maximum(v3["volume_max"] - v3["volume_min"], F(1e-5))
    vmin = F(p["value_min"])
    vmax = max(F(p["value_max"]), F(vmin + F(1e-5)))
    signed = vmin < 0 and vmax > 0
    abs_max = max(abs(vmin), abs(vmax))
    trans = np.ones((H, W), F)
    color = np.zeros((H, W, 3), F)
    active = hit.copy()
    for i in range(steps):
        travel = t0 + (F(i) + F(0.5)) * step_len
        w = origin + d * travel[..., None]
        uvw = (w - v3["volume_min"]) / extent
        value = _sample_field(field, uvw) * F(p["value_scale"])
        if signed:
            level = np.clip(np.abs(value) / F(abs_max), F(0.0), F(1.0)) if abs_max > F(1e-5) else np.zeros_like(value)
            sample = np.where((value < 0)[..., None], v3["color_a"], v3["color_b"])
        else:
            level = np.clip((value - vmin) / (vmax - vmin), F(0.0), F(1.0))
            sample = v3["color_a"] + level[..., None] * (v3["color_b"] - v3["color_a"])
        upd = active & (level >= F(1e-4))
        alpha = F(1.0) - np.exp(-level * F(p["density"]) * step_len)
        color = np.where(upd[..., None], color + sample * (trans * alpha)[..., None], color)
        trans = np.where(upd, trans * (F(1.0) - alpha), trans)
        active = active & ~(upd & (trans < F(0.01)))
    out = np.zeros((H, W, 4), F)
    out[..., :3] = np.where(hit[..., None], color, F(0.0))
    out[..., 3] = np.where(hit, F(1.0) - trans, F(0.0))
    return out
