"""The colour-split layout of the red-black solves (sf_stencil.cu: k_rb_layout,
k_rb_half), restated in NumPy on the CPU: splitting a field into its red and
black arrays, updating one colour from the other through the split-layout
neighbour mapping, and merging back gives the same values as the colour
update on the interleaved field. This checks the index arithmetic of the
layout (row offsets s = (y + z) & 1, x neighbours k + s_u - 1 and k + s_u,
y and z neighbours at the same k) on every face kind the kernels handle by
wrap or ghost; the GPU tests hold the kernels themselves bit-equal to the
reference library."""

import numpy as np
import pytest


def split(f):
    """(nz, ny, nx) -> red, black arrays (nz, ny, nx/2): row (y, z) of red
    holds x = 2k + ((y + z) & 1)."""
    nz, ny, nx = f.shape
    z, y = np.meshgrid(np.arange(nz), np.arange(ny), indexing="ij")
    s = ((y + z) & 1)[..., None]
    k = np.arange(nx // 2)[None, None, :]
    red = np.take_along_axis(f, 2 * k + s, axis=2)
    black = np.take_along_axis(f, 2 * k + 1 - s, axis=2)
    return red, black


def merge(red, black):
    nz, ny, hx = red.shape
    f = np.empty((nz, ny, 2 * hx), red.dtype)
    z, y = np.meshgrid(np.arange(nz), np.arange(ny), indexing="ij")
    s = ((y + z) & 1)[..., None]
    k = np.arange(hx)[None, None, :]
    np.put_along_axis(f, 2 * k + s, red, axis=2)
    np.put_along_axis(f, 2 * k + 1 - s, black, axis=2)
    return f


def ghost(self_value, mode, const):
    """Face ghost of a cell from its own value: copy, constant, reflection."""
    if mode == "copy":
        return self_value
    if mode == "const":
        return np.full_like(self_value, const)
    return (np.float32(const) - self_value).astype(np.float32)


def neighbour(f, z, y, x, axis, step, periodic, mode, const):
    """Value of the neighbour of cells (z, y, x) one step along `axis` on the
    interleaved field, with the face rules of the stencils."""
    n = f.shape[axis]
    c = [z, y, x]
    c[axis] = c[axis] + step
    out = np.empty(z.shape, f.dtype)
    inside = (c[axis] >= 0) & (c[axis] < n)
    if periodic:
        c[axis] = c[axis] % n
        return f[c[0], c[1], c[2]]
    cc = list(c)
    cc[axis] = np.clip(c[axis], 0, n - 1)
    out = f[cc[0], cc[1], cc[2]]
    face = ~inside
    out = np.where(face, ghost(f[z, y, x], mode, const), out)
    return out


def update(nb, r, coef):
    """Pressure form of the update: (nb - h^2 div) / 6, rounded to FP32."""
    return ((nb.astype(np.float64) - np.float64(coef) * r) / 6.0).astype(np.float32)


def colour_interleaved(f, rhs, colour, coef, periodic, mode, const):
    nz, ny, nx = f.shape
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    sel = ((x + y + z + colour) & 1) == 0
    z, y, x = z[sel], y[sel], x[sel]
    acc = None
    for axis in (2, 1, 0):  # x-, x+, y-, y+, z-, z+
        for step in (-1, 1):
            v = neighbour(f, z, y, x, axis, step, periodic[axis], mode, const)
            acc = v if acc is None else (acc + v).astype(np.float32)
    out = f.copy()
    out[z, y, x] = update(acc, rhs[z, y, x], coef)
    return out


def colour_split(u, v, w, self_u, colour, coef, periodic, mode, const):
    """k_rb_half's mapping: u cells x = 2k + s_u, s_u = (y + z + colour) & 1;
    x neighbours v[k + s_u - 1], v[k + s_u] (wrapped or ghosted at the row
    ends), y / z neighbours v at the same k."""
    nz, ny, hx = u.shape
    z, y, k = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(hx), indexing="ij")
    s_u = (y + z + colour) & 1
    px, py, pz = periodic[2], periodic[1], periodic[0]

    def vx(kk):
        inside = (kk >= 0) & (kk < hx)
        if px:
            return v[z, y, kk % hx]
        return np.where(inside, v[z, y, np.clip(kk, 0, hx - 1)], ghost(self_u, mode, const))

    xm = vx(k + s_u - 1)
    xp = vx(k + s_u)
    # a cell's x- neighbour is a face ghost only at x = 0 (s_u = 0, k = 0),
    # its x+ neighbour only at x = nx - 1 (s_u = 1, k = hx - 1)
    def vyz(axis, step):
        c = [z, y, k]
        n = (nz, ny)[axis]
        c[axis] = c[axis] + step
        inside = (c[axis] >= 0) & (c[axis] < n)
        if (pz, py)[axis]:
            c[axis] = c[axis] % n
            return v[c[0], c[1], c[2]]
        c[axis] = np.clip(c[axis], 0, n - 1)
        return np.where(inside, v[c[0], c[1], c[2]], ghost(self_u, mode, const))

    acc = xm
    for val in (xp, vyz(1, -1), vyz(1, 1), vyz(0, -1), vyz(0, 1)):
        acc = (acc + val).astype(np.float32)
    return update(acc, w, coef)


CASES = [
    ((6, 5, 8), (False, False, False), "copy", 0.0),
    ((4, 6, 16), (True, False, True), "const", 0.25),
    ((5, 4, 8), (False, True, False), "reflect", 0.5),
    ((2, 6, 24), (True, True, True), "copy", 0.0),
]


@pytest.mark.parametrize("shape,periodic,mode,const", CASES)
def test_split_layout_matches_interleaved_colours(shape, periodic, mode, const):
    rng = np.random.default_rng(sum(shape))
    f = rng.standard_normal(shape).astype(np.float32)
    rhs = rng.standard_normal(shape).astype(np.float32)
    coef = np.float32(0.01)
    ref = f
    for colour in (0, 1):
        ref = colour_interleaved(ref, rhs, colour, coef, periodic, mode, const)
    red, black = split(f)
    rr, rb = split(rhs)
    assert np.array_equal(merge(red, black), f)
    red = colour_split(red, black, rr, red, 0, coef, periodic, mode, const)
    black = colour_split(black, red, rb, black, 1, coef, periodic, mode, const)
    got = merge(red, black)
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))
