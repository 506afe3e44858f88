// sf_device.cuh -- device-side ghost rules and trilinear sampling.
//
// The boundary semantics are those of the reference backend
// (backend-cuda.cu:62-189) because results must agree with it to 1e-5:
//   scalar   : per axis x, y, z in order -- periodic wraps, ZERO_FLUX clamps
//              and continues, FIXED_VALUE returns the face value.
//   pressure : periodic wraps, OUTFLOW returns the face pressure (Dirichlet),
//              walls clamp (Neumann).
//   velocity : periodic wraps and continues; any other face reads the cell on
//              the face with every other axis clamped and returns it directly
//              (OUTFLOW, or FREE_SLIP for a tangential component) or reflected
//              about the prescribed wall velocity (2 v_wall - v).
// Arithmetic that rounds is written in the same expression shapes as the
// reference so the compiler forms the same fused multiply-adds.
//
// Field storage: the advected fields (velocity, scalars) are FP32 (the
// reference's layout) or BF16 (half the bytes, FP32 arithmetic); the readers
// below are templates over the element type T (float or __nv_bfloat16) and
// the packed-velocity type P (float4, or Bf16x4 = four BF16 in 8 bytes).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "sf_types.h"
#include "stable-fluids-3d.h"

namespace sfb {

struct __align__(8) Bf16x4 {
    __nv_bfloat162 xy, zw;
};

__device__ __forceinline__ float to_f(float v) { return v; }
__device__ __forceinline__ float to_f(__nv_bfloat16 v) { return __bfloat162float(v); }
template <typename T>
__device__ __forceinline__ T from_f(float v);
template <>
__device__ __forceinline__ float from_f<float>(float v) { return v; }
template <>
__device__ __forceinline__ __nv_bfloat16 from_f<__nv_bfloat16>(float v) { return __float2bfloat16_rn(v); }

// read-only cached loads
__device__ __forceinline__ float ldg_f(const float* p) { return __ldg(p); }
__device__ __forceinline__ float ldg_f(const __nv_bfloat16* p) { return __bfloat162float(__ldg(p)); }
__device__ __forceinline__ float4 ldg4(const float4* p) { return __ldg(p); }
__device__ __forceinline__ float4 ldg4(const Bf16x4* p) {
    const uint2 u = __ldg(reinterpret_cast<const uint2*>(p));
    const float2 a = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&u.x));
    const float2 b = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&u.y));
    return make_float4(a.x, a.y, b.x, b.y);
}
template <typename P>
__device__ __forceinline__ P pack4(float x, float y, float z);
template <>
__device__ __forceinline__ float4 pack4<float4>(float x, float y, float z) { return make_float4(x, y, z, 0.0f); }
template <>
__device__ __forceinline__ Bf16x4 pack4<Bf16x4>(float x, float y, float z) { return Bf16x4{__floats2bfloat162_rn(x, y), __floats2bfloat162_rn(z, 0.0f)}; }

__device__ __forceinline__ size_t lin(int x, int y, int z, const Dims& d) {
    return static_cast<size_t>(x) + static_cast<size_t>(d.nx) * (static_cast<size_t>(y) + static_cast<size_t>(d.ny) * static_cast<size_t>(z));
}

__device__ __forceinline__ int wrap_index(int c, int n) {
    c %= n;
    return c < 0 ? c + n : c;
}

__device__ __forceinline__ int clamp_index(int c, int n) { return c < 0 ? 0 : (c >= n ? n - 1 : c); }

__device__ __forceinline__ bool inside(int x, int y, int z, const Dims& d) {
    return static_cast<unsigned>(x) < static_cast<unsigned>(d.nx) && static_cast<unsigned>(y) < static_cast<unsigned>(d.ny) && static_cast<unsigned>(z) < static_cast<unsigned>(d.nz);
}

// ---------------------------------------------------------------- scalars --
__device__ __forceinline__ bool scalar_resolve_axis(int& c, int n, int face_lo, const ScalarBC& b, int axis, float& value) {
    if (static_cast<unsigned>(c) < static_cast<unsigned>(n)) return true;
    const int face = face_lo + (c < 0 ? 0 : 1);
    if (b.periodic[axis]) {
        c = wrap_index(c, n);
        return true;
    }
    if (b.type[face] == STABLE_FLUIDS_SCALAR_BOUNDARY_ZERO_FLUX) {
        c = c < 0 ? 0 : n - 1;
        return true;
    }
    value = b.value[face];
    return false;
}

// Resolves (x, y, z) to an interior index, or returns false with the fixed
// face value in `value`.
__device__ __forceinline__ bool scalar_resolve(int& x, int& y, int& z, const Dims& d, const ScalarBC& b, float& value) {
    if (!scalar_resolve_axis(x, d.nx, XM, b, 0, value)) return false;
    if (!scalar_resolve_axis(y, d.ny, YM, b, 1, value)) return false;
    if (!scalar_resolve_axis(z, d.nz, ZM, b, 2, value)) return false;
    return true;
}

template <typename T>
__device__ __forceinline__ float load_scalar(const T* __restrict__ f, int x, int y, int z, const Dims& d, const ScalarBC& b) {
    if (inside(x, y, z, d)) return to_f(f[lin(x, y, z, d)]);
    float value;
    if (!scalar_resolve(x, y, z, d, b, value)) return value;
    return to_f(f[lin(x, y, z, d)]);
}

// --------------------------------------------------------------- pressure --
__device__ __forceinline__ bool pressure_resolve_axis(int& c, int n, int face_lo, const FlowBC& b, int axis, float& value) {
    if (static_cast<unsigned>(c) < static_cast<unsigned>(n)) return true;
    const int face = face_lo + (c < 0 ? 0 : 1);
    if (b.periodic[axis]) {
        c = wrap_index(c, n);
        return true;
    }
    if (b.type[face] == STABLE_FLUIDS_FLOW_BOUNDARY_OUTFLOW) {
        value = b.pressure[face];
        return false;
    }
    c = c < 0 ? 0 : n - 1;
    return true;
}

__device__ __forceinline__ float load_pressure(const float* __restrict__ f, int x, int y, int z, const Dims& d, const FlowBC& b) {
    if (inside(x, y, z, d)) return f[lin(x, y, z, d)];
    float value;
    if (!pressure_resolve_axis(x, d.nx, XM, b, 0, value)) return value;
    if (!pressure_resolve_axis(y, d.ny, YM, b, 1, value)) return value;
    if (!pressure_resolve_axis(z, d.nz, ZM, b, 2, value)) return value;
    return f[lin(x, y, z, d)];
}

// --------------------------------------------------------------- velocity --
// Ghost value of one component from the face cell `interior`.
__device__ __forceinline__ float velocity_ghost(float interior, int comp, int axis, int face, const FlowBC& b) {
    const int t = b.type[face];
    if (t == STABLE_FLUIDS_FLOW_BOUNDARY_OUTFLOW) return interior;
    if (t == STABLE_FLUIDS_FLOW_BOUNDARY_FREE_SLIP_WALL && comp != axis) return interior;
    return 2.0f * b.vel[face][comp] - interior;
}

// Component `comp` of a SoA velocity field at any integer position.
template <typename T>
__device__ __forceinline__ float load_velocity(const T* __restrict__ f, int comp, int x, int y, int z, const Dims& d, const FlowBC& b) {
    if (inside(x, y, z, d)) return to_f(f[lin(x, y, z, d)]);
    int c[3] = {x, y, z};
    const int n[3] = {d.nx, d.ny, d.nz};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if (static_cast<unsigned>(c[a]) < static_cast<unsigned>(n[a])) continue;
        if (b.periodic[a]) {
            c[a] = wrap_index(c[a], n[a]);
            continue;
        }
        const int face = 2 * a + (c[a] < 0 ? 0 : 1);
        int q[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) q[k] = clamp_index(c[k], n[k]);
        const float interior = to_f(f[lin(q[0], q[1], q[2], d)]);
        return velocity_ghost(interior, comp, a, face, b);
    }
    return to_f(f[lin(c[0], c[1], c[2], d)]);
}

// All three components from a packed (x, y, z, unused) field.
template <typename P>
__device__ __forceinline__ float3 load_velocity3(const P* __restrict__ f, int x, int y, int z, const Dims& d, const FlowBC& b) {
    if (inside(x, y, z, d)) {
        const float4 v = ldg4(&f[lin(x, y, z, d)]);
        return make_float3(v.x, v.y, v.z);
    }
    int c[3] = {x, y, z};
    const int n[3] = {d.nx, d.ny, d.nz};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if (static_cast<unsigned>(c[a]) < static_cast<unsigned>(n[a])) continue;
        if (b.periodic[a]) {
            c[a] = wrap_index(c[a], n[a]);
            continue;
        }
        const int face = 2 * a + (c[a] < 0 ? 0 : 1);
        int q[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) q[k] = clamp_index(c[k], n[k]);
        const float4 v = ldg4(&f[lin(q[0], q[1], q[2], d)]);
        return make_float3(velocity_ghost(v.x, 0, a, face, b), velocity_ghost(v.y, 1, a, face, b), velocity_ghost(v.z, 2, a, face, b));
    }
    const float4 v = ldg4(&f[lin(c[0], c[1], c[2], d)]);
    return make_float3(v.x, v.y, v.z);
}

// ----------------------------------------------------------- trilinear ----
// Periodic world wrap, backend-cuda.cu:195-206.
__device__ __forceinline__ float wrap_world(float p, float extent) {
    p = extent <= 0.0f ? 0.0f : fmodf(p, extent);
    if (p < 0.0f) p += extent;
    return p;
}

struct Cell {
    int x0, y0, z0;
    float tx, ty, tz;
};

// p / h, correctly rounded. When h is a power of two, 1 / h is exact and
// p * (1 / h) is the same correctly rounded value without a division.
__device__ __forceinline__ float div_h(float p, float h) {
    const unsigned u = __float_as_uint(h);
    const bool pow2 = (u & 0x007fffffu) == 0u && (u & 0x7f800000u) != 0u;  // normal, zero mantissa
    return pow2 ? __fmul_rn(p, __frcp_rn(h)) : p / h;
}

// Grid coordinates of a world position: g = p / h - 0.5, floor, fraction.
__device__ __forceinline__ Cell locate(float x, float y, float z, float h) {
    const float gx = div_h(x, h) - 0.5f;
    const float gy = div_h(y, h) - 0.5f;
    const float gz = div_h(z, h) - 0.5f;
    Cell c;
    c.x0 = static_cast<int>(floorf(gx));
    c.y0 = static_cast<int>(floorf(gy));
    c.z0 = static_cast<int>(floorf(gz));
    c.tx = gx - static_cast<float>(c.x0);
    c.ty = gy - static_cast<float>(c.y0);
    c.tz = gz - static_cast<float>(c.z0);
    return c;
}

// The 2x2x2 block of corners at (x0, y0, z0) lies inside the grid. Written
// as x0 < n - 1, not x0 + 1 < n: the position of a diverged (infinite)
// velocity saturates x0 to INT_MAX, and x0 + 1 would wrap to a negative.
__device__ __forceinline__ bool block_inside(const Cell& c, const Dims& d) {
    return c.x0 >= 0 && c.y0 >= 0 && c.z0 >= 0 && c.x0 < d.nx - 1 && c.y0 < d.ny - 1 && c.z0 < d.nz - 1;
}

// A corner block's base index for the boundary path, limited to [-2, n]:
// corners beyond a non-periodic face resolve to the same face value however
// far out they lie (positions on a periodic axis are wrapped first), and the
// limit keeps base + 1 from overflowing.
__device__ __forceinline__ int corner_base(int c, int n) { return c < -2 ? -2 : (c > n ? n : c); }

// Interpolation in x, then y, then z, each as a + (b - a) * t with the
// product and the sum rounded once (one FMA): the contraction the compiler
// applies to the reference's expression (backend-cuda.cu:231-237), written
// out so that it does not depend on the code the function is inlined into.
__device__ __forceinline__ float trilerp(float c000, float c100, float c010, float c110, float c001, float c101, float c011, float c111, const Cell& c) {
    const float c00 = __fmaf_rn(c100 - c000, c.tx, c000);
    const float c10 = __fmaf_rn(c110 - c010, c.tx, c010);
    const float c01 = __fmaf_rn(c101 - c001, c.tx, c001);
    const float c11 = __fmaf_rn(c111 - c011, c.tx, c011);
    const float c0 = __fmaf_rn(c10 - c00, c.ty, c00);
    const float c1 = __fmaf_rn(c11 - c01, c.ty, c01);
    return __fmaf_rn(c1 - c0, c.tz, c0);
}

// Velocity (3 components) at a world position from the packed field.
template <typename P>
__device__ __forceinline__ float3 sample_velocity3(const P* __restrict__ v, float x, float y, float z, const Dims& d, float h, const FlowBC& b) {
    if (b.periodic[0]) x = wrap_world(x, static_cast<float>(d.nx) * h);
    if (b.periodic[1]) y = wrap_world(y, static_cast<float>(d.ny) * h);
    if (b.periodic[2]) z = wrap_world(z, static_cast<float>(d.nz) * h);
    const Cell c = locate(x, y, z, h);
    float3 s[8];
    if (block_inside(c, d)) {
        const size_t i = lin(c.x0, c.y0, c.z0, d);
        const size_t sy = static_cast<size_t>(d.nx), sz = static_cast<size_t>(d.nx) * static_cast<size_t>(d.ny);
        const size_t off[8] = {0, 1, sy, sy + 1, sz, sz + 1, sz + sy, sz + sy + 1};
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const float4 q = ldg4(&v[i + off[k]]);
            s[k] = make_float3(q.x, q.y, q.z);
        }
    } else {
        const int bx = corner_base(c.x0, d.nx), by = corner_base(c.y0, d.ny), bz = corner_base(c.z0, d.nz);
#pragma unroll
        for (int k = 0; k < 8; ++k) s[k] = load_velocity3(v, bx + (k & 1), by + ((k >> 1) & 1), bz + (k >> 2), d, b);
    }
    return make_float3(trilerp(s[0].x, s[1].x, s[2].x, s[3].x, s[4].x, s[5].x, s[6].x, s[7].x, c),
                       trilerp(s[0].y, s[1].y, s[2].y, s[3].y, s[4].y, s[5].y, s[6].y, s[7].y, c),
                       trilerp(s[0].z, s[1].z, s[2].z, s[3].z, s[4].z, s[5].z, s[6].z, s[7].z, c));
}

// Midpoint RK2 back-trace in world units (backend-cuda.cu:295-300), from the
// centre (x, y, z) of cell (cx, cy, cz).
template <typename P>
__device__ __forceinline__ float3 trace_rk2(float x, float y, float z, int cx, int cy, int cz, const P* __restrict__ v, float dt, const Dims& d, float h, const FlowBC& b) {
    // The first sample is at the cell's own centre. Where its grid position
    // comes out exactly on the cell (all three fractions zero, as for a
    // power-of-two h) every interpolation weight of the other corners is
    // zero and the trilinear value is the cell's own velocity: read it
    // directly. (It can differ from the interpolated value only in the sign
    // of a zero, which x - (0.5 dt) v does not see.)
    float3 v0;
    const Cell c = locate(x, y, z, h);
    if (c.tx == 0.0f && c.ty == 0.0f && c.tz == 0.0f && c.x0 == cx && c.y0 == cy && c.z0 == cz) {
        const float4 q = ldg4(&v[lin(cx, cy, cz, d)]);
        v0 = make_float3(q.x, q.y, q.z);
    } else {
        v0 = sample_velocity3(v, x, y, z, d, h, b);
    }
    // x - (0.5 dt) v and x - dt v, each product and difference rounded once
    const float half_dt = __fmul_rn(0.5f, dt);
    const float mx = __fmaf_rn(-half_dt, v0.x, x);
    const float my = __fmaf_rn(-half_dt, v0.y, y);
    const float mz = __fmaf_rn(-half_dt, v0.z, z);
    const float3 v1 = sample_velocity3(v, mx, my, mz, d, h, b);
    return make_float3(__fmaf_rn(-dt, v1.x, x), __fmaf_rn(-dt, v1.y, y), __fmaf_rn(-dt, v1.z, z));
}

}  // namespace sfb
