// sf_stencil.cu -- the iterative 7-point solves of the step: implicit
// diffusion (I - alpha L) x = b for velocity components and scalars, and the
// pressure Poisson equation sum6(p) - 6 p = h^2 div.
//
// Update formulas (backend-cuda.cu:354-375, 398-407), neighbour sum order
// x-, x+, y-, y+, z-, z+:
//   diffusion: x = (b + alpha * nb) / (1 + 6 alpha)
//   pressure : p = (nb - h^2 * div) / 6
// RBGS updates (x+y+z) even cells, then odd ones, in place; JACOBI updates
// every cell from the previous iterate.

#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <climits>

#include "sf_batch.cuh"
#include "sf_device.cuh"
#include "sf_launch.h"
#include "sf_stencil_tb.cuh"
#include "sf_stencil_wave.cuh"

namespace sfb {

namespace {

template <int KIND, typename T>
__device__ __forceinline__ float neighbour(const T* __restrict__ f, int x, int y, int z, const Dims& d, const FlowBC& fb, const ScalarBC& sb) {
    if constexpr (KIND == KIND_PRESSURE) return load_pressure(reinterpret_cast<const float*>(f), x, y, z, d, fb);
    else if constexpr (KIND == KIND_SCALAR) return load_scalar(f, x, y, z, d, sb);
    else return load_velocity(f, KIND, x, y, z, d, fb);
}

template <int KIND, typename T>
__device__ __forceinline__ float neighbour_sum(const T* __restrict__ f, int x, int y, int z, const Dims& d, const FlowBC& fb, const ScalarBC& sb) {
    return neighbour<KIND>(f, x - 1, y, z, d, fb, sb) + neighbour<KIND>(f, x + 1, y, z, d, fb, sb) + neighbour<KIND>(f, x, y - 1, z, d, fb, sb) + neighbour<KIND>(f, x, y + 1, z, d, fb, sb) + neighbour<KIND>(f, x, y, z - 1, d, fb, sb)
         + neighbour<KIND>(f, x, y, z + 1, d, fb, sb);
}

// One colour of an RBGS iteration. Thread (hx, y) owns, in each of ZC
// consecutive planes, the cell x = 2 hx + ((y + z + parity) & 1) of the
// colour, so every thread is active. Cells of one colour never read each
// other, so the thread loads the neighbours of all its cells first, then
// updates, then stores (independent memory requests in flight). Interior
// cells read their six neighbours directly; cells on the boundary use the
// reference's ghost rules.
constexpr int kColourPlanes = 4;

template <int KIND, typename T = float>
__global__ void __launch_bounds__(256) k_rbgs_colour(T* x, const T* __restrict__ rhs, float coef, int parity, Dims d, FlowBC fb, ScalarBC sb) {
    const int hx = static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x);
    const int y = static_cast<int>(blockIdx.y * blockDim.y + threadIdx.y);
    const int z0 = static_cast<int>(blockIdx.z) * kColourPlanes;
    if (y >= d.ny) return;
    const size_t sy = static_cast<size_t>(d.nx), sz = static_cast<size_t>(d.nx) * static_cast<size_t>(d.ny);
    const float divisor = KIND == KIND_PRESSURE ? 6.0f : 1.0f + 6.0f * coef;
    const double recip = tb::recip64(divisor);
    float num[kColourPlanes];
    size_t idx[kColourPlanes];
    bool ok[kColourPlanes];
#pragma unroll
    for (int k = 0; k < kColourPlanes; ++k) {
        const int z = z0 + k;
        const int cx = 2 * hx + ((y + z + parity) & 1);
        ok[k] = z < d.nz && cx < d.nx;
        idx[k] = ok[k] ? lin(cx, y, z, d) : 0;
        float nb = 0.0f;
        if (ok[k]) {
            const bool interior = cx >= 1 && cx <= d.nx - 2 && y >= 1 && y <= d.ny - 2 && z >= 1 && z <= d.nz - 2;
            if (interior) {
                const T* c = x + idx[k];
                nb = to_f(c[-1]) + to_f(c[1]) + to_f(c[-static_cast<ptrdiff_t>(sy)]) + to_f(c[sy]) + to_f(c[-static_cast<ptrdiff_t>(sz)]) + to_f(c[sz]);
            } else {
                nb = neighbour_sum<KIND>(x, cx, y, z, d, fb, sb);
            }
        }
        num[k] = tb::numerator<KIND>(nb, ok[k] ? to_f(rhs[idx[k]]) : 0.0f, coef);
    }
#pragma unroll
    for (int k = 0; k < kColourPlanes; ++k) {
        if (!ok[k]) continue;
        x[idx[k]] = from_f<T>(tb::divide(num[k], divisor, recip));
    }
}

// One Jacobi sweep, dst = update(src): thread (x, y) owns the cells of
// kColourPlanes consecutive planes; interior cells read their neighbours
// directly, boundary cells use the ghost rules.
template <int KIND, typename T = float>
__global__ void __launch_bounds__(256) k_jacobi(T* __restrict__ dst, const T* __restrict__ src, const T* __restrict__ rhs, float coef, Dims d, FlowBC fb, ScalarBC sb) {
    const int cx = static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x);
    const int y = static_cast<int>(blockIdx.y * blockDim.y + threadIdx.y);
    const int z0 = static_cast<int>(blockIdx.z) * kColourPlanes;
    if (cx >= d.nx || y >= d.ny) return;
    const size_t sy = static_cast<size_t>(d.nx), sz = static_cast<size_t>(d.nx) * static_cast<size_t>(d.ny);
    const float inv = wave::jacobi_inverse(KIND, coef);
    const bool xy_interior = cx >= 1 && cx <= d.nx - 2 && y >= 1 && y <= d.ny - 2;
#pragma unroll
    for (int k = 0; k < kColourPlanes; ++k) {
        const int z = z0 + k;
        if (z >= d.nz) break;
        const size_t i = lin(cx, y, z, d);
        float nb;
        if (xy_interior && z >= 1 && z <= d.nz - 2) {
            const T* c = src + i;
            nb = to_f(c[-1]) + to_f(c[1]) + to_f(c[-static_cast<ptrdiff_t>(sy)]) + to_f(c[sy]) + to_f(c[-static_cast<ptrdiff_t>(sz)]) + to_f(c[sz]);
        } else {
            nb = neighbour_sum<KIND>(src, cx, y, z, d, fb, sb);
        }
        dst[i] = from_f<T>(wave::jacobi_update<KIND>(nb, to_f(rhs[i]), coef, inv));
    }
}

// ------------------------------------------------- vectorised z-marching --
// Both schemes again, for grids with nx % 4 == 0 and 16-byte aligned fields:
// a thread owns 4 consecutive cells of a row (one float4) and marches through
// kVecPlanes-deep z chunks, carrying the planes below / at / above in
// registers, so every field value is loaded once per sweep from L2/HBM (plus
// the x and y neighbours, which hit L1). Face ghosts come from the kind's
// GhostRule (periodic wrap, copy of the face cell, constant, reflection) --
// the same values as the load_* ghost rules for a face neighbour -- applied
// with selects, so boundary threads take the same path as interior ones.
// Arithmetic, neighbour order and division are those of k_rbgs_colour /
// k_jacobi, so results are bit-identical.
template <int KIND>
__device__ __forceinline__ float vec_update(float nb, float rhs, float coef, float divisor, double recip) {
    return tb::divide(tb::numerator<KIND>(nb, rhs, coef), divisor, recip);
}

constexpr int kVecRows = 4;  // rows per CTA; 32 x kVecRows threads

// ---- FP32 fields: float4 rows (4 cells per thread) ----------------------
struct VecGhost4 {
    int ox_lo, ox_hi;  // x offsets of the row's x- / x+ neighbours from x0 (wrap or self on a face)
    int oy_lo, oy_hi;  // y offsets of the y- / y+ rows
    bool gx_lo, gx_hi, gy_lo, gy_hi;  // apply the face ghost
};

__device__ __forceinline__ VecGhost4 vec_ghost4(int x0, int y, const Dims& d, const GhostRule& g) {
    const int sy = d.nx;
    VecGhost4 v{-1, 4, -sy, sy, false, false, false, false};
    if (x0 == 0) {
        v.ox_lo = g.periodic[0] ? d.nx - 1 : 0;
        v.gx_lo = !g.periodic[0];
    }
    if (x0 + 4 == d.nx) {
        v.ox_hi = g.periodic[0] ? -x0 : 3;
        v.gx_hi = !g.periodic[0];
    }
    if (y == 0) {
        v.oy_lo = g.periodic[1] ? (d.ny - 1) * sy : 0;
        v.gy_lo = !g.periodic[1];
    }
    if (y == d.ny - 1) {
        v.oy_hi = g.periodic[1] ? -(d.ny - 1) * sy : 0;
        v.gy_hi = !g.periodic[1];
    }
    return v;
}

__device__ __forceinline__ float4 ld4(const float* p) { return *reinterpret_cast<const float4*>(p); }

__device__ __forceinline__ float4 ghost4(const GhostRule& g, int face, float4 self) {
    return make_float4(tb::ghost(g, face, self.x), tb::ghost(g, face, self.y), tb::ghost(g, face, self.z), tb::ghost(g, face, self.w));
}


// The plane below the chunk's first plane (or its ghost at z = 0).
__device__ __forceinline__ float4 vec_below4(const float* x, int i, int z, const Dims& d, const GhostRule& g, float4 cur) {
    const int sz = d.nx * d.ny;
    if (z > 0) return ld4(x + i - sz);
    if (g.periodic[2]) return ld4(x + i + (d.nz - 1) * sz);
    return ghost4(g, ZM, cur);
}

__device__ __forceinline__ float4 vec_above4(const float* x, int i, int z, const Dims& d, const GhostRule& g, float4 cur) {
    const int sz = d.nx * d.ny;
    if (z + 1 < d.nz) return ld4(x + i + sz);
    if (g.periodic[2]) return ld4(x + i - (d.nz - 1) * sz);
    return ghost4(g, ZP, cur);
}


// One Jacobi sweep dst = update(src), block `blk` of the launch (blockIdx
// for one simulation, the work item's block in a batch). DOWN marches the
// chunk from its top plane down: a sweep that runs opposite to the one
// before starts on the planes that sweep wrote last, which are still in L2
// (the values are the same either way: a Jacobi sweep reads only src).
template <int KIND, bool DOWN = false>
__device__ __forceinline__ void jacobi_vec4_block(uint3 blk, float* __restrict__ dst, const float* __restrict__ src, const float* __restrict__ rhs, float coef, int z_chunk, const Dims& d, const GhostRule& g) {
    const int x0 = 4 * static_cast<int>(blk.x * 32 + threadIdx.x), y = static_cast<int>(blk.y * kVecRows + threadIdx.y);
    if (x0 >= d.nx || y >= d.ny) return;
    const int zb = static_cast<int>(blk.z) * z_chunk, ze = min(zb + z_chunk, d.nz);
    const float inv = wave::jacobi_inverse(KIND, coef);
    const VecGhost4 v = vec_ghost4(x0, y, d, g);
    const int sz = d.nx * d.ny;
    // the update of plane z at index i from its planes below / at / above
    const auto plane = [&](int i, float4 below, float4 cur, float4 above) {
        float a = src[i + v.ox_lo], b = src[i + v.ox_hi];
        float4 c = ld4(src + i + v.oy_lo), e = ld4(src + i + v.oy_hi);
        const float4 r = ld4(rhs + i);
        if (v.gx_lo) a = tb::ghost(g, XM, a);
        if (v.gx_hi) b = tb::ghost(g, XP, b);
        if (v.gy_lo) c = ghost4(g, YM, c);
        if (v.gy_hi) e = ghost4(g, YP, e);
        float4 o;
        o.x = wave::jacobi_update<KIND>(a + cur.y + c.x + e.x + below.x + above.x, r.x, coef, inv);
        o.y = wave::jacobi_update<KIND>(cur.x + cur.z + c.y + e.y + below.y + above.y, r.y, coef, inv);
        o.z = wave::jacobi_update<KIND>(cur.y + cur.w + c.z + e.z + below.z + above.z, r.z, coef, inv);
        o.w = wave::jacobi_update<KIND>(cur.z + b + c.w + e.w + below.w + above.w, r.w, coef, inv);
        *reinterpret_cast<float4*>(dst + i) = o;
    };
    if constexpr (!DOWN) {
        int i = x0 + d.nx * (y + d.ny * zb);
        float4 cur = ld4(src + i);
        float4 below = vec_below4(src, i, zb, d, g, cur);
#pragma unroll 2
        for (int z = zb; z < ze; ++z, i += sz) {
            const float4 above = vec_above4(src, i, z, d, g, cur);
            plane(i, below, cur, above);
            below = cur;
            cur = above;
        }
    } else {
        int i = x0 + d.nx * (y + d.ny * (ze - 1));
        float4 cur = ld4(src + i);
        float4 above = vec_above4(src, i, ze - 1, d, g, cur);
#pragma unroll 2
        for (int z = ze - 1; z >= zb; --z, i -= sz) {
            const float4 below = vec_below4(src, i, z, d, g, cur);
            plane(i, below, cur, above);
            above = cur;
            cur = below;
        }
    }
}

// One colour of an RBGS iteration, in place: in each float4 the two cells
// with (x + y + z + parity) even are updated; the other two are stored back
// unchanged (no thread of this launch changes them, so rewriting the value
// just read is harmless and keeps every store a full 16 bytes).
template <int KIND>
__device__ __forceinline__ void rbgs_vec4_block(uint3 blk, float* x, const float* __restrict__ rhs, float coef, int parity, int z_chunk, const Dims& d, const GhostRule& g) {
    const int x0 = 4 * static_cast<int>(blk.x * 32 + threadIdx.x), y = static_cast<int>(blk.y * kVecRows + threadIdx.y);
    if (x0 >= d.nx || y >= d.ny) return;
    const int zb = static_cast<int>(blk.z) * z_chunk, ze = min(zb + z_chunk, d.nz);
    const float divisor = KIND == KIND_PRESSURE ? 6.0f : 1.0f + 6.0f * coef;
    const double recip = tb::recip64(divisor);
    const VecGhost4 v = vec_ghost4(x0, y, d, g);
    const int sz = d.nx * d.ny;
    int i = x0 + d.nx * (y + d.ny * zb);
    float4 cur = ld4(x + i);
    float4 below = vec_below4(x, i, zb, d, g, cur);
#pragma unroll 2
    for (int z = zb; z < ze; ++z, i += sz) {
        const float4 above = vec_above4(x, i, z, d, g, cur);
        float a = x[i + v.ox_lo], b = x[i + v.ox_hi];
        float4 c = ld4(x + i + v.oy_lo), e = ld4(x + i + v.oy_hi);
        const float4 r = ld4(rhs + i);
        if (v.gx_lo) a = tb::ghost(g, XM, a);
        if (v.gx_hi) b = tb::ghost(g, XP, b);
        if (v.gy_lo) c = ghost4(g, YM, c);
        if (v.gy_hi) e = ghost4(g, YP, e);
        const bool even = ((y + z + parity) & 1) == 0;  // cells 0 and 2 of the float4 (else 1 and 3)
        const float n_lo = even ? a + cur.y + c.x + e.x + below.x + above.x : cur.x + cur.z + c.y + e.y + below.y + above.y;
        const float n_hi = even ? cur.y + cur.w + c.z + e.z + below.z + above.z : cur.z + b + c.w + e.w + below.w + above.w;
        const float q_lo = vec_update<KIND>(n_lo, even ? r.x : r.y, coef, divisor, recip);
        const float q_hi = vec_update<KIND>(n_hi, even ? r.z : r.w, coef, divisor, recip);
        const float4 o = even ? make_float4(q_lo, cur.y, q_hi, cur.w) : make_float4(cur.x, q_lo, cur.z, q_hi);
        *reinterpret_cast<float4*>(x + i) = o;
        below = cur;
        cur = above;
    }
}

// Consecutive sweeps are launched as programmatic dependents of the one
// before (launch_sweep): a dependent's CTAs become resident as the previous
// grid's CTAs retire and wait here, before their first global read, until
// that grid has completed and its writes are visible. Without the launch
// attribute the wait returns at once.
__device__ __forceinline__ void wait_for_previous_grid() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

template <int KIND, bool DOWN = false>
__global__ void __launch_bounds__(32 * kVecRows) k_jacobi_vec4(float* __restrict__ dst, const float* __restrict__ src, const float* __restrict__ rhs, float coef, int z_chunk, Dims d, GhostRule g) {
    wait_for_previous_grid();
    jacobi_vec4_block<KIND, DOWN>(blockIdx, dst, src, rhs, coef, z_chunk, d, g);
}

template <int KIND>
__global__ void __launch_bounds__(32 * kVecRows) k_rbgs_vec4(float* x, const float* __restrict__ rhs, float coef, int parity, int z_chunk, Dims d, GhostRule g) {
    wait_for_previous_grid();
    rbgs_vec4_block<KIND>(blockIdx, x, rhs, coef, parity, z_chunk, d, g);
}

// Launches a sweep kernel (one that starts with wait_for_previous_grid) as a
// programmatic dependent of the preceding kernel on the stream.
template <typename... P, typename... A>
cudaError_t launch_sweep(void (*kernel)(P...), dim3 grid, dim3 block, cudaStream_t s, A... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr{};
    attr.id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr.val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = &attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, static_cast<P>(args)...);
}


// ---- BF16 fields: 4 cells per thread (one 8-byte vector) ------------------
// The diffusion fields of a BF16-storage context. Same march, ghosts, sum
// order and division as the float4 kernels, in FP32 arithmetic on the
// unpacked values, rounded once to BF16 on the store. Half the bytes per cell
// means half the loads in flight per warp, so each thread issues the loads
// of the next plane (the row above it, the y- / y+ rows, the right-hand side
// and the two x-end cells) before it computes the current one. For RBGS that
// is safe in place: a colour launch reads only cells of the other colour
// (unchanged by the launch) or its own row before storing it.
__device__ __forceinline__ uint2 ld_bf4(const __nv_bfloat16* p) { return *reinterpret_cast<const uint2*>(p); }
__device__ __forceinline__ float4 unpack_bf4(uint2 u) {
    return make_float4(__uint_as_float(u.x << 16), __uint_as_float(u.x & 0xffff0000u), __uint_as_float(u.y << 16), __uint_as_float(u.y & 0xffff0000u));
}
__device__ __forceinline__ unsigned pack_bf2(float lo, float hi) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const unsigned*>(&h);
}
__device__ __forceinline__ float ld_bf1(const __nv_bfloat16* p) { return __uint_as_float(static_cast<unsigned>(*reinterpret_cast<const unsigned short*>(p)) << 16); }

// Raw loads of one plane for one thread.
struct Bf16Plane {
    uint2 up;        // the row above (plane z + 1, or the periodic wrap)
    uint2 ym, yp;    // the y- / y+ rows
    uint2 rhs;       // the right-hand side row
    float xm, xp;    // x- neighbour of cell 0, x+ neighbour of cell 3
};

__device__ __forceinline__ void fetch_bf16(Bf16Plane& q, const __nv_bfloat16* src, const __nv_bfloat16* rhs, int i, int z, const Dims& d, const GhostRule& g, const VecGhost4& v) {
    const int sz = d.nx * d.ny;
    if (z + 1 < d.nz) q.up = ld_bf4(src + i + sz);
    else if (g.periodic[2]) q.up = ld_bf4(src + i - (d.nz - 1) * sz);
    q.ym = ld_bf4(src + i + v.oy_lo);
    q.yp = ld_bf4(src + i + v.oy_hi);
    q.rhs = ld_bf4(rhs + i);
    q.xm = ld_bf1(src + i + v.ox_lo);
    q.xp = ld_bf1(src + i + v.ox_hi);
}

// RB: one colour of an RBGS iteration in place (dst == src); else one Jacobi
// sweep. DEPTH: planes of loads in flight ahead of the one computed.
template <int KIND, bool RB, int DEPTH>
__device__ __forceinline__ void march_bf16(__nv_bfloat16* dst, const __nv_bfloat16* src, const __nv_bfloat16* rhs, float coef, int parity, int z_chunk, const Dims& d, const GhostRule& g) {
    const int x0 = 4 * static_cast<int>(blockIdx.x * 32 + threadIdx.x), y = static_cast<int>(blockIdx.y * kVecRows + threadIdx.y);
    if (x0 >= d.nx || y >= d.ny) return;
    const int zb = static_cast<int>(blockIdx.z) * z_chunk, ze = min(zb + z_chunk, d.nz);
    const float divisor = KIND == KIND_PRESSURE ? 6.0f : 1.0f + 6.0f * coef;
    const double recip = tb::recip64(divisor);
    const float inv = wave::jacobi_inverse(KIND, coef);
    const VecGhost4 v = vec_ghost4(x0, y, d, g);
    const int sz = d.nx * d.ny;
    int i = x0 + d.nx * (y + d.ny * zb);
    float4 cur = unpack_bf4(ld_bf4(src + i));
    float4 below;
    if (zb > 0) below = unpack_bf4(ld_bf4(src + i - sz));
    else if (g.periodic[2]) below = unpack_bf4(ld_bf4(src + i + (d.nz - 1) * sz));
    else below = ghost4(g, ZM, cur);
    // one plane: q holds its raw loads; advances below / cur
    const auto plane = [&](const Bf16Plane& q, int z, int at) {
        const float4 above = (z + 1 < d.nz || g.periodic[2]) ? unpack_bf4(q.up) : ghost4(g, ZP, cur);
        float a = q.xm, b = q.xp;
        float4 c = unpack_bf4(q.ym), e = unpack_bf4(q.yp);
        const float4 r = unpack_bf4(q.rhs);
        if (v.gx_lo) a = tb::ghost(g, XM, a);
        if (v.gx_hi) b = tb::ghost(g, XP, b);
        if (v.gy_lo) c = ghost4(g, YM, c);
        if (v.gy_hi) e = ghost4(g, YP, e);
        uint2 o;
        if constexpr (RB) {
            if (((y + z + parity) & 1) == 0) {  // cells 0 and 2 (warp-uniform branch)
                o.x = pack_bf2(vec_update<KIND>(a + cur.y + c.x + e.x + below.x + above.x, r.x, coef, divisor, recip), cur.y);
                o.y = pack_bf2(vec_update<KIND>(cur.y + cur.w + c.z + e.z + below.z + above.z, r.z, coef, divisor, recip), cur.w);
            } else {  // cells 1 and 3
                o.x = pack_bf2(cur.x, vec_update<KIND>(cur.x + cur.z + c.y + e.y + below.y + above.y, r.y, coef, divisor, recip));
                o.y = pack_bf2(cur.z, vec_update<KIND>(cur.z + b + c.w + e.w + below.w + above.w, r.w, coef, divisor, recip));
            }
        } else {
            o.x = pack_bf2(wave::jacobi_update<KIND>(a + cur.y + c.x + e.x + below.x + above.x, r.x, coef, inv), wave::jacobi_update<KIND>(cur.x + cur.z + c.y + e.y + below.y + above.y, r.y, coef, inv));
            o.y = pack_bf2(wave::jacobi_update<KIND>(cur.y + cur.w + c.z + e.z + below.z + above.z, r.z, coef, inv), wave::jacobi_update<KIND>(cur.z + b + c.w + e.w + below.w + above.w, r.w, coef, inv));
        }
        *reinterpret_cast<uint2*>(dst + at) = o;
        below = cur;
        cur = above;
    };
    if constexpr (DEPTH == 1) {
        Bf16Plane nxt;
        fetch_bf16(nxt, src, rhs, i, zb, d, g, v);
        for (int z = zb; z < ze; ++z, i += sz) {
            const Bf16Plane q = nxt;  // waits for the loads issued one plane ago
            if (z + 1 < ze) fetch_bf16(nxt, src, rhs, i + sz, z + 1, d, g, v);
            plane(q, z, i);
        }
    } else {
        // two buffers, planes alternating: the copy out of one waits only for
        // loads issued two planes ago while the other's stay in flight
        static_assert(DEPTH == 2, "prefetch depth 1 or 2");
        Bf16Plane pa, pb;
        fetch_bf16(pa, src, rhs, i, zb, d, g, v);
        if (zb + 1 < ze) fetch_bf16(pb, src, rhs, i + sz, zb + 1, d, g, v);
        for (int z = zb; z < ze; z += 2, i += 2 * sz) {
            const Bf16Plane qa = pa;
            if (z + 2 < ze) fetch_bf16(pa, src, rhs, i + 2 * sz, z + 2, d, g, v);
            plane(qa, z, i);
            if (z + 1 < ze) {
                const Bf16Plane qb = pb;
                if (z + 3 < ze) fetch_bf16(pb, src, rhs, i + 3 * sz, z + 3, d, g, v);
                plane(qb, z + 1, i + sz);
            }
        }
    }
}

constexpr int kBf16Depth = 2;

template <int KIND, int DEPTH = kBf16Depth>
__global__ void __launch_bounds__(32 * kVecRows) k_jacobi_bf16(__nv_bfloat16* __restrict__ dst, const __nv_bfloat16* __restrict__ src, const __nv_bfloat16* __restrict__ rhs, float coef, int z_chunk, Dims d, GhostRule g) {
    march_bf16<KIND, false, DEPTH>(dst, src, rhs, coef, 0, z_chunk, d, g);
}

template <int KIND, int DEPTH = kBf16Depth>
__global__ void __launch_bounds__(32 * kVecRows) k_rbgs_bf16(__nv_bfloat16* x, const __nv_bfloat16* __restrict__ rhs, float coef, int parity, int z_chunk, Dims d, GhostRule g) {
    march_bf16<KIND, true, DEPTH>(x, x, rhs, coef, parity, z_chunk, d, g);
}

// ---- red-black solves in the split layout (FP32 and BF16 fields) ----------
// For an RBGS solve the iterate and the right-hand side are stored split by
// colour: two arrays (red, black), each [nz][ny][nx / 2], holding in row
// (y, z) the cells x = 2k + s, k = 0 .. nx/2 - 1, with s = (y + z) & 1 for
// the red array and 1 - s for the black one (red: x + y + z even). A colour
// update then reads only the other colour's array and the right-hand side of
// its own colour, and writes its own array, all dense: 3 values moved per
// updated cell, so 3 per cell per iteration, where a colour launch on the
// interleaved field moves whole lines (3 per cell per colour). In the split
// layout the six neighbours of the cell (x = 2k + s_u, y, z) of colour array
// u are, in the other array v: k + s_u - 1 and k + s_u of the same row
// (x - 1, x + 1), and k of rows y - 1, y + 1 and of planes z - 1, z + 1 (the
// other colour's offset in an adjacent row is s_u, so the cell beside sits
// at the same k). The update is the colour launch's: the same six values
// summed in the reference's order (x-, x+, y-, y+, z-, z+), the same
// numerator and exact division in FP32 (for BF16 storage: on the unpacked
// values, rounded once to BF16 on the store), so every cell gets the same
// bits. Face ghosts take the cell's own value from u (threads on a face read
// their own four cells); periodic axes wrap k or the row (even sizes only:
// an odd periodic size breaks the colouring and leaves the solve to the
// colour launches).

// Four consecutive cells as FP32, and back, for either element type.
__device__ __forceinline__ float4 ld4v(const float* p) { return ld4(p); }
__device__ __forceinline__ float4 ld4v(const __nv_bfloat16* p) { return unpack_bf4(ld_bf4(p)); }
__device__ __forceinline__ float ld1v(const float* p) { return *p; }
__device__ __forceinline__ float ld1v(const __nv_bfloat16* p) { return ld_bf1(p); }
__device__ __forceinline__ void st4v(float* p, float4 o) { *reinterpret_cast<float4*>(p) = o; }
__device__ __forceinline__ void st4v(__nv_bfloat16* p, float4 o) { *reinterpret_cast<uint2*>(p) = make_uint2(pack_bf2(o.x, o.y), pack_bf2(o.z, o.w)); }

// Eight cells of a row split into four of each colour (lo: the even cells,
// hi: the odd ones), or merged back; FP32 as float4 pairs, BF16 as the
// 16-bit halves of four words (little endian: the even cell in the low half).
struct Split8F { float4 even, odd; };
__device__ __forceinline__ Split8F split8(const float* p) {
    const float4 v0 = ld4(p), v1 = ld4(p + 4);
    return {make_float4(v0.x, v0.z, v1.x, v1.z), make_float4(v0.y, v0.w, v1.y, v1.w)};
}
__device__ __forceinline__ void merge8(float* p, float4 even, float4 odd) {
    *reinterpret_cast<float4*>(p) = make_float4(even.x, odd.x, even.y, odd.y);
    *reinterpret_cast<float4*>(p + 4) = make_float4(even.z, odd.z, even.w, odd.w);
}
__device__ __forceinline__ void st4raw(float* p, float4 v) { *reinterpret_cast<float4*>(p) = v; }
__device__ __forceinline__ float4 ld4raw(const float* p) { return ld4(p); }

struct Split8H { uint2 even, odd; };
__device__ __forceinline__ Split8H split8(const __nv_bfloat16* p) {
    const uint4 w = *reinterpret_cast<const uint4*>(p);
    return {make_uint2(__byte_perm(w.x, w.y, 0x5410), __byte_perm(w.z, w.w, 0x5410)), make_uint2(__byte_perm(w.x, w.y, 0x7632), __byte_perm(w.z, w.w, 0x7632))};
}
__device__ __forceinline__ void merge8(__nv_bfloat16* p, uint2 even, uint2 odd) {
    *reinterpret_cast<uint4*>(p) = make_uint4(__byte_perm(even.x, odd.x, 0x5410), __byte_perm(even.x, odd.x, 0x7632), __byte_perm(even.y, odd.y, 0x5410), __byte_perm(even.y, odd.y, 0x7632));
}
__device__ __forceinline__ void st4raw(__nv_bfloat16* p, uint2 v) { *reinterpret_cast<uint2*>(p) = v; }
__device__ __forceinline__ uint2 ld4raw(const __nv_bfloat16* p) { return ld_bf4(p); }
__device__ __forceinline__ float4 scale4(float4 v, float f) { return make_float4(__fmul_rn(v.x, f), __fmul_rn(v.y, f), __fmul_rn(v.z, f), __fmul_rn(v.w, f)); }
__device__ __forceinline__ uint2 scale4(uint2 v, float f) {
    const float4 u = scale4(unpack_bf4(v), f);  // FP32 product rounded once to BF16, as k_scale_field
    return make_uint2(pack_bf2(u.x, u.y), pack_bf2(u.z, u.w));
}

template <bool SPLIT, typename T>
__device__ __forceinline__ void rb_layout_group(size_t f, T* __restrict__ field, T* __restrict__ red, T* __restrict__ black, T* __restrict__ red2, T* __restrict__ black2, float scale, const Dims& d) {
    const int per_row = d.nx / 8;
    const size_t row = f / per_row;
    const int y = static_cast<int>(row % d.ny), z = static_cast<int>(row / d.ny);
    const bool odd = ((y + z) & 1) != 0;  // the row's red cells sit at odd x
    if constexpr (SPLIT) {
        const auto c = split8(field + 8 * f);
        st4raw(red + 4 * f, odd ? c.odd : c.even);
        st4raw(black + 4 * f, odd ? c.even : c.odd);
        if (red2 != nullptr) {
            st4raw(red2 + 4 * f, odd ? c.odd : c.even);
            st4raw(black2 + 4 * f, odd ? c.even : c.odd);
        }
    } else {
        auto r = ld4raw(red + 4 * f), b = ld4raw(black + 4 * f);
        if (scale != 1.0f) {
            r = scale4(r, scale);
            b = scale4(b, scale);
        }
        if (odd) merge8(field + 8 * f, b, r);
        else merge8(field + 8 * f, r, b);
    }
}

// Splits (or, with SPLIT false, merges and scales) a field: a thread moves
// eight cells of a row (a group f) and four of each colour array. `red2` /
// `black2` (split only, may be null) receive a second copy.
template <bool SPLIT, typename T>
__global__ void __launch_bounds__(256) k_rb_layout(T* __restrict__ field, T* __restrict__ red, T* __restrict__ black, T* __restrict__ red2, T* __restrict__ black2, float scale, Dims d) {
    const size_t n8 = static_cast<size_t>(d.nx / 8) * d.ny * d.nz;
    for (size_t f = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; f < n8; f += static_cast<size_t>(gridDim.x) * blockDim.x) rb_layout_group<SPLIT, T>(f, field, red, black, red2, black2, scale, d);
}

// One colour of an RBGS iteration in the split layout, in place: u (the
// colour's array) from v (the other colour's) and w (the right-hand side's
// array of u's colour); `colour` 0 = red, 1 = black. A thread owns four
// cells of a half row (k0 .. k0 + 3) and marches a z chunk with v's planes
// below, at and above in registers; y neighbours and the extra x neighbour
// come from L1. No thread reads another's cells of u, so the update is in
// place. Threads are numbered along the half plane (blockIdx.x, 128 groups
// of four a CTA; blockIdx.z the z chunk), so short rows still fill every
// lane of a warp.
template <int KIND, typename T>
__device__ __forceinline__ void rb_half_block(uint32_t bx, uint32_t bz, T* u, const T* __restrict__ v, const T* __restrict__ w, float coef, int colour, int z_chunk, const Dims& d, const GhostRule& g, bool down = false) {
    const int hx = d.nx / 2, q4 = hx / 4;
    const int j = static_cast<int>(bx) * (32 * kVecRows) + static_cast<int>(threadIdx.y * 32 + threadIdx.x);
    const int y = j / q4, k0 = 4 * (j - y * q4);
    if (y >= d.ny) return;
    const int zb = static_cast<int>(bz) * z_chunk, ze = min(zb + z_chunk, d.nz);
    const bool px = g.periodic[0] != 0, py = g.periodic[1] != 0, pz = g.periodic[2] != 0;
    const float divisor = KIND == KIND_PRESSURE ? 6.0f : 1.0f + 6.0f * coef;
    const double recip = tb::recip64(divisor);
    const int hsz = hx * d.ny;
    // rows y - 1, y + 1 (offsets in the half plane) and their face ghosts
    const bool gy_lo = !py && y == 0, gy_hi = !py && y == d.ny - 1;
    const int oy_lo = y > 0 ? -hx : (py ? (d.ny - 1) * hx : 0), oy_hi = y + 1 < d.ny ? hx : (py ? -(d.ny - 1) * hx : 0);
    // the extra x neighbour: k0 - 1 (rows whose u cells sit at even x) or
    // k0 + 4 (odd x), wrapped or replaced by a ghost at a face
    const bool gx_lo = !px && k0 == 0, gx_hi = !px && k0 + 4 == hx;
    const int ox_lo = k0 > 0 ? -1 : (px ? hx - 1 : 0), ox_hi = k0 + 4 < hx ? 4 : (px ? 4 - hx : 3);
    // x faces: one cell of the thread (cell 0 on rows whose cells sit at even
    // x, cell 3 on odd ones) takes its x ghost, from its own value in u;
    // y faces (the whole row) and z faces (the whole plane) sit behind a
    // branch interior threads skip, rather than selects every thread executes
    const bool y_face = gy_lo || gy_hi;
    const int off_up = pz ? -(d.nz - 1) * hsz : 0;  // plane z + 1 from the top plane (itself on a face)
    const int off_dn = pz ? (d.nz - 1) * hsz : 0;   // plane z - 1 from the bottom plane
    const auto update = [&](int z, int i, float4 below, float4 cur, float4 above) {
        const bool s_odd = ((y + z + colour) & 1) != 0;  // this row's cells of u sit at odd x
        float ext = ld1v(v + i + (s_odd ? ox_hi : ox_lo));
        float4 c = ld4v(v + i + oy_lo), e = ld4v(v + i + oy_hi);
        const float4 r = ld4v(w + i);
        if (s_odd ? gx_hi : gx_lo) ext = tb::ghost(g, s_odd ? XP : XM, ld1v(u + i + (s_odd ? 3 : 0)));
        float4 zm = below, zp = above;
        const bool z_lo = !pz && z == 0, z_hi = !pz && z == d.nz - 1;
        if (y_face || z_lo || z_hi) [[unlikely]] {
            const float4 self = ld4v(u + i);
            if (gy_lo) c = ghost4(g, YM, self);
            if (gy_hi) e = ghost4(g, YP, self);
            if (z_lo) zm = ghost4(g, ZM, self);
            if (z_hi) zp = ghost4(g, ZP, self);
        }
        const float xm0 = s_odd ? cur.x : ext, xm1 = s_odd ? cur.y : cur.x, xm2 = s_odd ? cur.z : cur.y, xm3 = s_odd ? cur.w : cur.z;
        const float xp0 = s_odd ? cur.y : cur.x, xp1 = s_odd ? cur.z : cur.y, xp2 = s_odd ? cur.w : cur.z, xp3 = s_odd ? ext : cur.w;
        float4 o;
        o.x = vec_update<KIND>(xm0 + xp0 + c.x + e.x + zm.x + zp.x, r.x, coef, divisor, recip);
        o.y = vec_update<KIND>(xm1 + xp1 + c.y + e.y + zm.y + zp.y, r.y, coef, divisor, recip);
        o.z = vec_update<KIND>(xm2 + xp2 + c.z + e.z + zm.z + zp.z, r.z, coef, divisor, recip);
        o.w = vec_update<KIND>(xm3 + xp3 + c.w + e.w + zm.w + zp.w, r.w, coef, divisor, recip);
        st4v(u + i, o);
    };
    // DOWN marches the chunk from its top plane (see jacobi_vec4_block)
    if (!down) {
        int i = k0 + hx * (y + d.ny * zb);
        float4 cur = ld4v(v + i);
        float4 below = ld4v(v + i + (zb > 0 ? -hsz : off_dn));
        for (int z = zb; z < ze; ++z, i += hsz) {
            const float4 above = ld4v(v + i + (z + 1 < d.nz ? hsz : off_up));
            update(z, i, below, cur, above);
            below = cur;
            cur = above;
        }
    } else {
        int i = k0 + hx * (y + d.ny * (ze - 1));
        float4 cur = ld4v(v + i);
        float4 above = ld4v(v + i + (ze < d.nz ? hsz : off_up));
        for (int z = ze - 1; z >= zb; --z, i -= hsz) {
            const float4 below = ld4v(v + i + (z > 0 ? -hsz : off_dn));
            update(z, i, below, cur, above);
            above = cur;
            cur = below;
        }
    }
}

template <int KIND, typename T>
__global__ void __launch_bounds__(32 * kVecRows) k_rb_half(T* u, const T* __restrict__ v, const T* __restrict__ w, float coef, int colour, int z_chunk, Dims d, GhostRule g, int down) {
    wait_for_previous_grid();
    rb_half_block<KIND, T>(blockIdx.x, blockIdx.z, u, v, w, coef, colour, z_chunk, d, g, down != 0);
}

// Launch shape of the vectorised kernels: as many z chunks as fit the
// resident CTA slots of all SMs in one wave (a partial second wave costs
// more than the longer march per CTA).
struct VecShape {
    dim3 grid;
    int z_chunk;
};

template <typename Kernel>
VecShape vec_shape(const Dims& d, Kernel kernel, int width = 4) {
    static int per_sm = [&] {
        int n = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, 32 * kVecRows, 0) != cudaSuccess || n < 1) n = 4;
        return n;
    }();
    int sms = 148;
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int bx = (d.nx / width + 31) / 32, by = (d.ny + kVecRows - 1) / kVecRows;
    const long long slots = static_cast<long long>(sms) * per_sm;
    long long chunks = slots / (static_cast<long long>(bx) * by);  // one wave: every CTA resident at once
    if (chunks < 1) chunks = 1;
    int z_chunk = static_cast<int>((d.nz + chunks - 1) / chunks);
    if (z_chunk < 4) z_chunk = d.nz < 4 ? d.nz : 4;
    const int bz = (d.nz + z_chunk - 1) / z_chunk;
    return {dim3(static_cast<unsigned>(bx), static_cast<unsigned>(by), static_cast<unsigned>(bz)), z_chunk};
}

// The grid of a kernel whose threads are numbered along a plane of
// `per_plane` float4 (128 a CTA) and whose CTAs march z chunks: one wave.
template <typename Kernel>
VecShape plane_shape(const Dims& d, Kernel kernel, long long per_plane) {
    static int per_sm = [&] {
        int n = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, 32 * kVecRows, 0) != cudaSuccess || n < 1) n = 4;
        return n;
    }();
    int sms = 148, dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const long long bxy = (per_plane + 32 * kVecRows - 1) / (32 * kVecRows);
    long long chunks = static_cast<long long>(sms) * per_sm / bxy;
    if (chunks < 1) chunks = 1;
    int z_chunk = static_cast<int>((d.nz + chunks - 1) / chunks);
    if (z_chunk < 4) z_chunk = d.nz < 4 ? d.nz : 4;
    const int bz = (d.nz + z_chunk - 1) / z_chunk;
    return {dim3(static_cast<unsigned>(bxy), 1, static_cast<unsigned>(bz)), z_chunk};
}

bool vec_ok(const StencilArgs& a, int width = 4) {
    const auto al = [](const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; };
    const size_t cells = static_cast<size_t>(a.dims.nx) * a.dims.ny * a.dims.nz;
    return a.dims.nx % width == 0 && cells < (1ull << 31) && al(a.x) && al(a.b) && (a.scratch == nullptr || al(a.scratch));
}

// FP64 sums of the pressure residual e = h^2 div - (sum6(p) - 6 p) and of
// b = h^2 div (the four sums of k_residual_sums, same per-cell arithmetic),
// with the z-marching float4 layout above; one atomic per sum per CTA.
__device__ __forceinline__ double vec_warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Every thread of the block must call it (block-wide reduction).
__device__ __forceinline__ void residual_vec_block(uint3 blk, const float* __restrict__ p, const float* __restrict__ div, float h2, int z_chunk, const Dims& d, const GhostRule& g, DeviceStats* stats) {
    const int x0 = 4 * static_cast<int>(blk.x * 32 + threadIdx.x), y = static_cast<int>(blk.y * kVecRows + threadIdx.y);
    double se = 0.0, se2 = 0.0, sb = 0.0, sb2 = 0.0;
    if (x0 < d.nx && y < d.ny) {
        const int zb = static_cast<int>(blk.z) * z_chunk, ze = min(zb + z_chunk, d.nz);
        const VecGhost4 v = vec_ghost4(x0, y, d, g);
        const int sz = d.nx * d.ny;
        int i = x0 + d.nx * (y + d.ny * zb);
        float4 cur = ld4(p + i);
        float4 below = vec_below4(p, i, zb, d, g, cur);
        // two planes per iteration, so the next plane's loads overlap this
        // plane's FP64 arithmetic (the sums keep their order)
#pragma unroll 2
        for (int z = zb; z < ze; ++z, i += sz) {
            const float4 above = vec_above4(p, i, z, d, g, cur);
            float a = p[i + v.ox_lo], b = p[i + v.ox_hi];
            float4 c = ld4(p + i + v.oy_lo), e = ld4(p + i + v.oy_hi);
            const float4 r = ld4(div + i);
            if (v.gx_lo) a = tb::ghost(g, XM, a);
            if (v.gx_hi) b = tb::ghost(g, XP, b);
            if (v.gy_lo) c = ghost4(g, YM, c);
            if (v.gy_hi) e = ghost4(g, YP, e);
            const float xm[4] = {a, cur.x, cur.y, cur.z}, xp[4] = {cur.y, cur.z, cur.w, b};
            const float ym[4] = {c.x, c.y, c.z, c.w}, yp[4] = {e.x, e.y, e.z, e.w};
            const float zm[4] = {below.x, below.y, below.z, below.w}, zp[4] = {above.x, above.y, above.z, above.w};
            const float pc[4] = {cur.x, cur.y, cur.z, cur.w}, rc[4] = {r.x, r.y, r.z, r.w};
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const double nb = static_cast<double>(xm[k]) + static_cast<double>(xp[k]) + static_cast<double>(ym[k]) + static_cast<double>(yp[k]) + static_cast<double>(zm[k]) + static_cast<double>(zp[k]);
                const double bb = static_cast<double>(h2) * static_cast<double>(rc[k]);
                const double ee = bb - (nb - 6.0 * static_cast<double>(pc[k]));
                se += ee;
                se2 += ee * ee;
                sb += bb;
                sb2 += bb * bb;
            }
            below = cur;
            cur = above;
        }
    }
    __shared__ double part[4][kVecRows];
    se = vec_warp_sum(se);
    se2 = vec_warp_sum(se2);
    sb = vec_warp_sum(sb);
    sb2 = vec_warp_sum(sb2);
    if (threadIdx.x == 0) {
        part[0][threadIdx.y] = se;
        part[1][threadIdx.y] = se2;
        part[2][threadIdx.y] = sb;
        part[3][threadIdx.y] = sb2;
    }
    __syncthreads();
    if (threadIdx.y == 0 && threadIdx.x < 4) {
        double t = 0.0;
#pragma unroll
        for (int w = 0; w < kVecRows; ++w) t += part[threadIdx.x][w];
        double* dst = threadIdx.x == 0 ? &stats->sum_e : threadIdx.x == 1 ? &stats->sum_e2 : threadIdx.x == 2 ? &stats->sum_b : &stats->sum_b2;
        atomicAdd(dst, t);
    }
}

__global__ void __launch_bounds__(32 * kVecRows) k_residual_vec(const float* __restrict__ p, const float* __restrict__ div, float h2, int z_chunk, Dims d, GhostRule g, DeviceStats* stats) {
    residual_vec_block(blockIdx, p, div, h2, z_chunk, d, g, stats);
}

// One Jacobi pressure sweep dst = update(src) that also adds the FP64
// residual sums of its input iterate src to stats (the sums of
// residual_vec_block, from the values the sweep loads anyway: no extra
// traffic). The residual-driven solve runs it as the last sweep of each
// check interval, so a check sees the residual of the iterate one sweep
// before the current one; the Jacobi residual's norm never increases from
// one sweep to the next (I - A/6 is symmetric with its spectrum in (-1, 1]),
// so that iterate meeting the tolerance means the current one does too.
__global__ void __launch_bounds__(32 * kVecRows) k_jacobi_vec4_residual(float* __restrict__ dst, const float* __restrict__ src, const float* __restrict__ rhs, float h2, int z_chunk, Dims d, GhostRule g, DeviceStats* stats) {
    wait_for_previous_grid();
    const int x0 = 4 * static_cast<int>(blockIdx.x * 32 + threadIdx.x), y = static_cast<int>(blockIdx.y * kVecRows + threadIdx.y);
    double se = 0.0, se2 = 0.0, sb = 0.0, sb2 = 0.0;
    if (x0 < d.nx && y < d.ny) {
        const int zb = static_cast<int>(blockIdx.z) * z_chunk, ze = min(zb + z_chunk, d.nz);
        const float inv = wave::jacobi_inverse(KIND_PRESSURE, h2);
        const VecGhost4 v = vec_ghost4(x0, y, d, g);
        const int sz = d.nx * d.ny;
        int i = x0 + d.nx * (y + d.ny * zb);
        float4 cur = ld4(src + i);
        float4 below = vec_below4(src, i, zb, d, g, cur);
        for (int z = zb; z < ze; ++z, i += sz) {
            const float4 above = vec_above4(src, i, z, d, g, cur);
            float a = src[i + v.ox_lo], b = src[i + v.ox_hi];
            float4 c = ld4(src + i + v.oy_lo), e = ld4(src + i + v.oy_hi);
            const float4 r = ld4(rhs + i);
            if (v.gx_lo) a = tb::ghost(g, XM, a);
            if (v.gx_hi) b = tb::ghost(g, XP, b);
            if (v.gy_lo) c = ghost4(g, YM, c);
            if (v.gy_hi) e = ghost4(g, YP, e);
            float4 o;
            o.x = wave::jacobi_update<KIND_PRESSURE>(a + cur.y + c.x + e.x + below.x + above.x, r.x, h2, inv);
            o.y = wave::jacobi_update<KIND_PRESSURE>(cur.x + cur.z + c.y + e.y + below.y + above.y, r.y, h2, inv);
            o.z = wave::jacobi_update<KIND_PRESSURE>(cur.y + cur.w + c.z + e.z + below.z + above.z, r.z, h2, inv);
            o.w = wave::jacobi_update<KIND_PRESSURE>(cur.z + b + c.w + e.w + below.w + above.w, r.w, h2, inv);
            *reinterpret_cast<float4*>(dst + i) = o;
            const float xm[4] = {a, cur.x, cur.y, cur.z}, xp[4] = {cur.y, cur.z, cur.w, b};
            const float ym[4] = {c.x, c.y, c.z, c.w}, yp[4] = {e.x, e.y, e.z, e.w};
            const float zm[4] = {below.x, below.y, below.z, below.w}, zp[4] = {above.x, above.y, above.z, above.w};
            const float pc[4] = {cur.x, cur.y, cur.z, cur.w}, rc[4] = {r.x, r.y, r.z, r.w};
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const double nb = static_cast<double>(xm[k]) + static_cast<double>(xp[k]) + static_cast<double>(ym[k]) + static_cast<double>(yp[k]) + static_cast<double>(zm[k]) + static_cast<double>(zp[k]);
                const double bb = static_cast<double>(h2) * static_cast<double>(rc[k]);
                const double ee = bb - (nb - 6.0 * static_cast<double>(pc[k]));
                se += ee;
                se2 += ee * ee;
                sb += bb;
                sb2 += bb * bb;
            }
            below = cur;
            cur = above;
        }
    }
    __shared__ double part[4][kVecRows];
    se = vec_warp_sum(se);
    se2 = vec_warp_sum(se2);
    sb = vec_warp_sum(sb);
    sb2 = vec_warp_sum(sb2);
    if (threadIdx.x == 0) {
        part[0][threadIdx.y] = se;
        part[1][threadIdx.y] = se2;
        part[2][threadIdx.y] = sb;
        part[3][threadIdx.y] = sb2;
    }
    __syncthreads();
    if (threadIdx.y == 0 && threadIdx.x < 4) {
        double t = 0.0;
#pragma unroll
        for (int w = 0; w < kVecRows; ++w) t += part[threadIdx.x][w];
        double* out = threadIdx.x == 0 ? &stats->sum_e : threadIdx.x == 1 ? &stats->sum_e2 : threadIdx.x == 2 ? &stats->sum_b : &stats->sum_b2;
        atomicAdd(out, t);
    }
}

template <typename T = float>
__global__ void k_scale_field(T* __restrict__ q, float factor, size_t n) {
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n; i += static_cast<size_t>(gridDim.x) * blockDim.x) q[i] = from_f<T>(to_f(q[i]) * factor);
}

GhostRule ghost_rule(int kind, const FlowBC& fb, const ScalarBC& sb);

// Vectorised sweep kernels per element type (4 cells per thread for both).
template <int KIND, typename T>
auto jacobi_vec_kernel() {
    if constexpr (sizeof(T) == sizeof(float)) return k_jacobi_vec4<KIND>;
    else return k_jacobi_bf16<KIND>;
}

template <int KIND, typename T>
auto rbgs_vec_kernel() {
    if constexpr (sizeof(T) == sizeof(float)) return k_rbgs_vec4<KIND>;
    else return k_rbgs_bf16<KIND>;
}

// True when a periodic axis of odd size breaks the red-black colouring
// across its wrap (the first and last cells of a line share a colour).
bool odd_periodic(const StencilArgs& a) {
    const bool sc = a.kind == KIND_SCALAR;
    const int per[3] = {sc ? a.scalar.periodic[0] : a.flow.periodic[0], sc ? a.scalar.periodic[1] : a.flow.periodic[1], sc ? a.scalar.periodic[2] : a.flow.periodic[2]};
    const int n[3] = {a.dims.nx, a.dims.ny, a.dims.nz};
    for (int k = 0; k < 3; ++k)
        if (per[k] && (n[k] & 1)) return true;
    return false;
}

// The split-layout red-black solve applies: rows of a multiple of 8 cells
// (four of each colour a thread), both scratch buffers, no odd periodic
// axis; per_pass 1 asks for the colour launches instead.
bool rb_split_ok(const StencilArgs& a) {
    if (a.scratch == nullptr || a.scratch2 == nullptr || a.per_pass == 1 || a.iterations < 1) return false;
    if (a.dims.nx % 8 != 0 || !vec_ok(a) || (reinterpret_cast<uintptr_t>(a.scratch2) & 15) != 0) return false;
    return !odd_periodic(a);
}

template <bool SPLIT, typename T>
cudaError_t launch_rb_layout(T* field, T* red, T* black, T* red2, T* black2, float scale, const Dims& d, cudaStream_t s) {
    const size_t n8 = static_cast<size_t>(d.nx / 8) * d.ny * d.nz;
    size_t blocks = (n8 + 255) / 256;
    if (blocks > 148u * 16u) blocks = 148u * 16u;
    k_rb_layout<SPLIT, T><<<static_cast<unsigned>(blocks), 256, 0, s>>>(field, red, black, red2, black2, scale, d);
    return cudaGetLastError();
}

// The solve in the split layout: the right-hand side split into scratch2,
// the iterate into scratch (from x, from b, or zero), the iterations as red
// and black half launches, then the iterate merged back into x, times
// out_scale. T: the element type of x, b and both scratch buffers.
template <int KIND, typename T>
cudaError_t run_rb_split(const StencilArgs& a, cudaStream_t s) {
    const Dims& d = a.dims;
    const size_t half = static_cast<size_t>(d.nx) * d.ny * d.nz / 2;
    T* const x = reinterpret_cast<T*>(a.x);
    T* const xr = reinterpret_cast<T*>(a.scratch);
    T* const xb = xr + half;
    T* const br = reinterpret_cast<T*>(a.scratch2);
    T* const bb = br + half;
    cudaError_t e = cudaSuccess;
    const bool from_b = a.init == INIT_FROM_B;
    if ((e = launch_rb_layout<true, T>(reinterpret_cast<T*>(const_cast<float*>(a.b)), br, bb, from_b ? xr : nullptr, from_b ? xb : nullptr, 1.0f, d, s)) != cudaSuccess) return e;
    int kernels = 2;  // the right-hand side's split and the final merge
    if (a.init == INIT_ZERO) {
        if ((e = cudaMemsetAsync(xr, 0, 2 * half * sizeof(T), s)) != cudaSuccess) return e;
    } else if (a.init == INIT_FROM_X) {
        if ((e = launch_rb_layout<true, T>(x, xr, xb, nullptr, nullptr, 1.0f, d, s)) != cudaSuccess) return e;
        ++kernels;
    }
    const GhostRule g = ghost_rule(KIND, a.flow, a.scalar);
    const auto kern = k_rb_half<KIND, T>;
    const VecShape vs = plane_shape(d, kern, static_cast<long long>(d.nx / 8) * d.ny);
    // the two colours march their z chunks in opposite directions, so each
    // launch starts on the planes the one before wrote last (still in L2)
    for (int it = 0; it < a.iterations; ++it) {
        if ((e = launch_sweep(kern, vs.grid, dim3(32, kVecRows), s, xr, static_cast<const T*>(xb), static_cast<const T*>(br), a.coef, 0, vs.z_chunk, d, g, 0)) != cudaSuccess) return e;
        if ((e = launch_sweep(kern, vs.grid, dim3(32, kVecRows), s, xb, static_cast<const T*>(xr), static_cast<const T*>(bb), a.coef, 1, vs.z_chunk, d, g, 1)) != cudaSuccess) return e;
    }
    if ((e = launch_rb_layout<false, T>(x, xr, xb, nullptr, nullptr, a.out_scale, d, s)) != cudaSuccess) return e;
    if (a.launches) *a.launches += 2 * a.iterations + kernels;
    return cudaSuccess;
}

// T: element type of x, b and scratch (BF16 only for the diffusion kinds of a
// BF16-storage context; the pressure is always FP32).
template <int KIND, typename T>
cudaError_t run_simple(const StencilArgs& a, cudaStream_t s) {
    const Dims& d = a.dims;
    const size_t n = static_cast<size_t>(d.nx) * d.ny * d.nz;
    const size_t bytes = n * sizeof(T);
    T* const ax = reinterpret_cast<T*>(a.x);
    T* const ascr = reinterpret_cast<T*>(a.scratch);
    const T* const ab = reinterpret_cast<const T*>(a.b);
    cudaError_t e = cudaSuccess;
    if (a.scheme == SCHEME_RBGS) {
        if (rb_split_ok(a)) return run_rb_split<KIND, T>(a, s);
        if (a.init == INIT_FROM_B) e = cudaMemcpyAsync(ax, ab, bytes, cudaMemcpyDeviceToDevice, s);
        else if (a.init == INIT_ZERO) e = cudaMemsetAsync(ax, 0, bytes, s);
        if (e != cudaSuccess) return e;
        if (vec_ok(a)) {
            const GhostRule g = ghost_rule(KIND, a.flow, a.scalar);
            const auto kernel = rbgs_vec_kernel<KIND, T>();
            const VecShape vs = vec_shape(d, kernel);
            for (int it = 0; it < a.iterations; ++it)
                for (int parity = 0; parity < 2; ++parity) {
                    if constexpr (sizeof(T) == sizeof(float)) launch_sweep(kernel, vs.grid, dim3(32, kVecRows), s, ax, ab, a.coef, parity, vs.z_chunk, d, g);
                    else kernel<<<vs.grid, dim3(32, kVecRows), 0, s>>>(ax, ab, a.coef, parity, vs.z_chunk, d, g);
                }
        } else {
            const dim3 cblock(32, 8, 1);
            const dim3 grid(static_cast<unsigned>(((d.nx + 1) / 2 + 31) / 32), static_cast<unsigned>((d.ny + 7) / 8), static_cast<unsigned>((d.nz + kColourPlanes - 1) / kColourPlanes));
            for (int it = 0; it < a.iterations; ++it)
                for (int parity = 0; parity < 2; ++parity) k_rbgs_colour<KIND, T><<<grid, cblock, 0, s>>>(ax, ab, a.coef, parity, d, a.flow, a.scalar);
        }
        if (a.launches) *a.launches += 2 * a.iterations;
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    } else {
        const bool vec = vec_ok(a);
        const GhostRule g = ghost_rule(KIND, a.flow, a.scalar);
        const auto jacobi_vec = jacobi_vec_kernel<KIND, T>();
        const VecShape vs = vec ? vec_shape(d, jacobi_vec) : VecShape{};
        const dim3 jblock(32, 8, 1);
        const dim3 grid(static_cast<unsigned>((d.nx + 31) / 32), static_cast<unsigned>((d.ny + 7) / 8), static_cast<unsigned>((d.nz + kColourPlanes - 1) / kColourPlanes));
        const int units = a.iterations;
        // Choose the first source so that the last launch lands in x.
        const T* src = ax;
        if (a.init == INIT_FROM_B) src = ab;
        else if (a.init == INIT_ZERO) {
            // Zero the buffer the first launch does not write.
            T* zero = (units & 1) ? ascr : ax;
            if ((e = cudaMemsetAsync(zero, 0, bytes, s)) != cudaSuccess) return e;
            src = zero;
        }
        if (a.iterations == 0) {
            if (src != ax) e = cudaMemcpyAsync(ax, src, bytes, cudaMemcpyDeviceToDevice, s);
            if (e != cudaSuccess) return e;
        }
        for (int u = 0; u < units; ++u) {
            const int left = units - u;  // launches still to run, this one included
            T* dst = (left & 1) ? ax : ascr;
            if (dst == src) dst = (dst == ax) ? ascr : ax;
            if (vec) {
                // consecutive sweeps march their z chunks in opposite directions (the last one upward)
                if constexpr (sizeof(T) == sizeof(float)) launch_sweep((left - 1) & 1 ? k_jacobi_vec4<KIND, true> : k_jacobi_vec4<KIND>, vs.grid, dim3(32, kVecRows), s, dst, static_cast<const T*>(src), ab, a.coef, vs.z_chunk, d, g);
                else jacobi_vec<<<vs.grid, dim3(32, kVecRows), 0, s>>>(dst, src, ab, a.coef, vs.z_chunk, d, g);
            } else {
                k_jacobi<KIND, T><<<grid, jblock, 0, s>>>(dst, src, ab, a.coef, d, a.flow, a.scalar);
            }
            src = dst;
        }
        if (a.launches) *a.launches += units;
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        if (src != ax && a.iterations > 0) {
            if ((e = cudaMemcpyAsync(ax, src, bytes, cudaMemcpyDeviceToDevice, s)) != cudaSuccess) return e;
        }
    }
    if (a.out_scale != 1.0f) {
        size_t g = (n + 255) / 256;
        if (g > 148u * 32u) g = 148u * 32u;
        k_scale_field<T><<<static_cast<unsigned>(g), 256, 0, s>>>(ax, a.out_scale, n);
        e = cudaGetLastError();
        if (a.launches) *a.launches += 1;
    }
    return e;
}


// ------------------------------------------------------ z-wavefront path --
// K stages per pass (sf_stencil_wave.cuh): Jacobi sweeps, or red-black
// half-iterations (two stages per iteration), for FP32 fields whose rows are
// 128 or 256 cells.
constexpr int kWaveRows = 16;  // rows per CTA (one warp each), halo rows included

// Stages per pass: 4 for rows of 128 cells; for rows of 256, 3 (Jacobi) or
// 2 (one red-black iteration): their shared-memory rings (4 input planes,
// two per intermediate stage, K + 3 right-hand-side planes of 16 KB) fill
// the 227 KB a CTA may use, and their register history the 128 registers a
// 512-thread CTA gives each thread.
template <int V, bool RB>
constexpr int wave_stages() { return V == 1 ? 4 : (RB ? 2 : 3); }

// Rows of 128 V cells: V, or 0 when the grid does not suit the kernel.
int wave_width(const StencilArgs& a) {
    if (a.bf16 || a.scratch == nullptr || !vec_ok(a)) return 0;
    if (a.dims.nx != 128 && a.dims.nx != 256) return 0;
    if (a.dims.nz <= 8) return 0;  // the chunk halo wraps a periodic z axis at most once
    if (a.scheme == SCHEME_RBGS && odd_periodic(a)) return 0;  // the colouring breaks across the wrap
    return a.dims.nx / 128;
}

template <int KIND, bool RB, int K, int V>
cudaError_t launch_wave_pass(const wave::WaveArgs& w, int sms, cudaStream_t s) {
    constexpr size_t smem = wave::WaveLayout<K, V, kWaveRows>::bytes;
    static_assert(smem <= 232448, "shared memory per CTA");
    auto kern = wave::k_wave<KIND, RB, K, V, kWaveRows>;
    static const cudaError_t attr = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (attr != cudaSuccess) return attr;
    constexpr int ty = kWaveRows - 2 * K;
    const int tiles = (w.d.ny + ty - 1) / ty;
    // one wave of CTAs (one per SM): z chunks per tile column
    int chunks = sms / tiles;
    if (chunks < 1) chunks = 1;
    wave::WaveArgs a = w;
    a.z_chunk = (w.d.nz + chunks - 1) / chunks;
    const dim3 grid(static_cast<unsigned>(tiles), static_cast<unsigned>((w.d.nz + a.z_chunk - 1) / a.z_chunk));
    kern<<<grid, 32 * kWaveRows, smem, s>>>(a);
    return cudaGetLastError();
}

// The solve as whole passes of K stages, the remainder as single sweeps
// (Jacobi) or single colour launches (red-black) of the same arithmetic.
template <int KIND, bool RB, int V>
cudaError_t run_wave(const StencilArgs& a, cudaStream_t s) {
    constexpr int K = wave_stages<V, RB>();
    const Dims& d = a.dims;
    const size_t bytes = static_cast<size_t>(d.nx) * d.ny * d.nz * sizeof(float);
    const int stages = RB ? 2 * a.iterations : a.iterations;
    const int passes = stages / K;
    if (passes == 0) return run_simple<KIND, float>(a, s);
    const int rest = stages - passes * K;  // Jacobi sweeps / red-black iterations x 2 left over
    cudaError_t e = cudaSuccess;
    const GhostRule g = ghost_rule(KIND, a.flow, a.scalar);
    wave::WaveArgs w{};
    w.rhs = a.b;
    w.coef = a.coef;
    w.d = d;
    w.g = g;
    int sms = 148, dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    // out-of-place units (Jacobi: the passes and the single sweeps; red-black:
    // the passes, the colour launches then run in place on x), the last in x
    const int units = RB ? passes : passes + rest;
    const float* src = a.init == INIT_ZERO ? nullptr : (a.init == INIT_FROM_B ? a.b : a.x);
    const bool scale_in_pass = rest == 0;
    const auto vs = vec_shape(d, k_jacobi_vec4<KIND>);
    for (int u = 0; u < units; ++u) {
        float* dst = ((units - 1 - u) % 2 == 0) ? a.x : a.scratch;
        if (src == dst) {  // warm start from x with an odd unit count: move it aside
            if ((e = cudaMemcpyAsync(a.scratch, a.x, bytes, cudaMemcpyDeviceToDevice, s)) != cudaSuccess) return e;
            src = a.scratch;
        }
        if (u < passes) {
            w.src = src;
            w.dst = dst;
            w.out_scale = (u == passes - 1 && scale_in_pass) ? a.out_scale : 1.0f;
            if ((e = launch_wave_pass<KIND, RB, K, V>(w, sms, s)) != cudaSuccess) return e;
        } else {
            k_jacobi_vec4<KIND><<<vs.grid, dim3(32, kVecRows), 0, s>>>(dst, src, a.b, a.coef, vs.z_chunk, d, g);
        }
        if (a.launches) *a.launches += 1;
        src = dst;
    }
    if (RB && rest > 0) {
        const auto rs = vec_shape(d, k_rbgs_vec4<KIND>);
        for (int it = 0; it < rest / 2; ++it)
            for (int parity = 0; parity < 2; ++parity) k_rbgs_vec4<KIND><<<rs.grid, dim3(32, kVecRows), 0, s>>>(a.x, a.b, a.coef, parity, rs.z_chunk, d, g);
        if (a.launches) *a.launches += rest;
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (!scale_in_pass && a.out_scale != 1.0f) {
        const size_t n = static_cast<size_t>(d.nx) * d.ny * d.nz;
        k_scale_field<<<148u * 32u, 256, 0, s>>>(a.x, a.out_scale, n);
        if (a.launches) *a.launches += 1;
        e = cudaGetLastError();
    }
    return e;
}

template <int KIND>
cudaError_t run_wave_kind(const StencilArgs& a, int v, cudaStream_t s) {
    const bool rb = a.scheme == SCHEME_RBGS;
    if (v == 1) return rb ? run_wave<KIND, true, 1>(a, s) : run_wave<KIND, false, 1>(a, s);
    return rb ? run_wave<KIND, true, 2>(a, s) : run_wave<KIND, false, 2>(a, s);
}

// ------------------------------------------------ temporally blocked path --
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) != cudaSuccess || q != cudaDriverEntryPointSuccess) p = nullptr;
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }();
    return fn;
}

// 3D map over a dense x-fastest FP32 field with a W x HH x 1 box.
bool plane_map(CUtensorMap* m, const float* base, const Dims& d, int w, int hh) {
    auto encode = tensor_map_encoder();
    if (encode == nullptr || base == nullptr) return false;
    const cuuint64_t dims[3] = {static_cast<cuuint64_t>(d.nx), static_cast<cuuint64_t>(d.ny), static_cast<cuuint64_t>(d.nz)};
    const cuuint64_t strides[2] = {static_cast<cuuint64_t>(d.nx) * 4u, static_cast<cuuint64_t>(d.nx) * static_cast<cuuint64_t>(d.ny) * 4u};
    const cuuint32_t box[3] = {static_cast<cuuint32_t>(w), static_cast<cuuint32_t>(hh), 1u};
    const cuuint32_t estr[3] = {1u, 1u, 1u};
    return encode(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Face ghost rules of a field kind, from the flattened boundary (the same
// rules as load_pressure / load_scalar / load_velocity for a face neighbour).
GhostRule ghost_rule(int kind, const FlowBC& fb, const ScalarBC& sb) {
    GhostRule g{};
    for (int f = 0; f < 6; ++f) {
        const int axis = f / 2;
        if (kind == KIND_PRESSURE) {
            g.mode[f] = fb.type[f] == STABLE_FLUIDS_FLOW_BOUNDARY_OUTFLOW ? GHOST_CONST : GHOST_COPY;
            g.k[f] = fb.pressure[f];
        } else if (kind == KIND_SCALAR) {
            g.mode[f] = sb.type[f] == STABLE_FLUIDS_SCALAR_BOUNDARY_FIXED_VALUE ? GHOST_CONST : GHOST_COPY;
            g.k[f] = sb.value[f];
        } else {
            const int comp = kind;
            const bool copy = fb.type[f] == STABLE_FLUIDS_FLOW_BOUNDARY_OUTFLOW || (fb.type[f] == STABLE_FLUIDS_FLOW_BOUNDARY_FREE_SLIP_WALL && comp != axis);
            g.mode[f] = copy ? GHOST_COPY : GHOST_REFLECT;
            g.k[f] = 2.0f * fb.vel[f][comp];
        }
    }
    for (int a = 0; a < 3; ++a) g.periodic[a] = kind == KIND_SCALAR ? sb.periodic[a] : fb.periodic[a];
    return g;
}

struct TbShape {
    int k, w, hh, nt, ctas_per_sm;
};

template <int KIND, int K, int W, int HH, int ZP, int NT>
cudaError_t launch_tb_pass(const TbArgs& args, const CUtensorMap& mx, const CUtensorMap& mb, int z_chunk, cudaStream_t s) {
    constexpr size_t smem = TbLayout<K, W, HH, ZP>::bytes;
    static_assert(smem <= 232448, "shared memory per CTA");
    auto kern = k_rbgs_tb<KIND, K, W, HH, ZP, NT>;
    static const cudaError_t attr = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (attr != cudaSuccess) return attr;
    constexpr int HX = ((K + 3) / 4) * 4;
    const dim3 grid(static_cast<unsigned>((args.d.nx + W - 2 * HX - 1) / (W - 2 * HX)), static_cast<unsigned>((args.d.ny + HH - 2 * K - 1) / (HH - 2 * K)), static_cast<unsigned>((args.d.nz + z_chunk - 1) / z_chunk));
    kern<<<grid, NT, smem, s>>>(mx, mb, args);
    return cudaGetLastError();
}

// Planes per CTA: minimise (waves x streamed planes per CTA).
int choose_z_chunk(const Dims& d, int tiles_xy, int k, int ctas_per_sm) {
    const int slots = 148 * ctas_per_sm;
    int best = d.nz;
    long long best_cost = LLONG_MAX;
    for (int c = 1; c <= d.nz; ++c) {
        const int z = (d.nz + c - 1) / c;
        if ((c - 1) * z >= d.nz) continue;
        const long long waves = (static_cast<long long>(tiles_xy) * c + slots - 1) / slots;
        const long long cost = waves * (z + 2 * k);
        if (cost < best_cost) {
            best_cost = cost;
            best = z;
        }
    }
    return best;
}

constexpr TbShape kTbShape{4, 96, 24, 384, 1};

template <int KIND>
cudaError_t run_tb(const StencilArgs& a, cudaStream_t s, unsigned* error_flag) {
    constexpr int K = 4, W = 96, HH = 24, ZP = 2, NT = 384;
    const Dims& d = a.dims;
    const size_t n = static_cast<size_t>(d.nx) * d.ny * d.nz;
    const size_t bytes = n * sizeof(float);
    const int per_pass = a.per_pass > 0 ? (a.per_pass < K / 2 ? a.per_pass : K / 2) : K / 2;
    cudaError_t e = cudaSuccess;
    if (a.iterations == 0) {
        if (a.init == INIT_ZERO) e = cudaMemsetAsync(a.x, 0, bytes, s);
        else if (a.init == INIT_FROM_B) e = cudaMemcpyAsync(a.x, a.b, bytes, cudaMemcpyDeviceToDevice, s);
        if (e != cudaSuccess) return e;
        if (a.out_scale != 1.0f) {
            k_scale_field<<<148u * 32u, 256, 0, s>>>(a.x, a.out_scale, n);
            if (a.launches) *a.launches += 1;
            return cudaGetLastError();
        }
        return cudaSuccess;
    }
    TbArgs t{};
    t.b = a.b;
    t.coef = a.coef;
    t.d = d;
    t.g = ghost_rule(a.kind, a.flow, a.scalar);
    t.error = error_flag;
    const bool aligned = d.nx % 4 == 0 && (reinterpret_cast<uintptr_t>(a.x) & 15) == 0 && (reinterpret_cast<uintptr_t>(a.scratch) & 15) == 0 && (reinterpret_cast<uintptr_t>(a.b) & 15) == 0;
    CUtensorMap map_b{}, map_x{}, map_s{};
    t.tma_ok = aligned && plane_map(&map_b, a.b, d, W, HH) && plane_map(&map_x, a.x, d, W, HH) && plane_map(&map_s, a.scratch, d, W, HH);
    constexpr int HX = ((K + 3) / 4) * 4;
    const int tiles_xy = ((d.nx + W - 2 * HX - 1) / (W - 2 * HX)) * ((d.ny + HH - 2 * K - 1) / (HH - 2 * K));
    const int passes = (a.iterations + per_pass - 1) / per_pass;
    const float* src = a.init == INIT_ZERO ? nullptr : (a.init == INIT_FROM_B ? a.b : a.x);
    const CUtensorMap* src_map = a.init == INIT_FROM_B ? &map_b : &map_x;
    for (int i = 0; i < passes; ++i) {
        float* dst = ((passes - 1 - i) % 2 == 0) ? a.x : a.scratch;
        const CUtensorMap* dst_map = dst == a.x ? &map_x : &map_s;
        if (src == dst) {  // warm start from x with an odd pass count: move it aside
            if ((e = cudaMemcpyAsync(a.scratch, a.x, bytes, cudaMemcpyDeviceToDevice, s)) != cudaSuccess) return e;
            src = a.scratch;
            src_map = &map_s;
        }
        const int iters = (i == passes - 1) ? a.iterations - per_pass * (passes - 1) : per_pass;
        t.src = src;
        t.dst = dst;
        t.k_run = 2 * iters;
        t.out_scale = (i == passes - 1) ? a.out_scale : 1.0f;
        t.z_chunk = choose_z_chunk(d, tiles_xy, t.k_run, kTbShape.ctas_per_sm);
        if ((e = launch_tb_pass<KIND, K, W, HH, ZP, NT>(t, *src_map, map_b, t.z_chunk, s)) != cudaSuccess) return e;
        if (a.launches) *a.launches += 1;
        src = dst;
        src_map = dst_map;
    }
    return cudaSuccess;
}

bool tb_supported(const StencilArgs& a) {
    if (a.scheme != SCHEME_RBGS || a.scratch == nullptr) return false;
    const int kind = a.kind;
    const int per[3] = {kind == KIND_SCALAR ? a.scalar.periodic[0] : a.flow.periodic[0], kind == KIND_SCALAR ? a.scalar.periodic[1] : a.flow.periodic[1], kind == KIND_SCALAR ? a.scalar.periodic[2] : a.flow.periodic[2]};
    const int n[3] = {a.dims.nx, a.dims.ny, a.dims.nz};
    // An odd periodic size breaks the red-black colouring across the wrap.
    for (int k = 0; k < 3; ++k)
        if (per[k] && (n[k] & 1)) return false;
    return true;
}

// ------------------------------------------------------- work-table batch --
// The sweeps of every simulation of a batch in one launch (sf_batch.h): work
// item w is block w - first[s] of simulation s's own vectorised launch, run
// by the same block body as a single-simulation sweep.
__device__ __forceinline__ uint3 vec_block_of(uint32_t local, const Dims& d) {
    return batch_block(local, static_cast<uint32_t>((d.nx / 4 + 31) / 32), static_cast<uint32_t>((d.ny + kVecRows - 1) / kVecRows));
}

template <int KIND>
__global__ void __launch_bounds__(32 * kVecRows) k_batch_rbgs(BatchTable t, int parity) {
    const uint32_t* first = t.first[SHAPE_VEC];
    for (uint32_t w = blockIdx.x; w < t.total[SHAPE_VEC]; w += gridDim.x) {
        const int si = batch_sim(first, t.nsims, w);
        const BatchSim& m = t.sims[si];
        const float coef = KIND == KIND_PRESSURE ? m.h * m.h : (KIND == KIND_SCALAR ? m.alpha_s : m.alpha_v);
        rbgs_vec4_block<KIND>(vec_block_of(w - first[si], m.d), batch_field(m, KIND, BF_X), batch_field(m, KIND, BF_B), coef, parity, m.z_chunk, m.d, m.ghost[KIND]);
    }
}

template <int KIND>
__global__ void __launch_bounds__(32 * kVecRows) k_batch_jacobi(BatchTable t, int dst, int src) {
    const uint32_t* first = t.first[SHAPE_VEC];
    for (uint32_t w = blockIdx.x; w < t.total[SHAPE_VEC]; w += gridDim.x) {
        const int si = batch_sim(first, t.nsims, w);
        const BatchSim& m = t.sims[si];
        const float coef = KIND == KIND_PRESSURE ? m.h * m.h : (KIND == KIND_SCALAR ? m.alpha_s : m.alpha_v);
        jacobi_vec4_block<KIND>(vec_block_of(w - first[si], m.d), batch_field(m, KIND, dst), batch_field(m, KIND, src), batch_field(m, KIND, BF_B), coef, m.z_chunk, m.d, m.ghost[KIND]);
    }
}

__global__ void __launch_bounds__(32 * kVecRows) k_batch_residual(BatchTable t) {
    const uint32_t* first = t.first[SHAPE_VEC];
    for (uint32_t w = blockIdx.x; w < t.total[SHAPE_VEC]; w += gridDim.x) {
        const int si = batch_sim(first, t.nsims, w);
        const BatchSim& m = t.sims[si];
        residual_vec_block(vec_block_of(w - first[si], m.d), m.pressure, m.divergence, m.h * m.h, m.z_chunk, m.d, m.ghost[KIND_PRESSURE], m.stats);
        __syncthreads();  // the block's reduction buffer is reused by the next item
    }
}

// dst <- src (src >= 0) or dst <- 0, over the linear shape.
__global__ void __launch_bounds__(256) k_batch_copy(BatchTable t, int kind, int dst, int src) {
    const uint32_t* first = t.first[SHAPE_LINEAR];
    for (uint32_t w = blockIdx.x; w < t.total[SHAPE_LINEAR]; w += gridDim.x) {
        const int si = batch_sim(first, t.nsims, w);
        const BatchSim& m = t.sims[si];
        const size_t n = static_cast<size_t>(m.d.nx) * m.d.ny * m.d.nz;
        const size_t i = static_cast<size_t>(w - first[si]) * 256u + threadIdx.x;
        if (i < n) batch_field(m, kind, dst)[i] = src >= 0 ? batch_field(m, kind, src)[i] : 0.0f;
    }
}

// Scalar dissipation after its diffusion: rho *= 1 / (1 + dt k) (k_scale_field).
__global__ void __launch_bounds__(256) k_batch_scale_scalar(BatchTable t) {
    const uint32_t* first = t.first[SHAPE_LINEAR];
    for (uint32_t w = blockIdx.x; w < t.total[SHAPE_LINEAR]; w += gridDim.x) {
        const int si = batch_sim(first, t.nsims, w);
        const BatchSim& m = t.sims[si];
        const size_t n = static_cast<size_t>(m.d.nx) * m.d.ny * m.d.nz;
        const size_t i = static_cast<size_t>(w - first[si]) * 256u + threadIdx.x;
        if (i < n) m.sdata[i] = m.sdata[i] * m.scale_s;
    }
}

// Colour-split red-black solves over the work table (rb_layout_group and
// rb_half_block per work item; the split buffers are the simulation's scratch
// and scratch2, red half first).
__global__ void __launch_bounds__(256) k_batch_rb_layout(BatchTable t, int kind, int which, int copy_iterate, int merge, int dissipate) {
    const uint32_t* first = t.first[SHAPE_OCT];
    for (uint32_t w = blockIdx.x; w < t.total[SHAPE_OCT]; w += gridDim.x) {
        const int si = batch_sim(first, t.nsims, w);
        const BatchSim& m = t.sims[si];
        const size_t n8 = static_cast<size_t>(m.d.nx / 8) * m.d.ny * m.d.nz, half = 4 * n8;
        const size_t f = static_cast<size_t>(w - first[si]) * 256u + threadIdx.x;
        if (f >= n8) continue;
        if (merge) {
            rb_layout_group<false, float>(f, batch_field(m, kind, BF_X), m.scratch, m.scratch + half, nullptr, nullptr, dissipate ? m.scale_s : 1.0f, m.d);
        } else {
            float* const dst = which == BF_B ? m.scratch2 : m.scratch;
            float* const dst2 = (which == BF_B && copy_iterate) ? m.scratch : nullptr;
            rb_layout_group<true, float>(f, batch_field(m, kind, which), dst, dst + half, dst2, dst2 != nullptr ? dst2 + half : nullptr, 1.0f, m.d);
        }
    }
}

template <int KIND>
__global__ void __launch_bounds__(32 * kVecRows) k_batch_rb_half(BatchTable t, int colour) {
    const uint32_t* first = t.first[SHAPE_HALF];
    for (uint32_t w = blockIdx.x; w < t.total[SHAPE_HALF]; w += gridDim.x) {
        const int si = batch_sim(first, t.nsims, w);
        const BatchSim& m = t.sims[si];
        const float coef = KIND == KIND_PRESSURE ? m.h * m.h : (KIND == KIND_SCALAR ? m.alpha_s : m.alpha_v);
        const uint32_t bxy = static_cast<uint32_t>((static_cast<size_t>(m.d.nx / 8) * m.d.ny + 127) / 128);
        const uint32_t local = w - first[si];
        const size_t half = static_cast<size_t>(m.d.nx) * m.d.ny * m.d.nz / 2;
        float* const xr = m.scratch;
        float* const xb = m.scratch + half;
        const float* const br = m.scratch2;
        const float* const bb = m.scratch2 + half;
        rb_half_block<KIND, float>(local % bxy, local / bxy, colour ? xb : xr, colour ? xr : xb, colour ? bb : br, coef, colour, m.z_chunk, m.d, m.ghost[KIND]);
    }
}

template <typename Kernel>
unsigned batch_grid_vec(uint32_t total, int sms, Kernel kernel) {
    static int per_sm = [&] {
        int n = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, 32 * kVecRows, 0) != cudaSuccess || n < 1) n = 4;
        return n;
    }();
    const uint32_t cap = static_cast<uint32_t>(sms) * static_cast<uint32_t>(per_sm);
    return total < cap ? (total == 0 ? 1u : total) : cap;
}

unsigned batch_grid_linear(uint32_t total, int sms) {
    const uint32_t cap = static_cast<uint32_t>(sms) * 8u;
    return total < cap ? (total == 0 ? 1u : total) : cap;
}

template <int KIND>
cudaError_t batch_sweep(const BatchTable& t, int scheme, int parity, int dst, int src, cudaStream_t s) {
    if (scheme == SCHEME_RBGS) k_batch_rbgs<KIND><<<batch_grid_vec(t.total[SHAPE_VEC], t.sms, k_batch_rbgs<KIND>), dim3(32, kVecRows), 0, s>>>(t, parity);
    else k_batch_jacobi<KIND><<<batch_grid_vec(t.total[SHAPE_VEC], t.sms, k_batch_jacobi<KIND>), dim3(32, kVecRows), 0, s>>>(t, dst, src);
    return cudaGetLastError();
}

}  // namespace

bool launch_pressure_interval_fused(const StencilArgs& a, DeviceStats* stats, cudaStream_t s) {
    if (a.kind != KIND_PRESSURE || a.scheme != SCHEME_JACOBI || a.init != INIT_FROM_X || a.bf16 || a.per_pass >= 2 || a.iterations < 1 || a.scratch == nullptr || !vec_ok(a)) return false;
    const Dims& d = a.dims;
    const size_t bytes = static_cast<size_t>(d.nx) * d.ny * d.nz * sizeof(float);
    const GhostRule g = ghost_rule(KIND_PRESSURE, a.flow, a.scalar);
    const VecShape vs = vec_shape(d, k_jacobi_vec4<KIND_PRESSURE>);
    const VecShape rs = vec_shape(d, k_jacobi_vec4_residual);
    const int units = a.iterations;
    const float* src = a.x;
    for (int u = 0; u < units; ++u) {
        float* dst = ((units - 1 - u) % 2 == 0) ? a.x : a.scratch;  // the last sweep lands in x
        if (src == dst) {  // odd sweep count: move the start aside (an error surfaces in the capture)
            cudaMemcpyAsync(a.scratch, a.x, bytes, cudaMemcpyDeviceToDevice, s);
            src = a.scratch;
        }
        // directions alternate, the last (residual) sweep upward, so each sweep
        // starts on the planes the one before wrote last (still in L2)
        if (u + 1 < units) launch_sweep((units - 1 - u) & 1 ? k_jacobi_vec4<KIND_PRESSURE, true> : k_jacobi_vec4<KIND_PRESSURE>, vs.grid, dim3(32, kVecRows), s, dst, src, a.b, a.coef, vs.z_chunk, d, g);
        else launch_sweep(k_jacobi_vec4_residual, rs.grid, dim3(32, kVecRows), s, dst, src, a.b, a.coef, rs.z_chunk, d, g, stats);
        src = dst;
    }
    if (a.launches) *a.launches += units;
    return true;  // launch errors stay pending for the caller's capture to report
}

bool launch_residual_sums_vec(const float* p, const float* div, Dims d, float h2, const FlowBC& b, DeviceStats* stats, cudaStream_t s) {
    const auto al = [](const void* q) { return (reinterpret_cast<uintptr_t>(q) & 15) == 0; };
    const size_t cells = static_cast<size_t>(d.nx) * d.ny * d.nz;
    if (d.nx % 4 != 0 || cells >= (1ull << 31) || !al(p) || !al(div)) return false;
    const VecShape vs = vec_shape(d, k_residual_vec);
    k_residual_vec<<<vs.grid, dim3(32, kVecRows), 0, s>>>(p, div, h2, vs.z_chunk, d, ghost_rule(KIND_PRESSURE, b, ScalarBC{}), stats);
    return true;
}

cudaError_t launch_stencil(const StencilArgs& a, cudaStream_t s) {
    // per_pass: 0 (default) = one launch per Jacobi sweep, red-black solves
    // in the colour-split layout where the rows allow (one launch per
    // colour); 1 = one launch per sweep or per colour on the interleaved
    // field; >= 2 = several sweeps per HBM pass: z-wavefront passes where the
    // rows suit them, else (red-black) the TMA pass. On B200 one launch per
    // sweep is the faster form: consecutive single sweeps in alternating z
    // directions stream their 12 B per cell at about the copy bandwidth,
    // while a 256-cell-row wavefront pass (16 warps per SM, one barrier per
    // plane) waits on its own instruction latencies.
    if (a.per_pass >= 2) {
        if (const int v = wave_width(a)) {
            switch (a.kind) {
            case KIND_VEL_X: return run_wave_kind<KIND_VEL_X>(a, v, s);
            case KIND_VEL_Y: return run_wave_kind<KIND_VEL_Y>(a, v, s);
            case KIND_VEL_Z: return run_wave_kind<KIND_VEL_Z>(a, v, s);
            case KIND_SCALAR: return run_wave_kind<KIND_SCALAR>(a, v, s);
            case KIND_PRESSURE: return run_wave_kind<KIND_PRESSURE>(a, v, s);
            default: return cudaErrorInvalidValue;
            }
        }
    }
    // the TMA red-black pass for other grids, when several iterations per pass are asked for
    if (a.blocked && a.per_pass >= 2 && !a.bf16 && tb_supported(a)) {
        switch (a.kind) {
        case KIND_VEL_X: return run_tb<KIND_VEL_X>(a, s, a.error_flag);
        case KIND_VEL_Y: return run_tb<KIND_VEL_Y>(a, s, a.error_flag);
        case KIND_VEL_Z: return run_tb<KIND_VEL_Z>(a, s, a.error_flag);
        case KIND_SCALAR: return run_tb<KIND_SCALAR>(a, s, a.error_flag);
        case KIND_PRESSURE: return run_tb<KIND_PRESSURE>(a, s, a.error_flag);
        default: return cudaErrorInvalidValue;
        }
    }
    if (a.bf16) {
        switch (a.kind) {
        case KIND_VEL_X: return run_simple<KIND_VEL_X, __nv_bfloat16>(a, s);
        case KIND_VEL_Y: return run_simple<KIND_VEL_Y, __nv_bfloat16>(a, s);
        case KIND_VEL_Z: return run_simple<KIND_VEL_Z, __nv_bfloat16>(a, s);
        case KIND_SCALAR: return run_simple<KIND_SCALAR, __nv_bfloat16>(a, s);
        default: return cudaErrorInvalidValue;  // the pressure is FP32
        }
    }
    switch (a.kind) {
    case KIND_VEL_X: return run_simple<KIND_VEL_X, float>(a, s);
    case KIND_VEL_Y: return run_simple<KIND_VEL_Y, float>(a, s);
    case KIND_VEL_Z: return run_simple<KIND_VEL_Z, float>(a, s);
    case KIND_SCALAR: return run_simple<KIND_SCALAR, float>(a, s);
    case KIND_PRESSURE: return run_simple<KIND_PRESSURE, float>(a, s);
    default: return cudaErrorInvalidValue;
    }
}

// ------------------------------------------------------ work-table batch --
GhostRule make_ghost_rule(int kind, const FlowBC& fb, const ScalarBC& sb) { return ghost_rule(kind, fb, sb); }

cudaError_t launch_batch_rb_split(const BatchTable& t, int kind, int which, int copy_iterate, cudaStream_t s) {
    k_batch_rb_layout<<<batch_grid_linear(t.total[SHAPE_OCT], t.sms), 256, 0, s>>>(t, kind, which, copy_iterate, 0, 0);
    return cudaGetLastError();
}

cudaError_t launch_batch_rb_merge(const BatchTable& t, int kind, int dissipate, cudaStream_t s) {
    k_batch_rb_layout<<<batch_grid_linear(t.total[SHAPE_OCT], t.sms), 256, 0, s>>>(t, kind, BF_X, 0, 1, dissipate);
    return cudaGetLastError();
}

template <int KIND>
cudaError_t batch_rb_half(const BatchTable& t, int colour, cudaStream_t s) {
    k_batch_rb_half<KIND><<<batch_grid_vec(t.total[SHAPE_HALF], t.sms, k_batch_rb_half<KIND>), dim3(32, kVecRows), 0, s>>>(t, colour);
    return cudaGetLastError();
}

cudaError_t launch_batch_rb_half(const BatchTable& t, int kind, int colour, cudaStream_t s) {
    switch (kind) {
    case KIND_VEL_X: return batch_rb_half<KIND_VEL_X>(t, colour, s);
    case KIND_VEL_Y: return batch_rb_half<KIND_VEL_Y>(t, colour, s);
    case KIND_VEL_Z: return batch_rb_half<KIND_VEL_Z>(t, colour, s);
    case KIND_SCALAR: return batch_rb_half<KIND_SCALAR>(t, colour, s);
    case KIND_PRESSURE: return batch_rb_half<KIND_PRESSURE>(t, colour, s);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_batch_sweep(const BatchTable& t, int kind, int scheme, int parity, int dst, int src, cudaStream_t s) {
    switch (kind) {
        case KIND_VEL_X: return batch_sweep<KIND_VEL_X>(t, scheme, parity, dst, src, s);
        case KIND_VEL_Y: return batch_sweep<KIND_VEL_Y>(t, scheme, parity, dst, src, s);
        case KIND_VEL_Z: return batch_sweep<KIND_VEL_Z>(t, scheme, parity, dst, src, s);
        case KIND_SCALAR: return batch_sweep<KIND_SCALAR>(t, scheme, parity, dst, src, s);
        case KIND_PRESSURE: return batch_sweep<KIND_PRESSURE>(t, scheme, parity, dst, src, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_batch_copy(const BatchTable& t, int kind, int dst, int src, cudaStream_t s) {
    k_batch_copy<<<batch_grid_linear(t.total[SHAPE_LINEAR], t.sms), 256, 0, s>>>(t, kind, dst, src);
    return cudaGetLastError();
}

cudaError_t launch_batch_scale_scalar(const BatchTable& t, cudaStream_t s) {
    k_batch_scale_scalar<<<batch_grid_linear(t.total[SHAPE_LINEAR], t.sms), 256, 0, s>>>(t);
    return cudaGetLastError();
}

cudaError_t launch_batch_residual_sums(const BatchTable& t, cudaStream_t s) {
    k_batch_residual<<<batch_grid_vec(t.total[SHAPE_VEC], t.sms, k_batch_residual), dim3(32, kVecRows), 0, s>>>(t);
    return cudaGetLastError();
}

}  // namespace sfb
