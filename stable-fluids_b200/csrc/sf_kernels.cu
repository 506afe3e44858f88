// sf_kernels.cu -- per-cell kernels of the step: force injection + velocity
// packing, fused RK2 advection, divergence, projection with the FP64
// residual, scalar source/advection, diagnostics.
//
// Layout in HBM: every field is a dense x-fastest array (the layout the ABI
// views expose); velocity additionally has a packed copy (x, y, z, 0) that
// the advection gathers read with one load per interpolation corner. The
// advected fields (velocity, scalar data) are FP32 or, with BF16 storage,
// BF16 (kernels are templates over the element type T and the packed type P;
// arithmetic is FP32 either way). Forces, sources, pressure, divergence and
// |u| are always FP32.

#include <cuda_runtime.h>

#include "sf_batch.cuh"
#include "sf_device.cuh"
#include "sf_launch.h"
#include "sf_stencil_tb.cuh"

namespace sfb {

namespace {

constexpr int kBX = 32, kBY = 4, kBZ = 2;

dim3 cell_block() { return dim3(kBX, kBY, kBZ); }
dim3 cell_grid(const Dims& d) {
    return dim3(static_cast<unsigned>((d.nx + kBX - 1) / kBX), static_cast<unsigned>((d.ny + kBY - 1) / kBY), static_cast<unsigned>((d.nz + kBZ - 1) / kBZ));
}
unsigned linear_grid(size_t n, int threads) {
    size_t g = (n + static_cast<size_t>(threads) - 1) / static_cast<size_t>(threads);
    const size_t cap = 148u * 32u;
    return static_cast<unsigned>(g < cap ? (g == 0 ? 1 : g) : cap);
}

// Cell of this thread in block `blk` of a (kBX, kBY, kBZ) launch over the grid
// (blockIdx for a single simulation, the work item's block in a batch).
__device__ __forceinline__ bool cell_coords(const Dims& d, uint3 blk, int& x, int& y, int& z) {
    x = static_cast<int>(blk.x * kBX + threadIdx.x);
    y = static_cast<int>(blk.y * kBY + threadIdx.y);
    z = static_cast<int>(blk.z * kBZ + threadIdx.z);
    return x < d.nx && y < d.ny && z < d.nz;
}

// ------------------------------------------------------------------ fill --
template <typename T>
__global__ void k_fill(T* __restrict__ f, float value, size_t n) {
    const T v = from_f<T>(value);
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n; i += static_cast<size_t>(gridDim.x) * blockDim.x) f[i] = v;
}

// Storage conversions for BF16 contexts (views, updates).
__global__ void k_bf16_to_f32(float* __restrict__ dst, const __nv_bfloat16* __restrict__ src, size_t n) {
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n; i += static_cast<size_t>(gridDim.x) * blockDim.x) dst[i] = __bfloat162float(src[i]);
}
__global__ void k_f32_to_bf16(__nv_bfloat16* __restrict__ dst, const float* __restrict__ src, size_t n) {
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n; i += static_cast<size_t>(gridDim.x) * blockDim.x) dst[i] = __float2bfloat16_rn(src[i]);
}

// ------------------------------------------------------- force + packing --
// v += dt * f for each force field in order (backend-cuda.cu:310-319 applied
// field after field), then writes the packed float4 copy.
template <typename T, typename P>
__global__ void k_force_pack(ForceArgs a) {
    T* vel[3] = {static_cast<T*>(a.vel[0]), static_cast<T*>(a.vel[1]), static_cast<T*>(a.vel[2])};
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < a.n; i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        float vx = to_f(vel[0][i]), vy = to_f(vel[1][i]), vz = to_f(vel[2][i]);
        for (int k = 0; k < a.force_count; ++k) {
            vx += a.dt * a.force[k][0][i];
            vy += a.dt * a.force[k][1][i];
            vz += a.dt * a.force[k][2][i];
        }
        if (a.write_soa) {
            vel[0][i] = from_f<T>(vx);
            vel[1][i] = from_f<T>(vy);
            vel[2][i] = from_f<T>(vz);
        }
        if (a.packed) static_cast<P*>(a.packed)[i] = pack4<P>(vx, vy, vz);
    }
}

// ------------------------------------------------------------- advection --
// One RK2 trace per cell for all three components (the reference re-traces
// per component, backend-cuda.cu:330-340; the trace is deterministic so the
// results are identical), then a trilinear sample of the packed velocity.
template <typename T, typename P>
__device__ __forceinline__ void advect_velocity_block(uint3 blk, const P* __restrict__ v, T* __restrict__ ox, T* __restrict__ oy, T* __restrict__ oz, float dt, const Dims& d, float h, const FlowBC& b) {
    int x, y, z;
    if (!cell_coords(d, blk, x, y, z)) return;
    const float px = __fmul_rn(static_cast<float>(x) + 0.5f, h);
    const float py = __fmul_rn(static_cast<float>(y) + 0.5f, h);
    const float pz = __fmul_rn(static_cast<float>(z) + 0.5f, h);
    const float3 t = trace_rk2(px, py, pz, x, y, z, v, dt, d, h, b);
    const float3 s = sample_velocity3(v, t.x, t.y, t.z, d, h, b);
    const size_t i = lin(x, y, z, d);
    ox[i] = from_f<T>(s.x);
    oy[i] = from_f<T>(s.y);
    oz[i] = from_f<T>(s.z);
}

template <typename T, typename P>
__global__ void __launch_bounds__(256, 5) k_advect_velocity(const P* __restrict__ v, T* __restrict__ ox, T* __restrict__ oy, T* __restrict__ oz, float dt, Dims d, float h, FlowBC b) { advect_velocity_block<T, P>(blockIdx, v, ox, oy, oz, dt, d, h, b); }

// Scalar value after the source injection rho + dt * S at an interior cell,
// or the fixed face value (the source never reaches a ghost).
template <typename T>
__device__ __forceinline__ float sourced_scalar(const T* __restrict__ q, const float* __restrict__ src, float dt, int x, int y, int z, const Dims& d, const ScalarBC& b) {
    if (!inside(x, y, z, d)) {
        float value;
        if (!scalar_resolve(x, y, z, d, b, value)) return value;
    }
    const size_t i = lin(x, y, z, d);
    return __fmaf_rn(dt, __ldg(&src[i]), ldg_f(&q[i]));  // rho + dt S, one rounding (backend-cuda.cu:326)
}

// Source injection fused into the advection gather (backend-cuda.cu:321-328
// followed by :342-352): each gathered corner is rho + dt * S, exactly the
// value the reference stores before it advects.
template <typename T, typename P>
__device__ __forceinline__ void scalar_source_advect_block(uint3 blk, const P* __restrict__ v, const T* __restrict__ q, const float* __restrict__ src, T* __restrict__ out, float dt, const Dims& d, float h, const FlowBC& fb, const ScalarBC& sb) {
    int x, y, z;
    if (!cell_coords(d, blk, x, y, z)) return;
    const float px = __fmul_rn(static_cast<float>(x) + 0.5f, h);
    const float py = __fmul_rn(static_cast<float>(y) + 0.5f, h);
    const float pz = __fmul_rn(static_cast<float>(z) + 0.5f, h);
    float3 t = trace_rk2(px, py, pz, x, y, z, v, dt, d, h, fb);
    if (sb.periodic[0]) t.x = wrap_world(t.x, static_cast<float>(d.nx) * h);
    if (sb.periodic[1]) t.y = wrap_world(t.y, static_cast<float>(d.ny) * h);
    if (sb.periodic[2]) t.z = wrap_world(t.z, static_cast<float>(d.nz) * h);
    const Cell c = locate(t.x, t.y, t.z, h);
    float s[8];
    if (block_inside(c, d)) {
        // the whole 2x2x2 block is inside: no ghost rule applies
        const size_t i = lin(c.x0, c.y0, c.z0, d);
        const size_t sy = static_cast<size_t>(d.nx), sz = static_cast<size_t>(d.nx) * static_cast<size_t>(d.ny);
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const size_t j = i + static_cast<size_t>(k & 1) + ((k >> 1) & 1 ? sy : 0) + (k >> 2 ? sz : 0);
            s[k] = __fmaf_rn(dt, __ldg(&src[j]), ldg_f(&q[j]));
        }
    } else {
        const int bx = corner_base(c.x0, d.nx), by = corner_base(c.y0, d.ny), bz = corner_base(c.z0, d.nz);
#pragma unroll
        for (int k = 0; k < 8; ++k) s[k] = sourced_scalar(q, src, dt, bx + (k & 1), by + ((k >> 1) & 1), bz + (k >> 2), d, sb);
    }
    out[lin(x, y, z, d)] = from_f<T>(trilerp(s[0], s[1], s[2], s[3], s[4], s[5], s[6], s[7], c));
}

template <typename T, typename P>
__global__ void __launch_bounds__(256) k_scalar_source_advect(const P* __restrict__ v, const T* __restrict__ q, const float* __restrict__ src, T* __restrict__ out, float dt, Dims d, float h, FlowBC fb, ScalarBC sb) { scalar_source_advect_block<T, P>(blockIdx, v, q, src, out, dt, d, h, fb, sb); }

template <typename T>
__global__ void k_scalar_source(T* __restrict__ q, const float* __restrict__ src, float dt, size_t n) {
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n; i += static_cast<size_t>(gridDim.x) * blockDim.x) q[i] = from_f<T>(__fmaf_rn(dt, src[i], to_f(q[i])));
}

// backend-cuda.cu:377-384
template <typename T>
__global__ void k_scale(T* __restrict__ q, float factor, size_t n) {
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n; i += static_cast<size_t>(gridDim.x) * blockDim.x) q[i] = from_f<T>(to_f(q[i]) * factor);
}

// ------------------------------------------------------------ divergence --
template <typename T>
__device__ __forceinline__ float divergence_at(const T* __restrict__ vx, const T* __restrict__ vy, const T* __restrict__ vz, int x, int y, int z, const Dims& d, float h, const FlowBC& b) {
    const float inv_2h = 0.5f / h;
    const float ddx = (load_velocity(vx, 0, x + 1, y, z, d, b) - load_velocity(vx, 0, x - 1, y, z, d, b)) * inv_2h;
    const float ddy = (load_velocity(vy, 1, x, y + 1, z, d, b) - load_velocity(vy, 1, x, y - 1, z, d, b)) * inv_2h;
    const float ddz = (load_velocity(vz, 2, x, y, z + 1, d, b) - load_velocity(vz, 2, x, y, z - 1, d, b)) * inv_2h;
    return ddx + ddy + ddz;
}

// backend-cuda.cu:386-396
template <typename T>
__device__ __forceinline__ void divergence_block(uint3 blk, float* __restrict__ div, const T* __restrict__ vx, const T* __restrict__ vy, const T* __restrict__ vz, const Dims& d, float h, const FlowBC& b) {
    int x, y, z;
    if (!cell_coords(d, blk, x, y, z)) return;
    div[lin(x, y, z, d)] = divergence_at(vx, vy, vz, x, y, z, d, h, b);
}

template <typename T>
__global__ void __launch_bounds__(256) k_divergence(float* __restrict__ div, const T* __restrict__ vx, const T* __restrict__ vy, const T* __restrict__ vz, Dims d, float h, FlowBC b) { divergence_block<T>(blockIdx, div, vx, vy, vz, d, h, b); }

// --------------------------------------------------- residual reductions --
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide sum of four doubles, then one atomicAdd per value per block.
__device__ __forceinline__ void block_accumulate4(double a, double b, double c, double e, DeviceStats* stats) {
    __shared__ double part[4][32];
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int nthreads = blockDim.x * blockDim.y * blockDim.z;
    const int lane = tid & 31, warp = tid >> 5;
    a = warp_sum(a);
    b = warp_sum(b);
    c = warp_sum(c);
    e = warp_sum(e);
    if (lane == 0) {
        part[0][warp] = a;
        part[1][warp] = b;
        part[2][warp] = c;
        part[3][warp] = e;
    }
    __syncthreads();
    if (warp == 0) {
        const int nw = (nthreads + 31) >> 5;
        a = lane < nw ? part[0][lane] : 0.0;
        b = lane < nw ? part[1][lane] : 0.0;
        c = lane < nw ? part[2][lane] : 0.0;
        e = lane < nw ? part[3][lane] : 0.0;
        a = warp_sum(a);
        b = warp_sum(b);
        c = warp_sum(c);
        e = warp_sum(e);
        if (lane == 0) {
            atomicAdd(&stats->sum_e, a);
            atomicAdd(&stats->sum_e2, b);
            atomicAdd(&stats->sum_b, c);
            atomicAdd(&stats->sum_b2, e);
        }
    }
}

// ------------------------------------------------------------ projection --
// u -= central gradient of p (backend-cuda.cu:409-422, in place), repacks the
// float4 velocity for the scalar advection, and (stats != nullptr) adds the
// FP64 residual terms of A p = b: e = h^2 div - (sum6(p) - 6 p).
template <typename T, typename P>
__device__ __forceinline__ void project_block(uint3 blk, T* __restrict__ vx, T* __restrict__ vy, T* __restrict__ vz, P* __restrict__ packed, const float* __restrict__ p, const float* __restrict__ div, const Dims& d, float h, float h2, const FlowBC& b, DeviceStats* stats) {
    int x, y, z;
    const bool ok = cell_coords(d, blk, x, y, z);
    double se = 0.0, se2 = 0.0, sb = 0.0, sb2 = 0.0;
    if (ok) {
        const float inv_2h = 0.5f / h;
        const size_t i = lin(x, y, z, d);
        const float pxp = load_pressure(p, x + 1, y, z, d, b), pxm = load_pressure(p, x - 1, y, z, d, b);
        const float pyp = load_pressure(p, x, y + 1, z, d, b), pym = load_pressure(p, x, y - 1, z, d, b);
        const float pzp = load_pressure(p, x, y, z + 1, d, b), pzm = load_pressure(p, x, y, z - 1, d, b);
        const float grad_x = (pxp - pxm) * inv_2h;
        const float grad_y = (pyp - pym) * inv_2h;
        const float grad_z = (pzp - pzm) * inv_2h;
        const float ux = to_f(vx[i]) - grad_x;
        const float uy = to_f(vy[i]) - grad_y;
        const float uz = to_f(vz[i]) - grad_z;
        vx[i] = from_f<T>(ux);
        vy[i] = from_f<T>(uy);
        vz[i] = from_f<T>(uz);
        if (packed) packed[i] = pack4<P>(ux, uy, uz);
        if (stats) {
            const double nb = static_cast<double>(pxm) + static_cast<double>(pxp) + static_cast<double>(pym) + static_cast<double>(pyp) + static_cast<double>(pzm) + static_cast<double>(pzp);
            const double bb = static_cast<double>(h2) * static_cast<double>(div[i]);
            const double e = bb - (nb - 6.0 * static_cast<double>(p[i]));
            se = e;
            se2 = e * e;
            sb = bb;
            sb2 = bb * bb;
        }
    }
    if (stats) block_accumulate4(se, se2, sb, sb2, stats);
}

template <typename T, typename P>
__global__ void __launch_bounds__(256) k_project(T* __restrict__ vx, T* __restrict__ vy, T* __restrict__ vz, P* __restrict__ packed, const float* __restrict__ p, const float* __restrict__ div, Dims d, float h, float h2, FlowBC b, DeviceStats* stats) { project_block<T, P>(blockIdx, vx, vy, vz, packed, p, div, d, h, h2, b, stats); }

__device__ __forceinline__ void residual_sums_block(uint3 blk, const float* __restrict__ p, const float* __restrict__ div, const Dims& d, float h2, const FlowBC& b, DeviceStats* stats) {
    int x, y, z;
    const bool ok = cell_coords(d, blk, x, y, z);
    double se = 0.0, se2 = 0.0, sb = 0.0, sb2 = 0.0;
    if (ok) {
        const size_t i = lin(x, y, z, d);
        const double nb = static_cast<double>(load_pressure(p, x - 1, y, z, d, b)) + static_cast<double>(load_pressure(p, x + 1, y, z, d, b)) + static_cast<double>(load_pressure(p, x, y - 1, z, d, b)) + static_cast<double>(load_pressure(p, x, y + 1, z, d, b))
                        + static_cast<double>(load_pressure(p, x, y, z - 1, d, b)) + static_cast<double>(load_pressure(p, x, y, z + 1, d, b));
        const double bb = static_cast<double>(h2) * static_cast<double>(div[i]);
        const double e = bb - (nb - 6.0 * static_cast<double>(p[i]));
        se = e;
        se2 = e * e;
        sb = bb;
        sb2 = bb * bb;
    }
    block_accumulate4(se, se2, sb, sb2, stats);
}

__global__ void __launch_bounds__(256) k_residual_sums(const float* __restrict__ p, const float* __restrict__ div, Dims d, float h2, FlowBC b, DeviceStats* stats) { residual_sums_block(blockIdx, p, div, d, h2, b, stats); }

// rel_res = ||b - A p|| / ||b||, with b's mean removed when the pressure
// operator is singular (no OUTFLOW face: constants are in its null space).
__device__ double relative_residual(const DeviceStats* s, double n, int singular, double* rhs_norm) {
    double r2 = s->sum_e2, b2 = s->sum_b2;
    if (singular) {
        const double mb = s->sum_b / n;
        r2 = s->sum_e2 - 2.0 * mb * s->sum_e + n * mb * mb;
        b2 = s->sum_b2 - n * mb * mb;
    }
    r2 = r2 < 0.0 ? 0.0 : r2;
    b2 = b2 < 0.0 ? 0.0 : b2;
    if (rhs_norm) *rhs_norm = sqrt(b2);
    return b2 > 0.0 ? sqrt(r2) / sqrt(b2) : 0.0;
}

__global__ void k_residual_finalize(DeviceStats* s, double n, int singular, int iterations) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double rhs = 0.0;
    s->rel_residual = relative_residual(s, n, singular, &rhs);
    s->rhs_norm = rhs;
    if (iterations >= 0) s->iterations = iterations;
}

// Residual-driven pressure solve: turns the accumulated sums into rel_res,
// counts the iterations run (reset: the count becomes `increment`), zeroes
// the sums for the next measurement, and continues the enclosing WHILE graph
// node while rel_res > tol and fewer than max_iterations have run.
__global__ void k_residual_check(DeviceStats* s, double n, int singular, int reset, int increment, double tol, int max_iterations, cudaGraphConditionalHandle handle) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double rhs = 0.0;
    const double rel = relative_residual(s, n, singular, &rhs);
    s->rhs_norm = rhs;
    s->rel_residual = rel;
    s->iterations = reset ? increment : s->iterations + increment;
    s->sum_e = s->sum_e2 = s->sum_b = s->sum_b2 = 0.0;
    const bool more = rel > tol && s->iterations < max_iterations;
    s->hit_cap = (rel > tol && !more) ? 1 : 0;
    s->keep_going = more ? 1 : 0;
    cudaGraphSetConditional(handle, more ? 1u : 0u);
}

// Learned warm start, after the trial sweeps on both candidates: the learned
// candidate (in p, sums in `learned`) is replaced by the plain one (in alt,
// sums in `plain`) when its relative residual is larger.
__global__ void k_warm_start_select(const DeviceStats* learned, const DeviceStats* plain, double n, int singular, float* __restrict__ p, const float* __restrict__ alt, size_t cells) {
    if (!(relative_residual(learned, n, singular, nullptr) > relative_residual(plain, n, singular, nullptr))) return;
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < cells; i += static_cast<size_t>(gridDim.x) * blockDim.x) p[i] = alt[i];
}

// Records the decision of k_warm_start_select and, on a fallback, adopts the
// plain candidate's residual sums (so that a residual-driven loop continues
// from the right value).
__global__ void k_warm_start_commit(DeviceStats* learned, const DeviceStats* plain, double n, int singular) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const bool fallback = relative_residual(learned, n, singular, nullptr) > relative_residual(plain, n, singular, nullptr);
    learned->used_fallback = fallback ? 1 : 0;
    if (fallback) {
        learned->sum_e = plain->sum_e;
        learned->sum_e2 = plain->sum_e2;
        learned->sum_b = plain->sum_b;
        learned->sum_b2 = plain->sum_b2;
    }
}

// ----------------------------------------------------------- diagnostics --
// Post-projection divergence (backend-cuda.cu:670) and |u| (:424-434) in one pass.
template <typename T>
__device__ __forceinline__ void post_diagnostics_block(uint3 blk, float* __restrict__ div, float* __restrict__ mag, const T* __restrict__ vx, const T* __restrict__ vy, const T* __restrict__ vz, const Dims& d, float h, const FlowBC& b) {
    int x, y, z;
    if (!cell_coords(d, blk, x, y, z)) return;
    const size_t i = lin(x, y, z, d);
    div[i] = divergence_at(vx, vy, vz, x, y, z, d, h, b);
    const float ux = to_f(vx[i]), uy = to_f(vy[i]), uz = to_f(vz[i]);
    mag[i] = sqrtf(ux * ux + uy * uy + uz * uz);
}

template <typename T>
__global__ void __launch_bounds__(256) k_post_diagnostics(float* __restrict__ div, float* __restrict__ mag, const T* __restrict__ vx, const T* __restrict__ vy, const T* __restrict__ vz, Dims d, float h, FlowBC b) { post_diagnostics_block<T>(blockIdx, div, mag, vx, vy, vz, d, h, b); }

// ------------------------------------- divergence / |u| on the z-march --
// The same values as divergence_block / post_diagnostics_block for FP32
// fields with nx % 4 == 0: a thread owns one float4 of a row and marches a z
// chunk, keeping the z component's planes below / at / above in registers;
// face ghosts come from the velocity components' GhostRules (copy for
// outflow and tangential free slip, reflection about the wall velocity
// otherwise -- load_velocity's rule for a face neighbour), periodic axes are
// read wrapped. The rounding is written out: central differences, then
// (dz * c) + ((dx * c) + (dy * c)) with the last two sums fused, and
// |u| = sqrt(w w + (u u + v v)) with the same fusing -- the contraction the
// reference's expressions take (backend-cuda.cu:391-395, 429-433).
constexpr int kDivRows = 4;

struct VelocityGhosts {
    GhostRule g[3];  // components x, y, z
};

__device__ __forceinline__ float4 ld4f(const float* p) { return *reinterpret_cast<const float4*>(p); }
__device__ __forceinline__ float4 ghost4f(const GhostRule& g, int face, float4 s) {
    return make_float4(tb::ghost(g, face, s.x), tb::ghost(g, face, s.y), tb::ghost(g, face, s.z), tb::ghost(g, face, s.w));
}
__device__ __forceinline__ float div_sum(float dx, float dy, float dz, float c) { return __fmaf_rn(dz, c, __fmaf_rn(dx, c, __fmul_rn(dy, c))); }
__device__ __forceinline__ float magnitude(float u, float v, float w) { return __fsqrt_rn(__fmaf_rn(w, w, __fmaf_rn(u, u, __fmul_rn(v, v)))); }

// Block `blk` of the launch (blockIdx for one simulation, the work item's
// block in a batch).
template <bool MAG>
__device__ __forceinline__ void divergence_vec4_block(uint3 blk, float* __restrict__ div, float* __restrict__ mag, const float* __restrict__ vx, const float* __restrict__ vy, const float* __restrict__ vz, int z_chunk, const Dims& d, float inv_2h, const GhostRule& gx, const GhostRule& gy, const GhostRule& gz) {
    const int x0 = 4 * static_cast<int>(blk.x * 32 + threadIdx.x), y = static_cast<int>(blk.y * kDivRows + threadIdx.y);
    if (x0 >= d.nx || y >= d.ny) return;
    const int zb = static_cast<int>(blk.z) * z_chunk, ze = min(zb + z_chunk, d.nz);
    const int sy = d.nx, sz = d.nx * d.ny;
    const bool px = gx.periodic[0] != 0, py = gy.periodic[1] != 0, pz = gz.periodic[2] != 0;
    int i = x0 + sy * (y + d.ny * zb);
    float4 zc = ld4f(vz + i);
    float4 zlo = zb > 0 ? ld4f(vz + i - sz) : (pz ? ld4f(vz + i + (d.nz - 1) * sz) : ghost4f(gz, ZM, zc));
    for (int z = zb; z < ze; ++z, i += sz) {
        const float4 zhi = z + 1 < d.nz ? ld4f(vz + i + sz) : (pz ? ld4f(vz + i - (d.nz - 1) * sz) : ghost4f(gz, ZP, zc));
        const float4 xc = ld4f(vx + i);
        const float xl = x0 > 0 ? vx[i - 1] : (px ? vx[i + d.nx - 1] : tb::ghost(gx, XM, xc.x));
        const float xr = x0 + 4 < d.nx ? vx[i + 4] : (px ? vx[i + 4 - d.nx] : tb::ghost(gx, XP, xc.w));
        const float4 yc = ld4f(vy + i);
        const float4 ylo = y > 0 ? ld4f(vy + i - sy) : (py ? ld4f(vy + i + (d.ny - 1) * sy) : ghost4f(gy, YM, yc));
        const float4 yhi = y + 1 < d.ny ? ld4f(vy + i + sy) : (py ? ld4f(vy + i - (d.ny - 1) * sy) : ghost4f(gy, YP, yc));
        float4 o;
        o.x = div_sum(xc.y - xl, yhi.x - ylo.x, zhi.x - zlo.x, inv_2h);
        o.y = div_sum(xc.z - xc.x, yhi.y - ylo.y, zhi.y - zlo.y, inv_2h);
        o.z = div_sum(xc.w - xc.y, yhi.z - ylo.z, zhi.z - zlo.z, inv_2h);
        o.w = div_sum(xr - xc.z, yhi.w - ylo.w, zhi.w - zlo.w, inv_2h);
        *reinterpret_cast<float4*>(div + i) = o;
        if constexpr (MAG) *reinterpret_cast<float4*>(mag + i) = make_float4(magnitude(xc.x, yc.x, zc.x), magnitude(xc.y, yc.y, zc.y), magnitude(xc.z, yc.z, zc.z), magnitude(xc.w, yc.w, zc.w));
        zlo = zc;
        zc = zhi;
    }
}

template <bool MAG>
__global__ void __launch_bounds__(32 * kDivRows) k_divergence_vec4(float* __restrict__ div, float* __restrict__ mag, const float* __restrict__ vx, const float* __restrict__ vy, const float* __restrict__ vz, int z_chunk, Dims d, float inv_2h, VelocityGhosts gh) {
    divergence_vec4_block<MAG>(blockIdx, div, mag, vx, vy, vz, z_chunk, d, inv_2h, gh.g[0], gh.g[1], gh.g[2]);
}

// ------------------------------------------------------- work-table batch --
// One launch per stage over every simulation of a batch (sf_batch.h); each
// work item runs the single-simulation block body above.

// v += dt f for the simulation's force fields in order, then the packed copy
// (the batch always advects, so the SoA velocity is not written here).
__global__ void __launch_bounds__(256) k_batch_force_pack(BatchTable t) {
    const uint32_t* first = t.first[SHAPE_LINEAR];
    for (uint32_t w = blockIdx.x; w < t.total[SHAPE_LINEAR]; w += gridDim.x) {
        const int si = batch_sim(first, t.nsims, w);
        const BatchSim& m = t.sims[si];
        const size_t n = static_cast<size_t>(m.d.nx) * m.d.ny * m.d.nz;
        const size_t i = static_cast<size_t>(w - first[si]) * 256u + threadIdx.x;
        if (i >= n) continue;
        float vx = m.vel[0][i], vy = m.vel[1][i], vz = m.vel[2][i];
        for (int k = 0; k < m.force_count; ++k) {
            vx += m.dt * m.force[k][0][i];
            vy += m.dt * m.force[k][1][i];
            vz += m.dt * m.force[k][2][i];
        }
        reinterpret_cast<float4*>(m.packed)[i] = pack4<float4>(vx, vy, vz);
    }
}

__device__ __forceinline__ uint3 cell_block_of(uint32_t local, const Dims& d) {
    return batch_block(local, static_cast<uint32_t>((d.nx + kBX - 1) / kBX), static_cast<uint32_t>((d.ny + kBY - 1) / kBY));
}

__global__ void __launch_bounds__(256) k_batch_advect_velocity(BatchTable t) {
    const uint32_t* first = t.first[SHAPE_CELL];
    for (uint32_t w = blockIdx.x; w < t.total[SHAPE_CELL]; w += gridDim.x) {
        const int si = batch_sim(first, t.nsims, w);
        const BatchSim& m = t.sims[si];
        advect_velocity_block<float, float4>(cell_block_of(w - first[si], m.d), reinterpret_cast<const float4*>(m.packed), m.temp[0], m.temp[1], m.temp[2], m.dt, m.d, m.h, m.flow);
    }
}

__global__ void __launch_bounds__(256) k_batch_scalar_source_advect(BatchTable t) {
    const uint32_t* first = t.first[SHAPE_CELL];
    for (uint32_t w = blockIdx.x; w < t.total[SHAPE_CELL]; w += gridDim.x) {
        const int si = batch_sim(first, t.nsims, w);
        const BatchSim& m = t.sims[si];
        scalar_source_advect_block<float, float4>(cell_block_of(w - first[si], m.d), reinterpret_cast<const float4*>(m.packed), m.sdata, m.source, m.stemp, m.dt, m.d, m.h, m.flow, m.sbc);
    }
}

// Divergence (MAG: and |u|) of every simulation with the z-marching body
// (the work table's fields are 256-byte aligned with nx % 4 == 0); each
// simulation's blocks use its sweep z chunk.
template <bool MAG>
__global__ void __launch_bounds__(32 * kDivRows) k_batch_divergence(BatchTable t) {
    const uint32_t* first = t.first[SHAPE_VEC];
    for (uint32_t w = blockIdx.x; w < t.total[SHAPE_VEC]; w += gridDim.x) {
        const int si = batch_sim(first, t.nsims, w);
        const BatchSim& m = t.sims[si];
        const uint3 blk = batch_block(w - first[si], static_cast<uint32_t>((m.d.nx / 4 + 31) / 32), static_cast<uint32_t>((m.d.ny + kDivRows - 1) / kDivRows));
        divergence_vec4_block<MAG>(blk, m.divergence, m.magnitude, m.vel[0], m.vel[1], m.vel[2], m.z_chunk, m.d, 0.5f / m.h, m.ghost[KIND_VEL_X], m.ghost[KIND_VEL_Y], m.ghost[KIND_VEL_Z]);
    }
}

__global__ void __launch_bounds__(256) k_batch_project(BatchTable t, int pack) {
    const uint32_t* first = t.first[SHAPE_CELL];
    for (uint32_t w = blockIdx.x; w < t.total[SHAPE_CELL]; w += gridDim.x) {
        const int si = batch_sim(first, t.nsims, w);
        const BatchSim& m = t.sims[si];
        project_block<float, float4>(cell_block_of(w - first[si], m.d), m.vel[0], m.vel[1], m.vel[2], pack ? reinterpret_cast<float4*>(m.packed) : nullptr, m.pressure, m.divergence, m.d, m.h, m.h * m.h, m.flow, nullptr);
    }
}

// Per simulation: zero the residual sums (before the batched residual sums)
// or turn them into rel_res (after), one thread per simulation.
__global__ void k_batch_stats(BatchTable t, int finalize, int iterations) {
    const int si = static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x);
    if (si >= t.nsims) return;
    const BatchSim& m = t.sims[si];
    DeviceStats* st = m.stats;
    if (!finalize) {
        st->sum_e = st->sum_e2 = st->sum_b = st->sum_b2 = 0.0;
        return;
    }
    double rhs = 0.0;
    const double n = static_cast<double>(m.d.nx) * m.d.ny * m.d.nz;
    st->rel_residual = relative_residual(st, n, m.flow.any_outflow ? 0 : 1, &rhs);
    st->rhs_norm = rhs;
    st->iterations = iterations;
}

// ----------------------------------------- coarse learned warm start --
// Mean of each 2x2x2 block (fine dims even).
__global__ void __launch_bounds__(256) k_restrict2(const float* __restrict__ fine, float* __restrict__ coarse, Dims f) {
    const Dims c{f.nx / 2, f.ny / 2, f.nz / 2, 0};
    int x, y, z;
    if (!cell_coords(c, blockIdx, x, y, z)) return;
    const size_t sy = static_cast<size_t>(f.nx), sz = static_cast<size_t>(f.nx) * f.ny;
    const size_t i = lin(2 * x, 2 * y, 2 * z, f);
    const float s = ((fine[i] + fine[i + 1]) + (fine[i + sy] + fine[i + sy + 1])) + ((fine[i + sz] + fine[i + sz + 1]) + (fine[i + sz + sy] + fine[i + sz + sy + 1]));
    coarse[lin(x, y, z, c)] = 0.125f * s;
}

// Cell-centred trilinear prolongation of the coarse correction: fine cell 2X
// sits at coarse coordinate X - 1/4 and 2X + 1 at X + 1/4 (weights 3/4, 1/4;
// clamped at the faces).
__global__ void __launch_bounds__(256) k_prolong_add(const float* __restrict__ cnew, const float* __restrict__ cold, float* __restrict__ p, Dims f) {
    const Dims c{f.nx / 2, f.ny / 2, f.nz / 2, 0};
    int x, y, z;
    if (!cell_coords(f, blockIdx, x, y, z)) return;
    const int X = x >> 1, Y = y >> 1, Z = z >> 1;
    const int X2 = (x & 1) ? min(X + 1, c.nx - 1) : max(X - 1, 0);
    const int Y2 = (y & 1) ? min(Y + 1, c.ny - 1) : max(Y - 1, 0);
    const int Z2 = (z & 1) ? min(Z + 1, c.nz - 1) : max(Z - 1, 0);
    const auto corr = [&](int a, int b, int d) {
        const size_t k = lin(a, b, d, c);
        return cnew[k] - cold[k];
    };
    const float c00 = 0.75f * corr(X, Y, Z) + 0.25f * corr(X2, Y, Z);
    const float c10 = 0.75f * corr(X, Y2, Z) + 0.25f * corr(X2, Y2, Z);
    const float c01 = 0.75f * corr(X, Y, Z2) + 0.25f * corr(X2, Y, Z2);
    const float c11 = 0.75f * corr(X, Y2, Z2) + 0.25f * corr(X2, Y2, Z2);
    const float v = 0.75f * (0.75f * c00 + 0.25f * c10) + 0.25f * (0.75f * c01 + 0.25f * c11);
    p[lin(x, y, z, f)] += v;
}

}  // namespace

// ------------------------------------------------------------- launchers --
// Storage dispatch: bf16 selects the BF16 element type (and the 8-byte packed velocity).
#define SFB_STORAGE(bf16, CALL_F32, CALL_BF16) \
    do {                                       \
        if (bf16) {                            \
            CALL_BF16;                         \
        } else {                               \
            CALL_F32;                          \
        }                                      \
    } while (0)

using bf16_t = __nv_bfloat16;

cudaError_t launch_fill(void* f, float value, size_t n, int bf16, cudaStream_t s) {
    SFB_STORAGE(bf16, (k_fill<float><<<linear_grid(n, 256), 256, 0, s>>>(static_cast<float*>(f), value, n)), (k_fill<bf16_t><<<linear_grid(n, 256), 256, 0, s>>>(static_cast<bf16_t*>(f), value, n)));
    return cudaGetLastError();
}

cudaError_t launch_convert(void* dst, const void* src, size_t n, int to_bf16, cudaStream_t s) {
    if (to_bf16) k_f32_to_bf16<<<linear_grid(n, 256), 256, 0, s>>>(static_cast<bf16_t*>(dst), static_cast<const float*>(src), n);
    else k_bf16_to_f32<<<linear_grid(n, 256), 256, 0, s>>>(static_cast<float*>(dst), static_cast<const bf16_t*>(src), n);
    return cudaGetLastError();
}

cudaError_t launch_force_pack(const ForceArgs& a, cudaStream_t s) {
    SFB_STORAGE(a.bf16, (k_force_pack<float, float4><<<linear_grid(a.n, 256), 256, 0, s>>>(a)), (k_force_pack<bf16_t, Bf16x4><<<linear_grid(a.n, 256), 256, 0, s>>>(a)));
    return cudaGetLastError();
}

cudaError_t launch_advect_velocity(const void* packed, void* ox, void* oy, void* oz, float dt, Dims d, float h, const FlowBC& b, int bf16, cudaStream_t s) {
    SFB_STORAGE(bf16, (k_advect_velocity<float, float4><<<cell_grid(d), cell_block(), 0, s>>>(static_cast<const float4*>(packed), static_cast<float*>(ox), static_cast<float*>(oy), static_cast<float*>(oz), dt, d, h, b)),
                (k_advect_velocity<bf16_t, Bf16x4><<<cell_grid(d), cell_block(), 0, s>>>(static_cast<const Bf16x4*>(packed), static_cast<bf16_t*>(ox), static_cast<bf16_t*>(oy), static_cast<bf16_t*>(oz), dt, d, h, b)));
    return cudaGetLastError();
}

cudaError_t launch_scalar_source_advect(const void* packed, const void* data, const float* source, void* out, float dt, Dims d, float h, const FlowBC& fb, const ScalarBC& sb, int bf16, cudaStream_t s) {
    SFB_STORAGE(bf16, (k_scalar_source_advect<float, float4><<<cell_grid(d), cell_block(), 0, s>>>(static_cast<const float4*>(packed), static_cast<const float*>(data), source, static_cast<float*>(out), dt, d, h, fb, sb)),
                (k_scalar_source_advect<bf16_t, Bf16x4><<<cell_grid(d), cell_block(), 0, s>>>(static_cast<const Bf16x4*>(packed), static_cast<const bf16_t*>(data), source, static_cast<bf16_t*>(out), dt, d, h, fb, sb)));
    return cudaGetLastError();
}

cudaError_t launch_scalar_source(void* data, const float* source, float dt, size_t n, int bf16, cudaStream_t s) {
    SFB_STORAGE(bf16, (k_scalar_source<float><<<linear_grid(n, 256), 256, 0, s>>>(static_cast<float*>(data), source, dt, n)), (k_scalar_source<bf16_t><<<linear_grid(n, 256), 256, 0, s>>>(static_cast<bf16_t*>(data), source, dt, n)));
    return cudaGetLastError();
}

cudaError_t launch_scale(void* data, float factor, size_t n, int bf16, cudaStream_t s) {
    SFB_STORAGE(bf16, (k_scale<float><<<linear_grid(n, 256), 256, 0, s>>>(static_cast<float*>(data), factor, n)), (k_scale<bf16_t><<<linear_grid(n, 256), 256, 0, s>>>(static_cast<bf16_t*>(data), factor, n)));
    return cudaGetLastError();
}

GhostRule make_ghost_rule(int kind, const FlowBC& fb, const ScalarBC& sb);

// The z-marching divergence for FP32 fields whose rows are whole float4s:
// false (nothing launched) when the grid or the pointers do not suit it.
bool launch_divergence_vec4(float* div, float* mag, const void* vx, const void* vy, const void* vz, Dims d, float h, const FlowBC& b, cudaStream_t s) {
    const auto al = [](const void* q) { return (reinterpret_cast<uintptr_t>(q) & 15) == 0; };
    const size_t cells = static_cast<size_t>(d.nx) * d.ny * d.nz;
    if (d.nx % 4 != 0 || cells >= (1ull << 31) || !al(div) || !al(vx) || !al(vy) || !al(vz) || (mag != nullptr && !al(mag))) return false;
    VelocityGhosts gh{};
    for (int c = 0; c < 3; ++c) gh.g[c] = make_ghost_rule(KIND_VEL_X + c, b, ScalarBC{});
    static int per_sm = [] {
        int n = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_divergence_vec4<true>, 32 * kDivRows, 0) != cudaSuccess || n < 1) n = 8;
        return n;
    }();
    int sms = 148, dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int bx = (d.nx / 4 + 31) / 32, by = (d.ny + kDivRows - 1) / kDivRows;
    long long chunks = static_cast<long long>(sms) * per_sm / (static_cast<long long>(bx) * by);  // one wave
    if (chunks < 1) chunks = 1;
    int z_chunk = static_cast<int>((d.nz + chunks - 1) / chunks);
    if (z_chunk < 4) z_chunk = d.nz < 4 ? d.nz : 4;
    const dim3 grid(static_cast<unsigned>(bx), static_cast<unsigned>(by), static_cast<unsigned>((d.nz + z_chunk - 1) / z_chunk));
    const float inv_2h = 0.5f / h;
    if (mag) k_divergence_vec4<true><<<grid, dim3(32, kDivRows), 0, s>>>(div, mag, static_cast<const float*>(vx), static_cast<const float*>(vy), static_cast<const float*>(vz), z_chunk, d, inv_2h, gh);
    else k_divergence_vec4<false><<<grid, dim3(32, kDivRows), 0, s>>>(div, nullptr, static_cast<const float*>(vx), static_cast<const float*>(vy), static_cast<const float*>(vz), z_chunk, d, inv_2h, gh);
    return true;
}

cudaError_t launch_divergence(float* div, const void* vx, const void* vy, const void* vz, Dims d, float h, const FlowBC& b, int bf16, cudaStream_t s) {
    if (!bf16 && launch_divergence_vec4(div, nullptr, vx, vy, vz, d, h, b, s)) return cudaGetLastError();
    SFB_STORAGE(bf16, (k_divergence<float><<<cell_grid(d), cell_block(), 0, s>>>(div, static_cast<const float*>(vx), static_cast<const float*>(vy), static_cast<const float*>(vz), d, h, b)),
                (k_divergence<bf16_t><<<cell_grid(d), cell_block(), 0, s>>>(div, static_cast<const bf16_t*>(vx), static_cast<const bf16_t*>(vy), static_cast<const bf16_t*>(vz), d, h, b)));
    return cudaGetLastError();
}
cudaError_t launch_project(void* vx, void* vy, void* vz, void* packed, const float* p, const float* div, Dims d, float h, float h2, const FlowBC& b, DeviceStats* stats, int bf16, cudaStream_t s) {
    SFB_STORAGE(bf16, (k_project<float, float4><<<cell_grid(d), cell_block(), 0, s>>>(static_cast<float*>(vx), static_cast<float*>(vy), static_cast<float*>(vz), static_cast<float4*>(packed), p, div, d, h, h2, b, stats)),
                (k_project<bf16_t, Bf16x4><<<cell_grid(d), cell_block(), 0, s>>>(static_cast<bf16_t*>(vx), static_cast<bf16_t*>(vy), static_cast<bf16_t*>(vz), static_cast<Bf16x4*>(packed), p, div, d, h, h2, b, stats)));
    return cudaGetLastError();
}

cudaError_t launch_residual_sums(const float* p, const float* div, Dims d, float h2, const FlowBC& b, DeviceStats* stats, cudaStream_t s) {
    if (launch_residual_sums_vec(p, div, d, h2, b, stats, s)) return cudaGetLastError();
    k_residual_sums<<<cell_grid(d), cell_block(), 0, s>>>(p, div, d, h2, b, stats);
    return cudaGetLastError();
}

cudaError_t launch_residual_finalize(DeviceStats* stats, Dims d, int singular, int iterations, cudaStream_t s) {
    const double n = static_cast<double>(d.nx) * static_cast<double>(d.ny) * static_cast<double>(d.nz);
    k_residual_finalize<<<1, 32, 0, s>>>(stats, n, singular, iterations);
    return cudaGetLastError();
}

cudaError_t launch_residual_check(DeviceStats* stats, Dims d, int singular, int reset, int increment, double tol, int max_iterations, cudaGraphConditionalHandle handle, cudaStream_t s) {
    const double n = static_cast<double>(d.nx) * static_cast<double>(d.ny) * static_cast<double>(d.nz);
    k_residual_check<<<1, 32, 0, s>>>(stats, n, singular, reset, increment, tol, max_iterations, handle);
    return cudaGetLastError();
}

cudaError_t launch_warm_start_select(DeviceStats* learned, const DeviceStats* plain, Dims d, int singular, float* p, const float* alt, cudaStream_t s) {
    const size_t cells = static_cast<size_t>(d.nx) * static_cast<size_t>(d.ny) * static_cast<size_t>(d.nz);
    const double n = static_cast<double>(cells);
    k_warm_start_select<<<linear_grid(cells, 256), 256, 0, s>>>(learned, plain, n, singular, p, alt, cells);
    k_warm_start_commit<<<1, 32, 0, s>>>(learned, plain, n, singular);
    return cudaGetLastError();
}

cudaError_t launch_post_diagnostics(float* div, float* mag, const void* vx, const void* vy, const void* vz, Dims d, float h, const FlowBC& b, int bf16, cudaStream_t s) {
    if (!bf16 && launch_divergence_vec4(div, mag, vx, vy, vz, d, h, b, s)) return cudaGetLastError();
    SFB_STORAGE(bf16, (k_post_diagnostics<float><<<cell_grid(d), cell_block(), 0, s>>>(div, mag, static_cast<const float*>(vx), static_cast<const float*>(vy), static_cast<const float*>(vz), d, h, b)),
                (k_post_diagnostics<bf16_t><<<cell_grid(d), cell_block(), 0, s>>>(div, mag, static_cast<const bf16_t*>(vx), static_cast<const bf16_t*>(vy), static_cast<const bf16_t*>(vz), d, h, b)));
    return cudaGetLastError();
}

// ------------------------------------------------------ work-table batch --
namespace {
unsigned batch_grid(uint32_t total, int sms, int per_sm) {
    const uint32_t cap = static_cast<uint32_t>(sms) * static_cast<uint32_t>(per_sm);
    return total < cap ? (total == 0 ? 1u : total) : cap;
}
}  // namespace

cudaError_t launch_batch_force_pack(const BatchTable& t, cudaStream_t s) {
    k_batch_force_pack<<<batch_grid(t.total[SHAPE_LINEAR], t.sms, 8), 256, 0, s>>>(t);
    return cudaGetLastError();
}

cudaError_t launch_batch_advect_velocity(const BatchTable& t, cudaStream_t s) {
    k_batch_advect_velocity<<<batch_grid(t.total[SHAPE_CELL], t.sms, 4), cell_block(), 0, s>>>(t);
    return cudaGetLastError();
}

cudaError_t launch_batch_scalar_source_advect(const BatchTable& t, cudaStream_t s) {
    k_batch_scalar_source_advect<<<batch_grid(t.total[SHAPE_CELL], t.sms, 4), cell_block(), 0, s>>>(t);
    return cudaGetLastError();
}

cudaError_t launch_batch_divergence(const BatchTable& t, cudaStream_t s) {
    k_batch_divergence<false><<<batch_grid(t.total[SHAPE_VEC], t.sms, 8), dim3(32, kDivRows), 0, s>>>(t);
    return cudaGetLastError();
}

cudaError_t launch_batch_project(const BatchTable& t, int pack, cudaStream_t s) {
    k_batch_project<<<batch_grid(t.total[SHAPE_CELL], t.sms, 8), cell_block(), 0, s>>>(t, pack);
    return cudaGetLastError();
}

cudaError_t launch_batch_post_diagnostics(const BatchTable& t, cudaStream_t s) {
    k_batch_divergence<true><<<batch_grid(t.total[SHAPE_VEC], t.sms, 8), dim3(32, kDivRows), 0, s>>>(t);
    return cudaGetLastError();
}

cudaError_t launch_batch_stats(const BatchTable& t, int finalize, int iterations, cudaStream_t s) {
    k_batch_stats<<<static_cast<unsigned>((t.nsims + 63) / 64), 64, 0, s>>>(t, finalize, iterations);
    return cudaGetLastError();
}

uint32_t batch_blocks(const Dims& d, int shape, int z_chunk) {
    if (shape == SHAPE_LINEAR) return static_cast<uint32_t>((static_cast<size_t>(d.nx) * d.ny * d.nz + 255) / 256);
    if (shape == SHAPE_CELL) {
        const dim3 g = cell_grid(d);
        return g.x * g.y * g.z;
    }
    const uint32_t zc = static_cast<uint32_t>(z_chunk < 1 ? 1 : z_chunk);
    const uint32_t chunks = (static_cast<uint32_t>(d.nz) + zc - 1) / zc;
    if (shape == SHAPE_HALF) return static_cast<uint32_t>((static_cast<size_t>(d.nx / 8) * d.ny + 127) / 128) * chunks;
    if (shape == SHAPE_OCT) return static_cast<uint32_t>((static_cast<size_t>(d.nx / 8) * d.ny * d.nz + 255) / 256);
    const uint32_t bx = static_cast<uint32_t>((d.nx / 4 + 31) / 32), by = static_cast<uint32_t>((d.ny + 3) / 4);
    return bx * by * chunks;
}

cudaError_t launch_restrict2(const float* fine, float* coarse, Dims fine_dims, cudaStream_t s) {
    const Dims c{fine_dims.nx / 2, fine_dims.ny / 2, fine_dims.nz / 2, 0};
    k_restrict2<<<cell_grid(c), cell_block(), 0, s>>>(fine, coarse, fine_dims);
    return cudaGetLastError();
}

cudaError_t launch_prolong_add(const float* coarse_new, const float* coarse_old, float* fine_p, Dims fine_dims, cudaStream_t s) {
    k_prolong_add<<<cell_grid(fine_dims), cell_block(), 0, s>>>(coarse_new, coarse_old, fine_p, fine_dims);
    return cudaGetLastError();
}

}  // namespace sfb
