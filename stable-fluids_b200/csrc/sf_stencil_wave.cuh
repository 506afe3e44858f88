// sf_stencil_wave.cuh -- K sweeps of the 7-point solves per HBM pass.
//
// A z-wavefront pipeline of K stages over an xy tile of full rows. The CTA
// owns R rows of the grid (one warp per row; a lane owns V float4 of the
// row, at x = 128 j + 4 lane, so a row is nx = 128 V cells) and a chunk of
// z planes, and marches up the chunk one plane per time step. At time step
// t, stage s (s = 1..K) updates plane q = t - s of its rows from stage s-1's
// values:
//   - x neighbours: the adjacent lanes' values (warp shuffles); the row's
//     ends take the face ghost or, on a periodic x axis, wrap;
//   - y neighbours: stage s-1's plane q in shared memory (a two-slot ring per
//     stage), written one time step earlier by the neighbouring warps;
//   - z neighbours: the lane's own registers -- stage s-1's planes q-1 and q
//     carried from earlier time steps, and plane q+1 produced by stage s-1
//     in this time step (stage 1 reads planes q and q+1 of the input from
//     the input ring and keeps plane q-1 in registers).
// Stage 0 is the input: plane t of the iterate and of the right-hand side,
// read from HBM once per pass by asynchronous copies (cp.async, 16 bytes per
// lane, cached in L2 only) straight into shared memory two time steps ahead
// of use: a ring of 4 input planes (t-1, t, and t+1, t+2 in flight) and one
// of K+3 right-hand-side planes (stage s reads plane q at time q + s). Every
// shared-memory value read in a time step was written -- or its copy waited
// for -- in an earlier one, so one barrier per time step orders everything.
//
// Each stage shrinks the rows whose values are exact by one at each side of
// the tile, and the planes by one at each end of the chunk: the tile carries
// K halo rows above and below its R - 2K output rows, and the chunk K halo
// planes at each end (fewer at a non-periodic face, where the face ghost
// rule applies instead). The rows and planes a stage cannot get right are
// skipped, warp-uniformly. Traffic: read x + b, write x = 12 B per cell per
// pass, whatever K.
//
// Schemes:
//   JACOBI : every stage is a Jacobi sweep with this library's Jacobi
//            arithmetic (jacobi_update); k_jacobi_vec4 computes the same, so
//            K sweeps here equal K single sweeps bit for bit;
//   RBGS   : stage s updates the cells of colour (s - 1) & 1 (red first) and
//            copies the others, with the reference's exact division
//            (backend-cuda.cu:354-375, 398-407): 2 stages = one red-black
//            iteration, bit-equal to the reference's two launches.
// Face ghosts are the GhostRule of the float4 sweeps (self value copied,
// reflected or replaced by a constant), so boundary cells take the same
// values as in k_rbgs_vec4 / k_jacobi_vec4.
#pragma once

#include <cuda_runtime.h>

#include "sf_device.cuh"
#include "sf_stencil_tb.cuh"
#include "sf_types.h"

namespace sfb {
namespace wave {

struct WaveArgs {
    const float* src;  // iterate at the start of the pass (null: zero)
    const float* rhs;  // right-hand side
    float* dst;        // iterate after the pass (never src)
    float coef;        // alpha or h^2
    float out_scale;   // multiplies the pass's result (dissipation; 1 = none)
    int z_chunk;       // output planes per CTA
    Dims d;
    GhostRule g;
};

// Shared memory of one CTA: the input ring of 4 planes, K-1 two-slot rings
// (stage s's output, s = 1..K-1), then the right-hand-side ring of K + 3
// planes; a plane holds the CTA's R rows of nx floats.
template <int K, int V, int R>
struct WaveLayout {
    static constexpr int NX = 128 * V;
    static constexpr int PLANE = R * NX;
    static constexpr int IN_PLANES = 4;
    static constexpr int RING_PLANES = IN_PLANES + 2 * (K - 1);
    static constexpr int RHS_PLANES = K + 3;
    static constexpr size_t bytes = static_cast<size_t>(RING_PLANES + RHS_PLANES) * PLANE * sizeof(float);
};

// 16-byte asynchronous copy global -> shared, L2 only; zero-fills when !valid.
__device__ __forceinline__ void cp_async16(float4* dst, const float* src, bool valid) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(tb::smem_addr(dst)), "l"(src), "r"(valid ? 16 : 0) : "memory");
}

__device__ __forceinline__ float4 ghost4v(const GhostRule& g, int face, float4 s) {
    return make_float4(tb::ghost(g, face, s.x), tb::ghost(g, face, s.y), tb::ghost(g, face, s.z), tb::ghost(g, face, s.w));
}

// The Jacobi update of this library (the reference has no Jacobi scheme):
// the numerator of the reference's update, rounded once (one fused
// multiply-add), times the correctly rounded reciprocal of the divisor:
//   pressure : RN(RN(nb - h^2 div) * RN(1 / 6))
//   diffusion: RN(RN(b + alpha nb) * RN(1 / RN(1 + 6 alpha)))
__device__ __forceinline__ float jacobi_inverse(int kind, float coef) { return __frcp_rn(kind == KIND_PRESSURE ? 6.0f : __fmaf_rn(6.0f, coef, 1.0f)); }

template <int KIND>
__device__ __forceinline__ float jacobi_update(float nb, float rhs, float coef, float inv) {
    const float num = KIND == KIND_PRESSURE ? __fmaf_rn(-coef, rhs, nb) : __fmaf_rn(coef, nb, rhs);
    return __fmul_rn(num, inv);
}

// One time step t of the pipeline (PH = t mod 3 selects which of the three
// history buffers of each stage holds planes q-1, q and q+1, so the history
// moves up a plane by renaming, without register copies).
template <int KIND, bool RB, int K, int V, int R>
struct WaveCta {
    using L = WaveLayout<K, V, R>;
    static constexpr int ROW4 = L::NX / 4;
    static constexpr int PLANE4 = L::PLANE / 4;
    static constexpr int RS = L::RHS_PLANES;
    static constexpr int TY = R - 2 * K;

    const WaveArgs& a;
    float4* in_ring;   // [4][R][ROW4]
    float4* rings;     // [K-1][2][R][ROW4], stage r's output at r-1
    float4* rhs_ring;  // [RS][R][ROW4]
    int lane, row, gy, z0, z1, nz;
    bool live, out_row, face_ylo, face_yhi, px, pz;
    bool xm_lane, xp_lane;          // this lane holds the row's first / last cell on a non-periodic x axis
    float4 h[K + 1][3][V];          // stage s's input planes (stage s-1's outputs; s = 1: the input)
    size_t row_off, sz;
    float inv;                      // Jacobi: RN(1 / divisor)
    float divisor;
    double recip;

    __device__ __forceinline__ int wrap_z(int z) const { return z < 0 ? z + nz : (z >= nz ? z - nz : z); }

    // the copies of input plane p (x and rhs) into ring slots p & 3 and ps
    __device__ __forceinline__ void issue(int p, int ps, int t_end) {
        if (p <= t_end) {
            const int pl = pz ? wrap_z(p) : p;
            if (pz || static_cast<unsigned>(pl) < static_cast<unsigned>(nz)) {
                const size_t i = static_cast<size_t>(pl) * sz + row_off + 4 * lane;
                float4* xs = in_ring + ((p & 3) * R + row) * ROW4 + lane;
                float4* rs = rhs_ring + (ps * R + row) * ROW4 + lane;
                const bool xv = live && a.src != nullptr;
#pragma unroll
                for (int j = 0; j < V; ++j) {
                    cp_async16(xs + 32 * j, xv ? a.src + i + 128 * j : a.rhs, xv);
                    cp_async16(rs + 32 * j, live ? a.rhs + i + 128 * j : a.rhs, live);
                }
            }
        }
        tb::cp_async_commit();
    }

    template <int PH>
    __device__ __forceinline__ void step(int t, int rt, int t_end) {
        constexpr int B = PH % 3, C = (PH + 1) % 3, N = (PH + 2) % 3;  // planes q-1, q, q+1 of each stage
        issue(t + 2, rt + 2 >= RS ? rt + 2 - RS : rt + 2, t_end);  // its slots held planes t - 2 and t - K - 1, last read at t - 1
        {   // stage 1's newest plane: the input plane t
            const float4* r0 = in_ring + ((t & 3) * R + row) * ROW4 + lane;
#pragma unroll
            for (int j = 0; j < V; ++j) h[1][N][j] = r0[32 * j];
        }
#pragma unroll
        for (int s = 1; s <= K; ++s) {
            const int q = t - s;
            const bool in_planes = q >= z0 - K + s && q <= z1 - 1 + K - s && (pz || static_cast<unsigned>(q) < static_cast<unsigned>(nz));
            float4 o[V];
            if (in_planes && live && row >= s && row < R - s) {  // warp-uniform
                const int pq = pz ? wrap_z(q) : q;
                const float4* ring_in = s == 1 ? in_ring + ((q & 3) * R) * ROW4 + lane : rings + (((s - 2) * 2 + (q & 1)) * R) * ROW4 + lane;
                const int rslot = rt - s < 0 ? rt - s + RS : rt - s;
                const float4* rhs_in = rhs_ring + (rslot * R + row) * ROW4 + lane;
                const bool zlo = !pz && pq == 0, zhi = !pz && pq == nz - 1;
                const bool edge = face_ylo || face_yhi || zlo || zhi;
                float lw[V], rx[V];
#pragma unroll
                for (int j = 0; j < V; ++j) {
                    lw[j] = __shfl_sync(0xffffffffu, h[s][C][j].w, (lane + 31) & 31);
                    rx[j] = __shfl_sync(0xffffffffu, h[s][C][j].x, (lane + 1) & 31);
                }
                const bool even = RB ? (((gy + pq + ((s - 1) & 1)) & 1) == 0) : true;
#pragma unroll
                for (int j = 0; j < V; ++j) {
                    const float4 c = h[s][C][j];
                    float4 ym = ring_in[(row - 1) * ROW4 + 32 * j];
                    float4 yp = ring_in[(row + 1) * ROW4 + 32 * j];
                    float4 zb = h[s][B][j], za = h[s][N][j];
                    if (edge) {  // a face row or plane (warp-uniform, rare)
                        if (face_ylo) ym = ghost4v(a.g, YM, c);
                        if (face_yhi) yp = ghost4v(a.g, YP, c);
                        if (zlo) zb = ghost4v(a.g, ZM, c);
                        if (zhi) za = ghost4v(a.g, ZP, c);
                    }
                    const float4 r = rhs_in[32 * j];
                    float left = lane == 0 ? lw[(j + V - 1) % V] : lw[j];
                    float right = lane == 31 ? rx[(j + 1) % V] : rx[j];
                    if (j == 0) left = xm_lane ? tb::ghost(a.g, XM, c.x) : left;
                    if (j == V - 1) right = xp_lane ? tb::ghost(a.g, XP, c.w) : right;
                    const float n0 = left + c.y + ym.x + yp.x + zb.x + za.x;
                    const float n1 = c.x + c.z + ym.y + yp.y + zb.y + za.y;
                    const float n2 = c.y + c.w + ym.z + yp.z + zb.z + za.z;
                    const float n3 = c.z + right + ym.w + yp.w + zb.w + za.w;
                    if constexpr (RB) {
                        if (even) o[j] = make_float4(tb::divide(tb::numerator<KIND>(n0, r.x, a.coef), divisor, recip), c.y, tb::divide(tb::numerator<KIND>(n2, r.z, a.coef), divisor, recip), c.w);
                        else o[j] = make_float4(c.x, tb::divide(tb::numerator<KIND>(n1, r.y, a.coef), divisor, recip), c.z, tb::divide(tb::numerator<KIND>(n3, r.w, a.coef), divisor, recip));
                    } else {
                        o[j] = make_float4(jacobi_update<KIND>(n0, r.x, a.coef, inv), jacobi_update<KIND>(n1, r.y, a.coef, inv), jacobi_update<KIND>(n2, r.z, a.coef, inv), jacobi_update<KIND>(n3, r.w, a.coef, inv));
                    }
                }
                if (s < K) {
                    float4* ring_out = rings + (((s - 1) * 2 + (q & 1)) * R + row) * ROW4 + lane;
#pragma unroll
                    for (int j = 0; j < V; ++j) ring_out[32 * j] = o[j];
                } else if (out_row && q >= z0 && q < z1) {
                    float* out = a.dst + static_cast<size_t>(pq) * sz + row_off + 4 * lane;
                    const float f = a.out_scale;  // 1 leaves every value unchanged
#pragma unroll
                    for (int j = 0; j < V; ++j) *reinterpret_cast<float4*>(out + 128 * j) = make_float4(__fmul_rn(o[j].x, f), __fmul_rn(o[j].y, f), __fmul_rn(o[j].z, f), __fmul_rn(o[j].w, f));
                }
            } else {
#pragma unroll
                for (int j = 0; j < V; ++j) o[j] = make_float4(0.f, 0.f, 0.f, 0.f);
            }
            if (s < K) {
#pragma unroll
                for (int j = 0; j < V; ++j) h[s + 1][N][j] = o[j];  // stage s+1's newest plane
            }
        }
        tb::cp_async_wait<1>();  // this thread's copies of plane t + 1 have landed
        __syncthreads();
    }
};

template <int KIND, bool RB, int K, int V, int R>
__global__ void __launch_bounds__(32 * R, 1) k_wave(WaveArgs a) {
    using W = WaveCta<KIND, RB, K, V, R>;
    using L = typename W::L;
    static_assert(R > 2 * K, "tile rows must exceed the halo");
    extern __shared__ __align__(16) float4 sm4[];
    W w{a};
    w.in_ring = sm4;
    w.rings = sm4 + L::IN_PLANES * W::PLANE4;
    w.rhs_ring = sm4 + L::RING_PLANES * W::PLANE4;
    const Dims d = a.d;
    w.lane = static_cast<int>(threadIdx.x & 31);
    w.row = static_cast<int>(threadIdx.x >> 5);
    w.nz = d.nz;
    const int gy_u = static_cast<int>(blockIdx.x) * W::TY - K + w.row;  // unwrapped global row
    w.px = a.g.periodic[0] != 0;
    const bool py = a.g.periodic[1] != 0;
    w.pz = a.g.periodic[2] != 0;
    w.gy = gy_u;
    w.live = true;
    if (gy_u < 0 || gy_u >= d.ny) {
        if (py) w.gy = wrap_index(gy_u, d.ny);
        else w.live = false;
    }
    w.out_row = w.row >= K && w.row < R - K && gy_u < d.ny;
    w.face_ylo = !py && gy_u == 0;
    w.face_yhi = !py && gy_u == d.ny - 1;
    w.xm_lane = !w.px && w.lane == 0;
    w.xp_lane = !w.px && w.lane == 31;
    w.z0 = static_cast<int>(blockIdx.y) * a.z_chunk;
    if (w.z0 >= d.nz) return;  // CTA-uniform, before any barrier
    w.z1 = min(w.z0 + a.z_chunk, d.nz);
    w.sz = static_cast<size_t>(d.nx) * d.ny;
    w.row_off = static_cast<size_t>(w.gy) * d.nx;
    w.divisor = KIND == KIND_PRESSURE ? 6.0f : 1.0f + 6.0f * a.coef;
    w.recip = tb::recip64(w.divisor);
    w.inv = jacobi_inverse(KIND, a.coef);
#pragma unroll
    for (int s = 0; s <= K; ++s)
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
            for (int j = 0; j < V; ++j) w.h[s][k][j] = make_float4(0.f, 0.f, 0.f, 0.f);

    const int t_begin = w.pz ? w.z0 - K : max(w.z0 - K, 0);
    const int t_end = w.z1 - 1 + K;
    // rhs ring slot of plane t_begin (the ring holds plane p at p mod RS)
    int rt = t_begin % W::RS;
    if (rt < 0) rt += W::RS;
    w.issue(t_begin, rt, t_end);
    w.issue(t_begin + 1, rt + 1 >= W::RS ? rt + 1 - W::RS : rt + 1, t_end);
    tb::cp_async_wait<1>();
    __syncthreads();
    // three time steps per iteration: planes t, t+1, t+2 in phases 0, 1, 2 of
    // the history buffers (CTA-uniform bounds)
    const auto next = [](int r) { return r + 1 == W::RS ? 0 : r + 1; };
    for (int t = t_begin; t <= t_end; t += 3) {
        w.template step<0>(t, rt, t_end);
        rt = next(rt);
        if (t + 1 > t_end) break;
        w.template step<1>(t + 1, rt, t_end);
        rt = next(rt);
        if (t + 2 > t_end) break;
        w.template step<2>(t + 2, rt, t_end);
        rt = next(rt);
    }
    tb::cp_async_wait<0>();
}

}  // namespace wave
}  // namespace sfb
