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
//   RBGS   : stage s updates the cells of colour (parity0 + s - 1) & 1 and
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
    int k_run;         // stages run in this pass (1..K)
    int parity0;       // red-black: colour of stage 1
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

template <int KIND, bool RB, int K, int V, int R>
__global__ void __launch_bounds__(32 * R, 1) k_wave(WaveArgs a) {
    using L = WaveLayout<K, V, R>;
    constexpr int PLANE = L::PLANE;
    constexpr int ROW4 = L::NX / 4;  // float4 per row
    static_assert(R > 2 * K, "tile rows must exceed the halo");
    extern __shared__ __align__(16) float4 sm4[];
    float4* const in_ring = sm4;                                // [4][R][ROW4]
    float4* const rings = sm4 + L::IN_PLANES * PLANE / 4;       // [K-1][2][R][ROW4]: stage s's output at s-1
    float4* const rhs_ring = sm4 + L::RING_PLANES * PLANE / 4;  // [K+3][R][ROW4]
    constexpr int RS = L::RHS_PLANES;

    const Dims d = a.d;
    const GhostRule& g = a.g;
    const int lane = static_cast<int>(threadIdx.x & 31), row = static_cast<int>(threadIdx.x >> 5);
    constexpr int TY = R - 2 * K;
    const int gy_u = static_cast<int>(blockIdx.x) * TY - K + row;  // unwrapped global row
    const bool px = g.periodic[0] != 0, py = g.periodic[1] != 0, pz = g.periodic[2] != 0;
    int gy = gy_u;
    bool live = true;
    if (gy < 0 || gy >= d.ny) {
        if (py) gy = wrap_index(gy, d.ny);
        else live = false;
    }
    const bool out_row = row >= K && row < R - K && gy_u < d.ny;
    const bool face_ylo = !py && gy_u == 0, face_yhi = !py && gy_u == d.ny - 1;
    const int z0 = static_cast<int>(blockIdx.y) * a.z_chunk;
    if (z0 >= d.nz) return;  // CTA-uniform, before any barrier
    const int z1 = min(z0 + a.z_chunk, d.nz);
    const int k_run = a.k_run;
    const int t_begin = pz ? z0 - K : max(z0 - K, 0);
    const int t_end = z1 - 1 + k_run;
    const size_t sz = static_cast<size_t>(d.nx) * d.ny;
    const size_t row_off = static_cast<size_t>(gy) * d.nx;
    const float divisor = KIND == KIND_PRESSURE ? 6.0f : 1.0f + 6.0f * a.coef;
    const double recip = tb::recip64(divisor);
    const float inv = jacobi_inverse(KIND, a.coef);

    // plane index of unwrapped z (z0 - 2K <= z <= z1 - 1 + K: a few
    // additions wrap it), or -1 outside a non-periodic axis
    const auto plane_of = [&](int z) {
        if (!pz) return static_cast<unsigned>(z) < static_cast<unsigned>(d.nz) ? z : -1;
        while (z < 0) z += d.nz;
        while (z >= d.nz) z -= d.nz;
        return z;
    };

    // index s (2..K): stage s-1's planes q and q-1 for stage s; below[1]:
    // input plane q-1 of stage 1
    float4 cur[K + 1][V], below[K + 1][V];
#pragma unroll
    for (int s = 0; s <= K; ++s)
#pragma unroll
        for (int j = 0; j < V; ++j) cur[s][j] = below[s][j] = make_float4(0.f, 0.f, 0.f, 0.f);

    // copies of input plane t (x and rhs) into their ring slots, one commit
    // group per time step (empty past the chunk's last plane)
    const auto issue = [&](int t) {
        const int pl = (t <= t_end) ? plane_of(t) : -1;
        if (pl >= 0) {
            float4* xs = in_ring + (wrap_index(t, 4) * R + row) * ROW4;
            float4* rs = rhs_ring + (wrap_index(t, RS) * R + row) * ROW4;
            const size_t i0 = static_cast<size_t>(pl) * sz + row_off + 4 * lane;
#pragma unroll
            for (int j = 0; j < V; ++j) {
                const size_t i = i0 + 128 * j;
                cp_async16(xs + 32 * j + lane, live && a.src != nullptr ? a.src + i : a.rhs, live && a.src != nullptr);
                cp_async16(rs + 32 * j + lane, live ? a.rhs + i : a.rhs, live);
            }
        }
        tb::cp_async_commit();
    };
    issue(t_begin);
    issue(t_begin + 1);
    tb::cp_async_wait<1>();
    __syncthreads();

    for (int t = t_begin; t <= t_end; ++t) {
        issue(t + 2);  // its slots held planes t - 2 (input) and t - K - 1 (rhs), last read at t - 1
        // stage 1's newest plane: the input plane t
        float4 above[V];
        {
            const float4* r0 = in_ring + (wrap_index(t, 4) * R + row) * ROW4;
#pragma unroll
            for (int j = 0; j < V; ++j) above[j] = r0[32 * j + lane];
        }

#pragma unroll
        for (int s = 1; s <= K; ++s) {
            if (s > k_run) break;
            const int q = t - s;
            const int pq = plane_of(q);
            const bool active = pq >= 0 && q >= z0 - K + s && q <= z1 - 1 + K - s && live && row >= s && row < R - s;  // warp-uniform
            const bool to_ring = s < k_run, to_dst = s == k_run && out_row && q >= z0 && q < z1;
            const float4* ring_in = s == 1 ? in_ring + wrap_index(q, 4) * R * ROW4 : rings + (((s - 2) * 2 + (q & 1)) * R) * ROW4;
            const float4* rhs_in = rhs_ring + (wrap_index(q, RS) * R + row) * ROW4;
            float4* ring_out = rings + (((s - 1) * 2 + (q & 1)) * R + row) * ROW4;
            const bool even = RB ? (((gy + pq + ((a.parity0 + s - 1) & 1)) & 1) == 0) : true;
            const bool zlo = !pz && pq == 0, zhi = !pz && pq == d.nz - 1;
            const bool edge = face_ylo || face_yhi || zlo || zhi;
            float lw[V], rx[V];
            float4 cs[V];  // stage s-1's plane q, this lane's cells
#pragma unroll
            for (int j = 0; j < V; ++j) cs[j] = s == 1 ? ring_in[row * ROW4 + 32 * j + lane] : cur[s][j];
            if (active) {
#pragma unroll
                for (int j = 0; j < V; ++j) {
                    lw[j] = __shfl_sync(0xffffffffu, cs[j].w, (lane + 31) & 31);
                    rx[j] = __shfl_sync(0xffffffffu, cs[j].x, (lane + 1) & 31);
                }
            }
            // one float4 segment at a time: update, store, move up one plane
#pragma unroll
            for (int j = 0; j < V; ++j) {
                float4 o = make_float4(0.f, 0.f, 0.f, 0.f);
                if (active) {
                    const float4 c = cs[j];
                    float4 ym, yp, zb, za;
                    if (!edge) {  // interior rows and planes: no ghost (warp-uniform)
                        ym = ring_in[(row - 1) * ROW4 + 32 * j + lane];
                        yp = ring_in[(row + 1) * ROW4 + 32 * j + lane];
                        zb = below[s][j];
                        za = above[j];
                    } else {
                        ym = face_ylo ? ghost4v(g, YM, c) : ring_in[(row - 1) * ROW4 + 32 * j + lane];
                        yp = face_yhi ? ghost4v(g, YP, c) : ring_in[(row + 1) * ROW4 + 32 * j + lane];
                        zb = zlo ? ghost4v(g, ZM, c) : below[s][j];
                        za = zhi ? ghost4v(g, ZP, c) : above[j];
                    }
                    const float4 r = rhs_in[32 * j + lane];
                    float left = lane == 0 ? lw[(j + V - 1) % V] : lw[j];
                    float right = lane == 31 ? rx[(j + 1) % V] : rx[j];
                    if (!px) {  // x faces: the row's first and last cell (lanes 0 and 31)
                        if (j == 0 && lane == 0) left = tb::ghost(g, XM, c.x);
                        if (j == V - 1 && lane == 31) right = tb::ghost(g, XP, c.w);
                    }
                    const float n0 = left + c.y + ym.x + yp.x + zb.x + za.x;
                    const float n1 = c.x + c.z + ym.y + yp.y + zb.y + za.y;
                    const float n2 = c.y + c.w + ym.z + yp.z + zb.z + za.z;
                    const float n3 = c.z + right + ym.w + yp.w + zb.w + za.w;
                    if constexpr (RB) {
                        if (even) o = make_float4(tb::divide(tb::numerator<KIND>(n0, r.x, a.coef), divisor, recip), c.y, tb::divide(tb::numerator<KIND>(n2, r.z, a.coef), divisor, recip), c.w);
                        else o = make_float4(c.x, tb::divide(tb::numerator<KIND>(n1, r.y, a.coef), divisor, recip), c.z, tb::divide(tb::numerator<KIND>(n3, r.w, a.coef), divisor, recip));
                    } else {
                        o = make_float4(jacobi_update<KIND>(n0, r.x, a.coef, inv), jacobi_update<KIND>(n1, r.y, a.coef, inv), jacobi_update<KIND>(n2, r.z, a.coef, inv), jacobi_update<KIND>(n3, r.w, a.coef, inv));
                    }
                    if (to_ring) {
                        ring_out[32 * j + lane] = o;
                    } else if (to_dst) {
                        float4 w = o;
                        if (a.out_scale != 1.0f) w = make_float4(__fmul_rn(w.x, a.out_scale), __fmul_rn(w.y, a.out_scale), __fmul_rn(w.z, a.out_scale), __fmul_rn(w.w, a.out_scale));
                        *reinterpret_cast<float4*>(a.dst + static_cast<size_t>(pq) * sz + row_off + 128 * j + 4 * lane) = w;
                    }
                }
                if (s == 1) {
                    below[1][j] = cs[j];
                } else {
                    below[s][j] = cur[s][j];
                    cur[s][j] = above[j];
                }
                above[j] = o;  // stage s+1's newest plane
            }
        }
        tb::cp_async_wait<1>();  // this thread's copies of plane t + 1 have landed
        __syncthreads();
    }
    tb::cp_async_wait<0>();
}

}  // namespace wave
}  // namespace sfb
