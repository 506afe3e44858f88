// sf_stencil_tb.cuh -- temporally blocked red-black Gauss-Seidel pass.
//
// One launch runs K_run colour half-sweeps (K_run/2 full RBGS iterations)
// over the whole field while reading x and b from HBM once and writing x
// once (12 B per cell per pass instead of ~12 B per cell per half-sweep).
//
// Tiling (2.5D): each CTA owns an xy tile of TX x TY output cells and a
// chunk of Z planes. It loads the tile plus a halo of HX (x, rounded up to 4
// cells for 16-byte TMA alignment) and K (y) cells, and streams the planes of
// its chunk (plus K halo planes at each chunk end) through a ring of shared
// memory planes. At stream time j plane j is loaded and colour stage s
// (s = 1..K_run) updates plane j - s in place:
//   - stage s - 1 finished plane j - s + 1 earlier in the same time step,
//   - stage s + 1 has not yet touched plane j - s - 1,
// so every stage reads exactly the values the global half-sweep would see.
// Each stage shrinks the region of correct values by one cell in x and y
// (and one plane at each chunk end), which the halo absorbs. The updates use
// the reference's arithmetic (backend-cuda.cu:354-375, 398-407), so the
// result equals K_run/2 reference iterations bit for bit.
//
// Shared-memory mapping: a warp updates 16 cells of one colour in each of two
// adjacent rows. Because the row pitch W is even and adjacent rows hold
// opposite colours, the 32 lanes address 32 distinct banks for the cell, its
// x, y and z neighbours and b: no bank conflicts with a plain row-major plane,
// which is what a TMA box writes.
//
// Loads: one elected thread issues a 3D TMA box per plane for x and for b
// (cp.async.bulk.tensor, mbarrier completion, prefetch distance D planes).
// CTAs whose halo wraps around a periodic x or y boundary (TMA fills outside
// the tensor instead of wrapping) and grids whose rows are not 16-byte
// aligned load with cp.async instead. Every mbarrier wait is bounded: on
// timeout the kernel records an error flag and returns.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include "sf_device.cuh"
#include "sf_launch.h"

namespace sfb {

// Ghost value of a face in a stencil: self (Neumann / copy), a constant
// (Dirichlet), or k - self (reflection about a prescribed wall value).
enum GhostMode : int32_t { GHOST_COPY = 0, GHOST_CONST = 1, GHOST_REFLECT = 2 };

struct GhostRule {
    int32_t mode[6];
    float k[6];
    int32_t periodic[3];
    int32_t pad;
};

struct TbArgs {
    const float* src;  // x at the start of the pass (null: zero)
    const float* b;    // right-hand side
    float* dst;        // x after the pass
    float coef;
    float out_scale;
    Dims d;
    GhostRule g;
    int k_run;         // colour half-sweeps in this pass (even, <= K)
    int z_chunk;       // output planes per CTA
    int tma_ok;        // tensor maps usable (rows 16-byte aligned)
    unsigned* error;   // set to 1 if a bounded wait gives up
};

namespace tb {

constexpr int kPrefetch = 2;  // planes in flight ahead of the one being consumed

__device__ __forceinline__ unsigned smem_addr(const void* p) { return static_cast<unsigned>(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}

// Bounded wait for the phase with the given parity; false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity) {
    const unsigned addr = smem_addr(bar);
    for (unsigned it = 0; it < (1u << 26); ++it) {
        unsigned done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(addr), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void tma_load_plane(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_addr(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void cp_async4(void* dst, const float* src, bool valid) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(smem_addr(dst)), "l"(src), "r"(valid ? 4 : 0) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

template <int KIND>
__device__ __forceinline__ float ghost(const GhostRule& g, int face, float self) {
    const int m = g.mode[face];
    if (m == GHOST_COPY) return self;
    if (m == GHOST_CONST) return g.k[face];
    return g.k[face] - self;
}

template <int KIND>
__device__ __forceinline__ float update(float nb, float rhs, float coef) {
    if constexpr (KIND == KIND_PRESSURE) return (nb - coef * rhs) / 6.0f;
    else return (rhs + coef * nb) / (1.0f + 6.0f * coef);
}

}  // namespace tb

// K: halo (max colour half-sweeps per pass); W, HH: loaded plane size;
// NT: threads per CTA.
template <int KIND, int K, int W, int HH, int NT>
__global__ void __launch_bounds__(NT, 1) k_rbgs_tb(const __grid_constant__ CUtensorMap map_x, const __grid_constant__ CUtensorMap map_b, TbArgs a) {
    constexpr int HX = ((K + 3) / 4) * 4;
    constexpr int TX = W - 2 * HX;
    constexpr int TY = HH - 2 * K;
    constexpr int D = tb::kPrefetch;
    constexpr int R = K + D + 2;   // x planes: j-K-1 .. j+D
    constexpr int RB = K + D + 1;  // b planes: j-K .. j+D
    constexpr int NB = D + 1;      // barriers: planes j .. j+D
    constexpr int PLANE = W * HH;
    constexpr int SEGS = W / 32;
    constexpr int NWARPS = NT / 32;
    static_assert(W % 32 == 0 && TX > 0 && TY > 0, "tile shape");

    extern __shared__ __align__(128) float smem[];
    float* xs = smem;                 // R planes
    float* bs = smem + R * PLANE;     // RB planes
    uint64_t* bars = reinterpret_cast<uint64_t*>(bs + RB * PLANE);

    const Dims d = a.d;
    const int x0 = static_cast<int>(blockIdx.x) * TX;
    const int y0 = static_cast<int>(blockIdx.y) * TY;
    const int z0 = static_cast<int>(blockIdx.z) * a.z_chunk;
    if (z0 >= d.nz) return;
    const int z1 = min(z0 + a.z_chunk, d.nz);
    const int xo = x0 - HX, yo = y0 - K;  // plane origin in grid coordinates
    const bool px = a.g.periodic[0] != 0, py = a.g.periodic[1] != 0, pz = a.g.periodic[2] != 0;
    const int k_run = a.k_run;
    const int zs = pz ? z0 - k_run : max(z0 - k_run, 0);
    const int ze = pz ? z1 - 1 + k_run : min(z1 - 1 + k_run, d.nz - 1);  // inclusive
    const int nplanes = ze - zs + 1;
    const bool wraps = (px && (xo < 0 || xo + W > d.nx)) || (py && (yo < 0 || yo + HH > d.ny));
    const bool use_tma = a.tma_ok && !wraps;
    const bool zero_x = a.src == nullptr;
    const int tid = static_cast<int>(threadIdx.x);
    const int warp = tid >> 5, lane = tid & 31;

    if (tid == 0) {
        for (int i = 0; i < NB; ++i) tb::mbar_init(&bars[i], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    auto plane_z = [&](int pi) {  // grid z of stream plane pi
        int z = zs + pi;
        return pz ? wrap_index(z, d.nz) : z;
    };

    // Enqueue the loads of stream plane pi (x into its ring slot, b into its).
    auto issue = [&](int pi) {
        if (pi >= nplanes) {
            if (!use_tma) tb::cp_async_commit();
            return;
        }
        float* xdst = xs + (pi % R) * PLANE;
        float* bdst = bs + (pi % RB) * PLANE;
        const int z = plane_z(pi);
        if (zero_x)
            for (int i = tid; i < PLANE; i += NT) xdst[i] = 0.0f;
        if (use_tma) {
            if (tid == 0) {
                tb::fence_proxy_async();
                uint64_t* bar = &bars[pi % NB];
                tb::mbar_expect_tx(bar, (zero_x ? 1u : 2u) * PLANE * 4u);
                if (!zero_x) tb::tma_load_plane(xdst, &map_x, xo, yo, z, bar);
                tb::tma_load_plane(bdst, &map_b, xo, yo, z, bar);
            }
        } else {
            const size_t zoff = static_cast<size_t>(z) * d.ny * d.nx;
            for (int i = tid; i < PLANE; i += NT) {
                int gx = xo + i % W, gy = yo + i / W;
                if (px) gx = wrap_index(gx, d.nx);
                if (py) gy = wrap_index(gy, d.ny);
                const bool in = static_cast<unsigned>(gx) < static_cast<unsigned>(d.nx) && static_cast<unsigned>(gy) < static_cast<unsigned>(d.ny);
                const size_t off = in ? zoff + static_cast<size_t>(gy) * d.nx + gx : 0;
                if (!zero_x) tb::cp_async4(xdst + i, a.src + off, in);
                tb::cp_async4(bdst + i, a.b + off, in);
            }
            tb::cp_async_commit();
        }
    };

    for (int p = 0; p < D && p < nplanes; ++p) issue(p);
    if (!use_tma)
        for (int p = nplanes; p < D; ++p) tb::cp_async_commit();

    const int row_lo_x = HX - K;  // first column inside the dependency cone
    for (int j = 0; j < nplanes + k_run; ++j) {
        // prefetch plane j + D (its slots held planes no longer needed)
        issue(j + D);
        if (j < nplanes) {
            if (use_tma) {
                if (!tb::mbar_wait(&bars[j % NB], static_cast<unsigned>((j / NB) & 1))) {
                    if (tid == 0) atomicExch(a.error, 1u);
                    return;
                }
            } else {
                tb::cp_async_wait<D>();
            }
        }
        __syncthreads();

        for (int s = 1; s <= k_run; ++s) {
            const int pi = j - s;
            if (pi >= 0 && pi < nplanes) {
                const int colour = (s - 1) & 1;
                const int gz = plane_z(pi);
                float* P = xs + (pi % R) * PLANE;
                const float* Pm = xs + ((pi + R - 1) % R) * PLANE;
                const float* Pp = xs + ((pi + 1) % R) * PLANE;
                const float* B = bs + (pi % RB) * PLANE;
                const bool gz_lo = !pz && gz == 0, gz_hi = !pz && gz == d.nz - 1;
                const int rows = HH - 2 * s;
                const int tasks = ((rows + 1) >> 1) * SEGS;
                for (int t = warp; t < tasks; t += NWARPS) {
                    const int row = s + 2 * (t / SEGS) + (lane >> 4);
                    const int seg = t % SEGS;
                    const int gy = yo + row;
                    const int h = (colour + gy + gz) & 1;  // x parity of this colour in this row (xo is even)
                    const int lx = 32 * seg + 2 * (lane & 15) + h;
                    const int gx = xo + lx;
                    if (row >= HH - s || lx < row_lo_x + s || lx >= W - row_lo_x - s) continue;
                    if (!px && static_cast<unsigned>(gx) >= static_cast<unsigned>(d.nx)) continue;
                    if (!py && static_cast<unsigned>(gy) >= static_cast<unsigned>(d.ny)) continue;
                    const int c = row * W + lx;
                    const float self = P[c];
                    const float xm = (!px && gx == 0) ? tb::ghost<KIND>(a.g, XM, self) : P[c - 1];
                    const float xp = (!px && gx == d.nx - 1) ? tb::ghost<KIND>(a.g, XP, self) : P[c + 1];
                    const float ym = (!py && gy == 0) ? tb::ghost<KIND>(a.g, YM, self) : P[c - W];
                    const float yp = (!py && gy == d.ny - 1) ? tb::ghost<KIND>(a.g, YP, self) : P[c + W];
                    const float zm = gz_lo ? tb::ghost<KIND>(a.g, ZM, self) : Pm[c];
                    const float zp = gz_hi ? tb::ghost<KIND>(a.g, ZP, self) : Pp[c];
                    const float nb = xm + xp + ym + yp + zm + zp;
                    P[c] = tb::update<KIND>(nb, B[c], a.coef);
                }
            }
            __syncthreads();
        }

        // plane j - k_run is final: write its interior
        const int q = j - k_run;
        if (q >= 0 && q < nplanes) {
            const int zq = zs + q;
            if (zq >= z0 && zq < z1) {
                const float* P = xs + (q % R) * PLANE;
                const size_t zoff = static_cast<size_t>(zq) * d.ny * d.nx;
                if (use_tma) {  // rows 16-byte aligned: float4 stores
                    constexpr int V = TX / 4;
                    for (int i = tid; i < TY * V; i += NT) {
                        const int row = K + i / V, lx = HX + 4 * (i % V);
                        const int gx = xo + lx, gy = yo + row;
                        if (gy >= d.ny || gx >= d.nx) continue;
                        float4 v = *reinterpret_cast<const float4*>(P + row * W + lx);
                        v.x *= a.out_scale;
                        v.y *= a.out_scale;
                        v.z *= a.out_scale;
                        v.w *= a.out_scale;
                        *reinterpret_cast<float4*>(a.dst + zoff + static_cast<size_t>(gy) * d.nx + gx) = v;
                    }
                } else {
                    for (int i = tid; i < TY * TX; i += NT) {
                        const int row = K + i / TX, lx = HX + i % TX;
                        const int gx = xo + lx, gy = yo + row;
                        if (gy >= d.ny || gx >= d.nx) continue;
                        a.dst[zoff + static_cast<size_t>(gy) * d.nx + gx] = P[row * W + lx] * a.out_scale;
                    }
                }
            }
        }
        __syncthreads();
    }
    if (!use_tma) tb::cp_async_wait<0>();
}

}  // namespace sfb
