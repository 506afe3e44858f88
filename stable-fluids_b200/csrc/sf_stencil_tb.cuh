// sf_stencil_tb.cuh -- temporally blocked red-black Gauss-Seidel pass.
//
// One launch runs k_run colour half-sweeps (k_run/2 full RBGS iterations)
// over the whole field while reading x and b from HBM once and writing x
// once: 12 B per cell per pass instead of ~12 B per cell per half-sweep.
//
// Tiling (2.5D): each CTA owns an xy tile of TX x TY output cells and a chunk
// of planes. It loads the tile plus a halo of HX (x, a multiple of 4 cells for
// 16-byte TMA alignment) and K (y) cells, and streams its planes (plus k_run
// halo planes at each chunk end) through a ring of shared-memory planes, ZP
// planes per time step. At time step j colour stage s (s = 1..k_run) updates
// planes ZP*j - s - k (k = 0..ZP-1) in place:
//   - stage s-1 finished plane ZP*j - s + 1 earlier in the same time step,
//   - stage s+1 has not yet touched the planes below,
// so every stage reads exactly the values the global half-sweep would see.
// Each stage shrinks the region of correct values by one cell in x and y (and
// one plane at each chunk end), which the halo absorbs. The updates use the
// reference's arithmetic (backend-cuda.cu:354-375, 398-407), so the result
// equals k_run/2 reference iterations bit for bit.
//
// Work split: warp w owns x segment w % 3 (32 columns) and every PG-th row
// pair from w / 3; lanes 0-15 take the lower row of a pair, lanes 16-31 the
// upper one, each lane the cell of the stage's colour in its column pair.
// Because the row pitch W is even and adjacent rows hold opposite colours,
// the 32 lanes hit 32 distinct banks for the cell, its x, y, z neighbours and
// b: no bank conflicts on a plain row-major plane, which is what a TMA box
// writes. Within a stage every load reads the other colour and every store
// writes this colour, so a lane issues all loads of the stage first, then
// computes, then stores; all addresses are immediate offsets from one base
// per plane.
//
// Boundaries: x/y ghost values are written into the halo cells just outside
// the domain before each stage (fill_ghosts); z ghosts are applied on the
// first and last plane of a non-periodic z axis. Periodic axes need no
// ghosts: the halo holds the wrapped cells.
//
// Loads: one elected thread issues a 3D TMA box per plane for x and for b
// (cp.async.bulk.tensor, mbarrier completion, D time steps ahead). CTAs whose
// halo wraps around a periodic x or y boundary (a TMA box fills outside the
// tensor instead of wrapping) and grids whose rows are not 16-byte aligned
// load with cp.async instead. The mbarrier wait is bounded: on timeout the
// kernel sets an error flag and returns.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include "sf_device.cuh"
#include "sf_launch.h"

namespace sfb {

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

#ifdef SFB_TB_PROFILE
// Per-CTA cycle counters of a profiling build: [0] waits, [1] stages,
// [2] output, [3] TMA path used, [4] time steps.
__device__ unsigned long long g_tb_profile[4096][5];
#define SFB_TB_MARK(var) const long long var = clock64()
#define SFB_TB_ADD(slot, from) \
    if (threadIdx.x == 0) g_tb_profile[blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)][slot] += clock64() - (from)
#else
#define SFB_TB_MARK(var)
#define SFB_TB_ADD(slot, from)
#endif

namespace tb {

constexpr int kPrefetch = 2;  // time steps of loads in flight ahead of the one consumed
constexpr int kSlackFloats = 1536;  // read-only slack after the rings for masked lanes

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

__device__ __forceinline__ float ghost(const GhostRule& g, int face, float self) {
    const int m = g.mode[face];
    if (m == GHOST_COPY) return self;
    if (m == GHOST_CONST) return g.k[face];
    return g.k[face] - self;
}

// Correctly rounded FP32 n / d for every FP32 n and the stencil divisors:
// the quotient is formed in FP64 by Markstein's correction (P. Markstein,
// IBM J. Res. Dev. 34(1), 1990) from y = RN64(1 / d) -- q = RN(n y),
// r = n - q d (exact with an FMA), q' = RN(q + r y) = RN64(n / d) -- and
// rounded once to FP32. For a normal FP32 quotient that double rounding is
// innocuous (53 >= 2 * 24 + 2; S. Figueroa, "When is double rounding
// innocuous?", SIGNUM Newsl. 30(3), 1995). For a quotient in the subnormal
// range, an exact FP32 midpoint n / d is representable in FP64 and every
// other quotient lies at least 2^-175 from a midpoint, farther than the FP64
// error (<= 2^-179), so the FP32 rounding is right there too. Checked against
// IEEE FP32 division for all finite FP32 numerators with d = 6 and with
// diffusion divisors 1 + 6 alpha. There is no data-dependent branch: tiny and
// subnormal numerators (common where a field decays to zero) cost the same as
// any other, and B200 issues FP64 FMAs at half its FP32 rate. Zeros keep
// their sign.
__device__ __forceinline__ double recip64(float d) { return __drcp_rn(static_cast<double>(d)); }

__device__ __forceinline__ float divide(float n, float d, double y) {
    const double a = static_cast<double>(n);
    const double q = __dmul_rn(a, y);
    const double r = __fma_rn(-q, static_cast<double>(d), a);
    const double q1 = __fma_rn(r, y, q);
    return n == 0.0f ? n : __double2float_rn(q1);
}

// Numerator of the update in the reference's expression shape
// (backend-cuda.cu:363, :406), so the compiler fuses it the same way.
template <int KIND>
__device__ __forceinline__ float numerator(float nb, float rhs, float coef) {
    if constexpr (KIND == KIND_PRESSURE) return nb - coef * rhs;
    else return rhs + coef * nb;
}

}  // namespace tb

// CTA-uniform values of one (stage, plane) of a time step.
struct Combo {
    int x, xm, xp, b;  // ring offsets (floats) of the plane, its z neighbours and its b plane; x < 0: no plane
    int parity;        // x parity of the stage's colour in the tile's even rows
    int zflags;        // 1: first plane of a non-periodic z axis, 2: last plane
    int pad0, pad1;
};

// One colour stage for one warp: NPL planes x MP row pairs, loads first,
// then the updates, then predicated stores.
template <int KIND, int W, int MP, int PG, int NPL>
__device__ __forceinline__ void stage_all(const Combo* combo, float* xs, const float* bs, int s, int npairs, int pg, int hi, int lane_off, int lx_lane, int lo_x, bool mask_x, int gx_base, int nx, bool mask_y, int gy_base, int ny, const TbArgs& a,
                                          float divisor, double recip) {
    constexpr int STEP = 2 * PG * W;  // floats between this lane's row pairs
    float num[NPL][MP];
    float* cell[NPL];
    bool lane_ok[NPL];
#pragma unroll
    for (int k = 0; k < NPL; ++k) {
        const Combo e = combo[k];
        const bool plane_ok = e.x >= 0;
        const int par = e.parity ^ hi;
        const int c0 = lane_off + s * W + par;  // this lane's first cell
        const int lx = lx_lane + par;
        bool ok = plane_ok && lx >= lo_x + s && lx < W - lo_x - s;
        if (mask_x) ok = ok && static_cast<unsigned>(gx_base + par) < static_cast<unsigned>(nx);
        lane_ok[k] = ok;
        const float* P = xs + (plane_ok ? e.x : 0) + c0;
        const float* Pm = xs + (plane_ok ? e.xm : 0) + c0;
        const float* Pp = xs + (plane_ok ? e.xp : 0) + c0;
        const float* B = bs + (plane_ok ? e.b : 0) + c0;
        cell[k] = xs + (plane_ok ? e.x : 0) + c0;
        if (e.zflags == 0) {  // CTA-uniform
#pragma unroll
            for (int m = 0; m < MP; ++m) {
                const int o = m * STEP;
                const float nb = P[o - 1] + P[o + 1] + P[o - W] + P[o + W] + Pm[o] + Pp[o];
                num[k][m] = tb::numerator<KIND>(nb, B[o], a.coef);
            }
        } else {
            const bool zlo = (e.zflags & 1) != 0, zhi = (e.zflags & 2) != 0;
#pragma unroll
            for (int m = 0; m < MP; ++m) {
                const int o = m * STEP;
                const float self = P[o];
                const float zm = zlo ? tb::ghost(a.g, ZM, self) : Pm[o];
                const float zp = zhi ? tb::ghost(a.g, ZP, self) : Pp[o];
                const float nb = P[o - 1] + P[o + 1] + P[o - W] + P[o + W] + zm + zp;
                num[k][m] = tb::numerator<KIND>(nb, B[o], a.coef);
            }
        }
    }
#pragma unroll
    for (int k = 0; k < NPL; ++k)
#pragma unroll
        for (int m = 0; m < MP; ++m) {
            const int pair = pg + PG * m;
            bool ok = lane_ok[k] && pair < npairs;
            if (mask_y) ok = ok && static_cast<unsigned>(gy_base + s + 2 * PG * m) < static_cast<unsigned>(ny);
            const float q = tb::divide(num[k][m], divisor, recip);
            if (ok) cell[k][m * STEP] = q;
        }
}

// Writes the x/y ghost values of the boundary cells of one colour into the
// halo cells just outside the domain (non-periodic faces only). A ghost cell
// is the face neighbour of exactly one domain cell, so it can hold that
// cell's ghost value (a function of the cell itself: copy, constant or
// reflection, backend-cuda.cu:62-189 for a face neighbour) for as long as the
// cell keeps its value, i.e. until the stage that updates it.
template <int W, int HH>
__device__ __forceinline__ void fill_ghosts(float* P, int gz, int colour, int xo, int yo, const TbArgs& a, int tid, int nt) {
    const Dims& d = a.d;
    const bool px = a.g.periodic[0] != 0, py = a.g.periodic[1] != 0;
    if (!px) {
        const int lb0 = -xo, lb1 = d.nx - 1 - xo;  // local columns of x = 0 and x = nx - 1
        const bool lo = lb0 >= 1 && lb0 < W, hi = lb1 >= 0 && lb1 + 1 < W;
        if (lo || hi)
            for (int row = tid; row < HH; row += nt) {
                const int gy = yo + row;
                if (!py && static_cast<unsigned>(gy) >= static_cast<unsigned>(d.ny)) continue;
                if (lo && ((gy + gz) & 1) == colour) P[row * W + lb0 - 1] = tb::ghost(a.g, XM, P[row * W + lb0]);
                if (hi && ((d.nx - 1 + gy + gz) & 1) == colour) P[row * W + lb1 + 1] = tb::ghost(a.g, XP, P[row * W + lb1]);
            }
    }
    if (!py) {
        const int rb0 = -yo, rb1 = d.ny - 1 - yo;  // local rows of y = 0 and y = ny - 1
        const bool lo = rb0 >= 1 && rb0 < HH, hi = rb1 >= 0 && rb1 + 1 < HH;
        if (lo || hi)
            for (int lx = tid; lx < W; lx += nt) {
                const int gx = xo + lx;
                if (!px && static_cast<unsigned>(gx) >= static_cast<unsigned>(d.nx)) continue;
                if (lo && ((gx + gz) & 1) == colour) P[(rb0 - 1) * W + lx] = tb::ghost(a.g, YM, P[rb0 * W + lx]);
                if (hi && ((gx + d.ny - 1 + gz) & 1) == colour) P[(rb1 + 1) * W + lx] = tb::ghost(a.g, YP, P[rb1 * W + lx]);
            }
    }
}

// Shared memory of one CTA: x ring, b ring, read-only slack (masked lanes
// may read past the last plane), barriers, combo table, abort flag.
template <int K, int W, int HH, int ZP>
struct TbLayout {
    static constexpr int D = tb::kPrefetch;
    static constexpr int R = ZP * D + 2 * ZP + K;  // x planes resident or in flight
    static constexpr int RB = R - 1;               // b planes
    static constexpr int NB = D + 1;               // one barrier per time step in flight
    static constexpr int PLANE = W * HH;
    static constexpr size_t slack_off = static_cast<size_t>(R + RB) * PLANE * 4;
    static constexpr size_t bars_off = slack_off + tb::kSlackFloats * 4;
    static constexpr size_t combo_off = bars_off + 8 * ((NB + 1) / 2 * 2);
    static constexpr size_t abort_off = combo_off + sizeof(Combo) * K * ZP;
    static constexpr size_t bytes = abort_off + 16;
};

// K: halo (max colour half-sweeps per pass); W, HH: loaded plane size;
// ZP: planes per time step; NT: threads per CTA.
template <int KIND, int K, int W, int HH, int ZP, int NT>
__global__ void __launch_bounds__(NT, 1) k_rbgs_tb(const __grid_constant__ CUtensorMap map_x, const __grid_constant__ CUtensorMap map_b, TbArgs a) {
    using L = TbLayout<K, W, HH, ZP>;
    constexpr int HX = ((K + 3) / 4) * 4;
    constexpr int TX = W - 2 * HX;
    constexpr int TY = HH - 2 * K;
    constexpr int D = L::D, R = L::R, RB = L::RB, NB = L::NB, PLANE = L::PLANE;
    constexpr int SEGS = W / 32;
    constexpr int NWARPS = NT / 32;
    constexpr int PG = NWARPS / SEGS;
    constexpr int MP = ((HH - 2) / 2 + PG - 1) / PG;  // row pairs per warp per stage, at most
    static_assert(W % 32 == 0 && TX > 0 && TY > 0 && TX % 4 == 0 && HH % 2 == 0, "tile shape");
    static_assert(NWARPS % SEGS == 0, "warps must split evenly over x segments");
    // a masked lane reads at most row 2 PG MP + K of a plane (its last pair's
    // upper row plus one): that many rows must fit in a plane plus the slack
    static_assert((2 * PG * MP + K + 1) * W <= PLANE + tb::kSlackFloats, "slack for masked reads");

    extern __shared__ __align__(128) float smem[];
    float* xs = smem;
    float* bs = smem + R * PLANE;
    char* base = reinterpret_cast<char*>(smem);
    uint64_t* bars = reinterpret_cast<uint64_t*>(base + L::bars_off);
    Combo* combo = reinterpret_cast<Combo*>(base + L::combo_off);
    int* abort_flag = reinterpret_cast<int*>(base + L::abort_off);

    const Dims d = a.d;
    const int x0 = static_cast<int>(blockIdx.x) * TX;
    const int y0 = static_cast<int>(blockIdx.y) * TY;
    const int z0 = static_cast<int>(blockIdx.z) * a.z_chunk;
    if (z0 >= d.nz) return;
    const int z1 = min(z0 + a.z_chunk, d.nz);
    const int xo = x0 - HX, yo = y0 - K;
    const bool px = a.g.periodic[0] != 0, py = a.g.periodic[1] != 0, pz = a.g.periodic[2] != 0;
    const int k_run = a.k_run;
    const int zs = pz ? z0 - k_run : max(z0 - k_run, 0);
    const int ze = pz ? z1 - 1 + k_run : min(z1 - 1 + k_run, d.nz - 1);
    const int nplanes = ze - zs + 1;
    const bool out_x = xo < 0 || xo + W > d.nx, out_y = yo < 0 || yo + HH > d.ny;
    const bool wraps = (px && out_x) || (py && out_y);
    const bool mask_x = !px && out_x, mask_y = !py && out_y;
    const bool fill = mask_x || mask_y;
    const bool use_tma = a.tma_ok && !wraps;
    const bool zero_x = a.src == nullptr;
    const int tid = static_cast<int>(threadIdx.x);
    const int warp = tid >> 5, lane = tid & 31;
    const float divisor = KIND == KIND_PRESSURE ? 6.0f : 1.0f + 6.0f * a.coef;
    const double recip = tb::recip64(divisor);

    if (tid == 0) {
        for (int i = 0; i < NB; ++i) tb::mbar_init(&bars[i], 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // the slack is read by masked lanes only; keep it finite
    for (int i = tid; i < tb::kSlackFloats; i += NT) reinterpret_cast<float*>(base + L::slack_off)[i] = 0.0f;
    __syncthreads();

    auto plane_z = [&](int pi) {
        const int z = zs + pi;
        return pz ? wrap_index(z, d.nz) : z;
    };

    // Enqueue the loads of time step `step` (stream planes ZP*step ..).
    auto issue = [&](int step) {
        const int first = ZP * step;
        if (first >= nplanes) {
            if (!use_tma) tb::cp_async_commit();
            return;
        }
        const int count = min(ZP, nplanes - first);
        if (zero_x)
            for (int k = 0; k < count; ++k) {
                float* xdst = xs + ((first + k) % R) * PLANE;
                for (int i = tid; i < PLANE; i += NT) xdst[i] = 0.0f;
            }
        if (use_tma) {
            if (tid == 0) {
                tb::fence_proxy_async();
                uint64_t* bar = &bars[step % NB];
                tb::mbar_expect_tx(bar, static_cast<unsigned>(count) * (zero_x ? 1u : 2u) * PLANE * 4u);
                for (int k = 0; k < count; ++k) {
                    const int pi = first + k, z = plane_z(pi);
                    if (!zero_x) tb::tma_load_plane(xs + (pi % R) * PLANE, &map_x, xo, yo, z, bar);
                    tb::tma_load_plane(bs + (pi % RB) * PLANE, &map_b, xo, yo, z, bar);
                }
            }
        } else {
            for (int k = 0; k < count; ++k) {
                const int pi = first + k;
                float* xdst = xs + (pi % R) * PLANE;
                float* bdst = bs + (pi % RB) * PLANE;
                const size_t zoff = static_cast<size_t>(plane_z(pi)) * d.ny * d.nx;
                for (int i = tid; i < PLANE; i += NT) {
                    int gx = xo + i % W, gy = yo + i / W;
                    if (px) gx = wrap_index(gx, d.nx);
                    if (py) gy = wrap_index(gy, d.ny);
                    const bool in = static_cast<unsigned>(gx) < static_cast<unsigned>(d.nx) && static_cast<unsigned>(gy) < static_cast<unsigned>(d.ny);
                    const size_t off = in ? zoff + static_cast<size_t>(gy) * d.nx + gx : 0;
                    if (!zero_x) tb::cp_async4(xdst + i, a.src + off, in);
                    tb::cp_async4(bdst + i, a.b + off, in);
                }
            }
            tb::cp_async_commit();
        }
    };

    // fixed work split and per-lane constants
    const int seg = warp % SEGS, pg = warp / SEGS, hi = lane >> 4;
    const int lx_lane = 32 * seg + 2 * (lane & 15);
    const int lane_off = (hi + 2 * pg) * W + lx_lane;  // row hi + 2 pg, column lx_lane
    const int lo_x = HX - K;                           // first column inside the dependency cone
    const int gx_base = xo + lx_lane;
    const int gy_base = yo + hi + 2 * pg;

    // ghost cells for colour stage t of time step jj (its planes are resident)
    auto fill_stage = [&](int jj, int t) {
#pragma unroll
        for (int k = 0; k < ZP; ++k) {
            const int pi = ZP * jj - t - k;
            if (pi < 0 || pi >= nplanes) continue;
            fill_ghosts<W, HH>(xs + (pi % R) * PLANE, plane_z(pi), (t - 1) & 1, xo, yo, a, tid, NT);
        }
    };

    const int steps = (nplanes - 1 + k_run + ZP - 1) / ZP + 1;  // the last plane leaves stage k_run at step ceil((nplanes-1+k_run)/ZP)
    for (int t = 0; t < D; ++t) issue(t);

    for (int j = 0; j < steps; ++j) {
        issue(j + D);
        // table of the CTA-uniform values of each (stage, plane) of this step
        if (tid < k_run * ZP) {
            const int s = tid / ZP + 1, k = tid % ZP;
            const int pi = ZP * j - s - k;
            Combo e{-1, 0, 0, 0, 0, 0, 0, 0};
            if (pi >= 0 && pi < nplanes) {
                const int gz = plane_z(pi);
                e.x = (pi % R) * PLANE;
                e.xm = ((pi + R - 1) % R) * PLANE;
                e.xp = ((pi + 1) % R) * PLANE;
                e.b = (pi % RB) * PLANE;
                e.parity = ((s - 1) + yo + s + gz) & 1;  // colour + y parity of row s + z
                e.zflags = (!pz && gz == 0 ? 1 : 0) | (!pz && gz == d.nz - 1 ? 2 : 0);
            }
            combo[tid] = e;
        }
        SFB_TB_MARK(t_wait);
        if (ZP * j < nplanes) {
            if (use_tma) {
                // one thread polls; the barrier below publishes the data
                if (tid == 0 && !tb::mbar_wait(&bars[j % NB], static_cast<unsigned>((j / NB) & 1))) {
                    atomicExch(a.error, 1u);
                    *abort_flag = 1;
                }
            } else {
                tb::cp_async_wait<D>();
            }
        }
        __syncthreads();
        if (*abort_flag) return;
        SFB_TB_ADD(0, t_wait);
        SFB_TB_MARK(t_stage);

        for (int s = 1; s <= k_run; ++s) {
            const int npairs = (HH - 2 * s) >> 1;
            stage_all<KIND, W, MP, PG, ZP>(combo + (s - 1) * ZP, xs, bs, s, npairs, pg, hi, lane_off, lx_lane, lo_x, mask_x, gx_base, d.nx, mask_y, gy_base, d.ny, a, divisor, recip);
            // the next stage's colour is untouched by this one: fill its ghosts now
            if (fill && s < k_run) fill_stage(j, s + 1);
            __syncthreads();
        }
        SFB_TB_ADD(1, t_stage);
        SFB_TB_MARK(t_out);

        // ghosts of the first stage of the next time step (its planes arrived
        // in this one); the output below reads other planes
        if (fill) fill_stage(j + 1, 1);
        // planes ZP*j - k_run - k are final: write their interiors
#pragma unroll
        for (int k = 0; k < ZP; ++k) {
            const int q = ZP * j - k_run - k;
            if (q < 0 || q >= nplanes) continue;
            const int zq = zs + q;
            if (zq < z0 || zq >= z1) continue;
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
        __syncthreads();
        SFB_TB_ADD(2, t_out);
    }
#ifdef SFB_TB_PROFILE
    if (threadIdx.x == 0) {
        g_tb_profile[blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)][3] = use_tma;
        g_tb_profile[blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)][4] += steps;
    }
#endif
    if (!use_tma) tb::cp_async_wait<0>();
}

}  // namespace sfb
