// sf_unet_tc.cuh -- 3x3x3 convolution of the warm-start network on the
// 5th-generation tensor cores: tcgen05.mma (BF16 x BF16 -> FP32) with the
// accumulators in tensor memory, operands brought into shared memory by TMA.
//
// Implicit GEMM. A CTA owns an output tile of TX = 32 columns x TY rows of
// ZO consecutive z planes. The input halo of the tile (ZO + 2 planes x
// (TY + 2) rows x P = TX + 2 columns) is stored per 8-channel chunk as rows
// of 16 bytes, row index r = hy * P + hx -- exactly the order in which a TMA
// box of 8 channels x P x (TY + 2) voxels lands -- so that the halo row of
// output voxel (y, x) shifted by tap (dy, dx) is r = m + dy * P + dx with
// m = y * P + x: the A operand of one in-plane shift is a contiguous run of
// rows. GEMM row m walks the tile with a pitch of P (the two extra columns per
// row are computed and dropped), and M-blocks of 128 rows cover TY * P rows.
// In the no-swizzle K-major canonical layout that is a descriptor with 16-byte
// rows, 128-byte core-matrix groups (SBO) and the chunk stride as LBO, whose
// start address moves by 16 bytes per row of shift.
//
// Several output planes per MMA. Input plane ip (z = z0 - 1 + ip) meets
// output plane o (z = z0 + o) through tap dz = ip - o, so one MMA per input
// plane and in-plane shift (dy, dx) serves every output plane o with
// 0 <= ip - o <= 2 at once: its B operand stacks the weights of those taps
// (N = COUT per plane) and its D columns are those planes' accumulators. The
// weights are kept as [dy][dx][dz][cout] rows per 8-channel chunk, so the
// taps of one (dy, dx) are adjacent rows; output plane o's accumulator sits at
// column (ZO - 1 - o) * COUT, so increasing dz meets increasing columns. Each
// output still sums its taps in (dz, dy, dx) order, one K = 16 MMA step per
// tap and channel group. Every MMA reads its 4 KB A tile from shared memory
// whatever its N, so wider MMAs amortise it: layers with COUT = 16 use ZO = 4
// (tiles of 32 x 7 x 4 voxels, 1.8x fewer MMAs per voxel than one plane of
// 32 x 15); wider layers use ZO = 1.
//
// Channels are processed in groups of 16 (one K = 16 MMA step); a pipeline
// item is (tile, group). Warp-specialised, persistent CTA (one per SM):
//   warp 0 (one thread) : TMA loads of items into S shared-memory stages
//                         (and of the weights, once, when they fit);
//   warp 1              : walks the items as a converged warp; one elected
//                         lane issues (ZO + 2) x 9 x M-blocks MMAs per item
//                         (fully unrolled, compile-time operand offsets) into
//                         one of two TMEM accumulator buffers, and
//                         tcgen05.commit to release the stage and, after a
//                         tile's last group, its buffer;
//   warps 2-5           : epilogue -- tcgen05.ld of the accumulators (warp w
//                         reads TMEM lanes 32 (w % 4) .. +31), bias,
//                         activation, channels-last BF16 (or FP32 channel 0)
//                         stores -- overlapping the next tile's MMAs.
// Every wait on an mbarrier is bounded; a role that gives up raises a shared
// abort flag, so the others stop too, and records the failure in *error
// (results are then invalid) instead of hanging the GPU.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "sf_types.h"

namespace sfb::net::tc {

constexpr int TX = 32, P = TX + 2;
constexpr uint32_t kSpinLimit = 1u << 26;

template <int TY>
struct Geo {
    static constexpr int MB = (TY * P + 127) / 128;                    // M blocks of 128 GEMM rows
    static constexpr int HALO_ROWS = (TY + 2) * P;                      // rows holding input data
    static constexpr int R = ((MB * 128 + 2 * P + 2) + 7) / 8 * 8;      // rows per plane chunk (reads stay inside)
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) { asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory"); }
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    return done != 0;
}
// Bounded wait. Gives up (false) after kSpinLimit polls or as soon as
// another role of the CTA has given up (*abort); the first to give up sets
// *abort and records the failure in *error.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int* abort, unsigned* error) {
    for (uint32_t i = 0; i < kSpinLimit; ++i) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((i & 1023u) == 1023u && *abort) return false;
    }
    *abort = 1;
    if (error) atomicOr(error, 2u);
    return false;
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) { asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) { asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory"); }

__device__ __forceinline__ void tma_load_4d(uint32_t dst, const CUtensorMap* map, int c0, int c1, int c2, int c3, uint32_t bar) {
    asm volatile("cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(bar)
                 : "memory");
}
__device__ __forceinline__ void tma_load_5d(uint32_t dst, const CUtensorMap* map, int c0, int c1, int c2, int c3, int c4, uint32_t bar) {
    asm volatile("cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(bar)
                 : "memory");
}

// The weights of one 8-channel chunk c (input channels 8c .. 8c + 7) into
// shared memory as rows [dy][dx][dz][cout]: one box of the 3 dz taps per
// (dy, dx). The tensor map views the [dz][dy][dx][cout][cin] weights as
// (cin, cout, dx, dy, dz).
__device__ __forceinline__ void tma_load_weight_chunk(uint32_t dst, const CUtensorMap* map, int c, uint32_t box_bytes, uint32_t bar) {
    for (int dy = 0; dy < 3; ++dy)
        for (int dx = 0; dx < 3; ++dx) tma_load_5d(dst + static_cast<uint32_t>(dy * 3 + dx) * box_bytes, map, c * 8, 0, dx, dy, 0, bar);
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// No-swizzle K-major shared-memory matrix descriptor (sm_100 format).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return static_cast<uint64_t>((addr & 0x3FFFFu) >> 4) | (static_cast<uint64_t>((lbo & 0x3FFFFu) >> 4) << 16) | (static_cast<uint64_t>((sbo & 0x3FFFFu) >> 4) << 32) | (1ull << 46);
}

// Instruction descriptor: kind::f16, A = B = BF16 (K-major), D = F32, M = 128.
// N must be a multiple of 16 in [16, 256].
__host__ __device__ constexpr uint32_t instr_desc(uint32_t n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((n >> 3) << 17) | (static_cast<uint32_t>(128 >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        :
        : "r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
        : "memory");
}
__device__ __forceinline__ void mma_commit(uint32_t bar) { asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory"); }

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                 : "r"(taddr)
                 : "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// One lane of a converged warp (elect.sync over the full mask).
__device__ __forceinline__ bool elect_one() {
    uint32_t pred;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "elect.sync _|p, 0xffffffff;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(pred));
    return pred != 0;
}

enum Epilogue : int { RELU_BF16 = 0, LINEAR_BF16 = 1, LINEAR_F32_CH0 = 2 };

// Shared-memory plan of one (CIN, COUT) convolution. ZO output planes per
// tile (ZO + 2 input planes per stage). The weights of all taps and channels
// stay resident when they fit beside two input stages; otherwise each stage
// carries the weights of its channel group. TY = 15 (4 M-blocks) when it
// fits, else 7 (2 M-blocks); three stages when they fit.
template <int CIN, int COUT>
struct Cfg {
    static constexpr int ZO = COUT == 16 ? 4 : 1;
    static constexpr int PLANES = ZO + 2;
    static constexpr int LIMIT = 232448 - 1024;
    static constexpr int W_ALL = 27 * CIN * COUT * 2;
    static constexpr int IN15 = 2 * PLANES * Geo<15>::R * 16, IN7 = 2 * PLANES * Geo<7>::R * 16;
    static constexpr bool RES = W_ALL + 2 * IN7 <= LIMIT;
    static constexpr int TY = (!RES || W_ALL + 2 * IN15 <= LIMIT) ? 15 : 7;
    static constexpr int MB = Geo<TY>::MB;
    static constexpr int R = Geo<TY>::R;
    static constexpr int PLANE_CHUNK = R * 16;               // one 8-channel chunk of one plane (a multiple of 128 bytes)
    static constexpr int IN = 2 * PLANES * PLANE_CHUNK;      // PLANES planes x 2 chunks
    static constexpr int WCHUNK = 27 * COUT * 16;            // one 8-channel chunk of all taps' weights, rows [dy][dx][dz][cout]
    static constexpr int STAGE = IN + (RES ? 0 : 2 * WCHUNK);
    static constexpr int S = (RES && W_ALL + 3 * IN <= LIMIT) ? 3 : 2;
    static constexpr int STAGE_OFF = RES ? W_ALL : 0;
    static constexpr int BAR_OFF = STAGE_OFF + S * STAGE;    // full[S], empty[S], acc_full[2], acc_empty[2], weights, tmem slot, abort
    static constexpr int BIAS_OFF = BAR_OFF + 128;
    static constexpr int BYTES = BIAS_OFF + COUT * 4;
    static constexpr int BOX_BYTES = 8 * 2 * P * (TY + 2);   // one input TMA box
    static constexpr int WBOX_BYTES = 8 * 2 * 3 * COUT;      // one weight TMA box: the 3 dz taps of one (dy, dx)
    static constexpr int ITEM_TX = 2 * PLANES * BOX_BYTES + (RES ? 0 : 2 * WCHUNK);
    static constexpr int TILE_COLS = ZO * COUT;              // accumulator columns of one M-block
    static constexpr int COLS = 2 * MB * TILE_COLS;          // two accumulator buffers
    static constexpr int ALLOC = COLS <= 32 ? 32 : COLS <= 64 ? 64 : COLS <= 128 ? 128 : COLS <= 256 ? 256 : 512;
    static_assert(BYTES <= 232448, "shared memory");
    static_assert(COLS <= 512, "tensor memory");
    static_assert(COUT % 16 == 0 && (ZO == 1 ? COUT : 3 * COUT) <= 256, "MMA N");
    static_assert(9 * WBOX_BYTES == WCHUNK && WBOX_BYTES % 128 == 0, "weight boxes fill a chunk, 128-byte aligned");
    static_assert(BOX_BYTES <= PLANE_CHUNK && PLANE_CHUNK % 128 == 0 && WCHUNK % 128 == 0 && W_ALL % 128 == 0 && STAGE % 128 == 0, "layout");
};

struct ConvArgs {
    void* out;                 // channels-last, out_ch channels (or FP32 channel 0)
    const float* bias;         // COUT (may be null)
    int out_ch, out_off;
    Dims d;
    int tiles_x, tiles_y, tiles_z;  // tiles per axis (tiles_z = ceil(nz / ZO))
    unsigned* error;
};

// The MMAs of one pipeline item (one tile, one 16-channel group), fully
// unrolled so that every operand is a compile-time offset from the stage,
// weight and accumulator bases. Input plane ip meets output planes
// o_lo .. o_hi through taps dz = ip - o; the block of plane o_hi = ip is
// written for the first time at shift (0, 0) of group 0 (`first`), so it
// gets its own MMA that overwrites instead of accumulating.
template <typename C, int COUT>
__device__ __forceinline__ void issue_item(uint64_t da0, uint64_t db0, uint32_t d0, bool first) {
    constexpr int ZO = C::ZO;
    const uint32_t acc0 = first ? 0u : 1u;
#pragma unroll
    for (int ip = 0; ip < C::PLANES; ++ip) {
        const int o_hi = ip < ZO - 1 ? ip : ZO - 1, o_lo = ip > 2 ? ip - 2 : 0;
        const int nblk = o_hi - o_lo + 1, dz_lo = ip - o_hi;
        const uint32_t col = static_cast<uint32_t>((ZO - 1 - o_hi) * COUT);
#pragma unroll
        for (int sh = 0; sh < 9; ++sh) {
            const int dy = sh / 3, dx = sh % 3;
            const uint64_t db = db0 + static_cast<uint64_t>((sh * 3 + dz_lo) * COUT);  // rows of 16 bytes
#pragma unroll
            for (int mb = 0; mb < C::MB; ++mb) {
                const uint64_t da = da0 + static_cast<uint64_t>(ip * 2 * (C::PLANE_CHUNK / 16) + mb * 128 + dy * P + dx);
                const uint32_t dm = d0 + static_cast<uint32_t>(mb * C::TILE_COLS) + col;
                if (o_hi == ip && sh == 0) {
                    mma_bf16(dm, da, db, instr_desc(COUT), acc0);
                    if (nblk > 1) mma_bf16(dm + COUT, da, db + COUT, instr_desc(static_cast<uint32_t>((nblk - 1) * COUT)), 1u);
                } else {
                    mma_bf16(dm, da, db, instr_desc(static_cast<uint32_t>(nblk * COUT)), 1u);
                }
            }
        }
    }
}

// Roles: warp 0 loads (one thread issues the TMA boxes), warp 1 issues the
// MMAs (the converged warp, one elected lane), warps 2..5 run the epilogue
// (warp w reads TMEM lanes 32 (w % 4) .. +31). Pipeline items are (tile,
// 16-channel group) in order; stage i % S holds item i; accumulator buffer
// k % 2 holds tile k.
constexpr int kThreadsTC = 192;

template <int CIN, int COUT, int EPI>
__global__ void __launch_bounds__(kThreadsTC, 1) k_conv3d_tc(const __grid_constant__ CUtensorMap map_in, const __grid_constant__ CUtensorMap map_w, ConvArgs a) {
    static_assert(CIN % 16 == 0, "channel groups of 16");
    using C = Cfg<CIN, COUT>;
    constexpr int GROUPS = CIN / 16;
    constexpr int S = C::S, MB = C::MB, TY = C::TY, ZO = C::ZO;
    extern __shared__ __align__(1024) unsigned char smem[];
    const int warp = static_cast<int>(threadIdx.x) >> 5, lane = static_cast<int>(threadIdx.x) & 31;
    const uint32_t sbase = smem_u32(smem);
    const uint32_t bars = sbase + C::BAR_OFF;
    const auto full = [&](int s) { return bars + 8u * static_cast<uint32_t>(s); };
    const auto empty = [&](int s) { return bars + 8u * static_cast<uint32_t>(S + s); };
    const auto acc_full = [&](int k) { return bars + 8u * static_cast<uint32_t>(2 * S + k); };
    const auto acc_empty = [&](int k) { return bars + 8u * static_cast<uint32_t>(2 * S + 2 + k); };
    const uint32_t wbar = bars + 8u * static_cast<uint32_t>(2 * S + 4);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + C::BAR_OFF + 8 * (2 * S + 5));
    volatile int* abort = reinterpret_cast<volatile int*>(smem + C::BAR_OFF + 8 * (2 * S + 5) + 4);
    float* bias_s = reinterpret_cast<float*>(smem + C::BIAS_OFF);

    // rows past the halo are read by the shifted A operands: zero them once
    for (int s = 0; s < S; ++s)
        for (int i = static_cast<int>(threadIdx.x); i < 2 * C::PLANES * (C::PLANE_CHUNK - C::BOX_BYTES) / 16; i += kThreadsTC) {
            const int chunk = i / ((C::PLANE_CHUNK - C::BOX_BYTES) / 16), r = i % ((C::PLANE_CHUNK - C::BOX_BYTES) / 16);
            *reinterpret_cast<uint4*>(smem + C::STAGE_OFF + s * C::STAGE + chunk * C::PLANE_CHUNK + C::BOX_BYTES + r * 16) = make_uint4(0, 0, 0, 0);
        }
    for (int c = static_cast<int>(threadIdx.x); c < COUT; c += kThreadsTC) bias_s[c] = a.bias ? a.bias[c] : 0.0f;
    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(full(s), 1);
            mbar_init(empty(s), 1);
        }
        for (int k = 0; k < 2; ++k) {
            mbar_init(acc_full(k), 1);
            mbar_init(acc_empty(k), 128);
        }
        mbar_init(wbar, 1);
        *abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)), "r"(static_cast<uint32_t>(C::ALLOC)) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_proxy_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    const int tiles = a.tiles_x * a.tiles_y * a.tiles_z;
    const int my_tiles = tiles > static_cast<int>(blockIdx.x) ? (tiles - 1 - static_cast<int>(blockIdx.x)) / static_cast<int>(gridDim.x) + 1 : 0;
    const int items = my_tiles * GROUPS;
    const auto tile_of = [&](int k) { return static_cast<int>(blockIdx.x) + k * static_cast<int>(gridDim.x); };

    if (warp == 0 && lane == 0) {
        // ---- producer
        if constexpr (C::RES) {
            mbar_expect_tx(wbar, static_cast<uint32_t>(C::W_ALL));
            for (int c = 0; c < CIN / 8; ++c) tma_load_weight_chunk(sbase + static_cast<uint32_t>(c * C::WCHUNK), &map_w, c, C::WBOX_BYTES, wbar);
        }
        for (int i = 0; i < items; ++i) {
            const int s = i % S, u = i / S;
            if (u >= 1 && !mbar_wait(empty(s), static_cast<uint32_t>((u - 1) & 1), abort, a.error)) break;
            const int tile = tile_of(i / GROUPS), g = i % GROUPS;
            const int tx = tile % a.tiles_x, rest = tile / a.tiles_x;
            const int ty = rest % a.tiles_y, z0 = (rest / a.tiles_y) * ZO;
            const uint32_t st = sbase + static_cast<uint32_t>(C::STAGE_OFF + s * C::STAGE);
            mbar_expect_tx(full(s), static_cast<uint32_t>(C::ITEM_TX));
            // input planes z0 - 1 .. z0 + ZO (out-of-range planes read as zeros)
            for (int plane = 0; plane < C::PLANES; ++plane)
                for (int ch = 0; ch < 2; ++ch) tma_load_4d(st + static_cast<uint32_t>((plane * 2 + ch) * C::PLANE_CHUNK), &map_in, g * 16 + ch * 8, tx * TX - 1, ty * TY - 1, z0 - 1 + plane, full(s));
            if constexpr (!C::RES)
                for (int ch = 0; ch < 2; ++ch) tma_load_weight_chunk(st + static_cast<uint32_t>(C::IN + ch * C::WCHUNK), &map_w, 2 * g + ch, C::WBOX_BYTES, full(s));
        }
    } else if (warp == 1) {
        // ---- MMA issuer: the whole warp walks the items (its values stay
        // warp-uniform); one elected lane issues the MMAs and the commits
        const auto wait_all = [&](uint32_t bar, uint32_t parity) { return __all_sync(0xffffffffu, mbar_wait(bar, parity, abort, a.error)); };
        bool ok = true;
        if constexpr (C::RES) ok = wait_all(wbar, 0);
        for (int i = 0; i < items && ok; ++i) {
            const int s = i % S, u = i / S;
            const int k = i / GROUPS, g = i % GROUPS, ab = k & 1;
            if (g == 0 && k >= 2 && !wait_all(acc_empty(ab), static_cast<uint32_t>(((k >> 1) - 1) & 1))) break;
            if (!wait_all(full(s), static_cast<uint32_t>(u & 1))) break;
            tc_fence_after();
            const uint32_t st = sbase + static_cast<uint32_t>(C::STAGE_OFF + s * C::STAGE);
            const uint32_t wb = C::RES ? sbase + static_cast<uint32_t>(2 * g * C::WCHUNK) : st + static_cast<uint32_t>(C::IN);
            const uint64_t da0 = smem_desc(st, C::PLANE_CHUNK, 128);
            const uint64_t db0 = smem_desc(wb, C::WCHUNK, 128);
            const uint32_t d0 = tmem + static_cast<uint32_t>(ab * MB * C::TILE_COLS);
            if (elect_one()) {
                issue_item<C, COUT>(da0, db0, d0, g == 0);
                mma_commit(empty(s));
                if (g == GROUPS - 1) mma_commit(acc_full(ab));
            }
            __syncwarp();
        }
    } else if (warp >= 2) {
        // ---- epilogue
        const int q = warp & 3;  // TMEM lane quarter of this warp
        for (int k = 0; k < my_tiles; ++k) {
            const int ab = k & 1;
            if (!mbar_wait(acc_full(ab), static_cast<uint32_t>((k >> 1) & 1), abort, a.error)) break;
            tc_fence_after();
            const int tile = tile_of(k);
            const int tx = tile % a.tiles_x, rest = tile / a.tiles_x;
            const int ty = rest % a.tiles_y, z0 = (rest / a.tiles_y) * ZO;
#pragma unroll 1
            for (int mo = 0; mo < MB * ZO; ++mo) {
                const int mb = mo / ZO, o = mo % ZO, z = z0 + o;
                const int m = mb * 128 + q * 32 + lane;
                const int y = m / P, x = m % P;
                const int gx = tx * TX + x, gy = ty * TY + y;
                const bool live = x < TX && y < TY && gx < a.d.nx && gy < a.d.ny && z < a.d.nz;
                const size_t v = live ? static_cast<size_t>(gx) + static_cast<size_t>(a.d.nx) * (gy + static_cast<size_t>(a.d.ny) * z) : 0;
                const uint32_t col = static_cast<uint32_t>(ab * MB * C::TILE_COLS + mb * C::TILE_COLS + (ZO - 1 - o) * COUT);
#pragma unroll
                for (int c0 = 0; c0 < COUT; c0 += 16) {
                    float acc[16];
                    tmem_ld16(tmem + (static_cast<uint32_t>(q * 32) << 16) + col + static_cast<uint32_t>(c0), acc);
                    tmem_wait_ld();
                    if (!live) continue;
                    if constexpr (EPI == LINEAR_F32_CH0) {
                        if (c0 == 0) static_cast<float*>(a.out)[v] = acc[0] + bias_s[0];
                    } else {
                        uint32_t packed[8];
#pragma unroll
                        for (int j = 0; j < 8; ++j) {
                            float r0 = acc[2 * j] + bias_s[c0 + 2 * j];
                            float r1 = acc[2 * j + 1] + bias_s[c0 + 2 * j + 1];
                            if constexpr (EPI == RELU_BF16) {
                                r0 = fmaxf(r0, 0.0f);
                                r1 = fmaxf(r1, 0.0f);
                            }
                            __nv_bfloat162 h = __floats2bfloat162_rn(r0, r1);
                            packed[j] = *reinterpret_cast<uint32_t*>(&h);
                        }
                        uint4* dst = reinterpret_cast<uint4*>(static_cast<__nv_bfloat16*>(a.out) + v * a.out_ch + a.out_off + c0);
                        dst[0] = make_uint4(packed[0], packed[1], packed[2], packed[3]);
                        dst[1] = make_uint4(packed[4], packed[5], packed[6], packed[7]);
                    }
                }
            }
            tc_fence_before();
            mbar_arrive(acc_empty(ab));
        }
    }
    __syncthreads();
    tc_fence_after();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(static_cast<uint32_t>(C::ALLOC)) : "memory");
}

}  // namespace sfb::net::tc
