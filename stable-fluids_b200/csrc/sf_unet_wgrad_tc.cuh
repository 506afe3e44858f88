// sf_unet_wgrad_tc.cuh -- weight gradient of a 3x3x3 convolution of the
// warm-start network on the tcgen05 tensor cores (BF16 x BF16 -> FP32 in
// tensor memory).
//
//   dw[tap][co][ci] += sum_v dout[v][co] * in[v + off(tap)][ci]
//
// Per tap a GEMM D (co x ci) = A (co x K) B^T (ci x K) whose K runs over the
// voxels. A CTA owns one tap and a contiguous range of voxels (linear index
// x + nx (y + ny z)), taken in chunks of 128. For each chunk the threads copy
// (cp.async, 16 bytes = 8 channels of one voxel) the chunk's dout rows and
// the in rows of the voxels shifted by the tap -- zeros where the shifted
// voxel is outside the grid (the convolution's zero padding) or past the
// last voxel -- into shared memory as the activations lie in memory,
// channels-last per 8-channel group: group g holds [voxel][8 channels].
// That is the MN-major canonical layout of both operands (8 M or N elements
// contiguous in a 16-byte row, K = voxel rows 16 bytes apart, 8-voxel core
// matrices 128 bytes apart, 8-channel groups one group apart), so nothing is
// transposed. One elected thread issues eight K = 16 MMAs per chunk,
// M = 128, N = CIN, accumulating in tensor memory. Only the COUT/8 groups of
// A are stored: the MMA's rows past COUT read whatever follows in shared
// memory (the B groups, the next stage, a pad at the end), and those rows of
// the accumulator are never read. Four stages: the copies of chunks i + 1
// and i + 2 are in flight while chunk i is multiplied, the latter into the
// stage chunk i - 2 was multiplied from. At the end warp w reads
// accumulator lanes 32 w .. 32 w + 31 (the output channels) and adds them to
// dw with FP32 atomics; the centre tap's CTAs also sum dout into the bias
// gradient. Every wait on an mbarrier is
// bounded (tc::mbar_wait); a CTA that gives up records it in *error.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "sf_types.h"
#include "sf_unet_tc.cuh"

namespace sfb::net::tc {

constexpr int kWgK = 128;        // voxels per chunk
constexpr int kWgThreads = 128;  // four warps: copies, one MMA issuer, the epilogue
constexpr int kWgStages = 4;
constexpr int kWgAhead = kWgStages - 2;  // chunks in flight ahead of the one multiplied

template <int CIN, int COUT>
struct WgCfg {
    static constexpr int GROUP = kWgK * 16;  // one 8-channel group of a chunk (2 KB)
    static constexpr int A = COUT / 8 * GROUP;
    static constexpr int B = CIN / 8 * GROUP;
    static constexpr int STAGE = A + B;
    static constexpr int REACH = 16 * GROUP;  // what the M = 128 operand spans from a stage's A
    static constexpr int PAD = REACH > STAGE ? REACH - STAGE : 0;
    static constexpr int BAR_OFF = kWgStages * STAGE + PAD;  // done[stages], TMEM slot, abort flag
    static constexpr int BYTES = BAR_OFF + 64;
    static constexpr int ALLOC = CIN <= 32 ? 32 : (CIN <= 64 ? 64 : 128);
    static_assert(COUT % 8 == 0 && COUT <= 128, "output channels: 8-channel groups, M = 128");
    static_assert(CIN % 16 == 0 && CIN <= 128, "MMA N: a multiple of 16, within the accumulator allocation");
};

// kind::f16, BF16 operands, FP32 accumulator, M = 128, N = n, A and B MN-major.
__host__ __device__ constexpr uint32_t instr_desc_mn(uint32_t n) { return instr_desc(n) | (1u << 15) | (1u << 16); }

__device__ __forceinline__ void cp_async16_zfill(uint32_t dst, const void* src, bool valid) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(valid ? 16 : 0) : "memory");
}

// The copies of chunk c into stage st (all threads; one cp.async group):
// thread t copies voxel v0 + t of the chunk, all its channel groups.
static_assert(kWgThreads == kWgK, "one voxel of the chunk per thread");

template <int CIN, int COUT>
__device__ __forceinline__ void wgrad_load(uint32_t st, int c, const __nv_bfloat16* __restrict__ in, const __nv_bfloat16* __restrict__ dout, const Dims& d, int nvox, int dx, int dy, int dz) {
    using C = WgCfg<CIN, COUT>;
    const int k = static_cast<int>(threadIdx.x);
    const int v = c * kWgK + k;
    const bool live = v < nvox;
    const int vv = live ? v : 0;
    const int x = vv % d.nx + dx, y = (vv / d.nx) % d.ny + dy, z = vv / (d.nx * d.ny) + dz;
    const bool inside = live && static_cast<unsigned>(x) < static_cast<unsigned>(d.nx) && static_cast<unsigned>(y) < static_cast<unsigned>(d.ny) && static_cast<unsigned>(z) < static_cast<unsigned>(d.nz);
    const size_t sv = inside ? static_cast<size_t>(x) + static_cast<size_t>(d.nx) * (y + static_cast<size_t>(d.ny) * z) : 0;
    const uint32_t row = st + static_cast<uint32_t>(k * 16);
#pragma unroll
    for (int g = 0; g < COUT / 8; ++g) cp_async16_zfill(row + static_cast<uint32_t>(g * C::GROUP), dout + static_cast<size_t>(vv) * COUT + g * 8, live);
#pragma unroll
    for (int g = 0; g < CIN / 8; ++g) cp_async16_zfill(row + static_cast<uint32_t>(C::A + g * C::GROUP), in + sv * CIN + g * 8, inside);
    asm volatile("cp.async.commit_group;" ::: "memory");
}

template <int CIN, int COUT>
__global__ void __launch_bounds__(kWgThreads) k_conv3d_wgrad_tc(const __nv_bfloat16* __restrict__ in, const __nv_bfloat16* __restrict__ dout, float* __restrict__ dw, float* __restrict__ dbias, Dims d, int chunks_per_cta, unsigned* error) {
    using C = WgCfg<CIN, COUT>;
    constexpr int S = kWgStages;
    extern __shared__ __align__(1024) unsigned char smem[];
    const int tid = static_cast<int>(threadIdx.x), warp = tid >> 5, lane = tid & 31;
    const int tap = static_cast<int>(blockIdx.x);
    const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
    const int nvox = d.nx * d.ny * d.nz;  // grids of the network stay below 2^31 voxels
    const int nchunks = (nvox + kWgK - 1) / kWgK;
    const int c_begin = static_cast<int>(blockIdx.y) * chunks_per_cta;
    const int c_end = c_begin + chunks_per_cta < nchunks ? c_begin + chunks_per_cta : nchunks;
    const int n = c_end > c_begin ? c_end - c_begin : 0;
    const uint32_t sbase = smem_u32(smem);
    const uint32_t done0 = sbase + C::BAR_OFF;  // done[s] = done0 + 8 s: the MMAs that read stage s
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + C::BAR_OFF + 8 * S);
    volatile int* abort = reinterpret_cast<volatile int*>(smem + C::BAR_OFF + 8 * S + 4);
    const auto stage = [&](int i) { return sbase + static_cast<uint32_t>((i % S) * C::STAGE); };

    // the pad past the last stage is read only into accumulator rows that are never used; keep it finite
    for (int i = tid; i < C::PAD / 16; i += kWgThreads) reinterpret_cast<uint4*>(smem + S * C::STAGE)[i] = make_uint4(0, 0, 0, 0);
    if (tid == 0) {
        for (int s = 0; s < S; ++s) mbar_init(done0 + 8u * static_cast<uint32_t>(s), 1);
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

    // kWgAhead chunks in flight ahead of the one multiplied; a stage is
    // refilled two chunks after its MMAs were issued, so the wait for them is short
    for (int i = 0; i < kWgAhead; ++i) {
        if (i < n) wgrad_load<CIN, COUT>(stage(i), c_begin + i, in, dout, d, nvox, dx, dy, dz);
        else asm volatile("cp.async.commit_group;" ::: "memory");
    }
    float bsum = 0.0f;  // centre tap: thread co < COUT sums dout[.][co]
    bool ok = true;
    for (int i = 0; i < n; ++i) {
        // chunk i + kWgAhead goes into the stage chunk i - 2 was multiplied from
        const int j = i + kWgAhead;
        if (j < n) {
            if (j >= S && !mbar_wait(done0 + 8u * static_cast<uint32_t>(j % S), static_cast<uint32_t>((j / S - 1) & 1), abort, error)) ok = false;
            if (ok) wgrad_load<CIN, COUT>(stage(j), c_begin + j, in, dout, d, nvox, dx, dy, dz);
            else asm volatile("cp.async.commit_group;" ::: "memory");
        } else {
            asm volatile("cp.async.commit_group;" ::: "memory");
        }
        asm volatile("cp.async.wait_group %0;" ::"n"(kWgAhead) : "memory");  // chunk i has landed
        fence_proxy_async_smem();  // this thread's copies, visible to the tensor core
        if (!__syncthreads_and(ok ? 1 : 0)) {
            ok = false;
            break;
        }
        const uint32_t st = stage(i);
        if (tap == 13 && tid < COUT) {
            const __nv_bfloat16* a = reinterpret_cast<const __nv_bfloat16*>(smem + (i % S) * C::STAGE + (tid / 8) * C::GROUP) + (tid % 8);
            for (int k = 0; k < kWgK; ++k) bsum += __bfloat162float(a[8 * k]);
        }
        if (warp == 0) {
            tc_fence_after();
            if (elect_one()) {
#pragma unroll
                for (int kk = 0; kk < kWgK / 16; ++kk) {
                    const uint64_t da = smem_desc(st + static_cast<uint32_t>(kk * 256), 128, C::GROUP);
                    const uint64_t db = smem_desc(st + static_cast<uint32_t>(C::A + kk * 256), 128, C::GROUP);
                    mma_bf16(tmem, da, db, instr_desc_mn(CIN), (i > 0 || kk > 0) ? 1u : 0u);
                }
                mma_commit(done0 + 8u * static_cast<uint32_t>(i % S));
            }
            __syncwarp();
        }
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    // the last commit covers every MMA before it
    if (ok && n > 0 && !mbar_wait(done0 + 8u * static_cast<uint32_t>((n - 1) % S), static_cast<uint32_t>(((n - 1) / S) & 1), abort, error)) ok = false;
    tc_fence_after();
    if (__syncthreads_and(ok ? 1 : 0) && n > 0 && warp * 32 < COUT) {
        const int co = warp * 32 + lane;
#pragma unroll 1
        for (int c0 = 0; c0 < CIN; c0 += 16) {
            float acc[16];
            tmem_ld16(tmem + (static_cast<uint32_t>(warp * 32) << 16) + static_cast<uint32_t>(c0), acc);
            tmem_wait_ld();
            if (co < COUT)
#pragma unroll
                for (int jj = 0; jj < 16; ++jj) atomicAdd(&dw[(static_cast<size_t>(tap) * COUT + co) * CIN + c0 + jj], acc[jj]);
        }
    }
    if (tap == 13 && tid < COUT && dbias != nullptr && n > 0) atomicAdd(dbias + tid, bsum);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(static_cast<uint32_t>(C::ALLOC)) : "memory");
}

}  // namespace sfb::net::tc
