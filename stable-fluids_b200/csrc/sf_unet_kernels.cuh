// sf_unet_kernels.cuh -- kernels of the warm-start network besides the
// tcgen05 convolution (sf_unet_tc.cuh): the weight gradient of a 3x3x3
// convolution (mma.sync BF16 x BF16 -> FP32), 2x average pooling, 2x nearest
// upsampling, and the element-wise pieces of training.
//
// Activations are channels-last BF16: element (voxel v, channel c) at
// v * C + c, v = x + nx (y + ny z), C a multiple of 16 (padded with zeros).
// Weights are BF16 [tap][cout][cin] with tap = (dz+1)*9 + (dy+1)*3 + (dx+1),
// plus an FP32 master copy for the optimizer. Zero padding at the grid edge.
//
// Weight-gradient GEMM instruction: mma.sync m16n8k16 BF16 x BF16 -> FP32.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "sf_types.h"

namespace sfb::net {

__device__ __forceinline__ void mma_bf16(float (&c)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0, uint32_t b1) {
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, {%0, %1, %2, %3};"
                 : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
                 : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t ld32(const __nv_bfloat16* p) { return *reinterpret_cast<const uint32_t*>(p); }

// Weight gradient: dw[tap][co][ci] += sum_v dout[v][co] in[v + off(tap)][ci],
// dbias[co] += sum_v dout[v][co]. GEMM per tap with M = COUT, N = CIN,
// K = voxels; the operand tiles are stored channel-major in shared memory so
// that K pairs are contiguous. Grid: (27, chunks); each CTA covers a z range
// of the grid for its tap and adds its FP32 partial sums atomically.
template <int CIN, int COUT>
__global__ void __launch_bounds__(128) k_conv3d_wgrad(const __nv_bfloat16* __restrict__ in, const __nv_bfloat16* __restrict__ dout, float* __restrict__ dw, float* __restrict__ dbias, Dims d, int z_per_cta) {
    static_assert(CIN % 8 == 0 && COUT % 16 == 0, "channel padding");
    constexpr int MT = COUT / 16, NTL = CIN / 8;  // m tiles, n tiles
    constexpr int TILES = MT * NTL;
    constexpr int PER_WARP = (TILES + 3) / 4;
    constexpr int V = 64;  // voxels per chunk: one row of 64 x (K = 4 x 16)
    __shared__ __align__(16) __nv_bfloat16 sa[COUT][V + 8];
    __shared__ __align__(16) __nv_bfloat16 sb[CIN][V + 8];
    const int tap = static_cast<int>(blockIdx.x);
    const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
    const int tid = static_cast<int>(threadIdx.x), warp = tid >> 5, lane = tid & 31;
    const int g = lane >> 2, t = lane & 3;
    float acc[PER_WARP][4];
#pragma unroll
    for (int i = 0; i < PER_WARP; ++i) acc[i][0] = acc[i][1] = acc[i][2] = acc[i][3] = 0.0f;
    float bsum = 0.0f;
    const int zb = static_cast<int>(blockIdx.y) * z_per_cta, ze = min(zb + z_per_cta, d.nz);
    for (int z = zb; z < ze; ++z)
        for (int y = 0; y < d.ny; ++y)
            for (int xc = 0; xc < d.nx; xc += V) {
                __syncthreads();
                for (int i = tid; i < V * COUT; i += 128) {
                    const int c = i % COUT, vx = i / COUT, gx = xc + vx;
                    sa[c][vx] = gx < d.nx ? dout[(static_cast<size_t>(gx) + static_cast<size_t>(d.nx) * (y + static_cast<size_t>(d.ny) * z)) * COUT + c] : __float2bfloat16(0.0f);
                }
                const int sy = y + dy, sz = z + dz;
                for (int i = tid; i < V * CIN; i += 128) {
                    const int c = i % CIN, vx = i / CIN, sx = xc + vx + dx;
                    const bool inb = xc + vx < d.nx && static_cast<unsigned>(sx) < static_cast<unsigned>(d.nx) && static_cast<unsigned>(sy) < static_cast<unsigned>(d.ny) && static_cast<unsigned>(sz) < static_cast<unsigned>(d.nz);
                    sb[c][vx] = inb ? in[(static_cast<size_t>(sx) + static_cast<size_t>(d.nx) * (sy + static_cast<size_t>(d.ny) * sz)) * CIN + c] : __float2bfloat16(0.0f);
                }
                __syncthreads();
                if (tap == 13 && tid < COUT)
                    for (int vx = 0; vx < V; ++vx) bsum += __bfloat162float(sa[tid][vx]);
#pragma unroll
                for (int kc = 0; kc < V / 16; ++kc) {
#pragma unroll
                    for (int i = 0; i < PER_WARP; ++i) {
                        const int tile_id = warp * PER_WARP + i;
                        if (tile_id >= TILES) continue;
                        const int mt = tile_id / NTL, nt = tile_id % NTL;
                        const int k0 = kc * 16 + 2 * t;
                        const uint32_t a0 = ld32(&sa[mt * 16 + g][k0]), a1 = ld32(&sa[mt * 16 + g + 8][k0]);
                        const uint32_t a2 = ld32(&sa[mt * 16 + g][k0 + 8]), a3 = ld32(&sa[mt * 16 + g + 8][k0 + 8]);
                        const uint32_t b0 = ld32(&sb[nt * 8 + g][k0]), b1 = ld32(&sb[nt * 8 + g][k0 + 8]);
                        mma_bf16(acc[i], a0, a1, a2, a3, b0, b1);
                    }
                }
            }
#pragma unroll
    for (int i = 0; i < PER_WARP; ++i) {
        const int tile_id = warp * PER_WARP + i;
        if (tile_id >= TILES) continue;
        const int mt = tile_id / NTL, nt = tile_id % NTL;
        float* base = dw + static_cast<size_t>(tap) * COUT * CIN;
        const int co = mt * 16 + g, ci = nt * 8 + 2 * t;
        atomicAdd(base + co * CIN + ci, acc[i][0]);
        atomicAdd(base + co * CIN + ci + 1, acc[i][1]);
        atomicAdd(base + (co + 8) * CIN + ci, acc[i][2]);
        atomicAdd(base + (co + 8) * CIN + ci + 1, acc[i][3]);
    }
    if (tap == 13 && tid < COUT && dbias) atomicAdd(dbias + tid, bsum);
}


// ------------------------------------------------------ element-wise pieces --

// Network input: channel 0 = b * scale, channel 1 = p_prev * scale, the
// other 14 channels zero (16-channel padded tensor). scale = 1 / rms(b) is
// read from *scale.
__global__ void k_pack_input(const float* __restrict__ b, const float* __restrict__ p_prev, const float* __restrict__ scale, float b_factor, __nv_bfloat16* __restrict__ out, size_t n) {
    const float s = *scale;
    for (size_t v = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; v < n; v += static_cast<size_t>(gridDim.x) * blockDim.x) {
        __nv_bfloat162 pair = __floats2bfloat162_rn(b[v] * b_factor * s, p_prev ? p_prev[v] * s : 0.0f);
        uint4 z4 = make_uint4(0, 0, 0, 0);
        uint4 first = z4;
        first.x = *reinterpret_cast<uint32_t*>(&pair);
        reinterpret_cast<uint4*>(out + v * 16)[0] = first;
        reinterpret_cast<uint4*>(out + v * 16)[1] = z4;
    }
}

// scale = 1 / rms(b_factor * b) from the FP64 sum of squares in *sumsq.
__global__ void k_finish_scale(const double* __restrict__ sumsq, double n, float* __restrict__ scale) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        const double rms = sqrt(*sumsq / n);
        *scale = rms > 0.0 ? static_cast<float>(1.0 / rms) : 1.0f;
    }
}

__global__ void k_sum_squares(const float* __restrict__ b, float b_factor, size_t n, double* __restrict__ out) {
    double acc = 0.0;
    for (size_t v = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; v < n; v += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const double x = static_cast<double>(b[v]) * b_factor;
        acc += x * x;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(out, acc);
}

// p0 = p_prev + delta / scale (the network predicts the scaled correction).
// p_prev may alias p0 (element-wise, each thread reads before it writes).
__global__ void k_unpack_output(const float* __restrict__ delta, const float* p_prev, const float* __restrict__ scale, float* p0, size_t n) {
    const float inv = 1.0f / *scale;
    for (size_t v = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; v < n; v += static_cast<size_t>(gridDim.x) * blockDim.x) p0[v] = (p_prev ? p_prev[v] : 0.0f) + delta[v] * inv;
}

// The pooling / upsampling / copy kernels below move 8 channels (16 bytes)
// per thread; channel counts, strides and offsets are multiples of 8. The
// 2-D launches give blockIdx.y = y and blockIdx.z = z of the output grid and
// threads over (x, 8-channel chunk) of one row.
struct Bf8 {
    float v[8];
};
__device__ __forceinline__ Bf8 load8(const __nv_bfloat16* p) {
    const uint4 u = *reinterpret_cast<const uint4*>(p);
    const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&u);
    Bf8 r;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const float2 f = __bfloat1622float2(h[k]);
        r.v[2 * k] = f.x;
        r.v[2 * k + 1] = f.y;
    }
    return r;
}
__device__ __forceinline__ void store8(__nv_bfloat16* p, const Bf8& r) {
    uint4 u;
    __nv_bfloat162* h = reinterpret_cast<__nv_bfloat162*>(&u);
#pragma unroll
    for (int k = 0; k < 4; ++k) h[k] = __floats2bfloat162_rn(r.v[2 * k], r.v[2 * k + 1]);
    *reinterpret_cast<uint4*>(p) = u;
}

inline dim3 row_grid(int nx, int chunks_per_voxel, int ny, int nz) { return dim3(static_cast<unsigned>((nx * chunks_per_voxel + 255) / 256), static_cast<unsigned>(ny), static_cast<unsigned>(nz)); }

// 2x2x2 average pooling (even dims of the fine grid); channel stride in_ch.
// Launch: row_grid(coarse.nx, C / 8, coarse.ny, coarse.nz), 256 threads.
__global__ void k_pool2(const __nv_bfloat16* __restrict__ in, int in_ch, int in_off, __nv_bfloat16* __restrict__ out, int C, Dims coarse) {
    const int c8n = C / 8;
    const int i = static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x);
    if (i >= coarse.nx * c8n) return;
    const int x = i / c8n, c = (i % c8n) * 8, y = static_cast<int>(blockIdx.y), z = static_cast<int>(blockIdx.z);
    const int fnx = coarse.nx * 2, fny = coarse.ny * 2;
    Bf8 s{};
    for (int k = 0; k < 8; ++k) {
        const size_t fv = static_cast<size_t>(2 * x + (k & 1)) + static_cast<size_t>(fnx) * (2 * y + ((k >> 1) & 1) + static_cast<size_t>(fny) * (2 * z + (k >> 2)));
        const Bf8 a = load8(in + fv * in_ch + in_off + c);
#pragma unroll
        for (int j = 0; j < 8; ++j) s.v[j] += a.v[j];
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) s.v[j] *= 0.125f;
    const size_t v = static_cast<size_t>(x) + static_cast<size_t>(coarse.nx) * (y + static_cast<size_t>(coarse.ny) * z);
    store8(out + v * C + c, s);
}

// Backward of the pooling: each fine voxel gets 1/8 of its parent's gradient,
// added to (accumulate) or written into the fine gradient tensor.
// Launch: row_grid(fine nx, C / 8, fine ny, fine nz).
__global__ void k_pool2_backward(const __nv_bfloat16* __restrict__ gcoarse, int C, Dims coarse, __nv_bfloat16* __restrict__ gfine, int fine_ch, int fine_off, int accumulate) {
    const int c8n = C / 8, fnx = coarse.nx * 2, fny = coarse.ny * 2;
    const int i = static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x);
    if (i >= fnx * c8n) return;
    const int x = i / c8n, c = (i % c8n) * 8, y = static_cast<int>(blockIdx.y), z = static_cast<int>(blockIdx.z);
    const size_t cv = static_cast<size_t>(x / 2) + static_cast<size_t>(coarse.nx) * (y / 2 + static_cast<size_t>(coarse.ny) * (z / 2));
    Bf8 g = load8(gcoarse + cv * C + c);
    __nv_bfloat16* dst = gfine + (static_cast<size_t>(x) + static_cast<size_t>(fnx) * (y + static_cast<size_t>(fny) * z)) * fine_ch + fine_off + c;
    const Bf8 old = accumulate ? load8(dst) : Bf8{};
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        g.v[j] = 0.125f * g.v[j];
        if (accumulate) g.v[j] += old.v[j];
    }
    store8(dst, g);
}

// Nearest 2x upsampling of a coarse tensor into channels [out_off, out_off+C)
// of a fine tensor with channel stride out_ch. Launch: row_grid(fine nx, C / 8,
// fine ny, fine nz).
__global__ void k_upsample2(const __nv_bfloat16* __restrict__ in, int C, Dims coarse, __nv_bfloat16* __restrict__ out, int out_ch, int out_off) {
    const int c8n = C / 8, fnx = coarse.nx * 2, fny = coarse.ny * 2;
    const int i = static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x);
    if (i >= fnx * c8n) return;
    const int x = i / c8n, c = (i % c8n) * 8, y = static_cast<int>(blockIdx.y), z = static_cast<int>(blockIdx.z);
    const size_t cv = static_cast<size_t>(x / 2) + static_cast<size_t>(coarse.nx) * (y / 2 + static_cast<size_t>(coarse.ny) * (z / 2));
    const size_t fv = static_cast<size_t>(x) + static_cast<size_t>(fnx) * (y + static_cast<size_t>(fny) * z);
    *reinterpret_cast<uint4*>(out + fv * out_ch + out_off + c) = *reinterpret_cast<const uint4*>(in + cv * C + c);
}

// Backward of the upsampling: the coarse gradient is the sum over its 8
// children of channels [off, off + C) of the fine gradient. Launch:
// row_grid(coarse.nx, C / 8, coarse.ny, coarse.nz).
__global__ void k_upsample2_backward(const __nv_bfloat16* __restrict__ gfine, int fine_ch, int off, int C, Dims coarse, __nv_bfloat16* __restrict__ gcoarse) {
    const int c8n = C / 8, fnx = coarse.nx * 2, fny = coarse.ny * 2;
    const int i = static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x);
    if (i >= coarse.nx * c8n) return;
    const int x = i / c8n, c = (i % c8n) * 8, y = static_cast<int>(blockIdx.y), z = static_cast<int>(blockIdx.z);
    Bf8 s{};
    for (int k = 0; k < 8; ++k) {
        const size_t fv = static_cast<size_t>(2 * x + (k & 1)) + static_cast<size_t>(fnx) * (2 * y + ((k >> 1) & 1) + static_cast<size_t>(fny) * (2 * z + (k >> 2)));
        const Bf8 a = load8(gfine + fv * fine_ch + off + c);
#pragma unroll
        for (int j = 0; j < 8; ++j) s.v[j] += a.v[j];
    }
    const size_t v = static_cast<size_t>(x) + static_cast<size_t>(coarse.nx) * (y + static_cast<size_t>(coarse.ny) * z);
    store8(gcoarse + v * C + c, s);
}

// Copies channels [src_off, src_off + C) of src into [dst_off, ...) of dst
// (adding to dst when accumulate), 8 channels per thread.
__global__ void k_copy_channels(const __nv_bfloat16* __restrict__ src, int src_ch, int src_off, __nv_bfloat16* __restrict__ dst, int dst_ch, int dst_off, int C, size_t voxels, int accumulate) {
    const size_t c8n = static_cast<size_t>(C / 8), n = voxels * c8n;
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n; i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const size_t v = i / c8n, c = (i % c8n) * 8;
        __nv_bfloat16* d = dst + v * dst_ch + dst_off + c;
        if (accumulate) {
            Bf8 a = load8(src + v * src_ch + src_off + c);
            const Bf8 b = load8(d);
#pragma unroll
            for (int j = 0; j < 8; ++j) a.v[j] += b.v[j];
            store8(d, a);
        } else {
            *reinterpret_cast<uint4*>(d) = *reinterpret_cast<const uint4*>(src + v * src_ch + src_off + c);
        }
    }
}

// g *= (act > 0): the gradient through a ReLU whose output is act; n is a
// multiple of 8.
__global__ void k_relu_backward(__nv_bfloat16* __restrict__ g, const __nv_bfloat16* __restrict__ act, size_t n) {
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n / 8; i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const Bf8 a = load8(act + 8 * i);
        Bf8 v = load8(g + 8 * i);
#pragma unroll
        for (int j = 0; j < 8; ++j)
            if (!(a.v[j] > 0.0f)) v.v[j] = 0.0f;
        store8(g + 8 * i, v);
    }
}

// Mean squared error of the FP32 output against the target; writes the
// gradient (channel 0 of a 16-channel BF16 tensor) and adds the loss sum.
__global__ void k_mse(const float* __restrict__ out, const float* __restrict__ target, size_t n, __nv_bfloat16* __restrict__ grad16, double* __restrict__ loss_sum) {
    double acc = 0.0;
    const float k = 2.0f / static_cast<float>(n);
    for (size_t v = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; v < n; v += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const float e = out[v] - target[v];
        acc += static_cast<double>(e) * e;
        uint4 z4 = make_uint4(0, 0, 0, 0);
        __nv_bfloat162 first = __floats2bfloat162_rn(k * e, 0.0f);
        uint4 f = z4;
        f.x = *reinterpret_cast<uint32_t*>(&first);
        reinterpret_cast<uint4*>(grad16 + v * 16)[0] = f;
        reinterpret_cast<uint4*>(grad16 + v * 16)[1] = z4;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss_sum, acc);
}

// Adam on FP32 master weights; refreshes the BF16 copy and the transposed,
// tap-flipped BF16 copy used by the data-gradient convolution.
__global__ void k_adam(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v, __nv_bfloat16* __restrict__ w16, __nv_bfloat16* __restrict__ w16t, int cout, int cin, size_t n, float lr, float b1, float b2, float eps, float bc1, float bc2) {
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n; i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float wi = w[i] - lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
        w[i] = wi;
        if (w16) {
            w16[i] = __float2bfloat16(wi);
            const int tap = static_cast<int>(i / (static_cast<size_t>(cout) * cin));
            const int co = static_cast<int>((i / cin) % cout), ci = static_cast<int>(i % cin);
            w16t[(static_cast<size_t>(26 - tap) * cin + ci) * cout + co] = __float2bfloat16(wi);
        }
    }
}

}  // namespace sfb::net
