// sf_unet.cu -- the learned pressure warm start: a 3-level 3D U-Net
// (16/32/64 channels, 3x3x3 convolutions, ReLU, BF16 weights and
// activations, FP32 accumulation) mapping (h^2 divergence, previous pressure)
// to a warm-start pressure, with its own training (forward, backward, Adam)
// on the GPU.
//
//   in(2 -> padded 16) -> e0a(16) -> e0b(16) = s0 ----------------------.
//        pool -> e1a(32) -> e1b(32) = s1 ------------------.            |
//             pool -> ba(64) -> bb(64) -> up -> [up|s1](96) -> d1a(32) -> d1b(32)
//                                                   up -> [up|s0](48) -> d0a(16) -> d0b(16) -> out(1)
//
// Inputs are scaled by 1 / rms(h^2 div); the network predicts the scaled
// correction to the previous pressure: p0 = p_prev + out / scale. Grid sides
// must be multiples of 4 (two poolings).

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <new>
#include <random>
#include <set>
#include <vector>

#include "sf_types.h"
#include "sf_unet.h"
#include "sf_unet_kernels.cuh"
#include "sf_unet_tc.cuh"
#include "sf_unet_wgrad_tc.cuh"
#include "stable-fluids-b200.h"

namespace sfb::net {

unsigned blocks_for(size_t n) {
    size_t b = (n + 255) / 256;
    return static_cast<unsigned>(b < 148u * 32u ? (b == 0 ? 1 : b) : 148u * 32u);
}

struct Layer {
    int cin, cout;  // padded channel counts
    int cin_real;   // channels carrying data (fan-in of the initialisation)
    size_t wn = 0;  // 27 * cout * cin
    size_t off = 0; // offset of the weights in the parameter vector (then cout biases)
};

// The layer table of the network, in forward order.
enum LayerId { E0A, E0B, E1A, E1B, BA, BB, D1A, D1B, D0A, D0B, OUT, NLAYERS };
constexpr int kCin[NLAYERS] = {16, 16, 16, 32, 32, 64, 96, 32, 48, 16, 16};
constexpr int kCinReal[NLAYERS] = {2, 16, 16, 32, 32, 64, 96, 32, 48, 16, 16};
constexpr int kCout[NLAYERS] = {16, 16, 32, 32, 64, 64, 32, 32, 16, 16, 16};

struct Buffers {
    const void* owner = nullptr;  // the context predicting with it (inference only), or null
    Dims d0{}, d1{}, d2{};
    size_t n0 = 0, n1 = 0, n2 = 0;
    void* mem = nullptr;
    size_t bytes = 0;
    // activations (BF16, channels-last)
    __nv_bfloat16 *in = nullptr, *e0a = nullptr, *e0b = nullptr, *p0 = nullptr, *e1a = nullptr, *e1b = nullptr, *p1 = nullptr, *ba = nullptr, *bb = nullptr;
    __nv_bfloat16 *cat1 = nullptr, *d1a = nullptr, *d1b = nullptr, *cat0 = nullptr, *d0a = nullptr, *d0b = nullptr;
    float* out = nullptr;     // FP32 network output (channel 0)
    float* target = nullptr;  // FP32 scaled training target
    // gradients (BF16)
    __nv_bfloat16 *g16 = nullptr, *gd0b = nullptr, *gd0a = nullptr, *gcat0 = nullptr, *gd1b = nullptr, *gd1a = nullptr, *gcat1 = nullptr, *gbb = nullptr, *gba = nullptr, *gp1 = nullptr, *ge1b = nullptr, *ge1a = nullptr, *gp0 = nullptr, *ge0b = nullptr, *ge0a = nullptr;
    double* sums = nullptr;  // [0] sum of squares of b, [1] loss sum
    float* scale = nullptr;

    Buffers() = default;
    Buffers(const Buffers&) = delete;
    Buffers& operator=(const Buffers&) = delete;
    ~Buffers() {
        if (mem) cudaFree(mem);
    }
};

struct Net {
    Layer layers[NLAYERS];
    size_t nparams = 0;
    float* w = nullptr;             // FP32 master parameters
    float* g = nullptr;             // gradients
    float* m = nullptr;             // Adam moments
    float* v = nullptr;
    __nv_bfloat16* w16 = nullptr;   // BF16 weights [tap][cout][cin] per layer
    __nv_bfloat16* w16t = nullptr;  // BF16 transposed, tap-flipped weights [tap][cin][cout] (data gradient)
    unsigned* error = nullptr;      // set by a convolution whose bounded wait gave up
    int adam_t = 0;
    // Buffer sets by grid size and owner, kept until the network is
    // destroyed (or the owner releases them) so that step graphs holding
    // their addresses stay valid: the network's own set per size (training
    // and direct predictions, with the gradient buffers), and one
    // inference-only set per attached context, so that contexts sharing the
    // network can step at the same time.
    std::vector<std::unique_ptr<Buffers>> sets;
    Buffers* buf = nullptr;

    Net() = default;
    Net(const Net&) = delete;
    Net& operator=(const Net&) = delete;
    ~Net() {
        cudaFree(w);
        cudaFree(g);
        cudaFree(m);
        cudaFree(v);
        cudaFree(w16);
        cudaFree(w16t);
        cudaFree(error);
    }
};

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) != cudaSuccess || q != cudaDriverEntryPointSuccess) p = nullptr;
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }();
    return fn;
}

int sm_count() {
    static const int n = [] {
        int dev = 0, v = 148;
        if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) v = 148;
        return v;
    }();
    return n;
}

// 3x3x3 convolution on the tensor cores (tc::k_conv3d_tc): tensor maps for
// the channels-last input (boxes of 8 channels x (TX + 2) x (TY + 2) x 1
// voxels) and the [dz][dy][dx][COUT][CIN] weights, viewed as (cin, cout, dx,
// dy, dz) with boxes of 8 input channels x COUT x 1 x 1 x 3 (the dz taps of
// one in-plane shift), then one persistent CTA per SM.
template <int CIN, int COUT, int EPI>
cudaError_t conv(const __nv_bfloat16* in, const __nv_bfloat16* w, const float* bias, void* out, int out_ch, int out_off, Dims d, cudaStream_t s, unsigned* error) {
    using C = tc::Cfg<CIN, COUT>;
    auto encode = tensor_map_encoder();
    if (encode == nullptr) return cudaErrorNotSupported;
    CUtensorMap map_in{}, map_w{};
    const cuuint64_t gd[4] = {static_cast<cuuint64_t>(CIN), static_cast<cuuint64_t>(d.nx), static_cast<cuuint64_t>(d.ny), static_cast<cuuint64_t>(d.nz)};
    const cuuint64_t gs[3] = {static_cast<cuuint64_t>(CIN) * 2, static_cast<cuuint64_t>(d.nx) * CIN * 2, static_cast<cuuint64_t>(d.ny) * d.nx * CIN * 2};
    const cuuint32_t box[4] = {8u, static_cast<cuuint32_t>(tc::P), static_cast<cuuint32_t>(C::TY + 2), 1u};
    const cuuint32_t es[4] = {1u, 1u, 1u, 1u};
    if (encode(&map_in, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<__nv_bfloat16*>(in), gd, gs, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return cudaErrorInvalidValue;
    const cuuint64_t tap = static_cast<cuuint64_t>(COUT) * CIN * 2;  // bytes per tap
    const cuuint64_t wd[5] = {static_cast<cuuint64_t>(CIN), static_cast<cuuint64_t>(COUT), 3u, 3u, 3u};
    const cuuint64_t ws[4] = {static_cast<cuuint64_t>(CIN) * 2, tap, 3 * tap, 9 * tap};
    const cuuint32_t wbox[5] = {8u, static_cast<cuuint32_t>(COUT), 1u, 1u, 3u};
    const cuuint32_t wes[5] = {1u, 1u, 1u, 1u, 1u};
    if (encode(&map_w, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<__nv_bfloat16*>(w), wd, ws, wbox, wes, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return cudaErrorInvalidValue;
    auto kern = tc::k_conv3d_tc<CIN, COUT, EPI>;
    const cudaError_t attr = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, C::BYTES);
    if (attr != cudaSuccess) return attr;
    tc::ConvArgs a{out, bias, out_ch, out_off, d, (d.nx + tc::TX - 1) / tc::TX, (d.ny + C::TY - 1) / C::TY, (d.nz + C::ZO - 1) / C::ZO, error};
    const int tiles = a.tiles_x * a.tiles_y * a.tiles_z;
    const int grid = tiles < sm_count() ? tiles : sm_count();
    kern<<<grid, tc::kThreadsTC, C::BYTES, s>>>(map_in, map_w, a);
    return cudaGetLastError();
}

// Runtime dispatch of the (cin, cout) combinations the network uses.
cudaError_t conv_any(int cin, int cout, int epi, const __nv_bfloat16* in, const __nv_bfloat16* w, const float* bias, void* out, int out_ch, int out_off, Dims d, cudaStream_t s, unsigned* error) {
#define SFB_CONV(CI, CO)                                                                                                     \
    if (cin == CI && cout == CO) {                                                                                           \
        if (epi == tc::RELU_BF16) return conv<CI, CO, tc::RELU_BF16>(in, w, bias, out, out_ch, out_off, d, s, error);          \
        if (epi == tc::LINEAR_BF16) return conv<CI, CO, tc::LINEAR_BF16>(in, w, bias, out, out_ch, out_off, d, s, error);      \
        return conv<CI, CO, tc::LINEAR_F32_CH0>(in, w, bias, out, out_ch, out_off, d, s, error);                               \
    }
    SFB_CONV(16, 16) SFB_CONV(16, 32) SFB_CONV(32, 32) SFB_CONV(32, 64) SFB_CONV(64, 64) SFB_CONV(96, 32) SFB_CONV(48, 16)  // forward
    SFB_CONV(32, 16) SFB_CONV(64, 32) SFB_CONV(32, 96) SFB_CONV(16, 48)                                                     // data gradients
#undef SFB_CONV
    return cudaErrorInvalidValue;
}

// The weight gradient on the tcgen05 tensor cores (sf_unet_wgrad_tc.cuh);
// STABLE_FLUIDS_B200_WGRAD=mma selects the mma.sync GEMM per tap instead.
bool wgrad_on_mma_sync() {
    static const bool v = [] {
        const char* e = std::getenv("STABLE_FLUIDS_B200_WGRAD");
        return e != nullptr && std::strcmp(e, "mma") == 0;
    }();
    return v;
}

template <int CIN, int COUT>
cudaError_t wgrad(const __nv_bfloat16* in, const __nv_bfloat16* dout, float* dw, float* db, Dims d, cudaStream_t s, unsigned* error) {
    if (wgrad_on_mma_sync() || static_cast<long long>(d.nx) * d.ny * d.nz >= (1ll << 31)) {  // the tensor-core form indexes voxels in 32 bits
        const int zper = d.nz >= 64 ? 4 : (d.nz >= 16 ? 2 : 1);
        const dim3 grid(27, static_cast<unsigned>((d.nz + zper - 1) / zper));
        k_conv3d_wgrad<CIN, COUT><<<grid, 128, 0, s>>>(in, dout, dw, db, d, zper);
        return cudaGetLastError();
    }
    using C = tc::WgCfg<CIN, COUT>;
    const auto kern = tc::k_conv3d_wgrad_tc<CIN, COUT>;
    static const cudaError_t attr = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, C::BYTES);
    if (attr != cudaSuccess) return attr;
    static const int per_sm = [&] {
        int k = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&k, kern, tc::kWgThreads, C::BYTES) != cudaSuccess || k < 1) k = 1;
        return k;
    }();
    int sms = 148, dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const long long nvox = static_cast<long long>(d.nx) * d.ny * d.nz;
    const long long nchunks = (nvox + tc::kWgK - 1) / tc::kWgK;
    long long per_tap = static_cast<long long>(sms) * per_sm / 27;  // one wave of CTAs over the 27 taps
    if (per_tap < 1) per_tap = 1;
    const long long chunks = (nchunks + per_tap - 1) / per_tap;
    const dim3 grid(27, static_cast<unsigned>((nchunks + chunks - 1) / chunks));
    kern<<<grid, tc::kWgThreads, C::BYTES, s>>>(in, dout, dw, db, d, static_cast<int>(chunks), error);
    return cudaGetLastError();
}

cudaError_t wgrad_any(int cin, int cout, const __nv_bfloat16* in, const __nv_bfloat16* dout, float* dw, float* db, Dims d, cudaStream_t s, unsigned* error) {
#define SFB_WG(CI, CO) \
    if (cin == CI && cout == CO) return wgrad<CI, CO>(in, dout, dw, db, d, s, error);
    SFB_WG(16, 16) SFB_WG(16, 32) SFB_WG(32, 32) SFB_WG(32, 64) SFB_WG(64, 64) SFB_WG(96, 32) SFB_WG(48, 16)
#undef SFB_WG
    return cudaErrorInvalidValue;
}

// Copies FP32 master parameters from the host and refreshes the BF16 copies.
cudaError_t set_parameters(Net* n, const float* host) {
    cudaError_t e = cudaMemcpy(n->w, host, n->nparams * sizeof(float), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return e;
    n->adam_t = 0;
    // An Adam pass with lr = 0 and zero gradients leaves w unchanged and
    // rewrites both BF16 copies.
    const size_t fb = n->nparams * sizeof(float);
    if ((e = cudaMemset(n->g, 0, fb)) != cudaSuccess || (e = cudaMemset(n->m, 0, fb)) != cudaSuccess || (e = cudaMemset(n->v, 0, fb)) != cudaSuccess) return e;
    for (int l = 0; l < NLAYERS; ++l) {
        const Layer& L = n->layers[l];
        k_adam<<<blocks_for(L.wn), 256>>>(n->w + L.off, n->g + L.off, n->m + L.off, n->v + L.off, n->w16 + L.off, n->w16t + L.off, L.cout, L.cin, L.wn, 0.0f, 0.9f, 0.999f, 1e-8f, 1.0f, 1.0f);
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    return cudaDeviceSynchronize();
}

Net* create_net(uint32_t seed) {
    std::unique_ptr<Net> n{new (std::nothrow) Net{}};
    if (!n) return nullptr;
    size_t off = 0;
    for (int l = 0; l < NLAYERS; ++l) {
        Layer& L = n->layers[l];
        L.cin = kCin[l];
        L.cout = kCout[l];
        L.cin_real = kCinReal[l];
        L.wn = static_cast<size_t>(27) * L.cout * L.cin;
        L.off = off;
        off += L.wn + static_cast<size_t>(L.cout);
    }
    n->nparams = off;
    const size_t fb = off * sizeof(float);
    if (cudaMalloc(&n->w, fb) != cudaSuccess || cudaMalloc(&n->g, fb) != cudaSuccess || cudaMalloc(&n->m, fb) != cudaSuccess || cudaMalloc(&n->v, fb) != cudaSuccess) return nullptr;
    if (cudaMalloc(&n->w16, off * sizeof(__nv_bfloat16)) != cudaSuccess || cudaMalloc(&n->w16t, off * sizeof(__nv_bfloat16)) != cudaSuccess) return nullptr;
    if (cudaMalloc(&n->error, sizeof(unsigned)) != cudaSuccess || cudaMemset(n->error, 0, sizeof(unsigned)) != cudaSuccess) return nullptr;
    // He initialisation over the real fan-in (the output layer 10x smaller);
    // padded input channels and padded output channels of the last layer are
    // zero; biases zero.
    std::vector<float> host(off, 0.0f);
    std::mt19937_64 rng(seed);
    for (int l = 0; l < NLAYERS; ++l) {
        const Layer& L = n->layers[l];
        const float stdv = (l == OUT ? 0.1f : 1.0f) * std::sqrt(2.0f / (27.0f * static_cast<float>(L.cin_real)));
        std::normal_distribution<float> nd(0.0f, stdv);
        for (int tap = 0; tap < 27; ++tap)
            for (int co = 0; co < L.cout; ++co)
                for (int ci = 0; ci < L.cin; ++ci) {
                    const bool live = ci < L.cin_real && (l != OUT || co == 0);
                    host[L.off + (static_cast<size_t>(tap) * L.cout + co) * L.cin + ci] = live ? nd(rng) : 0.0f;
                }
    }
    if (set_parameters(n.get(), host.data()) != cudaSuccess) return nullptr;
    return n.release();
}

cudaError_t ensure_buffers(Net* n, Dims d, const void* owner = nullptr) {
    if (d.nx % 4 || d.ny % 4 || d.nz % 4 || d.nx < 4 || d.ny < 4 || d.nz < 4) return cudaErrorInvalidValue;
    for (auto& set : n->sets)
        if (set->owner == owner && set->d0.nx == d.nx && set->d0.ny == d.ny && set->d0.nz == d.nz) {
            n->buf = set.get();
            return cudaSuccess;
        }
    auto b = std::make_unique<Buffers>();
    b->owner = owner;
    b->d0 = d;
    b->d1 = Dims{d.nx / 2, d.ny / 2, d.nz / 2, 0};
    b->d2 = Dims{d.nx / 4, d.ny / 4, d.nz / 4, 0};
    b->n0 = static_cast<size_t>(d.nx) * d.ny * d.nz;
    b->n1 = b->n0 / 8;
    b->n2 = b->n1 / 8;
    struct Item {
        void** p;
        size_t bytes;
    };
    std::vector<Item> items;
    auto bf = [&](__nv_bfloat16** p, size_t voxels, int ch) { items.push_back({reinterpret_cast<void**>(p), voxels * ch * sizeof(__nv_bfloat16)}); };
    bf(&b->in, b->n0, 16);
    bf(&b->e0a, b->n0, 16);
    bf(&b->e0b, b->n0, 16);
    bf(&b->p0, b->n1, 16);
    bf(&b->e1a, b->n1, 32);
    bf(&b->e1b, b->n1, 32);
    bf(&b->p1, b->n2, 32);
    bf(&b->ba, b->n2, 64);
    bf(&b->bb, b->n2, 64);
    bf(&b->cat1, b->n1, 96);
    bf(&b->d1a, b->n1, 32);
    bf(&b->d1b, b->n1, 32);
    bf(&b->cat0, b->n0, 48);
    bf(&b->d0a, b->n0, 16);
    bf(&b->d0b, b->n0, 16);
    const bool training = owner == nullptr;
    if (training) {
    bf(&b->g16, b->n0, 16);
    bf(&b->gd0b, b->n0, 16);
    bf(&b->gd0a, b->n0, 16);
    bf(&b->gcat0, b->n0, 48);
    bf(&b->gd1b, b->n1, 32);
    bf(&b->gd1a, b->n1, 32);
    bf(&b->gcat1, b->n1, 96);
    bf(&b->gbb, b->n2, 64);
    bf(&b->gba, b->n2, 64);
    bf(&b->gp1, b->n2, 32);
    bf(&b->ge1b, b->n1, 32);
    bf(&b->ge1a, b->n1, 32);
    bf(&b->gp0, b->n1, 16);
    bf(&b->ge0b, b->n0, 16);
    bf(&b->ge0a, b->n0, 16);
    items.push_back({reinterpret_cast<void**>(&b->target), b->n0 * sizeof(float)});
    }
    items.push_back({reinterpret_cast<void**>(&b->out), b->n0 * sizeof(float)});
    items.push_back({reinterpret_cast<void**>(&b->sums), 2 * sizeof(double)});
    items.push_back({reinterpret_cast<void**>(&b->scale), sizeof(float)});
    size_t total = 0;
    for (const auto& it : items) total += (it.bytes + 255) & ~static_cast<size_t>(255);
    if (cudaMalloc(&b->mem, total) != cudaSuccess) {
        b->mem = nullptr;
        cudaGetLastError();
        return cudaErrorMemoryAllocation;
    }
    b->bytes = total;
    char* p = static_cast<char*>(b->mem);
    for (const auto& it : items) {
        *it.p = p;
        p += (it.bytes + 255) & ~static_cast<size_t>(255);
    }
    if (cudaMemset(b->mem, 0, total) != cudaSuccess) return cudaErrorMemoryAllocation;
    n->buf = b.get();
    n->sets.push_back(std::move(b));
    return cudaSuccess;
}

namespace {

const __nv_bfloat16* W(const Net* n, int l) { return n->w16 + n->layers[l].off; }
const __nv_bfloat16* WT(const Net* n, int l) { return n->w16t + n->layers[l].off; }
const float* Bias(const Net* n, int l) { return n->w + n->layers[l].off + n->layers[l].wn; }
float* GW(Net* n, int l) { return n->g + n->layers[l].off; }
float* GB(Net* n, int l) { return n->g + n->layers[l].off + n->layers[l].wn; }

#define SFB_TRY(x)                              \
    do {                                        \
        if ((e = (x)) != cudaSuccess) return e; \
    } while (0)

// Forward pass from b (scaled inside) and p_prev; leaves the FP32 output in
// buf->out and every activation in place for the backward pass. 20 kernels.
cudaError_t forward(Net* n, const float* b, float b_factor, const float* p_prev, cudaStream_t s) {
    Buffers& B = *n->buf;
    cudaError_t e;
    SFB_TRY(cudaMemsetAsync(B.sums, 0, sizeof(double), s));
    k_sum_squares<<<blocks_for(B.n0), 256, 0, s>>>(b, b_factor, B.n0, B.sums);
    k_finish_scale<<<1, 32, 0, s>>>(B.sums, static_cast<double>(B.n0), B.scale);
    k_pack_input<<<blocks_for(B.n0), 256, 0, s>>>(b, p_prev, B.scale, b_factor, B.in, B.n0);
    SFB_TRY(cudaGetLastError());
    SFB_TRY(conv_any(16, 16, tc::RELU_BF16, B.in, W(n, E0A), Bias(n, E0A), B.e0a, 16, 0, B.d0, s, n->error));
    SFB_TRY(conv_any(16, 16, tc::RELU_BF16, B.e0a, W(n, E0B), Bias(n, E0B), B.e0b, 16, 0, B.d0, s, n->error));
    k_pool2<<<row_grid(B.d1.nx, 2, B.d1.ny, B.d1.nz), 256, 0, s>>>(B.e0b, 16, 0, B.p0, 16, B.d1);
    SFB_TRY(conv_any(16, 32, tc::RELU_BF16, B.p0, W(n, E1A), Bias(n, E1A), B.e1a, 32, 0, B.d1, s, n->error));
    SFB_TRY(conv_any(32, 32, tc::RELU_BF16, B.e1a, W(n, E1B), Bias(n, E1B), B.e1b, 32, 0, B.d1, s, n->error));
    k_pool2<<<row_grid(B.d2.nx, 4, B.d2.ny, B.d2.nz), 256, 0, s>>>(B.e1b, 32, 0, B.p1, 32, B.d2);
    SFB_TRY(conv_any(32, 64, tc::RELU_BF16, B.p1, W(n, BA), Bias(n, BA), B.ba, 64, 0, B.d2, s, n->error));
    SFB_TRY(conv_any(64, 64, tc::RELU_BF16, B.ba, W(n, BB), Bias(n, BB), B.bb, 64, 0, B.d2, s, n->error));
    k_upsample2<<<row_grid(B.d1.nx, 8, B.d1.ny, B.d1.nz), 256, 0, s>>>(B.bb, 64, B.d2, B.cat1, 96, 0);
    k_copy_channels<<<blocks_for(B.n1 * 4), 256, 0, s>>>(B.e1b, 32, 0, B.cat1, 96, 64, 32, B.n1, 0);
    SFB_TRY(conv_any(96, 32, tc::RELU_BF16, B.cat1, W(n, D1A), Bias(n, D1A), B.d1a, 32, 0, B.d1, s, n->error));
    SFB_TRY(conv_any(32, 32, tc::RELU_BF16, B.d1a, W(n, D1B), Bias(n, D1B), B.d1b, 32, 0, B.d1, s, n->error));
    k_upsample2<<<row_grid(B.d0.nx, 4, B.d0.ny, B.d0.nz), 256, 0, s>>>(B.d1b, 32, B.d1, B.cat0, 48, 0);
    k_copy_channels<<<blocks_for(B.n0 * 2), 256, 0, s>>>(B.e0b, 16, 0, B.cat0, 48, 32, 16, B.n0, 0);
    SFB_TRY(conv_any(48, 16, tc::RELU_BF16, B.cat0, W(n, D0A), Bias(n, D0A), B.d0a, 16, 0, B.d0, s, n->error));
    SFB_TRY(conv_any(16, 16, tc::RELU_BF16, B.d0a, W(n, D0B), Bias(n, D0B), B.d0b, 16, 0, B.d0, s, n->error));
    SFB_TRY(conv_any(16, 16, tc::LINEAR_F32_CH0, B.d0b, W(n, OUT), Bias(n, OUT), B.out, 1, 0, B.d0, s, n->error));
    return cudaGetLastError();
}

// Backward pass from d loss / d out (in B.g16, channel 0): parameter
// gradients into n->g (zeroed first). Each convolution's data gradient is a
// convolution of the output gradient with the transposed, tap-flipped
// weights; the ReLU masks use the stored (post-ReLU) activations.
cudaError_t backward(Net* n, cudaStream_t s) {
    Buffers& B = *n->buf;
    cudaError_t e;
    SFB_TRY(cudaMemsetAsync(n->g, 0, n->nparams * sizeof(float), s));
    // out layer (linear)
    SFB_TRY(wgrad_any(16, 16, B.d0b, B.g16, GW(n, OUT), GB(n, OUT), B.d0, s, n->error));
    SFB_TRY(conv_any(16, 16, tc::LINEAR_BF16, B.g16, WT(n, OUT), nullptr, B.gd0b, 16, 0, B.d0, s, n->error));
    // d0b, d0a (input of d0a: cat0 = [up(d1b) | e0b])
    k_relu_backward<<<blocks_for(B.n0 * 16 / 8), 256, 0, s>>>(B.gd0b, B.d0b, B.n0 * 16);
    SFB_TRY(wgrad_any(16, 16, B.d0a, B.gd0b, GW(n, D0B), GB(n, D0B), B.d0, s, n->error));
    SFB_TRY(conv_any(16, 16, tc::LINEAR_BF16, B.gd0b, WT(n, D0B), nullptr, B.gd0a, 16, 0, B.d0, s, n->error));
    k_relu_backward<<<blocks_for(B.n0 * 16 / 8), 256, 0, s>>>(B.gd0a, B.d0a, B.n0 * 16);
    SFB_TRY(wgrad_any(48, 16, B.cat0, B.gd0a, GW(n, D0A), GB(n, D0A), B.d0, s, n->error));
    SFB_TRY(conv_any(16, 48, tc::LINEAR_BF16, B.gd0a, WT(n, D0A), nullptr, B.gcat0, 48, 0, B.d0, s, n->error));
    k_upsample2_backward<<<row_grid(B.d1.nx, 4, B.d1.ny, B.d1.nz), 256, 0, s>>>(B.gcat0, 48, 0, 32, B.d1, B.gd1b);
    // d1b, d1a (input of d1a: cat1 = [up(bb) | e1b])
    k_relu_backward<<<blocks_for(B.n1 * 32 / 8), 256, 0, s>>>(B.gd1b, B.d1b, B.n1 * 32);
    SFB_TRY(wgrad_any(32, 32, B.d1a, B.gd1b, GW(n, D1B), GB(n, D1B), B.d1, s, n->error));
    SFB_TRY(conv_any(32, 32, tc::LINEAR_BF16, B.gd1b, WT(n, D1B), nullptr, B.gd1a, 32, 0, B.d1, s, n->error));
    k_relu_backward<<<blocks_for(B.n1 * 32 / 8), 256, 0, s>>>(B.gd1a, B.d1a, B.n1 * 32);
    SFB_TRY(wgrad_any(96, 32, B.cat1, B.gd1a, GW(n, D1A), GB(n, D1A), B.d1, s, n->error));
    SFB_TRY(conv_any(32, 96, tc::LINEAR_BF16, B.gd1a, WT(n, D1A), nullptr, B.gcat1, 96, 0, B.d1, s, n->error));
    k_upsample2_backward<<<row_grid(B.d2.nx, 8, B.d2.ny, B.d2.nz), 256, 0, s>>>(B.gcat1, 96, 0, 64, B.d2, B.gbb);
    // bottleneck
    k_relu_backward<<<blocks_for(B.n2 * 64 / 8), 256, 0, s>>>(B.gbb, B.bb, B.n2 * 64);
    SFB_TRY(wgrad_any(64, 64, B.ba, B.gbb, GW(n, BB), GB(n, BB), B.d2, s, n->error));
    SFB_TRY(conv_any(64, 64, tc::LINEAR_BF16, B.gbb, WT(n, BB), nullptr, B.gba, 64, 0, B.d2, s, n->error));
    k_relu_backward<<<blocks_for(B.n2 * 64 / 8), 256, 0, s>>>(B.gba, B.ba, B.n2 * 64);
    SFB_TRY(wgrad_any(32, 64, B.p1, B.gba, GW(n, BA), GB(n, BA), B.d2, s, n->error));
    SFB_TRY(conv_any(64, 32, tc::LINEAR_BF16, B.gba, WT(n, BA), nullptr, B.gp1, 32, 0, B.d2, s, n->error));
    // e1b receives the skip (channels 64..95 of cat1) and the pooled path
    k_copy_channels<<<blocks_for(B.n1 * 4), 256, 0, s>>>(B.gcat1, 96, 64, B.ge1b, 32, 0, 32, B.n1, 0);
    k_pool2_backward<<<row_grid(B.d1.nx, 4, B.d1.ny, B.d1.nz), 256, 0, s>>>(B.gp1, 32, B.d2, B.ge1b, 32, 0, 1);
    k_relu_backward<<<blocks_for(B.n1 * 32 / 8), 256, 0, s>>>(B.ge1b, B.e1b, B.n1 * 32);
    SFB_TRY(wgrad_any(32, 32, B.e1a, B.ge1b, GW(n, E1B), GB(n, E1B), B.d1, s, n->error));
    SFB_TRY(conv_any(32, 32, tc::LINEAR_BF16, B.ge1b, WT(n, E1B), nullptr, B.ge1a, 32, 0, B.d1, s, n->error));
    k_relu_backward<<<blocks_for(B.n1 * 32 / 8), 256, 0, s>>>(B.ge1a, B.e1a, B.n1 * 32);
    SFB_TRY(wgrad_any(16, 32, B.p0, B.ge1a, GW(n, E1A), GB(n, E1A), B.d1, s, n->error));
    SFB_TRY(conv_any(32, 16, tc::LINEAR_BF16, B.ge1a, WT(n, E1A), nullptr, B.gp0, 16, 0, B.d1, s, n->error));
    // e0b: skip (channels 32..47 of cat0) + pooled path
    k_copy_channels<<<blocks_for(B.n0 * 2), 256, 0, s>>>(B.gcat0, 48, 32, B.ge0b, 16, 0, 16, B.n0, 0);
    k_pool2_backward<<<row_grid(B.d0.nx, 2, B.d0.ny, B.d0.nz), 256, 0, s>>>(B.gp0, 16, B.d1, B.ge0b, 16, 0, 1);
    k_relu_backward<<<blocks_for(B.n0 * 16 / 8), 256, 0, s>>>(B.ge0b, B.e0b, B.n0 * 16);
    SFB_TRY(wgrad_any(16, 16, B.e0a, B.ge0b, GW(n, E0B), GB(n, E0B), B.d0, s, n->error));
    SFB_TRY(conv_any(16, 16, tc::LINEAR_BF16, B.ge0b, WT(n, E0B), nullptr, B.ge0a, 16, 0, B.d0, s, n->error));
    k_relu_backward<<<blocks_for(B.n0 * 16 / 8), 256, 0, s>>>(B.ge0a, B.e0a, B.n0 * 16);
    SFB_TRY(wgrad_any(16, 16, B.in, B.ge0a, GW(n, E0A), GB(n, E0A), B.d0, s, n->error));
    return cudaGetLastError();
}

// Target of the training: (p_target - p_prev) * scale.
__global__ void k_make_target(const float* __restrict__ pt, const float* __restrict__ pp, const float* __restrict__ scale, float* __restrict__ out, size_t n) {
    const float s = *scale;
    for (size_t v = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; v < n; v += static_cast<size_t>(gridDim.x) * blockDim.x) out[v] = (pt[v] - (pp ? pp[v] : 0.0f)) * s;
}

cudaError_t loss_and_gradients(Net* n, const float* b, float b_factor, const float* p_prev, const float* p_target, double* loss, cudaStream_t s) {
    cudaError_t e;
    SFB_TRY(forward(n, b, b_factor, p_prev, s));
    Buffers& B = *n->buf;
    k_make_target<<<blocks_for(B.n0), 256, 0, s>>>(p_target, p_prev, B.scale, B.target, B.n0);
    SFB_TRY(cudaMemsetAsync(B.sums + 1, 0, sizeof(double), s));
    k_mse<<<blocks_for(B.n0), 256, 0, s>>>(B.out, B.target, B.n0, B.g16, B.sums + 1);
    SFB_TRY(backward(n, s));
    double sum = 0.0;
    SFB_TRY(cudaMemcpyAsync(&sum, B.sums + 1, sizeof(double), cudaMemcpyDeviceToHost, s));
    SFB_TRY(cudaStreamSynchronize(s));
    if (loss) *loss = sum / static_cast<double>(B.n0);
    return cudaSuccess;
}

#undef SFB_TRY

}  // namespace

cudaError_t prepare(Net* n, Dims d, const void* owner) { return ensure_buffers(n, d, owner); }

// Networks created and not yet destroyed: a context destroyed after the
// network it was attached to must not touch it.
std::mutex g_live_mu;
std::set<const Net*> g_live;

void register_live(const Net* n, bool live) {
    std::lock_guard<std::mutex> lock(g_live_mu);
    if (live) g_live.insert(n);
    else g_live.erase(n);
}

void release(Net* n, const void* owner) {
    if (n == nullptr || owner == nullptr) return;
    std::lock_guard<std::mutex> lock(g_live_mu);
    if (g_live.count(n) == 0) return;
    for (auto it = n->sets.begin(); it != n->sets.end();) {
        if ((*it)->owner == owner) {
            if (n->buf == it->get()) n->buf = nullptr;
            it = n->sets.erase(it);
        } else {
            ++it;
        }
    }
}

cudaError_t predict(Net* n, const float* b, float b_factor, const float* p_prev, float* p0, Dims d, cudaStream_t s, int* launches, const void* owner) {
    cudaError_t e = ensure_buffers(n, d, owner);
    if (e != cudaSuccess) return e;
    if ((e = forward(n, b, b_factor, p_prev, s)) != cudaSuccess) return e;
    k_unpack_output<<<blocks_for(n->buf->n0), 256, 0, s>>>(n->buf->out, p_prev, n->buf->scale, p0, n->buf->n0);
    if (launches) *launches += kPredictKernels;
    return cudaGetLastError();
}

cudaError_t adam_step(Net* n, float lr, cudaStream_t s) {
    n->adam_t += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    const float bc1 = 1.0f - std::pow(b1, static_cast<float>(n->adam_t)), bc2 = 1.0f - std::pow(b2, static_cast<float>(n->adam_t));
    for (int l = 0; l < NLAYERS; ++l) {
        const Layer& L = n->layers[l];
        k_adam<<<blocks_for(L.wn), 256, 0, s>>>(n->w + L.off, n->g + L.off, n->m + L.off, n->v + L.off, n->w16 + L.off, n->w16t + L.off, L.cout, L.cin, L.wn, lr, b1, b2, 1e-8f, bc1, bc2);
        const size_t bo = L.off + L.wn;
        k_adam<<<1, 64, 0, s>>>(n->w + bo, n->g + bo, n->m + bo, n->v + bo, nullptr, nullptr, 1, 1, static_cast<size_t>(L.cout), lr, b1, b2, 1e-8f, bc1, bc2);
    }
    return cudaGetLastError();
}

}  // namespace sfb::net

using sfb::net::Net;

namespace {

StableFluidsResult status(cudaError_t e) {
    if (e == cudaSuccess) return STABLE_FLUIDS_RESULT_OK;
    cudaGetLastError();
    return e == cudaErrorMemoryAllocation ? STABLE_FLUIDS_RESULT_OUT_OF_MEMORY : STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
}

}  // namespace

extern "C" {

StableFluidsResult stable_fluids_b200_network_create(uint32_t seed, void** out_network) {
    if (out_network == nullptr) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    *out_network = nullptr;
    Net* n = sfb::net::create_net(seed);
    if (n == nullptr) {
        cudaGetLastError();
        return STABLE_FLUIDS_RESULT_OUT_OF_MEMORY;
    }
    sfb::net::register_live(n, true);
    *out_network = n;
    return STABLE_FLUIDS_RESULT_OK;
}

StableFluidsResult stable_fluids_b200_network_destroy(void* network) {
    if (network != nullptr) cudaDeviceSynchronize();
    sfb::net::register_live(static_cast<Net*>(network), false);
    delete static_cast<Net*>(network);
    return STABLE_FLUIDS_RESULT_OK;
}

StableFluidsResult stable_fluids_b200_network_parameters(void* network, uint64_t* out_count, float* out_host_values) {
    if (network == nullptr) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    auto* n = static_cast<Net*>(network);
    if (out_count) *out_count = n->nparams;
    if (out_host_values) return status(cudaMemcpy(out_host_values, n->w, n->nparams * sizeof(float), cudaMemcpyDeviceToHost));
    return STABLE_FLUIDS_RESULT_OK;
}

StableFluidsResult stable_fluids_b200_network_set_parameters(void* network, const float* host_values) {
    if (network == nullptr || host_values == nullptr) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    return status(sfb::net::set_parameters(static_cast<Net*>(network), host_values));
}

StableFluidsResult stable_fluids_b200_network_predict(void* network, const float* divergence, const float* previous_pressure, int32_t nx, int32_t ny, int32_t nz, float cell_size, float* out_pressure, void* stream) {
    if (network == nullptr || divergence == nullptr || out_pressure == nullptr) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    const sfb::Dims d{nx, ny, nz, 0};
    return status(sfb::net::predict(static_cast<Net*>(network), divergence, cell_size * cell_size, previous_pressure, out_pressure, d, static_cast<cudaStream_t>(stream), nullptr, nullptr));
}

StableFluidsResult stable_fluids_b200_network_gradients(void* network, const float* divergence, const float* previous_pressure, const float* target_pressure, int32_t nx, int32_t ny, int32_t nz, float cell_size, double* out_loss, float* out_host_gradients, void* stream) {
    if (network == nullptr || divergence == nullptr || target_pressure == nullptr) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    auto* n = static_cast<Net*>(network);
    const sfb::Dims d{nx, ny, nz, 0};
    const auto s = static_cast<cudaStream_t>(stream);
    cudaError_t e = sfb::net::ensure_buffers(n, d);
    if (e == cudaSuccess) e = sfb::net::loss_and_gradients(n, divergence, cell_size * cell_size, previous_pressure, target_pressure, out_loss, s);
    if (e == cudaSuccess && out_host_gradients) e = cudaMemcpy(out_host_gradients, n->g, n->nparams * sizeof(float), cudaMemcpyDeviceToHost);
    return status(e);
}

StableFluidsResult stable_fluids_b200_network_train_step(void* network, const float* divergence, const float* previous_pressure, const float* target_pressure, int32_t nx, int32_t ny, int32_t nz, float cell_size, float learning_rate, double* out_loss, void* stream) {
    if (network == nullptr || divergence == nullptr || target_pressure == nullptr) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    auto* n = static_cast<Net*>(network);
    const sfb::Dims d{nx, ny, nz, 0};
    const auto s = static_cast<cudaStream_t>(stream);
    cudaError_t e = sfb::net::ensure_buffers(n, d);
    if (e == cudaSuccess) e = sfb::net::loss_and_gradients(n, divergence, cell_size * cell_size, previous_pressure, target_pressure, out_loss, s);
    if (e == cudaSuccess) e = sfb::net::adam_step(n, learning_rate, s);
    return status(e);
}

}  // extern "C"
