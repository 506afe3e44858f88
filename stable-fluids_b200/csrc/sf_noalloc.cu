// sf_noalloc.cu -- the pressure-residual measurement without any allocation.
//
// Some callers cannot allocate device memory at the point where they want a
// number: code running inside a host callback or an allocation-free phase of
// a renderer's frame, a process whose device memory is fully reserved by its
// own pool, or an embedding that forbids cudaMalloc after start-up. For them
// stable_fluids_b200_pressure_residual_noalloc() computes the same FP64
// relative Poisson residual as the step's residual measurement, with its
// scratch (one set of partial sums per z plane) in a fixed, file-scope device
// array instead of context memory.
//
// Limits and sharing:
//   - at most kMaxPlanes z planes (nz <= 4096); larger grids are rejected;
//   - the array (4096 x 4 doubles = 128 KiB) lives on every device that
//     loads this library, until the process exits;
//   - every call on a device uses the same array: calls whose work overlaps
//     on the GPU (different streams, no ordering between them) race and give
//     wrong results; calls ordered on one stream are fine. Each call
//     overwrites the partial sums it reads, so nothing has to be cleared.
//   - every call looks up the array's device address on the current device
//     (cudaGetSymbolAddress); the first call on a device may load the
//     library's device code there, so make that first call before any
//     stream capture.
//   - every invalid argument is rejected before any CUDA call.

#include <cuda_runtime.h>

#include <cmath>

#include "sf_boundary.h"
#include "sf_device.cuh"
#include "sf_types.h"
#include "stable-fluids-b200.h"

namespace sfb {
namespace {

constexpr int kMaxPlanes = 4096;
constexpr int kThreads = 256;

// Partial sums per z plane: sum e, sum e^2, sum b, sum b^2 (e = b - A p).
static __device__ __align__(256) double g_residual_partials[kMaxPlanes][4];

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// One block per z plane: the plane's four sums, reduced in a fixed order.
__global__ void __launch_bounds__(kThreads) k_plane_partials(const float* __restrict__ p, const float* __restrict__ div, Dims d, float h2, FlowBC b, double (*partials)[4]) {
    const int z = static_cast<int>(blockIdx.x);
    double se = 0.0, se2 = 0.0, sb = 0.0, sb2 = 0.0;
    const int cells = d.nx * d.ny;
    for (int i = static_cast<int>(threadIdx.x); i < cells; i += kThreads) {
        const int x = i % d.nx, y = i / d.nx;
        const size_t c = lin(x, y, z, d);
        const double nb = static_cast<double>(load_pressure(p, x - 1, y, z, d, b)) + static_cast<double>(load_pressure(p, x + 1, y, z, d, b)) + static_cast<double>(load_pressure(p, x, y - 1, z, d, b)) + static_cast<double>(load_pressure(p, x, y + 1, z, d, b))
                        + static_cast<double>(load_pressure(p, x, y, z - 1, d, b)) + static_cast<double>(load_pressure(p, x, y, z + 1, d, b));
        const double bb = static_cast<double>(h2) * static_cast<double>(div[c]);
        const double e = bb - (nb - 6.0 * static_cast<double>(p[c]));
        se += e;
        se2 += e * e;
        sb += bb;
        sb2 += bb * bb;
    }
    __shared__ double part[4][kThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    se = warp_sum(se);
    se2 = warp_sum(se2);
    sb = warp_sum(sb);
    sb2 = warp_sum(sb2);
    if (lane == 0) {
        part[0][warp] = se;
        part[1][warp] = se2;
        part[2][warp] = sb;
        part[3][warp] = sb2;
    }
    __syncthreads();
    if (threadIdx.x < 4) {
        double s = 0.0;
        for (int w = 0; w < kThreads / 32; ++w) s += part[threadIdx.x][w];
        partials[z][threadIdx.x] = s;
    }
}

// Sums the planes in order and writes {rel_residual, rhs_norm}.
__global__ void k_finish(const double (*partials)[4], int nz, double n, int singular, double* out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double s[4] = {0.0, 0.0, 0.0, 0.0};
    for (int z = 0; z < nz; ++z)
        for (int k = 0; k < 4; ++k) s[k] += partials[z][k];
    double r2 = s[1], b2 = s[3];
    if (singular) {
        const double mb = s[2] / n;
        r2 = s[1] - 2.0 * mb * s[0] + n * mb * mb;
        b2 = s[3] - n * mb * mb;
    }
    r2 = r2 < 0.0 ? 0.0 : r2;
    b2 = b2 < 0.0 ? 0.0 : b2;
    out[0] = b2 > 0.0 ? sqrt(r2) / sqrt(b2) : 0.0;
    out[1] = sqrt(b2);
}

// Device address of the partials array on the current device and context.
// Looked up on every call (a cheap runtime query), so a reset device or a
// different context never sees a stale address.
double (*partials_address())[4] {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_residual_partials) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return static_cast<double (*)[4]>(p);
}

}  // namespace
}  // namespace sfb

extern "C" StableFluidsResult stable_fluids_b200_pressure_residual_noalloc(const float* pressure, const float* divergence, int32_t nx, int32_t ny, int32_t nz, float cell_size, const StableFluidsFlowBoundaryConfig* flow_boundary, double* out_residual, void* stream) {
    using namespace sfb;
    // every rejection happens here, before any CUDA call
    if (pressure == nullptr || divergence == nullptr || flow_boundary == nullptr || out_residual == nullptr) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    if (nx <= 0 || ny <= 0 || nz <= 0 || !(cell_size > 0.0f) || !std::isfinite(cell_size)) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    if (nz > kMaxPlanes) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;  // beyond the fixed scratch: rejected
    if (static_cast<long long>(nx) * ny > (1ll << 30)) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    FlowBC b{};
    if (!flatten_flow(*flow_boundary, b)) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    auto partials = partials_address();
    if (partials == nullptr) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    const Dims d{nx, ny, nz, 0};
    const float h2 = cell_size * cell_size;
    const auto s = static_cast<cudaStream_t>(stream);
    k_plane_partials<<<static_cast<unsigned>(nz), kThreads, 0, s>>>(pressure, divergence, d, h2, b, partials);
    const double n = static_cast<double>(nx) * static_cast<double>(ny) * static_cast<double>(nz);
    k_finish<<<1, 32, 0, s>>>(partials, nz, n, b.any_outflow ? 0 : 1, out_residual);
    return cudaGetLastError() == cudaSuccess ? STABLE_FLUIDS_RESULT_OK : STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
}
