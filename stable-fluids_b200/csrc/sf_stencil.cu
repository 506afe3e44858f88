// sf_stencil.cu -- the iterative 7-point solves of the step: implicit
// diffusion (I - alpha L) x = b for velocity components and scalars, and the
// pressure Poisson equation sum6(p) - 6 p = h^2 div.
//
// Update formulas (backend-cuda.cu:354-375, 398-407), neighbour sum order
// x-, x+, y-, y+, z-, z+:
//   diffusion: x = (b + alpha * nb) / (1 + 6 alpha)
//   pressure : p = (nb - h^2 * div) / 6
// RBGS updates (x+y+z) even cells, then odd ones, in place; JACOBI updates
// every cell from the previous iterate.

#include <cuda_runtime.h>

#include "sf_device.cuh"
#include "sf_launch.h"

namespace sfb {

namespace {

template <int KIND>
__device__ __forceinline__ float neighbour(const float* __restrict__ f, int x, int y, int z, const Dims& d, const FlowBC& fb, const ScalarBC& sb) {
    if constexpr (KIND == KIND_PRESSURE) return load_pressure(f, x, y, z, d, fb);
    else if constexpr (KIND == KIND_SCALAR) return load_scalar(f, x, y, z, d, sb);
    else return load_velocity(f, KIND, x, y, z, d, fb);
}

template <int KIND>
__device__ __forceinline__ float update(float nb, float rhs, float coef) {
    if constexpr (KIND == KIND_PRESSURE) return (nb - coef * rhs) / 6.0f;
    else return (rhs + coef * nb) / (1.0f + 6.0f * coef);
}

template <int KIND>
__device__ __forceinline__ float neighbour_sum(const float* __restrict__ f, int x, int y, int z, const Dims& d, const FlowBC& fb, const ScalarBC& sb) {
    return neighbour<KIND>(f, x - 1, y, z, d, fb, sb) + neighbour<KIND>(f, x + 1, y, z, d, fb, sb) + neighbour<KIND>(f, x, y - 1, z, d, fb, sb) + neighbour<KIND>(f, x, y + 1, z, d, fb, sb) + neighbour<KIND>(f, x, y, z - 1, d, fb, sb)
         + neighbour<KIND>(f, x, y, z + 1, d, fb, sb);
}

// One colour of an RBGS iteration; thread (hx, y, z) owns cell
// x = 2 hx + ((y + z + parity) & 1), so every thread is active.
template <int KIND>
__global__ void __launch_bounds__(256) k_rbgs_colour(float* x, const float* __restrict__ rhs, float coef, int parity, Dims d, FlowBC fb, ScalarBC sb) {
    const int hx = static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x);
    const int y = static_cast<int>(blockIdx.y * blockDim.y + threadIdx.y);
    const int z = static_cast<int>(blockIdx.z * blockDim.z + threadIdx.z);
    if (y >= d.ny || z >= d.nz) return;
    const int cx = 2 * hx + ((y + z + parity) & 1);
    if (cx >= d.nx) return;
    const float nb = neighbour_sum<KIND>(x, cx, y, z, d, fb, sb);
    const size_t i = lin(cx, y, z, d);
    x[i] = update<KIND>(nb, rhs[i], coef);
}

template <int KIND>
__global__ void __launch_bounds__(256) k_jacobi(float* __restrict__ dst, const float* __restrict__ src, const float* __restrict__ rhs, float coef, Dims d, FlowBC fb, ScalarBC sb) {
    const int cx = static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x);
    const int y = static_cast<int>(blockIdx.y * blockDim.y + threadIdx.y);
    const int z = static_cast<int>(blockIdx.z * blockDim.z + threadIdx.z);
    if (cx >= d.nx || y >= d.ny || z >= d.nz) return;
    const float nb = neighbour_sum<KIND>(src, cx, y, z, d, fb, sb);
    const size_t i = lin(cx, y, z, d);
    dst[i] = update<KIND>(nb, rhs[i], coef);
}

__global__ void k_scale_field(float* __restrict__ q, float factor, size_t n) {
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n; i += static_cast<size_t>(gridDim.x) * blockDim.x) q[i] = q[i] * factor;
}

template <int KIND>
cudaError_t run_simple(const StencilArgs& a, cudaStream_t s) {
    const Dims& d = a.dims;
    const size_t n = static_cast<size_t>(d.nx) * d.ny * d.nz;
    const size_t bytes = n * sizeof(float);
    const dim3 block(32, 4, 2);
    cudaError_t e = cudaSuccess;
    if (a.scheme == SCHEME_RBGS) {
        if (a.init == INIT_FROM_B) e = cudaMemcpyAsync(a.x, a.b, bytes, cudaMemcpyDeviceToDevice, s);
        else if (a.init == INIT_ZERO) e = cudaMemsetAsync(a.x, 0, bytes, s);
        if (e != cudaSuccess) return e;
        const dim3 grid(static_cast<unsigned>(((d.nx + 1) / 2 + 31) / 32), static_cast<unsigned>((d.ny + 3) / 4), static_cast<unsigned>((d.nz + 1) / 2));
        for (int it = 0; it < a.iterations; ++it) {
            k_rbgs_colour<KIND><<<grid, block, 0, s>>>(a.x, a.b, a.coef, 0, d, a.flow, a.scalar);
            k_rbgs_colour<KIND><<<grid, block, 0, s>>>(a.x, a.b, a.coef, 1, d, a.flow, a.scalar);
        }
        if (a.launches) *a.launches += 2 * a.iterations;
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    } else {
        const dim3 grid(static_cast<unsigned>((d.nx + 31) / 32), static_cast<unsigned>((d.ny + 3) / 4), static_cast<unsigned>((d.nz + 1) / 2));
        // Choose the first source so that the last sweep lands in x.
        const float* src = a.x;
        if (a.init == INIT_FROM_B) src = a.b;
        else if (a.init == INIT_ZERO) {
            // Zero the buffer the first sweep does not write.
            float* zero = (a.iterations & 1) ? a.scratch : a.x;
            if ((e = cudaMemsetAsync(zero, 0, bytes, s)) != cudaSuccess) return e;
            src = zero;
        }
        if (a.iterations == 0) {
            if (src != a.x) e = cudaMemcpyAsync(a.x, src, bytes, cudaMemcpyDeviceToDevice, s);
            if (e != cudaSuccess) return e;
        }
        for (int it = 0; it < a.iterations; ++it) {
            const int left = a.iterations - it;  // sweeps still to run, this one included
            float* dst = (left & 1) ? a.x : a.scratch;
            if (dst == src) dst = (dst == a.x) ? a.scratch : a.x;
            k_jacobi<KIND><<<grid, block, 0, s>>>(dst, src, a.b, a.coef, d, a.flow, a.scalar);
            src = dst;
        }
        if (a.launches) *a.launches += a.iterations;
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        if (src != a.x && a.iterations > 0) {
            if ((e = cudaMemcpyAsync(a.x, src, bytes, cudaMemcpyDeviceToDevice, s)) != cudaSuccess) return e;
        }
    }
    if (a.out_scale != 1.0f) {
        size_t g = (n + 255) / 256;
        if (g > 148u * 32u) g = 148u * 32u;
        k_scale_field<<<static_cast<unsigned>(g), 256, 0, s>>>(a.x, a.out_scale, n);
        e = cudaGetLastError();
        if (a.launches) *a.launches += 1;
    }
    return e;
}

}  // namespace

cudaError_t launch_stencil(const StencilArgs& a, cudaStream_t s) {
    switch (a.kind) {
    case KIND_VEL_X: return run_simple<KIND_VEL_X>(a, s);
    case KIND_VEL_Y: return run_simple<KIND_VEL_Y>(a, s);
    case KIND_VEL_Z: return run_simple<KIND_VEL_Z>(a, s);
    case KIND_SCALAR: return run_simple<KIND_SCALAR>(a, s);
    case KIND_PRESSURE: return run_simple<KIND_PRESSURE>(a, s);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace sfb
