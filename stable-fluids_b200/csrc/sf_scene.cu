// sf_scene.cu -- the interactive plume scene of the reference viewer
// (vulkan-app/scene_plume.cpp:241-335) generated on the device.
//
// The viewer builds three masks on the host (a swirl field around the plume
// axis and a drift blob above the source), and every step recomputes the
// force's x and z components on the host from them and three animated
// scalars, uploads them and copies them into the context. Here the masks are
// closed-form functions of the cell position, so one kernel evaluates them
// and writes the force components straight into the context's force field:
// 8 bytes written per cell, nothing read, no host work per cell. The
// arithmetic follows the viewer's float expressions operation by operation,
// each rounded once (no contraction), so the fields equal the viewer's.

#include <cuda_runtime.h>

#include "sf_launch.h"

namespace sfb {

namespace {

// 1 - |p - c|^2 / r^2 inside the sphere, else 0 (scene_plume.cpp:257-265).
__device__ __forceinline__ float radial_weight(float px, float py, float pz, float cx, float cy, float cz, float radius) {
    const float dx = __fsub_rn(px, cx);
    const float dy = __fsub_rn(py, cy);
    const float dz = __fsub_rn(pz, cz);
    const float radius2 = __fmul_rn(radius, radius);
    const float dist2 = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
    if (dist2 >= radius2 || radius2 <= 0.0f) return 0.0f;
    return __fsub_rn(1.0f, __fdiv_rn(dist2, radius2));
}

__device__ __forceinline__ float cell_centre(int i, float h) { return __fmul_rn(__fadd_rn(static_cast<float>(i), 0.5f), h); }

// The scene's constant inputs (scene_plume.cpp:267-300): density source
// 32 w_s, force y 7.6 w_s; force x and z start at zero.
__global__ void __launch_bounds__(256) k_plume_setup(float* __restrict__ source, float* __restrict__ fx, float* __restrict__ fy, float* __restrict__ fz, PlumeGeometry g, Dims d) {
    const int x = static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x), y = static_cast<int>(blockIdx.y * blockDim.y + threadIdx.y), z = static_cast<int>(blockIdx.z * blockDim.z + threadIdx.z);
    if (x >= d.nx || y >= d.ny || z >= d.nz) return;
    const size_t i = static_cast<size_t>(x) + static_cast<size_t>(d.nx) * (static_cast<size_t>(y) + static_cast<size_t>(d.ny) * static_cast<size_t>(z));
    const float w = radial_weight(cell_centre(x, g.h), cell_centre(y, g.h), cell_centre(z, g.h), g.source_x, g.source_y, g.source_z, g.source_r);
    source[i] = __fmul_rn(32.0f, w);
    fy[i] = __fmul_rn(7.6f, w);
    fx[i] = 0.0f;
    fz[i] = 0.0f;
}

// One step's force x and z (scene_plume.cpp:274-284 masks, :326-330 forces).
__global__ void __launch_bounds__(256) k_plume_forces(float* __restrict__ fx, float* __restrict__ fz, PlumeGeometry g, Dims d, float drift_x, float drift_z, float swirl) {
    const int x = static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x), y = static_cast<int>(blockIdx.y * blockDim.y + threadIdx.y), z = static_cast<int>(blockIdx.z * blockDim.z + threadIdx.z);
    if (x >= d.nx || y >= d.ny || z >= d.nz) return;
    const size_t i = static_cast<size_t>(x) + static_cast<size_t>(d.nx) * (static_cast<size_t>(y) + static_cast<size_t>(d.ny) * static_cast<size_t>(z));
    const float px = cell_centre(x, g.h), py = cell_centre(y, g.h), pz = cell_centre(z, g.h);
    const float swirl_w = radial_weight(px, py, pz, g.source_x, g.swirl_y, g.source_z, g.swirl_r);
    const float drift_w = radial_weight(px, py, pz, g.source_x, g.drift_y, g.source_z, g.drift_r);
    const float dx = __fsub_rn(px, g.source_x);
    const float dz = __fsub_rn(pz, g.source_z);
    const float radial = __fsqrt_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dz, dz)));
    const float inv_radial = radial > 1.0e-5f ? __fdiv_rn(1.0f, radial) : 0.0f;
    const float swirl_xm = __fmul_rn(__fmul_rn(-dz, inv_radial), swirl_w);
    const float swirl_zm = __fmul_rn(__fmul_rn(dx, inv_radial), swirl_w);
    fx[i] = __fadd_rn(__fmul_rn(drift_x, drift_w), __fmul_rn(swirl, swirl_xm));
    fz[i] = __fadd_rn(__fmul_rn(drift_z, drift_w), __fmul_rn(swirl, swirl_zm));
}

// One thread per cell, (32, 4, 2) blocks, x fastest (no index division).
dim3 scene_block() { return dim3(32, 4, 2); }
dim3 scene_grid(const Dims& d) { return dim3(static_cast<unsigned>((d.nx + 31) / 32), static_cast<unsigned>((d.ny + 3) / 4), static_cast<unsigned>((d.nz + 1) / 2)); }

}  // namespace

cudaError_t launch_plume_setup(float* source, float* fx, float* fy, float* fz, const PlumeGeometry& g, Dims d, cudaStream_t s) {
    k_plume_setup<<<scene_grid(d), scene_block(), 0, s>>>(source, fx, fy, fz, g, d);
    return cudaGetLastError();
}

cudaError_t launch_plume_forces(float* fx, float* fz, const PlumeGeometry& g, Dims d, float drift_x, float drift_z, float swirl, cudaStream_t s) {
    k_plume_forces<<<scene_grid(d), scene_block(), 0, s>>>(fx, fz, g, d, drift_x, drift_z, swirl);
    return cudaGetLastError();
}

}  // namespace sfb
