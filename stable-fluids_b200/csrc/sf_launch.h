// sf_launch.h -- host-callable launchers for the step kernels. Plain types
// only, so the C++23 host runtime (sf_context.cpp) can call them without
// compiling CUDA.
#pragma once

#include <cuda_runtime.h>

#include "sf_types.h"

namespace sfb {

constexpr int kMaxForcesPerLaunch = 8;

struct ForceArgs {
    void* vel[3];                           // SoA velocity, FP32 or BF16 (read; written when write_soa)
    const float* force[kMaxForcesPerLaunch][3];
    int force_count;
    float dt;
    size_t n;
    void* packed;                           // packed velocity, float4 or 4 x BF16 (written when non-null)
    int write_soa;
    int bf16;                               // advected fields stored in BF16
};

// How a stencil solve obtains its initial iterate.
enum InitMode : int { INIT_FROM_X = 0, INIT_FROM_B = 1, INIT_ZERO = 2 };

enum Scheme : int { SCHEME_RBGS = 0, SCHEME_JACOBI = 1 };

struct StencilArgs {
    int kind;            // StencilKind
    int scheme;          // Scheme
    int init;            // InitMode
    int iterations;      // RBGS iterations (red + black) or Jacobi sweeps
    int per_pass;        // iterations fused per HBM pass (temporal blocking); 0 = automatic
    float coef;          // alpha (diffusion) or h^2 (pressure)
    float out_scale;     // multiply the final iterate by this (1 = none)
    float* x;            // the iterate (result lands here); BF16 elements when bf16
    const float* b;      // right-hand side (diffusion: advected field; pressure: divergence); BF16 when bf16
    float* scratch;      // a field-sized buffer for out-of-place sweeps
    float* scratch2;     // a second field-sized buffer (a red-black solve's split right-hand side); may be null
    Dims dims;
    FlowBC flow;
    ScalarBC scalar;
    int* launches;       // incremented by the number of kernels enqueued (may be null)
    int blocked;         // 1: temporally blocked passes where supported; 0: one launch per sweep
    unsigned* error_flag;  // device word a kernel sets when a bounded wait gives up
    int bf16;            // x, b, scratch hold BF16 (diffusion kinds of a BF16-storage context)
};

// `bf16` arguments: the advected field arrays passed are BF16 (else FP32).
cudaError_t launch_fill(void* f, float value, size_t n, int bf16, cudaStream_t s);
// FP32 -> BF16 (to_bf16) or BF16 -> FP32 element conversion.
cudaError_t launch_convert(void* dst, const void* src, size_t n, int to_bf16, cudaStream_t s);
cudaError_t launch_force_pack(const ForceArgs& a, cudaStream_t s);
cudaError_t launch_advect_velocity(const void* packed, void* out_x, void* out_y, void* out_z, float dt, Dims d, float h, const FlowBC& b, int bf16, cudaStream_t s);
cudaError_t launch_scalar_source_advect(const void* packed, const void* data, const float* source, void* out, float dt, Dims d, float h, const FlowBC& fb, const ScalarBC& sb, int bf16, cudaStream_t s);
cudaError_t launch_scalar_source(void* data, const float* source, float dt, size_t n, int bf16, cudaStream_t s);
cudaError_t launch_scale(void* data, float factor, size_t n, int bf16, cudaStream_t s);
cudaError_t launch_stencil(const StencilArgs& a, cudaStream_t s);
cudaError_t launch_divergence(float* div, const void* vx, const void* vy, const void* vz, Dims d, float h, const FlowBC& b, int bf16, cudaStream_t s);
// u -= grad p (in place) and repack; with stats != nullptr also accumulates
// the FP64 residual sums of the pressure system into stats.
cudaError_t launch_project(void* vx, void* vy, void* vz, void* packed, const float* p, const float* div, Dims d, float h, float h2, const FlowBC& b, DeviceStats* stats, int bf16, cudaStream_t s);
cudaError_t launch_residual_sums(const float* p, const float* div, Dims d, float h2, const FlowBC& b, DeviceStats* stats, cudaStream_t s);
// The same sums with the vectorised z-marching layout; false (nothing
// launched) when the grid or the pointers do not suit it (nx % 4, 16-byte
// alignment).
bool launch_residual_sums_vec(const float* p, const float* div, Dims d, float h2, const FlowBC& b, DeviceStats* stats, cudaStream_t s);
// The Jacobi pressure sweeps of one check interval of the residual-driven
// solve (a.iterations sweeps from x, landing in x), the last of them adding
// the FP64 residual sums of its input iterate to stats; false (nothing
// launched) when the solve is not a plain FP32 Jacobi pressure solve on a
// vectorisable grid.
bool launch_pressure_interval_fused(const StencilArgs& a, DeviceStats* stats, cudaStream_t s);
cudaError_t launch_residual_finalize(DeviceStats* stats, Dims d, int singular, int iterations, cudaStream_t s);
// One check of the residual-driven pressure solve (see k_residual_check).
cudaError_t launch_residual_check(DeviceStats* stats, Dims d, int singular, int reset, int increment, double tol, int max_iterations, cudaGraphConditionalHandle handle, cudaStream_t s);
// Learned warm start: keeps the candidate in p or replaces it by alt,
// whichever has the smaller relative residual (two kernels).
cudaError_t launch_warm_start_select(DeviceStats* learned, const DeviceStats* plain, Dims d, int singular, float* p, const float* alt, cudaStream_t s);
// Learned warm start on the coarsened grid: coarse = mean of each 2x2x2
// block of fine (fine dims even); fine_p += trilinear prolongation of
// (coarse_new - coarse_old) to the fine cell centres.
cudaError_t launch_restrict2(const float* fine, float* coarse, Dims fine_dims, cudaStream_t s);
cudaError_t launch_prolong_add(const float* coarse_new, const float* coarse_old, float* fine_p, Dims fine_dims, cudaStream_t s);

// The reference viewer's plume scene (sf_scene.cu): geometry in world units,
// derived from the grid by plume_geometry (host).
struct PlumeGeometry {
    float h;
    float source_x, source_y, source_z, source_r;
    float swirl_y, swirl_r;
    float drift_y, drift_r;
};
cudaError_t launch_plume_setup(float* source, float* fx, float* fy, float* fz, const PlumeGeometry& g, Dims d, cudaStream_t s);
cudaError_t launch_plume_forces(float* fx, float* fz, const PlumeGeometry& g, Dims d, float drift_x, float drift_z, float swirl, cudaStream_t s);
// Volume ray-march of one FP32 field (sf_render.cu); the fields of
// StableFluidsB200VolumeRender.
struct RenderParams {
    float eye[3], right[3], up[3], forward[3];
    float volume_min[3], volume_max[3];
    float color_a[3], color_b[3];
    float aspect, tan_half_fov, value_scale, density;
    float value_min, value_max, ortho_height;
    uint32_t steps, projection;
    int32_t width, height;
};
cudaError_t launch_render_volume(const float* field, Dims d, const RenderParams& p, float* out_rgba, cudaStream_t s);
cudaError_t launch_post_diagnostics(float* div, float* mag, const void* vx, const void* vy, const void* vz, Dims d, float h, const FlowBC& b, int bf16, cudaStream_t s);

}  // namespace sfb
