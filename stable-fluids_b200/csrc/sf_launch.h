// sf_launch.h -- host-callable launchers for the step kernels. Plain types
// only, so the C++23 host runtime (sf_context.cpp) can call them without
// compiling CUDA.
#pragma once

#include <cuda_runtime.h>

#include "sf_types.h"

namespace sfb {

constexpr int kMaxForcesPerLaunch = 8;

struct ForceArgs {
    float* vel[3];                          // SoA velocity (read; written when write_soa)
    const float* force[kMaxForcesPerLaunch][3];
    int force_count;
    float dt;
    size_t n;
    void* packed;                           // float4 velocity (written when non-null)
    int write_soa;
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
    float* x;            // the iterate (result lands here)
    const float* b;      // right-hand side (diffusion: advected field; pressure: divergence)
    float* scratch;      // a field-sized buffer for out-of-place sweeps
    Dims dims;
    FlowBC flow;
    ScalarBC scalar;
    int* launches;       // incremented by the number of kernels enqueued (may be null)
    int blocked;         // 1: temporally blocked passes where supported; 0: one launch per sweep
    unsigned* error_flag;  // device word a kernel sets when a bounded wait gives up
};

cudaError_t launch_fill(float* f, float value, size_t n, cudaStream_t s);
cudaError_t launch_force_pack(const ForceArgs& a, cudaStream_t s);
cudaError_t launch_advect_velocity(const void* packed, float* out_x, float* out_y, float* out_z, float dt, Dims d, float h, const FlowBC& b, cudaStream_t s);
cudaError_t launch_scalar_source_advect(const void* packed, const float* data, const float* source, float* out, float dt, Dims d, float h, const FlowBC& fb, const ScalarBC& sb, cudaStream_t s);
cudaError_t launch_scalar_source(float* data, const float* source, float dt, size_t n, cudaStream_t s);
cudaError_t launch_scale(float* data, float factor, size_t n, cudaStream_t s);
cudaError_t launch_stencil(const StencilArgs& a, cudaStream_t s);
cudaError_t launch_divergence(float* div, const float* vx, const float* vy, const float* vz, Dims d, float h, const FlowBC& b, cudaStream_t s);
// u -= grad p (in place) and repack; with stats != nullptr also accumulates
// the FP64 residual sums of the pressure system into stats.
cudaError_t launch_project(float* vx, float* vy, float* vz, void* packed, const float* p, const float* div, Dims d, float h, float h2, const FlowBC& b, DeviceStats* stats, cudaStream_t s);
cudaError_t launch_residual_sums(const float* p, const float* div, Dims d, float h2, const FlowBC& b, DeviceStats* stats, cudaStream_t s);
// The same sums with the vectorised z-marching layout; false (nothing
// launched) when the grid or the pointers do not suit it (nx % 4, 16-byte
// alignment).
bool launch_residual_sums_vec(const float* p, const float* div, Dims d, float h2, const FlowBC& b, DeviceStats* stats, cudaStream_t s);
cudaError_t launch_residual_finalize(DeviceStats* stats, Dims d, int singular, int iterations, cudaStream_t s);
// One check of the residual-driven pressure solve (see k_residual_check).
cudaError_t launch_residual_check(DeviceStats* stats, Dims d, int singular, int reset, int increment, double tol, int max_iterations, cudaGraphConditionalHandle handle, cudaStream_t s);
// Learned warm start: keeps the candidate in p or replaces it by alt,
// whichever has the smaller relative residual (two kernels).
cudaError_t launch_warm_start_select(DeviceStats* learned, const DeviceStats* plain, Dims d, int singular, float* p, const float* alt, cudaStream_t s);
cudaError_t launch_post_diagnostics(float* div, float* mag, const float* vx, const float* vy, const float* vz, Dims d, float h, const FlowBC& b, cudaStream_t s);

}  // namespace sfb
