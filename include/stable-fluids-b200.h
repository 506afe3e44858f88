/*
 * stable-fluids-b200.h -- project-side extensions to the stable-fluids C ABI.
 *
 * The upstream ABI (stable-fluids-3d.h) fixes the simulation configuration at
 * create time and has no room for solver options, so the extra choices this
 * build offers live here, in an additive interface that an unmodified caller
 * never needs:
 *   - the pressure/diffusion iteration scheme (red-black Gauss-Seidel with the
 *     reference's exact arithmetic, or pure Jacobi sweeps),
 *   - the temporal-blocking depth of the stencil passes,
 *   - a residual-driven pressure solve (iterate until the FP64 relative
 *     Poisson residual drops below a tolerance, inside the step graph),
 *   - the pressure warm start (zero as upstream, previous step, or learned),
 *   - per-step solver statistics.
 * stable_fluids_create_context_cuda() is exactly
 * stable_fluids_b200_create_context() with the default options below, except
 * that the environment variables listed at stable_fluids_b200_default_options
 * can override them so that an unmodified caller can select a scheme.
 */
#ifndef STABLE_FLUIDS_B200_H
#define STABLE_FLUIDS_B200_H

#include "stable-fluids-3d.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef enum StableFluidsB200Scheme {
    /* In-place red-black Gauss-Seidel; each iteration updates the cells with
     * (x+y+z) even, then odd, with the reference's arithmetic (upstream
     * backend-cuda.cu:354-375, 398-407). Results match the reference. */
    STABLE_FLUIDS_B200_SCHEME_RBGS = 0,
    /* Out-of-place Jacobi sweeps; one iteration = one sweep of all cells. */
    STABLE_FLUIDS_B200_SCHEME_JACOBI = 1,
} StableFluidsB200Scheme;

typedef enum StableFluidsB200WarmStart {
    STABLE_FLUIDS_B200_WARM_START_ZERO     = 0, /* p0 = 0 every step (upstream :644) */
    STABLE_FLUIDS_B200_WARM_START_PREVIOUS = 1, /* p0 = pressure of the previous step */
    STABLE_FLUIDS_B200_WARM_START_LEARNED  = 2, /* p0 = network(divergence, previous pressure) */
} StableFluidsB200WarmStart;

typedef struct StableFluidsB200Options {
    uint32_t scheme;                  /* StableFluidsB200Scheme */
    uint32_t warm_start;              /* StableFluidsB200WarmStart */
    int32_t iterations_per_pass;      /* temporal-blocking depth (iterations per HBM pass); 0 = automatic */
    float residual_tolerance;         /* > 0: solve pressure until rel_res <= tolerance */
    int32_t max_pressure_iterations;  /* cap of the residual-driven solve */
    int32_t residual_check_interval;  /* iterations between residual checks (>= 1) */
    uint32_t compute_residual;        /* 1: measure rel_res after every pressure solve */
    uint32_t reserved[9];
} StableFluidsB200Options;

/* Statistics of the most recent step (device values copied to the host). */
typedef struct StableFluidsB200StepStats {
    double rel_residual;              /* ||b - A p||_2 / ||b||_2 after the pressure solve, FP64 */
    double rhs_norm;                  /* ||b||_2, b = h^2 div (mean removed when A is singular) */
    int32_t pressure_iterations;      /* iterations the last pressure solve ran */
    int32_t hit_cap;                  /* 1 if a residual-driven solve stopped at its cap */
    int32_t used_fallback;            /* 1 if the learned warm start was rejected for plain */
    int32_t reserved;
} StableFluidsB200StepStats;

/* Fills *options with the defaults: RBGS, zero warm start, automatic
 * blocking, fixed iteration counts, no residual measurement. */
STABLE_FLUIDS_API StableFluidsResult stable_fluids_b200_default_options(StableFluidsB200Options* options);

/* stable_fluids_create_context_cuda with explicit options (options may be
 * null for the defaults; environment overrides are NOT applied here). */
STABLE_FLUIDS_API StableFluidsResult stable_fluids_b200_create_context(const StableFluidsContextCreateDesc* desc, const StableFluidsB200Options* options, void** out_context, StableFluidsScalarFieldHandle* out_scalar_field_handles, uint32_t out_scalar_field_handle_capacity, StableFluidsVectorFieldHandle* out_vector_field_handles, uint32_t out_vector_field_handle_capacity);

/* Waits for the context stream and returns the statistics of the last step. */
STABLE_FLUIDS_API StableFluidsResult stable_fluids_b200_get_step_stats(void* context, StableFluidsB200StepStats* out_stats);

/* Stages of the step, for profiling one stage outside the step graph. */
typedef enum StableFluidsB200Stage {
    STABLE_FLUIDS_B200_STAGE_FORCES             = 0, /* v += dt f, velocity packing */
    STABLE_FLUIDS_B200_STAGE_VELOCITY_ADVECTION = 1, /* RK2 semi-Lagrangian advection */
    STABLE_FLUIDS_B200_STAGE_VELOCITY_DIFFUSION = 2, /* implicit viscosity, 3 components */
    STABLE_FLUIDS_B200_STAGE_DIVERGENCE         = 3,
    STABLE_FLUIDS_B200_STAGE_PRESSURE           = 4, /* the pressure solve */
    STABLE_FLUIDS_B200_STAGE_PROJECTION         = 5,
    STABLE_FLUIDS_B200_STAGE_SCALARS            = 6, /* source, advection, diffusion, dissipation */
    STABLE_FLUIDS_B200_STAGE_DIAGNOSTICS        = 7, /* post-projection divergence, |u| */
    STABLE_FLUIDS_B200_STAGE_STEP               = 8, /* the whole step (one graph launch) */
} StableFluidsB200Stage;

typedef struct StableFluidsB200StepInfo {
    int32_t kernels_per_step;         /* kernel launches in one step */
    uint32_t scheme;
    int32_t iterations_per_pass;
    int32_t blocked;                  /* 1: temporally blocked stencil passes */
    uint64_t device_bytes;            /* device memory the context holds */
} StableFluidsB200StepInfo;

/* Enqueues one stage of the step on the context stream, outside the step
 * graph (its inputs are whatever the fields hold), and reports how many
 * kernels it launched. Meant for timing a stage with events on the context
 * stream; running stages out of order changes the simulation state. */
STABLE_FLUIDS_API StableFluidsResult stable_fluids_b200_enqueue_stage(void* context, uint32_t stage, int32_t* out_kernel_launches);

STABLE_FLUIDS_API StableFluidsResult stable_fluids_b200_get_step_info(void* context, StableFluidsB200StepInfo* out_info);

/* No counterpart in the reference. The FP64 relative Poisson residual
 * ||b - A p|| / ||b|| (b = h^2 divergence, mean removed when no face is
 * OUTFLOW; A p = sum of the 6 neighbours - 6 p with the pressure ghost rules)
 * of caller-provided dense nx*ny*nz FP32 device arrays, written as
 * {rel_residual, ||b||} to out_residual (2 doubles of device-accessible
 * memory), enqueued on `stream`. It allocates nothing -- for callers that
 * cannot call cudaMalloc at that point (allocation-free frame phases, fully
 * pooled device memory, host callbacks): its scratch is a fixed 128 KiB
 * device array owned by the library on every device that loads it.
 * Limits: nz <= 4096 (larger grids return BACKEND_FAILURE); calls that
 * overlap on the GPU race on the shared scratch (order them on one stream);
 * the first call on a device looks up the scratch address, so make it before
 * any stream capture. Same numbers as the step's residual measurement up to
 * FP64 summation order. */
STABLE_FLUIDS_API StableFluidsResult stable_fluids_b200_pressure_residual_noalloc(const float* pressure, const float* divergence, int32_t nx, int32_t ny, int32_t nz, float cell_size, const StableFluidsFlowBoundaryConfig* flow_boundary, double* out_residual, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* STABLE_FLUIDS_B200_H */
