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

typedef enum StableFluidsB200Storage {
    STABLE_FLUIDS_B200_STORAGE_FP32 = 0, /* every field FP32 (the reference's layout) */
    /* velocity and scalar fields stored as BF16 (half the bytes of the
     * advection and diffusion passes), all arithmetic FP32; pressure,
     * divergence, forces and sources stay FP32. Views of velocity and scalar
     * data are FP32 copies converted at stable_fluids_get_view_cuda. */
    STABLE_FLUIDS_B200_STORAGE_BF16 = 1,
} StableFluidsB200Storage;

typedef struct StableFluidsB200Options {
    uint32_t scheme;                  /* StableFluidsB200Scheme */
    uint32_t warm_start;              /* StableFluidsB200WarmStart */
    int32_t iterations_per_pass;      /* 0 = automatic (single sweeps; red-black solves in the
                                       * colour-split layout where rows are a multiple of 8 cells);
                                       * 1 = one launch per sweep / colour on the interleaved field;
                                       * >= 2 = temporally blocked passes of that many iterations */
    float residual_tolerance;         /* > 0: solve pressure until rel_res <= tolerance */
    int32_t max_pressure_iterations;  /* cap of the residual-driven solve */
    int32_t residual_check_interval;  /* iterations between residual checks (>= 1) */
    uint32_t compute_residual;        /* 1: measure rel_res after every pressure solve */
    int32_t warm_start_trial_iterations; /* learned warm start: sweeps run on the learned and on the
                                          * previous-pressure start before the one with the smaller
                                          * rel_res is kept (0 = compare the starts themselves) */
    uint32_t storage;                 /* StableFluidsB200Storage */
    uint32_t warm_start_coarsening;   /* learned warm start: 1 = the network runs on the grid
                                       * coarsened 2x in each axis (cell averages of the
                                       * divergence and the previous pressure), and its
                                       * correction is prolonged trilinearly to the grid; needs
                                       * even nx, ny, nz (else the full grid is used) */
    uint32_t reserved[6];
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

/* Staged update of a vector field, for callers that upload a new field from
 * the host every step (no counterpart in the reference, whose
 * stable_fluids_update_vector_field_cuda copies on the context stream and so
 * holds the next step back until the copy is done). The values (host memory,
 * pinned for the copy to run asynchronously, or device memory; null
 * components zero-fill as in update_vector_field) are copied on copy_stream
 * into staging arrays of the context, so the copy can run while the current
 * step computes; the next stable_fluids_step_cuda waits for it and moves the
 * values into the field (a device-to-device copy on the context stream) before
 * the step. The caller keeps the host arrays unchanged until the copy has run
 * on copy_stream. The first call allocates the staging arrays (3 fields) and
 * must not be made during a stream capture. Staging again before a step
 * replaces the staged values, and staged values still pending at the next
 * step overwrite an update_vector_field made in between. Only
 * stable_fluids_step_cuda applies staged values (a batch step does not). */
STABLE_FLUIDS_API StableFluidsResult stable_fluids_b200_stage_vector_field(void* context, StableFluidsVectorFieldHandle field, const float* values_x, const float* values_y, const float* values_z, void* copy_stream);

/* Asynchronous read-back of a view (no counterpart in the reference): the
 * view's arrays (one, or three for SOA3 views) are copied on the context
 * stream into a snapshot buffer of the context, then from it to host_out*
 * on copy_stream, so the next step can start while the copy to the host
 * runs. The data is in host_out* once copy_stream has passed this call
 * (synchronize or record an event on it). The snapshot is reused: the next
 * read_view_async waits on the context stream until this one's copy to the
 * host is done. The first calls allocate the snapshot arrays and must not be
 * made during a stream capture. */
STABLE_FLUIDS_API StableFluidsResult stable_fluids_b200_read_view_async(void* context, const StableFluidsViewRequest* request, float* host_out0, float* host_out1, float* host_out2, void* copy_stream);

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
    int32_t kernels_per_check;        /* residual-driven solve: kernel launches of one
                                         pass of the loop body (the interval's sweeps,
                                         the residual sums and the check); counted once
                                         in kernels_per_step */
    int32_t reserved;
} StableFluidsB200StepInfo;

/* Enqueues one stage of the step on the context stream, outside the step
 * graph (its inputs are whatever the fields hold), and reports how many
 * kernels it launched. Meant for timing a stage with events on the context
 * stream; running stages out of order changes the simulation state. */
STABLE_FLUIDS_API StableFluidsResult stable_fluids_b200_enqueue_stage(void* context, uint32_t stage, int32_t* out_kernel_launches);

STABLE_FLUIDS_API StableFluidsResult stable_fluids_b200_get_step_info(void* context, StableFluidsB200StepInfo* out_info);

/* ---- Learned pressure warm start (no counterpart in the reference) ----
 *
 * A 3-level 3D U-Net (16/32/64 channels, two 3x3x3 convolutions + ReLU per
 * level and side, 2x average pooling, nearest upsampling with skip
 * concatenation, a final 3x3x3 convolution to one channel), BF16 weights and
 * activations, FP32 accumulation on the tensor cores. Input: the pressure
 * right-hand side b = h^2 div and the previous pressure, both scaled by
 * 1 / rms(b); output: the scaled correction, p0 = p_prev + out * rms(b).
 * Grid sides must be multiples of 4.
 *
 * Parameters are FP32, one block per layer in forward order (enc0a enc0b
 * enc1a enc1b bott_a bott_b dec1a dec1b dec0a dec0b out): weights
 * [27 taps][cout][cin] (tap = (dz+1)*9 + (dy+1)*3 + (dx+1)) then cout biases,
 * with (cin, cout) = (16,16) (16,16) (16,32) (32,32) (32,64) (64,64) (96,32)
 * (32,32) (48,16) (16,16) (16,16); input channels 2..15 of the first layer
 * and output channels 1..15 of the last are padding (zero, never updated).
 *
 * A network object serves one stream at a time (its activation buffers are
 * shared by every call); all entry points except predict are synchronous.
 */
STABLE_FLUIDS_API StableFluidsResult stable_fluids_b200_network_create(uint32_t seed, void** out_network);
STABLE_FLUIDS_API StableFluidsResult stable_fluids_b200_network_destroy(void* network);
/* Parameter count and (if out_host_values != null) a host copy of them. */
STABLE_FLUIDS_API StableFluidsResult stable_fluids_b200_network_parameters(void* network, uint64_t* out_count, float* out_host_values);
/* Loads parameters from host memory and resets the optimizer state. */
STABLE_FLUIDS_API StableFluidsResult stable_fluids_b200_network_set_parameters(void* network, const float* host_values);
/* out_pressure = the warm start computed from device arrays
 * (previous_pressure may be null = zero, and may equal out_pressure),
 * enqueued on `stream`. */
STABLE_FLUIDS_API StableFluidsResult stable_fluids_b200_network_predict(void* network, const float* divergence, const float* previous_pressure, int32_t nx, int32_t ny, int32_t nz, float cell_size, float* out_pressure, void* stream);
/* Mean squared error between the network output and the scaled correction
 * towards target_pressure, (target - previous) / rms(b), and (if
 * out_host_gradients != null) its gradient with respect to every parameter,
 * in the parameter layout. */
STABLE_FLUIDS_API StableFluidsResult stable_fluids_b200_network_gradients(void* network, const float* divergence, const float* previous_pressure, const float* target_pressure, int32_t nx, int32_t ny, int32_t nz, float cell_size, double* out_loss, float* out_host_gradients, void* stream);
/* One Adam step (beta 0.9 / 0.999, eps 1e-8) on that loss; *out_loss is the
 * loss before the step. */
STABLE_FLUIDS_API StableFluidsResult stable_fluids_b200_network_train_step(void* network, const float* divergence, const float* previous_pressure, const float* target_pressure, int32_t nx, int32_t ny, int32_t nz, float cell_size, float learning_rate, double* out_loss, void* stream);
/* Uses `network` for the pressure warm start of a context created with
 * warm_start = LEARNED and rebuilds its step graph (null detaches). Until a
 * network is attached such a context starts from the previous pressure and
 * reports used_fallback = 1. With a network, each step predicts a start,
 * runs warm_start_trial_iterations sweeps on it and on the previous
 * pressure, and continues from the one with the smaller residual
 * (used_fallback = 1 when that is the previous pressure); the sweeps of the
 * trial count towards the step's iterations. Several contexts may share one
 * network: each attached context predicts with activation buffers of its own
 * (allocated here, freed when it detaches or is destroyed) and only reads the
 * shared weights. The network must outlive the attachment, and must not be
 * trained while an attached context steps. */
STABLE_FLUIDS_API StableFluidsResult stable_fluids_b200_attach_network(void* context, void* network);

/* ---- Batched stepping (no counterpart in the reference) ----
 * A batch steps several contexts (each with its own grid size and fields)
 * together; one batch step advances every context by one step. Two layouts:
 *
 *  - WORK_TABLE: one persistent kernel launch per stage of the step covers
 *    every simulation, walking a table of (simulation, thread block) work
 *    items; the stencil sweeps' z chunk per grid size comes from an
 *    autotuner. Needs contexts with the same stage structure: FP32 storage,
 *    the same scheme, iteration counts and warm start (zero or previous, no
 *    residual-driven solve, no temporal blocking), one scalar field with
 *    diffusion > 0, viscosity > 0, at most 4 force fields, nx % 4 == 0.
 *  - GRAPHS: the contexts' own step graphs as children of one CUDA graph; the
 *    simulations' kernels run concurrently. Any contexts except ones with a
 *    residual-driven solve (conditional graph nodes); contexts attached to
 *    one warm-start network share it (each has its own activation buffers).
 *
 * Both give the same bits as stepping each context alone. WORK_TABLE packs
 * the simulations into L2-sized groups and runs the groups on `chains`
 * concurrent streams (default 4): ~250 launches per group instead of ~250
 * per simulation, each group's sweeps served from L2. On B200 with 64 uneven
 * simulations (32^3..128^3) it is the faster layout (35.7 against 31.8 batch
 * steps/s). The batch is
 * ordered after the work queued on each context's stream and each context's
 * stream after the batch, so update/view calls keep working as for a single
 * context. The batch reads the contexts' configuration and field addresses
 * when it is created: rebuild it after stable_fluids_b200_attach_network, and
 * destroy it before any of its contexts. */
typedef enum StableFluidsB200BatchMode {
    STABLE_FLUIDS_B200_BATCH_GRAPHS = 0,     /* the default; any batchable contexts */
    STABLE_FLUIDS_B200_BATCH_WORK_TABLE = 1, /* BACKEND_FAILURE when the contexts do not allow it */
} StableFluidsB200BatchMode;

typedef struct StableFluidsB200BatchOptions {
    uint32_t mode;           /* StableFluidsB200BatchMode */
    uint32_t autotune;       /* WORK_TABLE: 1 = time the sweep tile options per grid size at create */
    const char* tile_cache;  /* JSON file of tuned tiles, read and updated when autotuning; may be NULL */
    uint32_t chains;         /* WORK_TABLE: groups run on this many concurrent streams (0 = default 4, max 8) */
    uint32_t reserved[3];
} StableFluidsB200BatchOptions;

/* stable_fluids_b200_batch_create_ex with mode GRAPHS and no autotuning. */
STABLE_FLUIDS_API StableFluidsResult stable_fluids_b200_batch_create(void* const* contexts, uint32_t count, void** out_batch);
STABLE_FLUIDS_API StableFluidsResult stable_fluids_b200_batch_create_ex(void* const* contexts, uint32_t count, const StableFluidsB200BatchOptions* options, void** out_batch);
/* The layout in use (StableFluidsB200BatchMode); for WORK_TABLE the
 * number of L2-sized groups the contexts were partitioned into (each group's
 * whole step runs before the next group's, so its sweeps reread their fields
 * from L2) and the z chunk (planes per thread block) of each context's
 * sweeps, in batch order (up to `capacity` entries; 0 for GRAPHS). */
STABLE_FLUIDS_API StableFluidsResult stable_fluids_b200_batch_layout(void* batch, uint32_t* out_mode, uint32_t* out_groups, int32_t* out_z_chunks, uint32_t capacity);
STABLE_FLUIDS_API StableFluidsResult stable_fluids_b200_batch_step(void* batch);
/* Number of contexts, kernel launches per batch step, and the batch's stream. */
STABLE_FLUIDS_API StableFluidsResult stable_fluids_b200_batch_info(void* batch, uint32_t* out_count, int32_t* out_kernels_per_step, void** out_stream);
STABLE_FLUIDS_API StableFluidsResult stable_fluids_b200_batch_destroy(void* batch);

/* ---- The reference viewer's plume scene on the device ----
 * Replaces the per-step host work of vulkan-app/scene_plume.cpp:323-335 (a
 * loop over every cell building the force's x and z components from three
 * host masks, two host-to-device copies and an update_vector_field copy) with
 * one kernel that evaluates the masks in closed form and writes the force
 * straight into the context's force field: nothing crosses PCIe. The scene
 * geometry is the viewer's (source at (0.50, 0.13, 0.50) of the domain,
 * radius 6 cells; swirl and drift spheres above it), derived from the
 * context's grid; the arithmetic is the viewer's float arithmetic, one
 * rounding per operation, so the fields are the ones the viewer uploads.
 * Both calls are asynchronous on the context stream.
 *
 * setup (scene_plume.cpp:267-300): density source 32 w and force y 7.6 w for
 * the source sphere's weight w; force x and z zero.
 * forces (:323-330): force x and z of animation step `animation_step`
 * (phase = step * 0.045, drift_x = 1.15 sin(phase), drift_z =
 * 0.85 cos(0.71 phase), swirl = 1.65 cos(0.53 phase), evaluated on the host
 * with the C library's sinf / cosf as the viewer does). */
STABLE_FLUIDS_API StableFluidsResult stable_fluids_b200_plume_scene_setup(void* context, StableFluidsScalarFieldHandle density, StableFluidsVectorFieldHandle force);
STABLE_FLUIDS_API StableFluidsResult stable_fluids_b200_plume_scene_forces(void* context, StableFluidsVectorFieldHandle force, int32_t animation_step);

/* ---- Headless volume rendering of a field ----
 * The reference viewer's volume shader (vulkan-app/shaders/field_volume.slang)
 * restated as a CUDA kernel: one primary ray per pixel through the field's
 * box, `steps` equal steps, trilinear samples, emission/absorption
 * compositing front to back, early exit below 1 % transmittance. The image is
 * written to a caller-provided device buffer of width * height RGBA float4
 * texels (row 0 at the top; colour premultiplied by alpha), instead of a
 * swapchain image. The fields mirror the shader's push constants. */
typedef struct StableFluidsB200VolumeRender {
    float eye[3], right[3], up[3], forward[3];   /* camera basis (world units) */
    float volume_min[3], volume_max[3];          /* the field's box in world units */
    float color_a[3], color_b[3];                /* ramp ends (signed range: negative / positive colour) */
    float aspect;                                /* width / height (params0.x) */
    float tan_half_fov;                          /* perspective (params0.y) */
    float value_scale;                           /* field multiplier (params0.z) */
    float density;                               /* extinction per unit length (params0.w) */
    float value_min, value_max;                  /* mapped range (params3.xy); a range spanning 0 is signed */
    float ortho_height;                          /* orthographic view height (params3.w) */
    uint32_t steps;                              /* march steps (params1.w) */
    uint32_t projection;                         /* 0 perspective, else orthographic (params2.x) */
    int32_t width, height;                       /* image size in pixels */
    uint32_t reserved[4];
} StableFluidsB200VolumeRender;

/* Renders the field `field` selects (a single-array view kind: scalar data or
 * source, velocity magnitude, pressure, divergence; FP32 as get_view returns
 * it) into out_rgba (device memory, width * height * 4 floats), enqueued on
 * the context stream after the work queued there. */
STABLE_FLUIDS_API StableFluidsResult stable_fluids_b200_render_volume(void* context, const StableFluidsViewRequest* field, const StableFluidsB200VolumeRender* params, float* out_rgba);

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
