/*
 * stable-fluids-3d.h -- C ABI of the 3D stable-fluids step (B200 build).
 *
 * This header is binary-compatible with the upstream interface
 * (stable-fluids-3d.h:1-160 of Xayah-Graphics/stable-fluids): every enum value,
 * struct field order, field type and exported function signature is the same,
 * so a caller compiled against the upstream header (benchmark.cu, the Vulkan
 * viewer) links against libstable-fluids.so from this project unchanged.
 * tests/test_abi.py checks the layout field by field. The declarations below
 * (enums, structs, signatures, the STABLE_FLUIDS_API visibility block) are
 * therefore the upstream file's, which is distributed under the Mozilla Public
 * License 2.0; the comments are this project's.
 *
 * Semantics (all functions are asynchronous on the context stream):
 *   - update_* take DEVICE pointers (host pointers are also accepted: the copy
 *     uses cudaMemcpyDefault); a null pointer zero-fills the field.
 *   - step enqueues one whole simulation step (one CUDA graph launch).
 *   - get_view returns library-owned, dense, x-fastest FP32 arrays that stay
 *     valid until destroy and are overwritten by the next step.
 */
#ifndef STABLE_FLUIDS_3D_H
#define STABLE_FLUIDS_3D_H

#include <stdint.h>

#if defined(_WIN32)
#  if defined(STABLE_FLUIDS_BUILD_SHARED)
#    define STABLE_FLUIDS_API __declspec(dllexport)
#  else
#    define STABLE_FLUIDS_API __declspec(dllimport)
#  endif
#elif defined(__GNUC__) || defined(__clang__)
#  define STABLE_FLUIDS_API __attribute__((visibility("default")))
#else
#  define STABLE_FLUIDS_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Return codes (upstream stable-fluids-3d.h:22-26). */
typedef enum StableFluidsResult {
    STABLE_FLUIDS_RESULT_OK              = 0,
    STABLE_FLUIDS_RESULT_OUT_OF_MEMORY   = 1,
    STABLE_FLUIDS_RESULT_BACKEND_FAILURE = 2,
} StableFluidsResult;

/* Per-face velocity/pressure boundary kind (upstream :28-33). */
typedef enum StableFluidsFlowBoundaryType {
    STABLE_FLUIDS_FLOW_BOUNDARY_NO_SLIP_WALL   = 0,
    STABLE_FLUIDS_FLOW_BOUNDARY_FREE_SLIP_WALL = 1,
    STABLE_FLUIDS_FLOW_BOUNDARY_OUTFLOW        = 2,
    STABLE_FLUIDS_FLOW_BOUNDARY_PERIODIC       = 3,
} StableFluidsFlowBoundaryType;

/* Per-face scalar boundary kind (upstream :35-39). */
typedef enum StableFluidsScalarBoundaryType {
    STABLE_FLUIDS_SCALAR_BOUNDARY_FIXED_VALUE = 0,
    STABLE_FLUIDS_SCALAR_BOUNDARY_ZERO_FLUX   = 1,
    STABLE_FLUIDS_SCALAR_BOUNDARY_PERIODIC    = 2,
} StableFluidsScalarBoundaryType;

/* 1-based handles; 0 is never a valid handle (upstream :41-42). */
typedef uint32_t StableFluidsScalarFieldHandle;
typedef uint32_t StableFluidsVectorFieldHandle;

/* One face of the flow domain: kind, prescribed wall velocity, outflow
 * pressure (upstream :44-50). 20 bytes. */
typedef struct StableFluidsFlowBoundaryFaceDesc {
    uint32_t type;
    float velocity_x;
    float velocity_y;
    float velocity_z;
    float pressure;
} StableFluidsFlowBoundaryFaceDesc;

/* The six faces in the order -x, +x, -y, +y, -z, +z (upstream :52-59). */
typedef struct StableFluidsFlowBoundaryConfig {
    StableFluidsFlowBoundaryFaceDesc x_minus;
    StableFluidsFlowBoundaryFaceDesc x_plus;
    StableFluidsFlowBoundaryFaceDesc y_minus;
    StableFluidsFlowBoundaryFaceDesc y_plus;
    StableFluidsFlowBoundaryFaceDesc z_minus;
    StableFluidsFlowBoundaryFaceDesc z_plus;
} StableFluidsFlowBoundaryConfig;

/* One face of a scalar field: kind and fixed value (upstream :61-64). */
typedef struct StableFluidsScalarBoundaryFaceDesc {
    uint32_t type;
    float value;
} StableFluidsScalarBoundaryFaceDesc;

typedef struct StableFluidsScalarBoundaryConfig {
    StableFluidsScalarBoundaryFaceDesc x_minus;
    StableFluidsScalarBoundaryFaceDesc x_plus;
    StableFluidsScalarBoundaryFaceDesc y_minus;
    StableFluidsScalarBoundaryFaceDesc y_plus;
    StableFluidsScalarBoundaryFaceDesc z_minus;
    StableFluidsScalarBoundaryFaceDesc z_plus;
} StableFluidsScalarBoundaryConfig;

/* Grid, time step and solver iteration counts (upstream :75-85).
 * The iteration counts are red-black Gauss-Seidel iterations in the
 * reference-compatible scheme; see stable-fluids-b200.h for other schemes. */
typedef struct StableFluidsSimulationConfig {
    int32_t nx;
    int32_t ny;
    int32_t nz;
    float cell_size;
    float dt;
    float viscosity;
    int32_t diffuse_iterations;
    int32_t pressure_iterations;
    StableFluidsFlowBoundaryConfig flow_boundary;
} StableFluidsSimulationConfig;

/* A transported scalar such as density (upstream :86-91). */
typedef struct StableFluidsScalarFieldDesc {
    float diffusion;
    float dissipation;
    float initial_value;
    StableFluidsScalarBoundaryConfig boundary;
} StableFluidsScalarFieldDesc;

typedef enum StableFluidsVectorFieldUsage {
    STABLE_FLUIDS_VECTOR_FIELD_FORCE = 0,
} StableFluidsVectorFieldUsage;

/* An auxiliary vector field; FORCE fields are added as v += dt * f at the
 * start of every step (upstream :93-102). */
typedef struct StableFluidsVectorFieldDesc {
    StableFluidsVectorFieldUsage usage;
    float initial_value_x;
    float initial_value_y;
    float initial_value_z;
} StableFluidsVectorFieldDesc;

/* Everything create needs; stream may be null, in which case the context
 * owns a non-blocking stream (upstream :104-111). */
typedef struct StableFluidsContextCreateDesc {
    StableFluidsSimulationConfig config;
    void* stream;
    const StableFluidsScalarFieldDesc* scalar_fields;
    uint32_t scalar_field_count;
    const StableFluidsVectorFieldDesc* vector_fields;
    uint32_t vector_field_count;
} StableFluidsContextCreateDesc;

/* upstream :112 */
STABLE_FLUIDS_API StableFluidsResult stable_fluids_create_context_cuda(const StableFluidsContextCreateDesc* desc, void** out_context, StableFluidsScalarFieldHandle* out_scalar_field_handles, uint32_t out_scalar_field_handle_capacity, StableFluidsVectorFieldHandle* out_vector_field_handles, uint32_t out_vector_field_handle_capacity);
/* upstream :113 -- a null context is accepted and ignored here. */
STABLE_FLUIDS_API StableFluidsResult stable_fluids_destroy_context_cuda(void* context);
/* upstream :115 */
STABLE_FLUIDS_API StableFluidsResult stable_fluids_update_scalar_field_cuda(void* context, StableFluidsScalarFieldHandle field, const float* values);
/* upstream :116 */
STABLE_FLUIDS_API StableFluidsResult stable_fluids_update_scalar_field_source_cuda(void* context, StableFluidsScalarFieldHandle field, const float* values);
/* upstream :117 */
STABLE_FLUIDS_API StableFluidsResult stable_fluids_update_vector_field_cuda(void* context, StableFluidsVectorFieldHandle field, const float* values_x, const float* values_y, const float* values_z);
/* upstream :118 */
STABLE_FLUIDS_API StableFluidsResult stable_fluids_step_cuda(void* context);

/* What get_view returns (upstream :120-128). */
typedef enum StableFluidsViewKind {
    STABLE_FLUIDS_VIEW_SCALAR_FIELD_DATA       = 0,
    STABLE_FLUIDS_VIEW_SCALAR_FIELD_SOURCE     = 1,
    STABLE_FLUIDS_VIEW_VECTOR_FIELD            = 2,
    STABLE_FLUIDS_VIEW_FLOW_VELOCITY           = 3,
    STABLE_FLUIDS_VIEW_FLOW_VELOCITY_MAGNITUDE = 4,
    STABLE_FLUIDS_VIEW_FLOW_PRESSURE           = 5,
    STABLE_FLUIDS_VIEW_FLOW_DIVERGENCE         = 6,
} StableFluidsViewKind;

typedef enum StableFluidsViewLayout {
    STABLE_FLUIDS_VIEW_LAYOUT_F32_3D      = 0,
    STABLE_FLUIDS_VIEW_LAYOUT_F32_3D_SOA3 = 1,
} StableFluidsViewLayout;

/* upstream :135-140 */
typedef struct StableFluidsViewRequest {
    uint32_t kind;
    StableFluidsScalarFieldHandle scalar_field;
    StableFluidsVectorFieldHandle vector_field;
    void* consumer_stream;
} StableFluidsViewRequest;

/* upstream :142-152 -- data1/data2 are set only for the SOA3 layout. */
typedef struct StableFluidsView {
    uint32_t layout;
    int32_t nx;
    int32_t ny;
    int32_t nz;
    uint64_t row_stride_bytes;
    uint64_t slice_stride_bytes;
    const float* data0;
    const float* data1;
    const float* data2;
} StableFluidsView;

/* upstream :154 */
STABLE_FLUIDS_API StableFluidsResult stable_fluids_get_view_cuda(void* context, const StableFluidsViewRequest* request, StableFluidsView* out_view);

#ifdef __cplusplus
}
#endif

#endif /* STABLE_FLUIDS_3D_H */
