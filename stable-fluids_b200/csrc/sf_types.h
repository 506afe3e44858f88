// sf_types.h -- plain structs shared by the host runtime (C++23) and the CUDA
// kernels (C++20). No CUDA or torch types appear here.
#pragma once

#include <cstddef>
#include <cstdint>

namespace sfb {

// Face order used everywhere: -x, +x, -y, +y, -z, +z (the ABI's order,
// stable-fluids-3d.h:52-59).
enum Face : int32_t { XM = 0, XP = 1, YM = 2, YP = 3, ZM = 4, ZP = 5 };

struct Dims {
    int32_t nx = 0, ny = 0, nz = 0;
    int32_t pad = 0;
};

// Flow boundary, flattened from StableFluidsFlowBoundaryConfig.
struct FlowBC {
    int32_t type[6];      // StableFluidsFlowBoundaryType per face
    float vel[6][3];      // prescribed wall velocity per face
    float pressure[6];    // outflow (Dirichlet) pressure per face
    int32_t periodic[3];  // both faces of the axis periodic
    int32_t any_outflow;  // some face is OUTFLOW (pressure operator nonsingular)
};

// Scalar boundary, flattened from StableFluidsScalarBoundaryConfig.
struct ScalarBC {
    int32_t type[6];      // StableFluidsScalarBoundaryType per face
    float value[6];       // fixed value per face
    int32_t periodic[3];
    int32_t pad;
};

// Which field a stencil kernel iterates and therefore which ghost rule and
// update formula it uses.
enum StencilKind : int32_t {
    KIND_VEL_X = 0,   // diffusion of velocity component x (velocity ghosts)
    KIND_VEL_Y = 1,
    KIND_VEL_Z = 2,
    KIND_SCALAR = 3,  // diffusion of a scalar (scalar ghosts)
    KIND_PRESSURE = 4 // Poisson pressure (pressure ghosts)
};

// Ghost value of a face in a stencil: self (Neumann / copy), a constant
// (Dirichlet), or k - self (reflection about a prescribed wall value).
enum GhostMode : int32_t { GHOST_COPY = 0, GHOST_CONST = 1, GHOST_REFLECT = 2 };

// Face ghost rules of one field kind (see ghost_rule in sf_stencil.cu).
struct GhostRule {
    int32_t mode[6];
    float k[6];
    int32_t periodic[3];
    int32_t pad;
};

// Device-side solver statistics, one per context (global memory).
struct DeviceStats {
    double sum_e;       // sum of e = b - A p
    double sum_e2;      // sum of e^2
    double sum_b;       // sum of b = h^2 div
    double sum_b2;      // sum of b^2
    double rel_residual;
    double rhs_norm;
    int32_t iterations;
    int32_t hit_cap;
    int32_t used_fallback;
    int32_t keep_going;  // residual-driven loop: 1 while another block of sweeps is needed
    uint32_t error;      // set by a kernel whose bounded wait gave up
    uint32_t pad;
};

}  // namespace sfb
