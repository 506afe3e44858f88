// sf_boundary.h -- the flow boundary of the ABI flattened into the kernels'
// FlowBC, with the reference's validation (backend-cuda.cu:516-520: known
// face kinds, periodic faces in pairs). One definition shared by the context
// code (C++23, g++) and the CUDA sources (C++20, nvcc).
#pragma once

#include "sf_types.h"
#include "stable-fluids-3d.h"

namespace sfb {

// Fills `out` from `b`; false if a face kind is unknown or a periodic face
// lacks its partner (out is then unspecified).
inline bool flatten_flow(const StableFluidsFlowBoundaryConfig& b, FlowBC& out) {
    out = FlowBC{};
    const StableFluidsFlowBoundaryFaceDesc* f = &b.x_minus;
    for (int k = 0; k < 6; ++k) {
        if (f[k].type > STABLE_FLUIDS_FLOW_BOUNDARY_PERIODIC) return false;
        out.type[k] = static_cast<int32_t>(f[k].type);
        out.vel[k][0] = f[k].velocity_x;
        out.vel[k][1] = f[k].velocity_y;
        out.vel[k][2] = f[k].velocity_z;
        out.pressure[k] = f[k].pressure;
        if (f[k].type == STABLE_FLUIDS_FLOW_BOUNDARY_OUTFLOW) out.any_outflow = 1;
    }
    for (int a = 0; a < 3; ++a) {
        const bool lo = f[2 * a].type == STABLE_FLUIDS_FLOW_BOUNDARY_PERIODIC, hi = f[2 * a + 1].type == STABLE_FLUIDS_FLOW_BOUNDARY_PERIODIC;
        if (lo != hi) return false;
        out.periodic[a] = lo ? 1 : 0;
    }
    return true;
}

}  // namespace sfb
