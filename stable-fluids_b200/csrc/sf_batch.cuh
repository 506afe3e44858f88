// sf_batch.cuh -- device helpers of the work-table kernels (see sf_batch.h).
#pragma once

#include <cuda_runtime.h>

#include "sf_batch.h"

namespace sfb {

// The simulation owning work item w: the s with first[s] <= w < first[s + 1]
// (binary search; every thread of the block reads the same entries).
__device__ __forceinline__ int batch_sim(const uint32_t* __restrict__ first, int nsims, uint32_t w) {
    int lo = 0, hi = nsims;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(&first[mid]) <= w) lo = mid;
        else hi = mid;
    }
    return lo;
}

// Block `local` of a grid of (gx, gy, *) blocks, x fastest.
__device__ __forceinline__ uint3 batch_block(uint32_t local, uint32_t gx, uint32_t gy) {
    return make_uint3(local % gx, (local / gx) % gy, local / (gx * gy));
}

// The iterate, right-hand side or scratch of a field kind.
__device__ __forceinline__ float* batch_field(const BatchSim& m, int kind, int which) {
    if (which == BF_SCRATCH) return m.scratch;
    if (kind == KIND_PRESSURE) return which == BF_X ? m.pressure : m.divergence;
    if (kind == KIND_SCALAR) return which == BF_X ? m.sdata : m.stemp;
    return which == BF_X ? m.vel[kind] : m.temp[kind];
}

}  // namespace sfb
