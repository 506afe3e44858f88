// sf_batch.h -- the work table of a batch of simulations stepped together.
//
// One launch per stage covers every simulation of the batch: the table holds
// one BatchSim per simulation (its field pointers, coefficients, boundaries
// and the autotuned z chunk of its sweeps) and, per launch shape, the first
// work item of each simulation. A work item is one thread block of one
// simulation: item w belongs to simulation s with first[s] <= w < first[s+1]
// and is block w - first[s] of that simulation's own grid. The kernels are
// persistent: a grid of at most (resident blocks per SM) x (SMs) blocks walks
// the items with a stride of the grid size. Plain types only, so the C++23
// host runtime can build the table.
#pragma once

#include <cuda_runtime.h>

#include "sf_types.h"

namespace sfb {

constexpr int kBatchForces = 4;  // force fields per simulation in a work-table batch

struct BatchSim {
    Dims d;
    float h;            // cell size
    float dt;
    float alpha_v;      // dt * viscosity / h^2
    float alpha_s;      // dt * diffusion / h^2 of the scalar
    float scale_s;      // scalar dissipation factor 1 / (1 + dt * dissipation)
    int32_t z_chunk;    // planes per block of the vectorised sweeps
    int32_t force_count;
    FlowBC flow;
    ScalarBC sbc;
    GhostRule ghost[5];  // per StencilKind
    float* vel[3];
    float* temp[3];      // advected velocity: right-hand sides of the velocity diffusion
    float* packed;       // float4 (x, y, z, 0) velocity for the advection gathers
    float* pressure;
    float* divergence;
    float* magnitude;
    float* scratch;      // field-sized buffer of the Jacobi ping-pong; a red-black solve's split iterate
    float* scratch2;     // a red-black solve's split right-hand side (null: none)
    float* sdata;        // the scalar field
    float* stemp;        // its advected copy (right-hand side of its diffusion)
    const float* source; // its source
    const float* force[kBatchForces][3];
    DeviceStats* stats;
};

// Launch shapes: LINEAR = 256 cells per block; CELL = (32, 4, 2) blocks over
// the grid; VEC = (32, 4) threads x 4 cells per thread over x, z_chunk planes;
// HALF = 128 groups of 4 cells of a colour-split half plane per block,
// z_chunk planes; OCT = 256 groups of 8 cells per block.
enum BatchShape : int32_t { SHAPE_LINEAR = 0, SHAPE_CELL = 1, SHAPE_VEC = 2, SHAPE_HALF = 3, SHAPE_OCT = 4 };
constexpr int kBatchShapes = 5;

struct BatchTable {
    const BatchSim* sims;      // device array, nsims entries
    const uint32_t* first[kBatchShapes];  // device arrays per BatchShape, nsims + 1 entries
    uint32_t total[kBatchShapes];         // work items per BatchShape
    int32_t nsims;
    int32_t sms;               // multiprocessors of the device
};

// Buffers a batched sweep reads or writes, per StencilKind: X = the iterate
// (velocity component, scalar, pressure), B = its right-hand side, SCRATCH.
enum BatchField : int32_t { BF_X = 0, BF_B = 1, BF_SCRATCH = 2 };

// Host helpers.
uint32_t batch_blocks(const Dims& d, int shape, int z_chunk);
GhostRule make_ghost_rule(int kind, const FlowBC& fb, const ScalarBC& sb);

// Stage launches (FP32 fields).
cudaError_t launch_batch_force_pack(const BatchTable& t, cudaStream_t s);
cudaError_t launch_batch_advect_velocity(const BatchTable& t, cudaStream_t s);
cudaError_t launch_batch_scalar_source_advect(const BatchTable& t, cudaStream_t s);
cudaError_t launch_batch_divergence(const BatchTable& t, cudaStream_t s);
cudaError_t launch_batch_project(const BatchTable& t, int pack, cudaStream_t s);
cudaError_t launch_batch_post_diagnostics(const BatchTable& t, cudaStream_t s);
// dst <- src (both BatchField of `kind`), or dst <- 0 when src < 0.
cudaError_t launch_batch_copy(const BatchTable& t, int kind, int dst, int src, cudaStream_t s);
cudaError_t launch_batch_scale_scalar(const BatchTable& t, cudaStream_t s);
// One RBGS colour (scheme RBGS, in place on X) or one Jacobi sweep dst <- update(src).
cudaError_t launch_batch_sweep(const BatchTable& t, int kind, int scheme, int parity, int dst, int src, cudaStream_t s);
// Red-black solves in the colour-split layout (every simulation with a
// scratch2 buffer, rows of a multiple of 8 cells, even periodic sizes):
// split `which` (BF_B into scratch2 and, with copy_iterate, also into scratch
// as the starting iterate; BF_X into scratch), one colour of an iteration,
// and the merge of scratch into BF_X (times the scalar dissipation factor
// when `dissipate`).
cudaError_t launch_batch_rb_split(const BatchTable& t, int kind, int which, int copy_iterate, cudaStream_t s);
cudaError_t launch_batch_rb_half(const BatchTable& t, int kind, int colour, cudaStream_t s);
cudaError_t launch_batch_rb_merge(const BatchTable& t, int kind, int dissipate, cudaStream_t s);
// Per simulation: zero its residual sums (finalize 0) or turn them into
// rel_res with the iteration count (finalize 1).
cudaError_t launch_batch_stats(const BatchTable& t, int finalize, int iterations, cudaStream_t s);
// Adds the FP64 residual sums of every simulation's pressure solve to its
// DeviceStats (between launch_batch_stats 0 and 1).
cudaError_t launch_batch_residual_sums(const BatchTable& t, cudaStream_t s);

}  // namespace sfb
