// sf_unet.h -- host interface of the learned pressure warm start (the
// network lives in sf_unet.cu) for the step runtime. Plain CUDA runtime
// types only, so the C++23 host code can include it.
#pragma once

#include <cuda_runtime.h>

#include "sf_types.h"

namespace sfb::net {

struct Net;

// Kernels one predict() enqueues.
constexpr int kPredictKernels = 21;

// Sets the FP32 master parameters from host memory (synchronous) and
// refreshes the BF16 copies; resets the optimizer state.
cudaError_t set_parameters(Net* n, const float* host);

// Allocates the activation buffers for grid d and `owner` (synchronous; call
// it before a stream capture that will contain predict()). Each owner (an
// attached context) gets inference-only buffers of its own, so that contexts
// sharing the network can predict concurrently; owner null is the network's
// own set. Grid sides must be multiples of 4.
cudaError_t prepare(Net* n, Dims d, const void* owner);

// Frees the buffer sets of `owner` (its step graphs must be gone or rebuilt).
void release(Net* n, const void* owner);

// p0 = p_prev + net(b_factor * b, p_prev) / scale on stream s, with the
// buffers of (d, owner); p_prev may be null (zero) and may alias p0. Adds
// kPredictKernels to *launches.
cudaError_t predict(Net* n, const float* b, float b_factor, const float* p_prev, float* p0, Dims d, cudaStream_t s, int* launches, const void* owner);

}  // namespace sfb::net
