// Exhaustive check, on the GPU, of the correctly rounded division the
// stencil kernels use (tb::divide in sf_stencil_tb.cuh) against IEEE
// FP32 division (__fdiv_rn): every finite FP32 numerator for the pressure
// divisor 6; for a few diffusion divisors 1 + 6a every 61st numerator plus
// every tiny one (0 < |n| < 2^-99, including the subnormal quotients).
// Prints "<divisor> <checked> <mismatches>" per divisor; exit status 1 on a
// mismatch.
#include <cstdio>

#include "sf_stencil_tb.cuh"

using namespace sfb;

// Numerators u * stride for u < 2^32 / stride, then (tiny != 0) every
// numerator with 0 < |n| < 2^-99 of both signs.
__global__ void k_check(float divisor, unsigned long long stride, int tiny, unsigned long long* counts) {
    const double recip = tb::recip64(divisor);
    unsigned long long checked = 0, bad = 0;
    const unsigned long long tiny_bits = 0x0E000000ull;  // bit pattern of 2^-99
    const unsigned long long total = 0x100000000ull / stride + (tiny ? 2 * tiny_bits : 0);
    for (unsigned long long j = blockIdx.x * static_cast<unsigned long long>(blockDim.x) + threadIdx.x; j < total; j += static_cast<unsigned long long>(gridDim.x) * blockDim.x) {
        unsigned long long u = j * stride;
        if (j >= 0x100000000ull / stride) {
            const unsigned long long t = j - 0x100000000ull / stride;  // 0 .. 2 tiny_bits - 1
            u = (t < tiny_bits ? t : 0x80000000ull + (t - tiny_bits));
        }
        const float n = __uint_as_float(static_cast<unsigned>(u));
        if (!isfinite(n)) continue;
        const float want = __fdiv_rn(n, divisor);
        const float got = tb::divide(n, divisor, recip);
        bad += __float_as_uint(want) != __float_as_uint(got);
        ++checked;
    }
    atomicAdd(&counts[0], checked);
    atomicAdd(&counts[1], bad);
}

int main() {
    unsigned long long* counts = nullptr;
    if (cudaMallocManaged(&counts, 2 * sizeof(unsigned long long)) != cudaSuccess) return 2;
    const float diffusion[] = {1.0f + 6.0f * 1e-4f, 1.0f + 6.0f * 0.01f, 1.0f + 6.0f * 0.37f, 7.3f};
    int failed = 0;
    for (int k = 0; k < 5; ++k) {
        counts[0] = counts[1] = 0;
        const float d = k == 0 ? 6.0f : diffusion[k - 1];
        if (k == 0) k_check<<<148 * 8, 256>>>(d, 1, 0, counts);
        else k_check<<<148 * 8, 256>>>(d, 61, 1, counts);
        if (cudaDeviceSynchronize() != cudaSuccess) return 2;
        std::printf("%.9g %llu %llu\n", d, counts[0], counts[1]);
        failed |= counts[1] != 0;
    }
    cudaFree(counts);
    return failed;
}
