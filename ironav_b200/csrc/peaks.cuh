// peaks.cuh — a measured 32-bit integer issue rate, the denominator of the analysis kernel's roofline.
//
// The driver's measured peaks cover HBM bandwidth and bf16 tensor throughput only; the analysis
// kernel is bound by the integer pipes. This kernel runs 16 independent chains per thread of
// a = (a + k) ^ b (one 32-bit add and one 32-bit xor, which no instruction fuses), on every SM at
// full occupancy, and reports 32-bit integer operations per second.
#pragma once
#include <cuda_runtime.h>

namespace ironav {

__global__ void __launch_bounds__(256) int32_peak_kernel(unsigned* out, int iters, unsigned seed) {
    unsigned a[16];
#pragma unroll
    for (int k = 0; k < 16; k++) a[k] = seed * (threadIdx.x + 1) + k * 0x9E3779B9u;
    const unsigned b = seed ^ blockIdx.x, kk = seed * 3u + 1u;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int r = 0; r < 8; r++) {
#pragma unroll
            for (int k = 0; k < 16; k++) a[k] = (a[k] + (kk + k)) ^ (b + r);
        }
    }
    unsigned s = 0;
#pragma unroll
    for (int k = 0; k < 16; k++) s ^= a[k];
    if (s == 0x12345678u) out[blockIdx.x] = s;  // keeps the chains live
}

}  // namespace ironav
