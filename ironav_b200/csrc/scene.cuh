// scene.cuh — the scene-cut measure of the encoder (change_threads, codec/change.rs:56-90), on the device.
//
// LowRes (codec/change.rs:16-24): each low-resolution sample is the mean (sum >> 4) of a 4x4 block of
// the padded source. change: for every whole 8x8 block of low-resolution samples, intra = sum of |v - mean|
// (mean = sum / 64) and inter = the least SAD against the previous picture's low-resolution samples over
// displacements of -4..4 in each direction that stay inside the picture; the picture totals of both.
// Low-resolution samples fit in a byte (means of 8-bit samples), so the SADs run on packed bytes. One warp
// per 8x8 block: lanes take the 81 displacements (3 rounds), the block's 16 words sit in registers.
#pragma once
#include "common.cuh"

namespace ironav {

// Low-resolution luma (lw x lh) of a w x h picture whose rows are `stride` apart, edges repeated to whole
// macroblocks first (H264Encoder::low_res on the padded Source, enc/mod.rs:689-693).
static __global__ void lowres_kernel(const uint8_t* __restrict__ luma, int stride, int w, int h, int lw, int lh,
                                     uint8_t* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= lw * lh) return;
    const int x0 = (i % lw) * 4, y0 = (i / lw) * 4;
    int sum = 0;
#pragma unroll
    for (int k = 0; k < 16; k++) sum += luma[(size_t)min(y0 + k / 4, h - 1) * stride + min(x0 + k % 4, w - 1)];
    out[i] = (uint8_t)(sum >> 4);
}

// Bytes at any offset of a low-resolution row: two aligned words realigned.
__device__ __forceinline__ uint32_t lr_word(const uint8_t* p) {
    const uintptr_t a = reinterpret_cast<uintptr_t>(p);
    const uint32_t* q = reinterpret_cast<const uint32_t*>(a & ~uintptr_t(3));
    return __funnelshift_r(q[0], q[1], (unsigned)(a & 3) * 8u);
}

// sums[0] += inter, sums[1] += intra over the blocks this launch covers (one warp per block).
static __global__ void change_kernel(const uint8_t* __restrict__ prev, const uint8_t* __restrict__ cur, int lw, int lh,
                                     unsigned long long* sums) {
    const int lane = threadIdx.x & 31;
    const int nbx = (lw >= 8) ? (lw - 8) / 8 + 1 : 0, nby = (lh >= 8) ? (lh - 8) / 8 + 1 : 0;
    const int blk = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (blk >= nbx * nby) return;
    const int bx = (blk % nbx) * 8, by = (blk / nbx) * 8;
    // the block's 64 samples: lanes 0..15 hold word (row = lane / 2, half = lane % 2)
    uint32_t mine = 0;
    if (lane < 16) mine = lr_word(cur + (size_t)(by + lane / 2) * lw + bx + (lane & 1) * 4);
    uint32_t wv[16];
#pragma unroll
    for (int k = 0; k < 16; k++) wv[k] = __shfl_sync(0xffffffffu, mine, k);
    // intra: sum of |v - mean|, mean = sum / 64 (codec/change.rs:62-63)
    int sum = 0;
#pragma unroll
    for (int k = 0; k < 16; k++) sum += __dp4a(wv[k], 0x01010101u, 0u);
    const uint32_t mean = (uint32_t)(sum / 64);
    const uint32_t mean4 = mean * 0x01010101u;
    int intra = 0;
#pragma unroll
    for (int k = 0; k < 16; k++) intra += (int)__vsadu4(wv[k], mean4);
    // inter: least SAD over the displacements inside the picture (codec/change.rs:64-75)
    int best = 0x7fffffff;
    for (int d = lane; d < 81; d += 32) {
        const int dx = d % 9 - 4, dy = d / 9 - 4, ox = bx + dx, oy = by + dy;
        if (ox < 0 || oy < 0 || ox + 8 > lw || oy + 8 > lh) continue;
        const uint8_t* p = prev + (size_t)oy * lw + ox;
        int sad = 0;
#pragma unroll
        for (int r = 0; r < 8; r++) sad += (int)__vsadu4(wv[2 * r], lr_word(p + r * lw)) + (int)__vsadu4(wv[2 * r + 1], lr_word(p + r * lw + 4));
        best = min(best, sad);
    }
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) best = min(best, __shfl_xor_sync(0xffffffffu, best, off));
    if (lane == 0) {
        atomicAdd(&sums[0], (unsigned long long)best);
        atomicAdd(&sums[1], (unsigned long long)intra);
    }
}

}  // namespace ironav
