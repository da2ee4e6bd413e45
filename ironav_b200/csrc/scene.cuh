// scene.cuh — the scene-cut measure of the encoder (change_threads, codec/change.rs:56-90), on the device.
//
// LowRes (codec/change.rs:16-24): each low-resolution sample is the mean (sum >> 4) of a 4x4 block of
// the padded source. change: for every whole 8x8 block of low-resolution samples, intra = sum of |v - mean|
// (mean = sum / 64) and inter = the least SAD against the previous picture's low-resolution samples over
// displacements of -4..4 in each direction that stay inside the picture; the picture totals of both.
// Low-resolution samples keep the picture's sample type (bytes for 8-bit pictures, halfwords for 10-bit),
// so the SADs run on packed samples. One warp per 8x8 block: lanes take the 81 displacements (3 rounds),
// the block's samples sit in registers.
#pragma once
#include "common.cuh"

namespace ironav {

// Low-resolution luma (lw x lh) of a w x h picture whose rows are `stride` samples apart, edges repeated to
// whole macroblocks first (H264Encoder::low_res on the padded Source, enc/mod.rs:689-693). T is the sample
// type; a mean of 10-bit samples keeps 10 bits (the encoder does not scale it down).
template <class T>
static __global__ void lowres_kernel(const T* __restrict__ luma, int stride, int w, int h, int lw, int lh, T* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= lw * lh) return;
    const int x0 = (i % lw) * 4, y0 = (i / lw) * 4;
    int sum = 0;
#pragma unroll
    for (int k = 0; k < 16; k++) sum += luma[(size_t)min(y0 + k / 4, h - 1) * stride + min(x0 + k % 4, w - 1)];
    out[i] = (T)(sum >> 4);
}

// The 32-bit word at any byte offset of a low-resolution row: two aligned words realigned.
__device__ __forceinline__ uint32_t lr_word(const uint8_t* p) {
    const uintptr_t a = reinterpret_cast<uintptr_t>(p);
    const uint32_t* q = reinterpret_cast<const uint32_t*>(a & ~uintptr_t(3));
    return __funnelshift_r(q[0], q[1], (unsigned)(a & 3) * 8u);
}

// Packed-sample helpers: 4 bytes or 2 halfwords a word.
template <class T>
__device__ __forceinline__ int lr_sad(uint32_t a, uint32_t b) {
    if constexpr (sizeof(T) == 1) return (int)__vsadu4(a, b);
    else return (int)__vsadu2(a, b);
}
template <class T>
__device__ __forceinline__ int lr_sum(uint32_t a) {
    if constexpr (sizeof(T) == 1) return __dp4a(a, 0x01010101u, 0u);
    else return (int)(a & 0xffffu) + (int)(a >> 16);
}

// sums[0] += inter, sums[1] += intra over the blocks this launch covers (one warp per block). A row of 8
// low-resolution samples is W = 2 * sizeof(T) words; the block's 8 W words sit in registers.
template <class T>
static __global__ void change_kernel(const T* __restrict__ prev_s, const T* __restrict__ cur_s, int lw, int lh,
                                     unsigned long long* sums) {
    constexpr int B = sizeof(T), W = 2 * B, NW = 8 * W;
    const uint8_t* prev = reinterpret_cast<const uint8_t*>(prev_s);
    const uint8_t* cur = reinterpret_cast<const uint8_t*>(cur_s);
    const int lane = threadIdx.x & 31;
    const int nbx = (lw >= 8) ? (lw - 8) / 8 + 1 : 0, nby = (lh >= 8) ? (lh - 8) / 8 + 1 : 0;
    const int blk = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (blk >= nbx * nby) return;
    const int bx = (blk % nbx) * 8, by = (blk / nbx) * 8;
    // the block's samples: lane k < NW holds word k (row k / W, word k % W of the row)
    uint32_t mine = 0;
    if (lane < NW) mine = lr_word(cur + ((size_t)(by + lane / W) * lw + bx) * B + (lane % W) * 4);
    uint32_t wv[NW];
#pragma unroll
    for (int k = 0; k < NW; k++) wv[k] = __shfl_sync(0xffffffffu, mine, k);
    // intra: sum of |v - mean|, mean = sum / 64 (codec/change.rs:62-63)
    int sum = 0;
#pragma unroll
    for (int k = 0; k < NW; k++) sum += lr_sum<T>(wv[k]);
    const uint32_t mean = (uint32_t)(sum / 64);
    const uint32_t meanw = B == 1 ? mean * 0x01010101u : mean * 0x00010001u;
    int intra = 0;
#pragma unroll
    for (int k = 0; k < NW; k++) intra += lr_sad<T>(wv[k], meanw);
    // inter: least SAD over the displacements inside the picture (codec/change.rs:64-75)
    int best = 0x7fffffff;
    for (int d = lane; d < 81; d += 32) {
        const int dx = d % 9 - 4, dy = d / 9 - 4, ox = bx + dx, oy = by + dy;
        if (ox < 0 || oy < 0 || ox + 8 > lw || oy + 8 > lh) continue;
        const uint8_t* p = prev + ((size_t)oy * lw + ox) * B;
        int sad = 0;
#pragma unroll
        for (int r = 0; r < 8; r++)
#pragma unroll
            for (int k = 0; k < W; k++) sad += lr_sad<T>(wv[r * W + k], lr_word(p + (size_t)r * lw * B + k * 4));
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
