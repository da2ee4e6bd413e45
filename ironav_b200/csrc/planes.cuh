// planes.cuh — K1: the half-sample planes of one reference picture (HalfPel::build,
// enc/subpel.rs:57-115), for 8-bit (uint8_t samples) and 10-bit (uint16_t samples) pictures.
//
// Each CTA produces a TW x TH tile of the four padded planes (sw x sh each, PAD = 48 samples of
// border): G = the picture with its edges repeated, b = horizontal half samples, h = vertical half
// samples, j = diagonal half samples from the unrounded horizontal sums. The tile's integer samples
// plus a 2-left/3-right/2-above/3-below halo are staged in shared memory once, the unrounded
// horizontal sums (b1) of every staged row are kept in shared memory as int32, and each thread
// writes 4 consecutive samples of each plane as one 32-bit (8-bit) or 64-bit (16-bit) store. HBM-bound:
// one read of the luma (through L2, halo rows re-read by neighbouring tiles) and 4 samples written per
// padded sample.
#pragma once
#include "common.cuh"

namespace ironav {

constexpr int K1_TW = 64;  // tile width (samples)
constexpr int K1_TH = 16;  // tile height (rows)
constexpr int K1_THREADS = (K1_TW / 4) * K1_TH;

__device__ __forceinline__ int k1_tap6(int a, int b, int c, int d, int e, int f) {
    return a - 5 * b + 20 * c + 20 * d - 5 * e + f;
}

__device__ __forceinline__ uint32_t k1_clip(int v, int maxv) { return (uint32_t)min(max(v, 0), maxv); }

// One TW x TH tile of the four planes, whose top-left sample is (x0, y0). luma: w x h samples, rows
// `stride` samples apart, values up to maxv = 2^bd - 1 (the half samples are clipped to it). Samples
// outside it repeat its edges, which is both the macroblock padding of H264Encoder::source
// (enc/mod.rs:502-519) when w x h is the picture size and the plane border of round1
// (enc/subpel.rs:72-76). All K1_THREADS threads of the block take part.
template <class T>
__device__ __forceinline__ void planes_tile(const T* __restrict__ luma, int stride, int w, int h, T* __restrict__ out,
                                            long long psize, int sw, int sh, int x0, int y0, int maxv) {
    __shared__ int g[K1_TH + 5][K1_TW + 8];       // integer samples, column c <-> x0 - 2 + c
    __shared__ int b1[K1_TH + 5][K1_TW];          // unrounded horizontal sums at x0 + c
    const int tid = threadIdx.x;
    // stage rows y0-2 .. y0+TH+2 and columns x0-2 .. x0+TW+5 of G (clamped to the plane; values
    // outside it are never used by an output that is not forced to zero)
    for (int i = tid; i < (K1_TH + 5) * (K1_TW + 8); i += K1_THREADS) {
        int r = i / (K1_TW + 8), c = i % (K1_TW + 8);
        int gy = min(max(y0 - 2 + r, 0), sh - 1), gx = min(max(x0 - 2 + c, 0), sw - 1);
        int sy = min(max(gy - PAD, 0), h - 1), sx = min(max(gx - PAD, 0), w - 1);
        g[r][c] = luma[(size_t)sy * stride + sx];
    }
    __syncthreads();
    for (int i = tid; i < (K1_TH + 5) * K1_TW; i += K1_THREADS) {
        int r = i / K1_TW, c = i % K1_TW;
        int gx = x0 + c;
        // b1 is only written for 2 <= x < sw - 3 (enc/subpel.rs:78-82); elsewhere it stays 0
        b1[r][c] = (gx >= 2 && gx < sw - 3) ? k1_tap6(g[r][c], g[r][c + 1], g[r][c + 2], g[r][c + 3], g[r][c + 4], g[r][c + 5]) : 0;
    }
    __syncthreads();
    const int ty = tid / (K1_TW / 4), tx = (tid % (K1_TW / 4)) * 4;
    const int y = y0 + ty, xb = x0 + tx;
    if (y >= sh || xb >= sw) return;  // sw is a multiple of 16, so a 4-sample group is whole
    const bool rows_ok = y >= 2 && y < sh - 3;  // rows of h and j outside stay 0 (enc/subpel.rs:95-97)
    // 4 samples of each plane, packed little-endian: one word (8-bit) or two (16-bit)
    constexpr int B = sizeof(T), BITS = 8 * B;
    uint32_t pg[B] = {}, pb[B] = {}, ph[B] = {}, pj[B] = {};
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const int c = tx + k, x = xb + k, r = ty + 2;
        const int wd = (k * B) >> 2, bit = (k * BITS) & 31;
        pg[wd] |= (uint32_t)g[r][c + 2] << bit;
        if (x >= 2 && x < sw - 3) pb[wd] |= k1_clip((b1[r][c] + 16) >> 5, maxv) << bit;
        if (rows_ok) {
            int v = k1_tap6(g[r - 2][c + 2], g[r - 1][c + 2], g[r][c + 2], g[r + 1][c + 2], g[r + 2][c + 2], g[r + 3][c + 2]);
            ph[wd] |= k1_clip((v + 16) >> 5, maxv) << bit;
            v = k1_tap6(b1[r - 2][c], b1[r - 1][c], b1[r][c], b1[r + 1][c], b1[r + 2][c], b1[r + 3][c]);
            pj[wd] |= k1_clip((v + 512) >> 10, maxv) << bit;
        }
    }
    const size_t o = (size_t)y * sw + xb;
    if constexpr (B == 1) {
        *reinterpret_cast<uint32_t*>(out + o) = pg[0];
        *reinterpret_cast<uint32_t*>(out + psize + o) = pb[0];
        *reinterpret_cast<uint32_t*>(out + 2 * psize + o) = ph[0];
        *reinterpret_cast<uint32_t*>(out + 3 * psize + o) = pj[0];
    } else {
        *reinterpret_cast<uint2*>(out + o) = make_uint2(pg[0], pg[1]);
        *reinterpret_cast<uint2*>(out + psize + o) = make_uint2(pb[0], pb[1]);
        *reinterpret_cast<uint2*>(out + 2 * psize + o) = make_uint2(ph[0], ph[1]);
        *reinterpret_cast<uint2*>(out + 3 * psize + o) = make_uint2(pj[0], pj[1]);
    }
}

template <class T>
static __global__ void __launch_bounds__(K1_THREADS) halfpel_planes_kernel(const T* __restrict__ luma, int stride, int w, int h,
                                                                             T* __restrict__ out, long long psize, int sw, int sh, int maxv) {
    planes_tile(luma, stride, w, h, out, psize, sw, sh, blockIdx.x * K1_TW, blockIdx.y * K1_TH, maxv);
}

// The co-located vector of each macroblock (col_mv, enc/frame.rs:944-947) from the reference
// picture's own decisions; none when the picture was intra coded (states == nullptr).
static __global__ void col_extract_kernel(const ironav_mbstate* __restrict__ states, ColMv* __restrict__ col, int nmb) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nmb) return;
    ColMv c;
    c.mv[0] = 0;
    c.mv[1] = 0;
    c.valid = 0;
    if (states && states[i].inter) {
        c.mv[0] = states[i].mvs[5][0];
        c.mv[1] = states[i].mvs[5][1];
        c.valid = 1;
    }
    col[i] = c;
}

// Repeats the right and bottom edges of a w x h picture stored in a pw x ph buffer (rows pw apart)
// to whole macroblocks (H264Encoder::source, enc/mod.rs:502-519). Reads only the w x h part.
template <class T>
static __global__ void pad_edges_kernel(T* __restrict__ p, int w, int h, int pw, int ph) {
    int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= pw || y >= ph || (x < w && y < h)) return;
    p[(size_t)y * pw + x] = p[(size_t)min(y, h - 1) * pw + min(x, w - 1)];
}

}  // namespace ironav
