// planes.cuh — K1: the half-sample planes of one reference picture (HalfPel::build,
// enc/subpel.rs:57-115), for 8-bit (uint8_t samples) and 10-bit (uint16_t samples) pictures.
//
// Each CTA produces a TW x TH tile of the four padded planes (sw x sh each, PAD = 48 samples of
// border): G = the picture with its edges repeated, b = horizontal half samples, h = vertical half
// samples, j = diagonal half samples from the unrounded horizontal sums. The tile's integer samples
// plus a 2-left/3-right/2-above/3-below halo are staged in shared memory once, the unrounded
// horizontal sums (b1) of every staged row are kept in shared memory as int32, and each thread
// writes one column of 4 rows of each plane. HBM-bound: one read of the luma (through L2, halo rows
// re-read by neighbouring tiles) and 4 samples written per padded sample.
#pragma once
#include "common.cuh"

namespace ironav {

constexpr int K1_TW = 64;  // tile width (samples)
constexpr int K1_TH = 16;  // tile height (rows)
constexpr int K1_THREADS = 256;
constexpr int K1_RPT = K1_TH * K1_TW / K1_THREADS;  // rows per thread (4)

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
    // stage rows y0-2 .. y0+TH+2 and columns x0-2 .. x0+TW+5 of G (clamped to the plane; values outside it
    // are never used by an output that is not forced to zero): a thread keeps one column (its clamps worked
    // out once) and steps over the rows
    constexpr int GC = K1_TW + 8, GR = K1_TH + 5, GSPAN = K1_THREADS / GC;
    if (tid < GSPAN * GC) {
        const int c = tid % GC;
        const int sx = min(max(min(max(x0 - 2 + c, 0), sw - 1) - PAD, 0), w - 1);
        for (int r = tid / GC; r < GR; r += GSPAN) {
            const int sy = min(max(min(max(y0 - 2 + r, 0), sh - 1) - PAD, 0), h - 1);
            g[r][c] = luma[(size_t)sy * stride + sx];
        }
    }
    __syncthreads();
    {
        // b1 is only written for 2 <= x < sw - 3 (enc/subpel.rs:78-82); elsewhere it stays 0
        const int c = tid % K1_TW, gx = x0 + c;
        const bool ok = gx >= 2 && gx < sw - 3;
        for (int r = tid / K1_TW; r < GR; r += K1_THREADS / K1_TW)
            b1[r][c] = ok ? k1_tap6(g[r][c], g[r][c + 1], g[r][c + 2], g[r][c + 3], g[r][c + 4], g[r][c + 5]) : 0;
    }
    __syncthreads();
    // each thread: one column x of the tile, K1_RPT consecutive rows; lanes of a warp take consecutive columns,
    // so the shared-memory reads are conflict-free and the stores of a row are contiguous. The 6-tap vertical
    // windows of the thread's rows come from K1_RPT + 5 staged values of G and of b1 kept in registers.
    const int c = tid % K1_TW, r0 = (tid / K1_TW) * K1_RPT;
    const int x = x0 + c;
    if (x >= sw) return;  // sw is a multiple of 16, not of the tile width
    int gv[K1_RPT + 5], bv[K1_RPT + 5];
#pragma unroll
    for (int k = 0; k < K1_RPT + 5; k++) {
        gv[k] = g[r0 + k][c + 2];
        bv[k] = b1[r0 + k][c];
    }
    const bool col_ok = x >= 2 && x < sw - 3;  // columns of b outside stay 0 (enc/subpel.rs:78-82)
#pragma unroll
    for (int k = 0; k < K1_RPT; k++) {
        const int y = y0 + r0 + k;
        if (y >= sh) break;  // never taken while sh is a multiple of K1_TH (16 * mb_h + 96)
        const bool rows_ok = y >= 2 && y < sh - 3;  // rows of h and j outside stay 0 (enc/subpel.rs:95-97)
        const size_t o = (size_t)y * sw + x;
        out[o] = (T)gv[k + 2];
        out[psize + o] = (T)(col_ok ? k1_clip((bv[k + 2] + 16) >> 5, maxv) : 0u);
        out[2 * psize + o] = (T)(rows_ok ? k1_clip((k1_tap6(gv[k], gv[k + 1], gv[k + 2], gv[k + 3], gv[k + 4], gv[k + 5]) + 16) >> 5, maxv) : 0u);
        out[3 * psize + o] = (T)(rows_ok ? k1_clip((k1_tap6(bv[k], bv[k + 1], bv[k + 2], bv[k + 3], bv[k + 4], bv[k + 5]) + 512) >> 10, maxv) : 0u);
    }
}

// The co-located vector of macroblock i (col_mv, enc/frame.rs:944-947) from the reference picture's own
// decisions; none when the picture was intra coded (states == nullptr).
__device__ __forceinline__ void col_extract(const ironav_mbstate* __restrict__ states, ColMv* __restrict__ col, int i) {
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

// The planes of one reference picture, and its co-located vectors (nmb of them; the grid's first nmb
// threads, of at least sw * sh / 4 >= 64 * nmb, take one each).
template <class T>
static __global__ void __launch_bounds__(K1_THREADS) halfpel_planes_kernel(const T* __restrict__ luma, int stride, int w, int h,
                                                                             T* __restrict__ out, long long psize, int sw, int sh, int maxv,
                                                                             const ironav_mbstate* __restrict__ states,
                                                                             ColMv* __restrict__ col, int nmb) {
    const int gi = (blockIdx.y * gridDim.x + blockIdx.x) * K1_THREADS + threadIdx.x;
    if (col && gi < nmb) col_extract(states, col, gi);
    planes_tile(luma, stride, w, h, out, psize, sw, sh, blockIdx.x * K1_TW, blockIdx.y * K1_TH, maxv);
}

// Repeats the right and bottom edges of a w x h picture stored in a pw x ph buffer (rows pw apart)
// to whole macroblocks (H264Encoder::source, enc/mod.rs:502-519). Reads only the w x h part. Thread i
// writes the i-th padding sample: the bottom rows h..ph-1 (pw samples each), then the right columns
// w..pw-1 of rows 0..h-1 (pad_edges_count of them).
__host__ __device__ __forceinline__ long long pad_edges_count(int w, int h, int pw, int ph) {
    return (long long)(ph - h) * pw + (long long)h * (pw - w);
}
template <class T>
static __global__ void pad_edges_kernel(T* __restrict__ p, int w, int h, int pw, int ph) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x, nb = (long long)(ph - h) * pw;
    int x, y;
    if (i < nb) {
        y = h + (int)(i / pw);
        x = (int)(i % pw);
    } else if (i < pad_edges_count(w, h, pw, ph)) {  // pw > w here
        const long long j = i - nb;
        y = (int)(j / (pw - w));
        x = w + (int)(j % (pw - w));
    } else {
        return;
    }
    p[(size_t)y * pw + x] = p[(size_t)min(y, h - 1) * pw + min(x, w - 1)];
}

}  // namespace ironav
