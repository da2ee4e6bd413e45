// planes.cuh — K1: the half-sample planes of one reference picture (HalfPel::build,
// enc/subpel.rs:57-115), for 8-bit (uint8_t samples) and 10-bit (uint16_t samples) pictures.
//
// Each CTA produces a TW x TH tile of the four padded planes (sw x sh each, PAD = 48 samples of
// border): G = the picture with its edges repeated, b = horizontal half samples, h = vertical half
// samples, j = diagonal half samples from the unrounded horizontal sums. The tile's integer samples
// plus a halo are staged in shared memory once, packed (four 8-bit or two 16-bit samples a word), the
// unrounded horizontal sums (b1) of every staged row are kept there as int32, and each thread writes
// four columns of one row of each plane with one store a plane. HBM-bound in principle: one read of
// the luma (through L2, halo rows re-read by neighbouring tiles) and 4 samples written per padded sample.
#pragma once
#include "common.cuh"

namespace ironav {

constexpr int K1_TW = 64;  // tile width (samples)
constexpr int K1_TH = 16;  // tile height (rows)
constexpr int K1_THREADS = 256;  // 16 groups of four columns x 16 rows

__device__ __forceinline__ int k1_tap6(int a, int b, int c, int d, int e, int f) {
    return a - 5 * b + 20 * c + 20 * d - 5 * e + f;
}

__device__ __forceinline__ uint32_t k1_clip(int v, int maxv) { return (uint32_t)min(max(v, 0), maxv); }

// dp4a with unsigned bytes in a and signed bytes in b: c + sum of a_k * b_k.
__device__ __forceinline__ int k1_dp4a(uint32_t a, uint32_t b, int c) {
    int d;
    asm("dp4a.u32.s32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
    return d;
}
// tap6's weights as signed bytes: (1, -5, 20, 20) on four samples, then (-5, 1) on the next two
constexpr uint32_t K1_TAPS_A = 0x1414FB01u, K1_TAPS_B = 0x000001FBu;
constexpr int K1_GW = 48;  // staged row pitch in words: 48 = 16 mod 32 banks, so a warp's two rows never share one

// The same tile for 8-bit pictures, four columns a thread: the integer samples are staged as packed bytes
// (word k of a staged row holds samples x0 - 4 + 4k .. x0 - 1 + 4k), the horizontal taps of four columns
// are two dp4a each on byte windows of three words, the vertical taps of a column two dp4a on its bytes of
// six rows gathered with prmt, and the diagonal taps run on the unrounded horizontal sums in shared memory.
// Every plane is written a 32-bit word (four samples) at a time. Samples outside the w x h picture
// repeat its edges: both the macroblock padding of H264Encoder::source (enc/mod.rs:502-519) when w x h is
// the picture size and the plane border of round1 (enc/subpel.rs:72-76).
// TH: the tile's rows (16 by default; the batched form's tuner may pick 8), with 16 * TH threads.
template <int TH = K1_TH>
__device__ __forceinline__ void planes_tile8(const uint8_t* __restrict__ luma, int stride, int w, int h, uint8_t* __restrict__ out,
                                             long long psize, int sw, int sh, int x0, int y0) {
    constexpr int NT = 16 * TH;                           // threads: 16 groups of four columns x TH rows
    constexpr int GR = TH + 5, GWORDS = (K1_TW + 8) / 4;  // TH + 5 rows of 18 words: samples x0-4 .. x0+67
    __shared__ uint32_t g[GR][K1_GW];
    __shared__ __align__(16) int b1[GR][K1_TW];
    const int tid = threadIdx.x;
    // stage rows y0-2 .. y0+18, samples x0-4 .. x0+71: whole words straight from the luma when every one
    // of them lies inside the picture and the rows are word aligned, else sample by sample with the clamps
    const bool fast = x0 - 4 - PAD >= 0 && x0 + 4 * GWORDS - 5 - PAD <= w - 1 && x0 + 4 * GWORDS - 5 <= sw - 1 &&
                      y0 - 2 - PAD >= 0 && y0 + GR - 3 - PAD <= h - 1 &&
                      ((reinterpret_cast<uintptr_t>(luma) | (uintptr_t)stride) & 3) == 0;
    for (int i = tid; i < GR * GWORDS; i += NT) {
        const int r = i / GWORDS, k = i % GWORDS;
        uint32_t v = 0;
        if (fast) {
            v = *reinterpret_cast<const uint32_t*>(luma + (size_t)(y0 - 2 + r - PAD) * stride + (x0 - 4 + 4 * k - PAD));
        } else {
            const int sy = min(max(min(max(y0 - 2 + r, 0), sh - 1) - PAD, 0), h - 1);
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int sx = min(max(min(max(x0 - 4 + 4 * k + j, 0), sw - 1) - PAD, 0), w - 1);
                v |= (uint32_t)luma[(size_t)sy * stride + sx] << (8 * j);
            }
        }
        g[r][k] = v;
    }
    __syncthreads();
    // the unrounded horizontal sums of columns x0 + 4q .. +3 of every staged row (only 2 <= x < sw - 3,
    // enc/subpel.rs:78-82; elsewhere 0); the 6-tap window of column X + j starts at byte 2 + j of word q
    for (int i = tid; i < GR * (K1_TW / 4); i += NT) {
        const int r = i / (K1_TW / 4), q = i % (K1_TW / 4);
        const uint32_t w0 = g[r][q], w1 = g[r][q + 1], w2 = g[r][q + 2];
        int4 v;
        int* vp = reinterpret_cast<int*>(&v);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const uint32_t wa = __funnelshift_r(j < 2 ? w0 : w1, j < 2 ? w1 : w2, 8 * ((2 + j) & 3));
            const uint32_t wb = __funnelshift_r(j < 2 ? w1 : w2, j < 2 ? w2 : 0u, 8 * ((6 + j) & 3));
            const int gx = x0 + 4 * q + j;
            vp[j] = (gx >= 2 && gx < sw - 3) ? k1_dp4a(wa, K1_TAPS_A, k1_dp4a(wb, K1_TAPS_B, 0)) : 0;
        }
        *reinterpret_cast<int4*>(&b1[r][4 * q]) = v;
    }
    __syncthreads();
    // a thread: columns X .. X + 3 of one row
    const int q = tid % (K1_TW / 4), rr = tid / (K1_TW / 4);
    const int X = x0 + 4 * q, y = y0 + rr;
    if (X >= sw || y >= sh) return;  // sw is a multiple of 16: a group is all in or all out
    const bool rows_ok = y >= 2 && y < sh - 3;  // rows of h and j outside stay 0 (enc/subpel.rs:95-97)
    uint32_t gr[6];
#pragma unroll
    for (int k = 0; k < 6; k++) gr[k] = g[rr + k][q + 1];
    int4 bv[6];
#pragma unroll
    for (int k = 0; k < 6; k++) bv[k] = *reinterpret_cast<const int4*>(&b1[rr + k][4 * q]);
    uint32_t pb = 0, ph = 0, pj = 0;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const int* b2 = reinterpret_cast<const int*>(&bv[2]);
        pb |= k1_clip((b2[j] + 16) >> 5, 255) << (8 * j);
        if (rows_ok) {
            // byte j of rows y-2 .. y+1, then of rows y+2 .. y+3
            const unsigned sel = (unsigned)j | ((unsigned)(j + 4) << 4);
            const uint32_t t01 = __byte_perm(gr[0], gr[1], sel), t23 = __byte_perm(gr[2], gr[3], sel);
            const uint32_t ca = __byte_perm(t01, t23, 0x5410), cb = __byte_perm(gr[4], gr[5], sel);
            ph |= k1_clip((k1_dp4a(ca, K1_TAPS_A, k1_dp4a(cb, K1_TAPS_B, 0)) + 16) >> 5, 255) << (8 * j);
            const int v0 = reinterpret_cast<const int*>(&bv[0])[j], v1 = reinterpret_cast<const int*>(&bv[1])[j];
            const int v2 = reinterpret_cast<const int*>(&bv[2])[j], v3 = reinterpret_cast<const int*>(&bv[3])[j];
            const int v4 = reinterpret_cast<const int*>(&bv[4])[j], v5 = reinterpret_cast<const int*>(&bv[5])[j];
            pj |= k1_clip((k1_tap6(v0, v1, v2, v3, v4, v5) + 512) >> 10, 255) << (8 * j);
        }
    }
    const size_t o = (size_t)y * sw + X;
    *reinterpret_cast<uint32_t*>(out + o) = gr[2];
    *reinterpret_cast<uint32_t*>(out + psize + o) = pb;
    *reinterpret_cast<uint32_t*>(out + 2 * psize + o) = ph;
    *reinterpret_cast<uint32_t*>(out + 3 * psize + o) = pj;
}

// dp2a with unsigned 16-bit halves in a and signed bytes in b: c + a.h0 * b.b(2s) + a.h1 * b.b(2s+1), s = 0
// (lo) or 1 (hi).
__device__ __forceinline__ int k1_dp2a_lo(uint32_t a, uint32_t b, int c) {
    int d;
    asm("dp2a.lo.u32.s32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
    return d;
}
__device__ __forceinline__ int k1_dp2a_hi(uint32_t a, uint32_t b, int c) {
    int d;
    asm("dp2a.hi.u32.s32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
    return d;
}
// tap6 on three pairs of 16-bit samples (s0, s1) (s2, s3) (s4, s5): (1, -5) lo and (20, 20) hi of
// K1_TAPS_A, then (-5, 1) lo of K1_TAPS_B
__device__ __forceinline__ int k1_tap6_pairs(uint32_t p01, uint32_t p23, uint32_t p45) {
    return k1_dp2a_lo(p45, K1_TAPS_B, k1_dp2a_hi(p23, K1_TAPS_A, k1_dp2a_lo(p01, K1_TAPS_A, 0)));
}

// The same tile for 10-bit pictures (16-bit samples), four columns a thread: samples staged two a word
// (word k of a staged row holds samples x0 - 4 + 2k and x0 - 3 + 2k), each 6-tap three dp2a on sample
// pairs (realigned by a 16-bit funnel shift for odd columns, gathered across rows with prmt for the
// vertical taps), the diagonal taps on the unrounded horizontal sums, and one 64-bit store per plane.
// Same values as planes_tile8 at 8 bits; half samples are clipped to maxv = 2^bd - 1.
template <int TH = K1_TH>
__device__ __forceinline__ void planes_tile16(const uint16_t* __restrict__ luma, int stride, int w, int h, uint16_t* __restrict__ out,
                                              long long psize, int sw, int sh, int x0, int y0, int maxv) {
    constexpr int NT = 16 * TH;
    constexpr int GR = TH + 5, GWORDS = (K1_TW + 8) / 2;  // TH + 5 rows of 36 words: samples x0-4 .. x0+67
    __shared__ __align__(16) uint32_t g[GR][K1_GW];
    __shared__ __align__(16) int b1[GR][K1_TW];
    const int tid = threadIdx.x;
    const bool fast = x0 - 4 - PAD >= 0 && x0 + 2 * GWORDS - 5 - PAD <= w - 1 && x0 + 2 * GWORDS - 5 <= sw - 1 &&
                      y0 - 2 - PAD >= 0 && y0 + GR - 3 - PAD <= h - 1 &&
                      (reinterpret_cast<uintptr_t>(luma) & 3) == 0 && (stride & 1) == 0;
    for (int i = tid; i < GR * GWORDS; i += NT) {
        const int r = i / GWORDS, k = i % GWORDS;
        uint32_t v = 0;
        if (fast) {
            v = *reinterpret_cast<const uint32_t*>(luma + (size_t)(y0 - 2 + r - PAD) * stride + (x0 - 4 + 2 * k - PAD));
        } else {
            const int sy = min(max(min(max(y0 - 2 + r, 0), sh - 1) - PAD, 0), h - 1);
#pragma unroll
            for (int j = 0; j < 2; j++) {
                const int sx = min(max(min(max(x0 - 4 + 2 * k + j, 0), sw - 1) - PAD, 0), w - 1);
                v |= (uint32_t)luma[(size_t)sy * stride + sx] << (16 * j);
            }
        }
        g[r][k] = v;
    }
    __syncthreads();
    // the unrounded horizontal sums of columns X = x0 + 4q .. X + 3 (word 2q holds X - 4, X - 3): the taps
    // of column X + j start at sample X + j - 2, i.e. at half j + 2 of words 2q ..
    for (int i = tid; i < GR * (K1_TW / 4); i += NT) {
        const int r = i / (K1_TW / 4), q = i % (K1_TW / 4);
        uint32_t wv[6];  // words 2q .. 2q + 5 (the last pair of column X + 3 starts at half 9)
#pragma unroll
        for (int k = 0; k < 6; k += 2) {
            const uint2 t = *reinterpret_cast<const uint2*>(&g[r][2 * q + k]);  // 64-bit reads: no bank conflicts
            wv[k] = t.x;
            wv[k + 1] = t.y;
        }
        int4 v;
        int* vp = reinterpret_cast<int*>(&v);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            // sample pairs starting at half j + 2, j + 4, j + 6 of the words
            uint32_t p[3];
#pragma unroll
            for (int m = 0; m < 3; m++) {
                const int hpos = j + 2 + 2 * m;  // half index of the pair's first sample
                p[m] = (hpos & 1) ? __funnelshift_r(wv[hpos >> 1], wv[(hpos >> 1) + 1], 16) : wv[hpos >> 1];
            }
            const int gx = x0 + 4 * q + j;
            vp[j] = (gx >= 2 && gx < sw - 3) ? k1_tap6_pairs(p[0], p[1], p[2]) : 0;
        }
        *reinterpret_cast<int4*>(&b1[r][4 * q]) = v;
    }
    __syncthreads();
    const int q = tid % (K1_TW / 4), rr = tid / (K1_TW / 4);
    const int X = x0 + 4 * q, y = y0 + rr;
    if (X >= sw || y >= sh) return;
    const bool rows_ok = y >= 2 && y < sh - 3;
    // this thread's samples X .. X + 3 of rows y - 2 .. y + 3: words 2q + 2 and 2q + 3
    uint32_t ga[6], gb[6];
#pragma unroll
    for (int k = 0; k < 6; k++) {
        const uint2 t = *reinterpret_cast<const uint2*>(&g[rr + k][2 * q + 2]);
        ga[k] = t.x;
        gb[k] = t.y;
    }
    int4 bv[6];
#pragma unroll
    for (int k = 0; k < 6; k++) bv[k] = *reinterpret_cast<const int4*>(&b1[rr + k][4 * q]);
    uint32_t pb[2] = {0, 0}, ph[2] = {0, 0}, pj[2] = {0, 0};
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const int sh16 = 16 * (j & 1);
        pb[j >> 1] |= k1_clip((reinterpret_cast<const int*>(&bv[2])[j] + 16) >> 5, maxv) << sh16;
        if (rows_ok) {
            const uint32_t* col = (j < 2) ? ga : gb;
            // the column's samples of rows (y-2, y-1), (y, y+1), (y+2, y+3) as 16-bit pairs
            const unsigned sel = (j & 1) ? 0x7632u : 0x5410u;
            const int hv = k1_tap6_pairs(__byte_perm(col[0], col[1], sel), __byte_perm(col[2], col[3], sel), __byte_perm(col[4], col[5], sel));
            ph[j >> 1] |= k1_clip((hv + 16) >> 5, maxv) << sh16;
            const int v0 = reinterpret_cast<const int*>(&bv[0])[j], v1 = reinterpret_cast<const int*>(&bv[1])[j];
            const int v2 = reinterpret_cast<const int*>(&bv[2])[j], v3 = reinterpret_cast<const int*>(&bv[3])[j];
            const int v4 = reinterpret_cast<const int*>(&bv[4])[j], v5 = reinterpret_cast<const int*>(&bv[5])[j];
            pj[j >> 1] |= k1_clip((k1_tap6(v0, v1, v2, v3, v4, v5) + 512) >> 10, maxv) << sh16;
        }
    }
    const size_t o = (size_t)y * sw + X;
    *reinterpret_cast<uint2*>(out + o) = make_uint2(ga[2], gb[2]);
    *reinterpret_cast<uint2*>(out + psize + o) = make_uint2(pb[0], pb[1]);
    *reinterpret_cast<uint2*>(out + 2 * psize + o) = make_uint2(ph[0], ph[1]);
    *reinterpret_cast<uint2*>(out + 3 * psize + o) = make_uint2(pj[0], pj[1]);
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
    if constexpr (sizeof(T) == 1) planes_tile8(luma, stride, w, h, out, psize, sw, sh, blockIdx.x * K1_TW, blockIdx.y * K1_TH);
    else planes_tile16(luma, stride, w, h, out, psize, sw, sh, blockIdx.x * K1_TW, blockIdx.y * K1_TH, maxv);
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

// The padded source from a picture in device memory in one pass: sample (x, y) of the pw x ph buffer is
// picture sample (min(x, w - 1), min(y, h - 1)) (H264Encoder::source, enc/mod.rs:502-519). A thread writes
// 16 bytes; pw is a multiple of 16, so a thread's samples lie in one row.
template <class T>
static __global__ void copy_pad_kernel(T* __restrict__ dst, int pw, int ph, const T* __restrict__ src, int stride, int w, int h) {
    constexpr int PER = 16 / (int)sizeof(T);
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)pw * ph / PER) return;
    const long long e = i * PER;
    const int y = (int)(e / pw), x0 = (int)(e % pw);
    const T* row = src + (size_t)min(y, h - 1) * stride;
    alignas(16) T v[PER];
#pragma unroll
    for (int k = 0; k < PER; k++) v[k] = row[min(x0 + k, w - 1)];
    *reinterpret_cast<uint4*>(dst + e) = *reinterpret_cast<const uint4*>(v);
}

}  // namespace ironav
