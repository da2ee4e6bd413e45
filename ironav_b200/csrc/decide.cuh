// decide.cuh — K7: the P macroblock decision of the CAVLC encoder (code_mb, enc/frame.rs:715-790) on the
// device, one warp per macroblock in the auto mode's wavefront: P_Skip tests (the fast luma and chroma SADs,
// then code_inter's cbp == 0), best_i16, best_inter (K2's searches), code_i4 when intra is competitive, and
// the coding of the cheapest (code_inter, code_i16 or the Intra4x4 trial, code_intra_chroma) into the
// unfiltered reconstruction that later macroblocks' intra prediction reads.
//
// A macroblock's intra prediction reads the reconstruction of its left, top, top-left and top-right
// neighbours; the wavefront's waits (left and top-right, K2's auto mode) cover all four, and a macroblock
// publishes its flag after its reconstruction, code and state are written (fence, then release store).
//
// Lanes: best_i16 takes a 4x4 block and two modes a lane; the Intra4x4 trial goes block by block in
// decoding order (each block predicts from the ones before), its nine modes on lanes 0-8 and the chosen
// block's transform on the winning lane; code_i16 takes a lane per 4x4 block with the DC transform on lane
// 0; intra chroma takes a lane per (mode, component, 4x4 block) for the search and then code_chroma_mb.
#pragma once
#include "residual.cuh"

namespace ironav {

struct DecideParams {
    CodeParams C;          // C.A: the analysis' parameters and the wavefront's (order, ticket, flags, epoch, err)
    ironav_mbcode* codes;  // every macroblock's code (neighbours' Intra4x4 modes are read back from here)
    int fast_t, fast_tc;   // the fast mode's P_Skip bounds on the luma and chroma SADs
    int intra;             // an IDR picture: no reference, every macroblock intra (code_mb of an I slice)
    int flat_t;            // the fast mode's bound on a flat macroblock's Intra16x16 cost (enc/frame.rs:763)
};

constexpr int K7_WARPS = 4;
constexpr int K7_MIN_BLOCKS = 2;  // the wavefront keeps few macroblocks in flight: registers (255, no spills) over occupancy
constexpr int KIND_I4 = 1, KIND_I8 = 2, KIND_I16 = 3, KIND_INTER = 5;  // Kind, h264/mb.rs:21-30

template <class T>
struct DecideSmem {
    WarpSmem<T> a;         // the analysis' working set (source, neighbour table, searches)
    CodeSmem c;            // the coder's
    int top[21];           // luma row above the macroblock: x = -1 (top-left) .. 19 (the top-right macroblock's first 4)
    int left[16];          // luma column to its left
    int ctop[2][9];        // chroma rows above: x = -1 .. 7
    int cleft[2][8];       // chroma columns to the left
    int i4rec[256];        // the Intra4x4 trial's reconstruction
    int16_t i4lv[16][16];  // its levels: raster 4x4 blocks, scan order
    int edge[2][13];       // the Intra4x4 trial's two current 4x4 blocks' edges: top-left, 8 above, 4 to the left
    int dcs[16];           // Intra16x16: each block's DC coefficient, then its dequantised DC
    int nbm[8];            // pred_i4_mode: the left macroblock's modes down its right column, then the top's along its
                           // bottom row (2 for a macroblock that is not Intra4x4, -1 unavailable)
    uint8_t i4modes[16];
    uint8_t i4nnz[16];
};

// A source sample of the staged macroblock (WarpSmem::src: 16 rows of 16 samples, packed).
template <class T>
__device__ __forceinline__ int src_at(const WarpSmem<T>& S, int x, int y) {
    if (sizeof(T) == 1) return (int)((S.src[y * 4 + (x >> 2)] >> (8 * (x & 3))) & 0xffu);
    return (int)((S.src[y * 8 + (x >> 1)] >> (16 * (x & 1))) & 0xffffu);
}

// satd4, enc/frame.rs:144-161, of 16 differences (raster)
__device__ __forceinline__ int satd4_d(const int (&d)[16]) {
    int t[16];
#pragma unroll
    for (int r = 0; r < 4; r++) {
        const int a = d[r * 4], b = d[r * 4 + 1], c = d[r * 4 + 2], e = d[r * 4 + 3];
        const int s0 = a + b, s1 = c + e, d0 = a - b, d1 = c - e;
        t[r * 4] = s0 + s1;
        t[r * 4 + 1] = s0 - s1;
        t[r * 4 + 2] = d0 - d1;
        t[r * 4 + 3] = d0 + d1;
    }
    int sum = 0;
#pragma unroll
    for (int c = 0; c < 4; c++) {
        const int a = t[c], b = t[4 + c], cc = t[8 + c], e = t[12 + c];
        const int s0 = a + b, s1 = cc + e, d0 = a - b, d1 = cc - e;
        sum += abs(s0 + s1) + abs(s0 - s1) + abs(d0 - d1) + abs(d0 + d1);
    }
    return sum >> 1;
}

// The 4x4 intra predictors (predict_nxn, h264/intra.rs:30-128; ITU-T H.264 8.3.1.2) as a table: every sample
// of every mode other than DC is (E[a] + 2 E[b] + E[c] + 2) >> 2 over the block's edge array E (E[0] the
// top-left sample, E[1 + i] the 8 above, E[9 + j] the 4 to the left): a copy has a = b = c, a two-sample
// average (x + y + 1) >> 1 has a = c = x, b = y, and (x + 3y + 2) >> 2 has b = c = y. Entry: a | b << 4 | c << 8.
__device__ __forceinline__ unsigned i4_entry(int mode, int x, int y) {
    auto T = [](int i) { return 1 + i; };                 // i >= -1: i = -1 is the top-left sample
    auto L = [](int j) { return j < 0 ? 0 : 9 + j; };
    auto e3 = [](int a, int b, int c) { return (unsigned)(a | b << 4 | c << 8); };
    switch (mode) {
    case 0: return e3(T(x), T(x), T(x));
    case 1: return e3(L(y), L(y), L(y));
    case 3: return (x == 3 && y == 3) ? e3(T(6), T(7), T(7)) : e3(T(x + y), T(x + y + 1), T(x + y + 2));
    case 4:
        if (x > y) return e3(T(x - y - 2), T(x - y - 1), T(x - y));
        if (x < y) return e3(L(y - x - 2), L(y - x - 1), L(y - x));
        return e3(T(0), 0, L(0));
    case 5: {
        const int z = 2 * x - y, i = x - (y >> 1);
        if (z >= 0 && (z & 1) == 0) return e3(T(i - 1), T(i), T(i - 1));
        if (z >= 0) return e3(T(i - 2), T(i - 1), T(i));
        if (z == -1) return e3(L(0), 0, T(0));
        return e3(L(y - 2 * x - 1), L(y - 2 * x - 2), L(y - 2 * x - 3));
    }
    case 6: {
        const int z = 2 * y - x, j = y - (x >> 1);
        if (z >= 0 && (z & 1) == 0) return e3(L(j - 1), L(j), L(j - 1));
        if (z >= 0) return e3(L(j - 2), L(j - 1), L(j));
        if (z == -1) return e3(L(0), 0, T(0));
        return e3(T(x - 2 * y - 1), T(x - 2 * y - 2), T(x - 2 * y - 3));
    }
    case 7: {
        const int i = x + (y >> 1);
        return (y & 1) == 0 ? e3(T(i), T(i + 1), T(i)) : e3(T(i), T(i + 1), T(i + 2));
    }
    case 8: {
        const int z = x + 2 * y, j = y + (x >> 1);
        if (z > 5) return e3(L(3), L(3), L(3));
        if (z == 5) return e3(L(2), L(3), L(3));
        if ((z & 1) == 0) return e3(L(j), L(j + 1), L(j));
        return e3(L(j), L(j + 1), L(j + 2));
    }
    default: return 0;  // DC: not a table entry
    }
}

// fdct4 (enc/frame.rs:113-132) of a 4x4 block held one value a lane (lane 4r + c of each half-warp: a block
// a half): the lane's coefficient at raster position (r, c). Every lane takes part in the shuffles.
__device__ __forceinline__ int fdct4_lanes(int v) {
    const int lane = threadIdx.x & 31, r = (lane >> 2) & 3, c = lane & 3, base = lane & ~3, hb = (lane & 16) + c;
    const int a0 = __shfl_sync(FULL, v, base), a1 = __shfl_sync(FULL, v, base + 1), a2 = __shfl_sync(FULL, v, base + 2), a3 = __shfl_sync(FULL, v, base + 3);
    int s03 = a0 + a3, d03 = a0 - a3, s12 = a1 + a2, d12 = a1 - a2;
    const int t = c == 0 ? s03 + s12 : (c == 1 ? 2 * d03 + d12 : (c == 2 ? s03 - s12 : d03 - 2 * d12));
    const int b0 = __shfl_sync(FULL, t, hb), b1 = __shfl_sync(FULL, t, hb + 4), b2 = __shfl_sync(FULL, t, hb + 8), b3 = __shfl_sync(FULL, t, hb + 12);
    s03 = b0 + b3, d03 = b0 - b3, s12 = b1 + b2, d12 = b1 - b2;
    return r == 0 ? s03 + s12 : (r == 1 ? 2 * d03 + d12 : (r == 2 ? s03 - s12 : d03 - 2 * d12));
}

// idct4_add (h264/idct.rs:8-31) of raster coefficients held one a lane (a block a half-warp, as fdct4_lanes)
// onto the lane's prediction sample.
__device__ __forceinline__ int idct4_lanes(int co, int pred, int maxv) {
    const int lane = threadIdx.x & 31, r = (lane >> 2) & 3, c = lane & 3, base = lane & ~3, hb = (lane & 16) + c;
    const int c0 = __shfl_sync(FULL, co, base), c1 = __shfl_sync(FULL, co, base + 1), c2 = __shfl_sync(FULL, co, base + 2), c3 = __shfl_sync(FULL, co, base + 3);
    const int e0 = c0 + c2, e1 = c0 - c2, e2 = (c1 >> 1) - c3, e3 = c1 + (c3 >> 1);
    const int t = c == 0 ? e0 + e3 : (c == 1 ? e1 + e2 : (c == 2 ? e1 - e2 : e0 - e3));
    const int t0 = __shfl_sync(FULL, t, hb), t1 = __shfl_sync(FULL, t, hb + 4), t2 = __shfl_sync(FULL, t, hb + 8), t3 = __shfl_sync(FULL, t, hb + 12);
    const int g0 = t0 + t2, g1 = t0 - t2, g2 = (t1 >> 1) - t3, g3 = t1 + (t3 >> 1);
    const int h = r == 0 ? g0 + g3 : (r == 1 ? g1 + g2 : (r == 2 ? g1 - g2 : g0 - g3));
    return min(max(pred + ((h + 32) >> 6), 0), maxv);
}

// The scan position of raster coefficient p (the inverse of ZIGZAG4), as nibbles.
__device__ __forceinline__ int invzz4_at(int p) { return (int)((0xFEA9DB83C7426510ull >> (4 * p)) & 15); }

// The Intra16x16 prediction of sample (x, y) (predict_16x16, h264/intra.rs:161-209): dcv the DC value, (pa,
// pb, pc) the plane parameters.
template <class T>
__device__ __forceinline__ int i16_sample(const DecideSmem<T>& S, int mode, int x, int y, int dcv, int pa, int pb, int pc, int maxv) {
    if (mode == 0) return S.top[1 + x];
    if (mode == 1) return S.left[y];
    if (mode == 2) return dcv;
    return min(max((pa + pb * (x - 7) + pc * (y - 7) + 16) >> 5, 0), maxv);
}

// The DC value and plane parameters of the Intra16x16 prediction from the neighbours in S.
template <class T>
__device__ __forceinline__ void i16_params(const DecideSmem<T>& S, bool ta, bool la, int bd, int* dcv, int* pa, int* pb, int* pc) {
    int st = 0, sl = 0, h = 0, v = 0;
#pragma unroll
    for (int i = 0; i < 16; i++) {
        st += S.top[1 + i];
        sl += S.left[i];
    }
#pragma unroll
    for (int k = 0; k < 8; k++) {
        h += (k + 1) * (S.top[1 + 8 + k] - S.top[1 + 6 - k]);  // top[-1] is the top-left sample (S.top[0])
        v += (k + 1) * (S.left[8 + k] - (6 - k < 0 ? S.top[0] : S.left[6 - k]));
    }
    *dcv = (ta && la) ? (st + sl + 16) >> 5 : (la ? (sl + 8) >> 4 : (ta ? (st + 8) >> 4 : 1 << (bd - 1)));
    *pa = 16 * (S.left[15] + S.top[16]);
    *pb = (5 * h + 32) >> 6;
    *pc = (5 * v + 32) >> 6;
}

// The chroma prediction of sample (x, y) of component cc (predict_chroma, h264/intra.rs:212-287, 8x8).
template <class T>
__device__ __forceinline__ int chroma_sample(const DecideSmem<T>& S, int mode, int cc, int x, int y, bool ta, bool la, int bd) {
    if (mode == 1) return S.cleft[cc][y];
    if (mode == 2) return S.ctop[cc][1 + x];
    if (mode == 3) {
        int hh = 0, vv = 0;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            hh += (k + 1) * (S.ctop[cc][1 + 4 + k] - S.ctop[cc][1 + 2 - k]);
            vv += (k + 1) * (S.cleft[cc][4 + k] - (2 - k < 0 ? S.ctop[cc][0] : S.cleft[cc][2 - k]));
        }
        const int a = 16 * (S.cleft[cc][7] + S.ctop[cc][8]), b = (34 * hh + 32) >> 6, c = (34 * vv + 32) >> 6;
        return min(max((a + b * (x - 3) + c * (y - 3) + 16) >> 5, 0), (1 << bd) - 1);
    }
    const int bx = x >> 2, by = y >> 2, mid = 1 << (bd - 1);
    const int st = S.ctop[cc][1 + bx * 4] + S.ctop[cc][2 + bx * 4] + S.ctop[cc][3 + bx * 4] + S.ctop[cc][4 + bx * 4];
    const int sl = S.cleft[cc][by * 4] + S.cleft[cc][by * 4 + 1] + S.cleft[cc][by * 4 + 2] + S.cleft[cc][by * 4 + 3];
    if (bx == by) return (ta && la) ? (st + sl + 4) >> 3 : (la ? (sl + 2) >> 2 : (ta ? (st + 2) >> 2 : mid));
    if (bx > 0) return ta ? (st + 2) >> 2 : (la ? (sl + 2) >> 2 : mid);
    return la ? (sl + 2) >> 2 : (ta ? (st + 2) >> 2 : mid);
}

// Loads the reconstructed samples around the macroblock (luma row above with the top-left and top-right
// samples, luma column to the left, the same for both chroma components) and the neighbours' Intra4x4 modes.
template <class T>
__device__ void load_intra_neighbours(const DecideParams& P, DecideSmem<T>& S, int mb, int mbx, int mby, bool ta, bool la, bool tra) {
    const int lane = threadIdx.x & 31;
    const CodeParams& C = P.C;
    const T* Y = reinterpret_cast<const T*>(C.rec[0]);
    const int x0 = mbx * 16, y0 = mby * 16;
    if (lane < 21) {
        const int x = lane - 1;
        const bool ok = x < 0 ? (ta && la) : (x < 16 ? ta : tra);
        S.top[lane] = ok ? (int)Y[(size_t)(y0 - 1) * C.ys + x0 + x] : 0;
    }
    if (lane < 16) S.left[lane] = la ? (int)Y[(size_t)(y0 + lane) * C.ys + x0 - 1] : 0;
    const int cx0 = mbx * 8, cy0 = mby * 8;
    if (lane < 18) {
        const int cc = lane / 9, x = lane % 9 - 1;
        const T* Cp = reinterpret_cast<const T*>(C.rec[1 + cc]);
        const bool ok = x < 0 ? (ta && la) : ta;
        S.ctop[cc][x + 1] = ok ? (int)Cp[(size_t)(cy0 - 1) * C.cs + cx0 + x] : 0;
    }
    if (lane >= 16) {
        const int cc = (lane - 16) >> 3, y = lane & 7;
        const T* Cp = reinterpret_cast<const T*>(C.rec[1 + cc]);
        S.cleft[cc][y] = la ? (int)Cp[(size_t)(cy0 + y) * C.cs + cx0 - 1] : 0;
    }
    if (lane < 8) {
        // pred_i4_mode's neighbours (enc/frame.rs:619-629): not Intra4x4 counts as DC
        const bool left = lane < 4;
        const bool ok = left ? la : ta;
        int m = -1;
        if (ok) {
            const ironav_mbcode* n = &P.codes[left ? mb - 1 : mb - C.A.mb_w];
            // Intra8x8 macroblocks (CABAC with the 8x8 transform) give their modes too (MbState::i4, 2309)
            m = (n->kind == KIND_I4 || n->kind == KIND_I8) ? (int)n->modes[left ? lane * 4 + 3 : 12 + (lane - 4)] : 2;
        }
        S.nbm[lane] = m;
    }
    __syncwarp();
}

// best_i16, enc/frame.rs:812-835: the cheapest Intra16x16 mode by SATD + lambda (modes other than DC);
// returns (mode, cost) on every lane.
template <class T>
__device__ int2 best_i16_d(const DecideParams& P, DecideSmem<T>& S, bool ta, bool la) {
    const int lane = threadIdx.x & 31;
    const int bd = P.C.bd, maxv = (1 << bd) - 1;
    int dcv, pa, pb, pc;
    i16_params(S, ta, la, bd, &dcv, &pa, &pb, &pc);
    const int b = lane & 15, bx = b & 3, by = b >> 2, half = lane >> 4;
    int sums[2];
#pragma unroll
    for (int q = 0; q < 2; q++) {
        const int mode = half + 2 * q;  // lanes 0-15: modes 0 and 2; lanes 16-31: modes 1 and 3
        int d[16];
#pragma unroll
        for (int r = 0; r < 4; r++)
#pragma unroll
            for (int k = 0; k < 4; k++)
                d[r * 4 + k] = src_at(S.a, bx * 4 + k, by * 4 + r) - i16_sample(S, mode, bx * 4 + k, by * 4 + r, dcv, pa, pb, pc, maxv);
        int s = satd4_d(d);
#pragma unroll
        for (int off = 8; off >= 1; off >>= 1) s += __shfl_xor_sync(FULL, s, off);
        sums[q] = s;
    }
    const int c0 = __shfl_sync(FULL, sums[0], 0), c2 = __shfl_sync(FULL, sums[1], 0);
    const int c1 = __shfl_sync(FULL, sums[0], 16), c3 = __shfl_sync(FULL, sums[1], 16);
    const int lam = P.C.A.lambda;
    int bm = 2, bc = BIG;
    if (ta && c0 + lam < bc) bm = 0, bc = c0 + lam;
    if (la && c1 + lam < bc) bm = 1, bc = c1 + lam;
    if (c2 < bc) bm = 2, bc = c2;
    if (ta && la && c3 + lam < bc) bm = 3, bc = c3 + lam;
    return make_int2(bm, bc);
}

__device__ __forceinline__ int zorder_d(int bx, int by) { return ((by >> 1) << 3) | ((bx >> 1) << 2) | ((by & 1) << 1) | (bx & 1); }

// code_i4, enc/frame.rs:1050-1138, as a trial: each block predicted from the reconstruction so far
// (S.i4rec inside the macroblock, the neighbours' around it), its mode the cheapest by SATD + lambda * (1
// for the predicted mode, 4 otherwise; from the table tab), coded with the intra rounding and
// reconstructed into S.i4rec. A block reads only its left, top-left, top and top-right neighbours, so the
// blocks go by anti-diagonal t = bx + 2 * by (10 steps of one or two blocks, a block a half-warp: its modes
// on lanes 0-8 of the half, a coefficient a lane for the coding) rather than one at a time in decoding
// order; the top-right's availability stays the decoding order's (zorder), and the cost is the same sum.
// Returns the summed cost (every lane).
template <class T, bool STOPPABLE = false>
__device__ int code_i4_trial(const DecideParams& P, DecideSmem<T>& S, const unsigned* tab, bool ta, bool la, bool tra,
                             const volatile int* stop = nullptr, int seq = 0) {
    const int lane = threadIdx.x & 31, hl = lane & 15, half = lane >> 4;
    const unsigned hmask = half ? 0xffff0000u : 0x0000ffffu;
    const int bd = P.C.bd, maxv = (1 << bd) - 1, lam = P.C.A.lambda;
    const int qp = P.C.qp + 6 * (bd - 8), m6 = qp % 6, qbits = 15 + qp / 6, f = (1 << qbits) / 3;
    const bool tla = ta && la;
    if (lane < 16) S.i4modes[lane] = 2;
    __syncwarp();
    int total = 0;
    for (int t = 0; t < 10; t++) {
        if constexpr (STOPPABLE) {
            if (__shfl_sync(FULL, (int)(*stop == seq), 0)) return 0;  // not needed after all
        }
        // the half's block: the upper one of the diagonal (the one with the smaller by), or the lower one
        const int by0 = max(0, (t - 2) >> 1), bx0 = t - 2 * by0;
        const bool two = bx0 >= 2 && by0 < 3;  // the diagonal's second block, (bx0 - 2, by0 + 1)
        const bool act = half == 0 || two;
        const int bx = act ? bx0 - 2 * half : 0, by = act ? by0 + half : 0;
        const bool hlf = bx > 0 || la, ht = by > 0 || ta;
        const bool htl = bx > 0 ? (by > 0 ? true : ta) : (by > 0 ? la : tla);
        // above-right: the macroblocks above for the top row, else a block decoded earlier (zorder, 2363-2365)
        const bool htr = by == 0 ? (bx < 3 ? ta : tra) : (bx == 3 ? false : zorder_d(bx + 1, by - 1) < zorder_d(bx, by));
        int* edge = S.edge[half];
        if (hl < 13) {
            int v = 0;
            if (hl == 0) {
                if (htl) v = by == 0 ? S.top[bx * 4] : (bx == 0 ? S.left[by * 4 - 1] : S.i4rec[(by * 4 - 1) * 16 + bx * 4 - 1]);
            } else if (hl < 9) {
                const int i = hl - 1;
                const int xi = (i < 4 || htr) ? i : 3;  // above-right not available: the last sample above repeated
                if (ht) v = by == 0 ? S.top[1 + bx * 4 + xi] : S.i4rec[(by * 4 - 1) * 16 + bx * 4 + xi];
            } else {
                const int j = hl - 9;
                if (hlf) v = bx == 0 ? S.left[by * 4 + j] : S.i4rec[(by * 4 + j) * 16 + bx * 4 - 1];
            }
            edge[hl] = v;
        }
        __syncwarp();
        // pred_i4_mode, enc/frame.rs:619-629
        const int a = bx > 0 ? S.i4modes[by * 4 + bx - 1] : S.nbm[by];
        const int b = by > 0 ? S.i4modes[(by - 1) * 4 + bx] : S.nbm[4 + bx];
        const int predicted = (a >= 0 && b >= 0) ? min(a, b) : 2;
        // the DC value (8.3.1.2.3)
        const int st = edge[1] + edge[2] + edge[3] + edge[4], sl = edge[9] + edge[10] + edge[11] + edge[12];
        const int dcv = (ht && hlf) ? (st + sl + 4) >> 3 : (hlf ? (sl + 2) >> 2 : (ht ? (st + 2) >> 2 : 1 << (bd - 1)));
        unsigned key = 0xffffffffu;
        {
            const int mode = hl < 9 ? hl : 2;
            const bool ok = hl < 9 &&
                            ((mode == 0 || mode == 3 || mode == 7) ? ht : ((mode == 1 || mode == 8) ? hlf : (mode == 2 ? true : (ht && hlf && htl))));
            int d[16];
#pragma unroll
            for (int k = 0; k < 16; k++) {
                const unsigned e = tab[mode * 17 + k];
                const int pv = mode == 2 ? dcv : (edge[e & 15] + 2 * edge[(e >> 4) & 15] + edge[(e >> 8) & 15] + 2) >> 2;
                d[k] = src_at(S.a, bx * 4 + (k & 3), by * 4 + (k >> 2)) - pv;
            }
            const int cost = satd4_d(d) + lam * (mode == predicted ? 1 : 4);
            if (ok) key = ((unsigned)cost << 4) | (unsigned)mode;  // the cheapest, the lowest mode on ties
        }
#pragma unroll
        for (int off = 8; off >= 1; off >>= 1) key = min(key, __shfl_xor_sync(FULL, key, off));
        const int bm = (int)(key & 15u);
        {
            const unsigned k0 = __shfl_sync(FULL, key, 0), k1 = __shfl_sync(FULL, key, 16);
            total += (int)(k0 >> 4) + (two ? (int)(k1 >> 4) : 0);
        }
        // quant_block (intra), enc/frame.rs:1025-1046, and the reconstruction: a coefficient a lane
        const int p = hl, r = p >> 2, c = p & 3;
        const unsigned e = tab[bm * 17 + p];
        const int pv = bm == 2 ? dcv : (edge[e & 15] + 2 * edge[(e >> 4) & 15] + edge[(e >> 8) & 15] + 2) >> 2;
        const int coef = fdct4_lanes(src_at(S.a, bx * 4 + c, by * 4 + r) - pv);
        const int cls = q_class_d(p);
        const int l = q_quant_d(coef, c_q_mf[m6][cls], f, qbits);
        const int nz = __popc(__ballot_sync(FULL, l != 0) & hmask);
        const int rec = idct4_lanes((l * c_q_v[m6][cls]) << (qp / 6), pv, maxv);
        if (act) {
            S.i4lv[by * 4 + bx][invzz4_at(p)] = (int16_t)l;
            S.i4rec[(by * 4 + r) * 16 + bx * 4 + c] = nz > 0 ? rec : pv;
            if (hl == 0) {
                S.i4nnz[by * 4 + bx] = (uint8_t)nz;
                S.i4modes[by * 4 + bx] = (uint8_t)bm;
            }
        }
        __syncwarp();
    }
    return total;
}

// code_i16, enc/frame.rs:1140-1200: the AC of each 4x4 block (a lane per block), the DC through the
// Hadamard transform halved and quantised with doubled precision (lane 0), reconstructed as a decoder does.
// Returns the luma coded block pattern (every lane).
template <class T>
__device__ uint32_t code_i16_d(const DecideParams& P, DecideSmem<T>& S, int mbx, int mby, int mode, bool ta, bool la, ironav_mbcode* out) {
    const int lane = threadIdx.x & 31;
    const int bd = P.C.bd, maxv = (1 << bd) - 1;
    const int qp = P.C.qp + 6 * (bd - 8), m6 = qp % 6, sh = qp / 6;
    int dcv, pa, pb, pc;
    i16_params(S, ta, la, bd, &dcv, &pa, &pb, &pc);
    const int bx = lane & 3, by = (lane >> 2) & 3;
    bool any_ac = false;
    if (lane < 16) {
        int d[16], c[16];
#pragma unroll
        for (int r = 0; r < 4; r++)
#pragma unroll
            for (int k = 0; k < 4; k++)
                d[r * 4 + k] = src_at(S.a, bx * 4 + k, by * 4 + r) - i16_sample(S, mode, bx * 4 + k, by * 4 + r, dcv, pa, pb, pc, maxv);
        q_fdct4_d(d, c);
        const int qbits = 15 + qp / 6, f = (1 << qbits) / 3;
#pragma unroll
        for (int k = 0; k < 16; k++) {
            const int pz = zz4_at(k);
            const int l = pz != 0 ? q_quant_d(c[pz], c_q_mf[m6][q_class_d(pz)], f, qbits) : 0;
            S.c.lv4[lane][k] = (int16_t)l;
            any_ac |= l != 0;
        }
        S.dcs[lane] = c[0];
    }
    const bool ac = __ballot_sync(FULL, any_ac) != 0;
    __syncwarp();
    if (lane == 0) {
        // hadamard4 (h264/idct.rs:76-95) of the DC coefficients, quantised; then the decoder's inverse
        int h[16], t[16];
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const int s0 = S.dcs[i * 4] + S.dcs[i * 4 + 1], s1 = S.dcs[i * 4] - S.dcs[i * 4 + 1];
            const int s2 = S.dcs[i * 4 + 2] + S.dcs[i * 4 + 3], s3 = S.dcs[i * 4 + 2] - S.dcs[i * 4 + 3];
            t[i * 4] = s0 + s2;
            t[i * 4 + 1] = s0 - s2;
            t[i * 4 + 2] = s1 - s3;
            t[i * 4 + 3] = s1 + s3;
        }
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int s0 = t[j] + t[4 + j], s1 = t[j] - t[4 + j], s2 = t[8 + j] + t[12 + j], s3 = t[8 + j] - t[12 + j];
            h[j] = s0 + s2;
            h[4 + j] = s0 - s2;
            h[8 + j] = s1 - s3;
            h[12 + j] = s1 + s3;
        }
        const int qbits = 16 + qp / 6, f = (1 << qbits) / 3;
        int dl[16];
#pragma unroll
        for (int k = 0; k < 16; k++) {
            const int pz = zz4_at(k);
            const int l = q_quant_d(h[pz] >> 1, c_q_mf[m6][0], f, qbits);
            out->dc[k] = (int16_t)l;
            dl[pz] = l;
        }
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const int s0 = dl[i * 4] + dl[i * 4 + 1], s1 = dl[i * 4] - dl[i * 4 + 1], s2 = dl[i * 4 + 2] + dl[i * 4 + 3], s3 = dl[i * 4 + 2] - dl[i * 4 + 3];
            t[i * 4] = s0 + s2;
            t[i * 4 + 1] = s0 - s2;
            t[i * 4 + 2] = s1 - s3;
            t[i * 4 + 3] = s1 + s3;
        }
        const int lsd = 16 * c_q_v[m6][0];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int s0 = t[j] + t[4 + j], s1 = t[j] - t[4 + j], s2 = t[8 + j] + t[12 + j], s3 = t[8 + j] - t[12 + j];
            const int fv[4] = {s0 + s2, s0 - s2, s1 - s3, s1 + s3};
#pragma unroll
            for (int i = 0; i < 4; i++)
                S.dcs[i * 4 + j] = qp >= 36 ? (fv[i] * lsd) << (qp / 6 - 6) : (fv[i] * lsd + (1 << (5 - qp / 6))) >> (6 - qp / 6);
        }
    }
    __syncwarp();
    if (lane < 16) {
        int co[16], p[16], nz = 0, any = 0;
        uint32_t packed[8];
#pragma unroll
        for (int k = 0; k < 16; k++) {
            const int pz = zz4_at(k);
            const int l = ac ? S.c.lv4[lane][k] : 0;
            nz += l != 0;
            co[pz] = (l * c_q_v[m6][q_class_d(pz)]) << sh;
            if (k & 1) packed[k >> 1] |= (uint32_t)(l & 0xffff) << 16;
            else packed[k >> 1] = (uint32_t)(l & 0xffff);
        }
        co[0] = S.dcs[lane];
#pragma unroll
        for (int k = 0; k < 16; k++) any |= co[k];
#pragma unroll
        for (int r = 0; r < 4; r++)
#pragma unroll
            for (int k = 0; k < 4; k++) p[r * 4 + k] = i16_sample(S, mode, bx * 4 + k, by * 4 + r, dcv, pa, pb, pc, maxv);
        int rb[16];
        if (any) {
            q_idct4_d(co, p, maxv, rb);
        } else {
#pragma unroll
            for (int k = 0; k < 16; k++) rb[k] = p[k];
        }
        T* RY = reinterpret_cast<T*>(P.C.rec[0]);
#pragma unroll
        for (int r = 0; r < 4; r++)
#pragma unroll
            for (int k = 0; k < 4; k++) RY[(size_t)(mby * 16 + by * 4 + r) * P.C.ys + mbx * 16 + bx * 4 + k] = (T)rb[r * 4 + k];
        uint32_t* lw = reinterpret_cast<uint32_t*>(out->res.luma[lane]);
#pragma unroll
        for (int k = 0; k < 8; k++) lw[k] = packed[k];
        out->res.nnz[lane] = (uint8_t)nz;
    }
    __syncwarp();
    return ac ? 15u : 0u;
}

// code_intra_chroma, enc/frame.rs:1807-1854: the chroma mode of least lambda * (1 DC, 3 otherwise) + SATD
// of both components (a lane per mode, component and 4x4 block), then code_chroma with the intra rounding.
// Returns the chroma part of the coded block pattern (every lane).
template <class T>
__device__ uint32_t code_intra_chroma_d(const DecideParams& P, DecideSmem<T>& S, int mbx, int mby, bool ta, bool la, ironav_mbcode* out) {
    const int lane = threadIdx.x & 31;
    const CodeParams& C = P.C;
    const int mode = lane >> 3, cc = (lane >> 2) & 1, blk = lane & 3, bx = blk & 1, by = blk >> 1;
    const T* SC = reinterpret_cast<const T*>(C.src_c) + (size_t)cc * C.cw * C.ch;
    int pr[16], d[16];
#pragma unroll
    for (int r = 0; r < 4; r++)
#pragma unroll
        for (int k = 0; k < 4; k++) {
            pr[r * 4 + k] = chroma_sample(S, mode, cc, bx * 4 + k, by * 4 + r, ta, la, C.bd);
            d[r * 4 + k] = (int)SC[(size_t)(mby * 8 + by * 4 + r) * C.cw + mbx * 8 + bx * 4 + k] - pr[r * 4 + k];
        }
    int s = satd4_d(d);
#pragma unroll
    for (int off = 4; off >= 1; off >>= 1) s += __shfl_xor_sync(FULL, s, off);
    const int lam = C.A.lambda;
    int bm = 0, bc = BIG;
#pragma unroll
    for (int m = 0; m < 4; m++) {
        const int cm = __shfl_sync(FULL, s, m * 8) + lam * (m == 0 ? 1 : 3);
        const bool ok = m == 0 || (m == 1 && la) || (m == 2 && ta) || (m == 3 && la && ta);
        if (ok && cm < bc) bm = m, bc = cm;
    }
    if (mode == bm) {
#pragma unroll
        for (int r = 0; r < 4; r++)
#pragma unroll
            for (int k = 0; k < 4; k++) S.c.cpred[cc][(by * 4 + r) * 8 + bx * 4 + k] = pr[r * 4 + k];
    }
    if (lane == 0) out->chroma_mode = (uint8_t)bm;
    __syncwarp();
    return code_chroma_mb<T>(C, S.c, mbx, mby, &out->res, true);
}

// The rectangle (x, y, w, h in 4x4 blocks) of partition n of rects(part, sub) in coding order
// (enc/frame.rs:208-223), and its reference index slot (ref_of).
__device__ __forceinline__ int4 rect_n(int part, const uint8_t* sub, int n, int* rslot) {
    if (part < 3) {
        *rslot = part == 0 ? 0 : n;
        return make_int4(c_parts[part][n][0], c_parts[part][n][1], c_parts[part][n][2], c_parts[part][n][3]);
    }
    int k = 0;
    while (n >= c_nsub[sub[k]]) n -= c_nsub[sub[k++]];
    *rslot = k;
    const int s = sub[k];
    return make_int4((k & 1) * 2 + c_sub[s][n][0], (k >> 1) * 2 + c_sub[s][n][1], c_sub[s][n][2], c_sub[s][n][3]);
}

// part_mvps, enc/frame.rs:579-594: each partition's predictor with the partitions before it in place; writes
// the differences (every vector less its predictor; beyond the partitions, the vector itself) and the
// macroblock's state.
template <class T>
__device__ void inter_tail(const DecideParams& P, DecideSmem<T>& S, const ironav_interdec& D, ironav_mbcode* out) {
    const int lane = threadIdx.x & 31;
    const AnalyseParams& A = P.C.A;
    const int part = D.part;
    const int count = part == 0 ? 1 : (part < 3 ? 2 : c_nsub[D.sub[0]] + c_nsub[D.sub[1]] + c_nsub[D.sub[2]] + c_nsub[D.sub[3]]);
    const int dir = part == 1 ? 1 : (part == 2 ? 2 : 0);
    if (lane < 16) S.a.t[lane] = make_int4(0, 0, -1, 0);
    if (lane >= count && lane < 16) {
        out->mvds[lane][0] = D.mvs[lane][0];
        out->mvds[lane][1] = D.mvs[lane][1];
    }
    __syncwarp();
    for (int n = 0; n < count; n++) {
        int rs;
        const int4 r = rect_n(part, D.sub, n, &rs);
        const int rf = D.refs[rs];
        const int2 p = pred_mv(A, S.a, S.a.ext, S.a.t, r.x, r.y, r.z, dir, rf);
        if (lane == 0) {
            out->mvds[n][0] = (int16_t)(D.mvs[n][0] - p.x);
            out->mvds[n][1] = (int16_t)(D.mvs[n][1] - p.y);
        }
        blk_paint(A, S.a, S.a.t, r.x, r.y, r.z, r.w, D.mvs[n][0], D.mvs[n][1], rf);
    }
    // the state (finish_mb, enc/frame.rs:2281-2321): the vectors painted over the partitions, the reference
    // of each 8x8 block
    if (lane < 16) {
        const int bx = lane & 3, by = lane >> 2;
        int n, rs;
        rect_of(part, D.sub, bx, by, &n, &rs);
        S.a.out.mvs[lane][0] = D.mvs[n][0];
        S.a.out.mvs[lane][1] = D.mvs[n][1];
        if ((bx & 1) == 0 && (by & 1) == 0) S.a.out.refs[(by >> 1) * 2 + (bx >> 1)] = (int8_t)D.refs[rs];
    }
    if (lane == 0) {
        S.a.out.inter = 1;
        S.a.out.pad[0] = S.a.out.pad[1] = S.a.out.pad[2] = 0;
        out->kind = KIND_INTER;
        out->part = D.part;
        for (int k = 0; k < 4; k++) {
            out->sub[k] = D.sub[k];
            out->refs[k] = D.refs[k];
        }
    }
    if (lane < 16) {
        out->mvs[lane][0] = D.mvs[lane][0];
        out->mvs[lane][1] = D.mvs[lane][1];
    }
    __syncwarp();
}

// ---- warp pairs (one stream's latency-bound wavefront) -----------------------------------------------
// The second warp of a pair works out a macroblock's intra side, best_i16 and then the Intra4x4 trial,
// while the first runs best_inter. The reference tries Intra4x4 only when intra is competitive after
// best_inter (766-779); the first warp then takes the trial's result, and otherwise tells the second to
// stop. The warps meet through sequence words in shared memory (one command, then best_i16's result, then
// the end of the intra side, per macroblock that reaches the intra stage); every wait is bounded in wall
// time and gives up when the launch's error word is set.
struct PairSync {
    volatile int cmd_seq;   // first warp: its latest command (cmd: 1 the intra side, -1 exit)
    volatile int cmd;
    volatile int stop_seq;  // first warp: the trial of this command is not needed
    volatile int i16_seq;   // second warp: best_i16 of this command is in i16
    volatile int done_seq;  // second warp: the intra side of this command is finished (c4 when it ran through)
    int2 i16;
    int c4;
    int ta, la, tra;        // the macroblock's neighbour availability
    int seq;                // the first warp's command count
};
constexpr unsigned long long PAIR_WAIT_NS = 20000000000ull;

// Waits until *word == want; false when the launch's error word is set or after PAIR_WAIT_NS (which sets
// it). The warp polls in step (lane 0's read decides) and fences before it reads what the word guards.
static __device__ bool pair_wait(const AnalyseParams& A, const volatile int* word, int want) {
    const unsigned long long t0 = globaltimer();
    for (unsigned i = 0;; i++) {
        if (__shfl_sync(FULL, (int)(*word == want), 0)) break;
        if ((i & 63) == 63) {
            bool quit = false;
            if ((threadIdx.x & 31) == 0) {
                quit = ld_acquire(A.err) != 0;
                if (!quit && globaltimer() - t0 > PAIR_WAIT_NS) {
                    atomicOr(A.err, 1u);
                    quit = true;
                }
            }
            if (__shfl_sync(FULL, quit, 0)) return false;
        }
        __nanosleep(i < 64 ? 32 : 256);
    }
    __threadfence_block();
    return true;
}

// Makes the warp's shared-memory writes visible, then sets *word = v (lane 0).
static __device__ __forceinline__ void pair_publish(volatile int* word, int v) {
    __threadfence_block();
    __syncwarp();
    if ((threadIdx.x & 31) == 0) *word = v;
    __syncwarp();
}

// The first warp's command: returns its sequence number.
static __device__ __forceinline__ int pair_command(PairSync& X, int cmd) {
    const int seq = X.seq + 1;
    __syncwarp();
    if ((threadIdx.x & 31) == 0) {
        X.seq = seq;
        X.cmd = cmd;
    }
    pair_publish(&X.cmd_seq, seq);
    return seq;
}

// The second warp: the intra side of each macroblock the first warp sends, until told to exit.
template <class T>
__device__ void pair_helper(const DecideParams& P, DecideSmem<T>& S, PairSync& X, const unsigned* i4tab) {
    const AnalyseParams& A = P.C.A;
    for (int seq = 1;; seq++) {
        if (!pair_wait(A, &X.cmd_seq, seq) || __shfl_sync(FULL, X.cmd, 0) < 0) return;
        const bool ta = X.ta != 0, la = X.la != 0, tra = X.tra != 0;
        const int2 i16 = best_i16_d(P, S, ta, la);
        if ((threadIdx.x & 31) == 0) X.i16 = i16;
        pair_publish(&X.i16_seq, seq);
        const int c4 = code_i4_trial<T, true>(P, S, i4tab, ta, la, tra, &X.stop_seq, seq);
        if ((threadIdx.x & 31) == 0) X.c4 = c4;
        pair_publish(&X.done_seq, seq);
    }
}

// code_mb's P_Skip tests, enc/frame.rs:722-751: the fast one on the luma and chroma SADs (live coding), then
// code_inter with the skip vector when its SAD is under the threshold. Returns true (every lane) when the
// macroblock is P_Skip, its code, state and reconstruction written; else false with the skip vector in *sv_out
// and S.c.dec holding the skip vector's 16x16 decision (mode 2, the 4x4 transform).
template <class T>
__device__ bool skip_tests_d(const DecideParams& P, DecideSmem<T>& S, int mb, int mbx, int mby, ironav_mbcode* out, int2* sv_out) {
    const int lane = threadIdx.x & 31;
    const AnalyseParams& A = P.C.A;
    const CodeParams& C = P.C;
    ironav_interdec& D = *reinterpret_cast<ironav_interdec*>(S.c.dec);
    // P_Skip first (722-751)
    const int2 sv = skip_mv(A, S.a);
    if (lane == 0) S.a.cand[0] = sv;
    __syncwarp();
    pred_batch(A, S.a, 0, 0, 0, 2, 2, 1, true);
    const int sad = S.a.cost[0];
    __syncwarp();
    // the skip vector's decision: 16x16 from reference 0
    if (lane == 0) {
        D.mode = 2;
        D.part = 0;
        D.t8 = 0;
        for (int k = 0; k < 4; k++) D.sub[k] = D.refs[k] = 0;
        D.pad[0] = D.pad[1] = D.pad[2] = 0;
    }
    if (lane < 16) {
        D.mvs[lane][0] = (int16_t)sv.x;
        D.mvs[lane][1] = (int16_t)sv.y;
    }
    __syncwarp();
    if (A.fast && sad < P.fast_t) {
        // close to the reference: P_Skip when the chroma is too, nothing transformed
        if (lane == 0) D.mode = 1;
        __syncwarp();
        for (int i = lane; i < 128; i += 32) {
            const int cc = i >> 6, cy = (i >> 3) & 7, cx = i & 7;
            const T* rc = reinterpret_cast<const T*>(C.ref_c[0]) + (size_t)cc * C.cw * C.ch;
            const int fx = sv.x & 7, fy = sv.y & 7;
            const int xs = mbx * 8 + cx + (sv.x >> 3), ysm = mby * 8 + cy + (sv.y >> 3);
            const int xa = min(max(xs, 0), C.cw - 1), xb = min(max(xs + 1, 0), C.cw - 1);
            const int ya = min(max(ysm, 0), C.ch - 1), yb = min(max(ysm + 1, 0), C.ch - 1);
            const int v = ((8 - fx) * (8 - fy) * rc[(size_t)ya * C.cw + xa] + fx * (8 - fy) * rc[(size_t)ya * C.cw + xb] +
                           (8 - fx) * fy * rc[(size_t)yb * C.cw + xa] + fx * fy * rc[(size_t)yb * C.cw + xb] + 32) >> 6;
            const T* SC = reinterpret_cast<const T*>(C.src_c) + (size_t)cc * C.cw * C.ch;
            S.c.cpred[cc][cy * 8 + cx] = abs((int)SC[(size_t)(mby * 8 + cy) * C.cw + mbx * 8 + cx] - v);
        }
        __syncwarp();
        int csad = 0;
        for (int i = lane; i < 128; i += 32) csad += S.c.cpred[i >> 6][i & 63];
#pragma unroll
        for (int off = 16; off >= 1; off >>= 1) csad += __shfl_xor_sync(FULL, csad, off);
        __syncwarp();
        if (csad < P.fast_tc) {
            // put_pred (1397-1403): code_inter_mb with a P_Skip decision writes exactly the prediction
            code_inter_mb<T>(C, S.c, mb, &out->res);
            if (lane == 0) out->skip = 1;
            D.mode = 2;
            inter_tail(P, S, D, out);
            if (lane < 16) out->mvds[lane][0] = out->mvds[lane][1] = 0;  // a P_Skip code carries no differences
            return true;
        }
        if (lane == 0) D.mode = 2;
        __syncwarp();
    }
    if (sad < A.skip_thresh) {
        const uint32_t cbp = code_inter_mb<T>(C, S.c, mb, &out->res);
        if (cbp == 0) {
            inter_tail(P, S, D, out);
            if (lane == 0) out->skip = 1;
            return true;
        }
    }
    *sv_out = sv;
    return false;
}

// code_mb for one macroblock without CABAC, enc/frame.rs:715-790: of a P picture, or of an IDR picture
// (P.intra: no P_Skip tests and no best_inter; the Intra4x4 trial always runs, but for flat macroblocks in
// live coding, 762-765). X: the warp pair's meeting words, when the macroblock's intra side runs on the
// pair's second warp (PAIR).
template <class T, bool PAIR = false>
__device__ void decide_mb(const DecideParams& P, DecideSmem<T>& S, const unsigned* i4tab, int mb, int mbx, int mby, PairSync* X = nullptr) {
    const int lane = threadIdx.x & 31;
    const AnalyseParams& A = P.C.A;
    const CodeParams& C = P.C;
    const int lam = A.lambda, x0 = mbx * 16, y0 = mby * 16;
    const bool ta = mby > A.band_start[mby], la = mbx > 0, tra = ta && mbx + 1 < A.mb_w;
    ironav_mbcode* out = &P.codes[mb];
    // the code starts as MbCode::new: zero, Intra4x4 modes 2
    {
        uint32_t* w = reinterpret_cast<uint32_t*>(out);
        for (int k = lane; k < (int)(sizeof(ironav_mbcode) / 4); k += 32) w[k] = (k >= 371 && k < 375) ? 0x02020202u : 0u;
    }
    stage_source(A, S.a);
    __syncwarp();
    ironav_interdec& D = *reinterpret_cast<ironav_interdec*>(S.c.dec);
    int2 sv = make_int2(0, 0);
    if (!P.intra && skip_tests_d<T>(P, S, mb, mbx, mby, out, &sv)) return;
    load_intra_neighbours(P, S, mb, mbx, mby, ta, la, tra);
    int2 i16 = make_int2(2, 0);
    int seq = 0;
    if constexpr (PAIR) {
        if (lane == 0) {
            X->ta = ta;
            X->la = la;
            X->tra = tra;
        }
        seq = pair_command(*X, 1);
    } else {
        i16 = best_i16_d(P, S, ta, la);
    }
    // best_inter, enc/frame.rs:839-849 (none in an IDR picture: nact is 0 there)
    int part = 0, cost = BIG, bestr = 0;
    uint32_t sub = 0;
    for (int r = 0; r < A.nact; r++) {
        const int4 bi = best_inter_or_learned(A, S.a, r);
        if (r == 0 || bi.x < cost) {
            part = bi.y;
            cost = bi.x;
            bestr = r;
            sub = (uint32_t)bi.z;
            if (lane < 16) {
                S.a.win_mvs[lane][0] = S.a.best_mvs[lane][0];
                S.a.win_mvs[lane][1] = S.a.best_mvs[lane][1];
            }
            __syncwarp();
        }
    }
    if constexpr (PAIR) {
        // on a failed wait the launch's error word is set and the host discards the picture
        i16 = pair_wait(A, &X->i16_seq, seq) ? X->i16 : make_int2(2, 1 << 28);
    }
    int best_intra = i16.y + lam * 4;
    // Intra4x4 is tried by coding it when intra is competitive (766-779); in an IDR picture always, but for
    // a flat macroblock in live coding (762-765)
    bool i4 = false;
    if (P.intra ? !(A.fast && i16.y < P.flat_t) : best_intra < cost) {
        int c4;
        if constexpr (PAIR) {
            c4 = pair_wait(A, &X->done_seq, seq) ? X->c4 : (1 << 28);
        } else {
            c4 = code_i4_trial(P, S, i4tab, ta, la, tra);
        }
        c4 += lam * 6;
        if (c4 < best_intra) {
            best_intra = c4;
            i4 = true;
        }
    } else if constexpr (PAIR) {
        // the trial is not the reference's here: stop it, and keep the pair in step
        if (lane == 0) X->stop_seq = seq;
        pair_wait(A, &X->done_seq, seq);
    }
    if (!P.intra && cost <= best_intra) {
        if (lane == 0) {
            D.mode = 2;
            D.part = (uint8_t)part;
            for (int k = 0; k < 4; k++) {
                D.sub[k] = (uint8_t)((sub >> (8 * k)) & 0xff);
                D.refs[k] = (uint8_t)bestr;
            }
        }
        if (lane < 16) {
            D.mvs[lane][0] = S.a.win_mvs[lane][0];
            D.mvs[lane][1] = S.a.win_mvs[lane][1];
        }
        __syncwarp();
        const uint32_t cbp = code_inter_mb<T>(C, S.c, mb, &out->res);
        inter_tail(P, S, D, out);
        if (lane == 0 && cbp == 0 && part == 0 && D.mvs[0][0] == sv.x && D.mvs[0][1] == sv.y && bestr == 0) out->skip = 1;
        return;
    }
    uint32_t cbp;
    if (i4) {
        T* RY = reinterpret_cast<T*>(C.rec[0]);
        for (int i = lane; i < 256; i += 32) RY[(size_t)(y0 + (i >> 4)) * C.ys + x0 + (i & 15)] = (T)S.i4rec[i];
        if (lane < 16) {
            uint32_t* lw = reinterpret_cast<uint32_t*>(out->res.luma[lane]);
            const uint32_t* src = reinterpret_cast<const uint32_t*>(S.i4lv[lane]);
#pragma unroll
            for (int k = 0; k < 8; k++) lw[k] = src[k];
            out->res.nnz[lane] = S.i4nnz[lane];
            out->modes[lane] = S.i4modes[lane];
        }
        const bool coded = lane < 16 && S.i4nnz[lane] > 0;
        const unsigned bal = __ballot_sync(FULL, coded);
        cbp = 0;
#pragma unroll
        for (int i8 = 0; i8 < 4; i8++) {
            const unsigned mask = 0x33u << ((i8 >> 1) * 8 + (i8 & 1) * 2);
            if (bal & mask) cbp |= 1u << i8;
        }
        if (lane == 0) out->kind = KIND_I4;
    } else {
        cbp = code_i16_d(P, S, mbx, mby, i16.x, ta, la, out);
        if (lane == 0) {
            out->kind = KIND_I16;
            out->i16_mode = (uint8_t)i16.x;
        }
    }
    cbp |= code_intra_chroma_d(P, S, mbx, mby, ta, la, out);
    if (lane == 0) out->res.cbp = (uint8_t)cbp;
    // the state of an intra macroblock: no motion
    if (lane < 16) S.a.out.mvs[lane][0] = S.a.out.mvs[lane][1] = 0;
    if (lane == 0) {
        S.a.out.inter = 0;
        for (int k = 0; k < 4; k++) S.a.out.refs[k] = -1;
        S.a.out.pad[0] = S.a.out.pad[1] = S.a.out.pad[2] = 0;
    }
    __syncwarp();
}

// One macroblock of decide mode: waits for its left and top-right (top at the right edge) neighbours,
// decides and codes it, and publishes it. Returns false when a wait gave up (the launch is abandoned).
template <class T, bool PAIR = false>
__device__ bool decide_one(const DecideParams& P, DecideSmem<T>& S, const unsigned* i4tab, int mb, PairSync* X = nullptr) {
    const int lane = threadIdx.x & 31;
    const AnalyseParams& A = P.C.A;
    const int mbx = mb % A.mb_w, mby = mb / A.mb_w;
    if (lane == 0) {
        S.a.mb = mb;
        S.a.mbx = mbx;
        S.a.mby = mby;
    }
    __syncwarp();
    // their own waits cover the other neighbours
    const int start = A.band_start[mby];
    bool ok = true;
    if (mbx > 0) ok = wait_published(A, mb - 1);
    if (ok && mby > start) ok = wait_published(A, (mbx + 1 < A.mb_w) ? mb - A.mb_w + 1 : mb - A.mb_w);
    if (!__all_sync(FULL, ok)) return false;
    load_neighbours(A, S.a, A.states_out);
    decide_mb<T, PAIR>(P, S, i4tab, mb, mbx, mby, X);
    if (lane < 18) reinterpret_cast<uint32_t*>(&A.states_out[mb])[lane] = reinterpret_cast<const uint32_t*>(&S.a.out)[lane];
    // the reconstruction, code and state before the flag
    __threadfence();
    __syncwarp();
    if (lane == 0 && mb != A.withhold) st_release(&A.flags[mb], A.epoch);
    return true;
}

// The Intra4x4 predictor table of a CTA (i4_entry per mode and sample; rows padded against bank conflicts).
__device__ __forceinline__ void fill_i4tab(unsigned* tab) {
    for (int t = threadIdx.x; t < 9 * 16; t += blockDim.x) tab[(t >> 4) * 17 + (t & 15)] = i4_entry(t >> 4, t & 3, (t >> 2) & 3);
    __syncthreads();
}

// Decide mode for one stream on warp pairs: the first warp of a pair takes the tickets and decides, the
// second works out the intra side of the first's macroblock (PairSync). One stream's wavefront keeps far
// fewer macroblocks in flight than the launch has pairs, so the second warps shorten each macroblock's
// latency at no cost in concurrency.
template <class T>
__global__ void __launch_bounds__(K7_WARPS * 32, K7_MIN_BLOCKS) decide_kernel(const __grid_constant__ DecideParams P) {
    __shared__ DecideSmem<T> smem[K7_WARPS / 2];
    __shared__ PairSync sync[K7_WARPS / 2];
    __shared__ unsigned i4tab[9 * 17];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    PairSync& X = sync[w >> 1];
    if ((w & 1) == 0 && lane == 0) {
        X.cmd_seq = X.cmd = X.stop_seq = X.i16_seq = X.done_seq = 0;
        X.seq = 0;
    }
    fill_i4tab(i4tab);  // its __syncthreads also publishes the words above
    DecideSmem<T>& S = smem[w >> 1];
    if (w & 1) {
        pair_helper<T>(P, S, X, i4tab);
        return;
    }
    const AnalyseParams& A = P.C.A;
    for (;;) {
        unsigned t = 0;
        if (lane == 0) t = atomicAdd(A.ticket, 1u);
        t = __shfl_sync(FULL, t, 0);
        if (t >= (unsigned)A.nmb) break;
        if (!decide_one<T, true>(P, S, i4tab, A.order[t], &X)) break;
    }
    pair_command(X, -1);
}

// Decide mode for many streams in one launch: ticket t is order[t] = stream << 20 | macroblock, in the
// streams' merged wavefront order (the batched form's); each stream's parameters in table[stream], copied
// into the warp's shared memory when the warp moves to another stream.
template <class T>
__global__ void __launch_bounds__(K7_WARPS * 32, K7_MIN_BLOCKS) decide_batch_kernel(const DecideParams* __restrict__ table,
                                                                                  const uint32_t* __restrict__ order, unsigned ntickets,
                                                                                  unsigned* ticket, const unsigned* err) {
    __shared__ DecideSmem<T> smem[K7_WARPS];
    __shared__ DecideParams prm[K7_WARPS];
    __shared__ unsigned i4tab[9 * 17];
    fill_i4tab(i4tab);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    DecideSmem<T>& S = smem[wid];
    int cur = -1;
    for (;;) {
        unsigned t = 0;
        if (lane == 0) t = atomicAdd(ticket, 1u);
        t = __shfl_sync(FULL, t, 0);
        if (t >= ntickets || ld_acquire(err) != 0) break;
        const uint32_t e = order[t];
        const int stream = (int)(e >> 20);
        if (stream != cur) {
            const uint32_t* src = reinterpret_cast<const uint32_t*>(&table[stream]);
            uint32_t* dst = reinterpret_cast<uint32_t*>(&prm[wid]);
            for (int k = lane; k < (int)(sizeof(DecideParams) / 4); k += 32) dst[k] = src[k];
            __syncwarp();
            cur = stream;
        }
        if (!decide_one<T>(prm[wid], S, i4tab, (int)(e & 0xFFFFFu))) break;
    }
}

// finish_mb's MbInfo for the deblocking filter (enc/frame.rs:2323-2339), a thread per macroblock: slice id
// band + 1 (enc/mod.rs:608), inter or not, QP_Y, t8x8 and the luma counts of the code; an inter
// macroblock's list-0 reference per 8x8 block, its identity (1 + index) and vectors from its state.
static __global__ void dbk_records_kernel(const ironav_mbcode* __restrict__ codes, const ironav_mbstate* __restrict__ states,
                                          const int* __restrict__ band_start, int mb_w, int nmb, int qp, ironav_dbk_mb* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nmb) return;
    const int row = i / mb_w;
    // the band of the row: rows where a band starts, counted up to it
    int band = 0;
    for (int r = 1; r <= row; r++) band += band_start[r] == r;
    const ironav_mbcode& k = codes[i];
    const ironav_mbstate& st = states[i];
    ironav_dbk_mb m;
    m.slice = (uint16_t)(band + 1);
    m.inter = k.kind == KIND_INTER;
    m.qp = (int8_t)qp;
    m.t8x8 = k.res.t8x8;
    m.keep = 0;
    m.pad[0] = m.pad[1] = 0;
    for (int b = 0; b < 16; b++) m.nnz[b] = k.res.nnz[b];
    for (int b = 0; b < 4; b++) {
        m.ref_idx[0][b] = m.inter ? st.refs[b] : (int8_t)-1;
        m.ref_id[0][b] = m.inter ? 1 + st.refs[b] : -1;
        m.ref_idx[1][b] = -1;
        m.ref_id[1][b] = -1;
    }
    for (int b = 0; b < 16; b++) {
        m.mv[0][b][0] = m.inter ? st.mvs[b][0] : (int16_t)0;
        m.mv[0][b][1] = m.inter ? st.mvs[b][1] : (int16_t)0;
        m.mv[1][b][0] = m.mv[1][b][1] = 0;
    }
    out[i] = m;
}

// Fills decide mode's parameters for the context's current picture (host side, ironav_inter.cu): the
// coding and the analysis parameters, the outputs; the caller sets the wavefront's fields (order, ticket,
// flags, epoch, err). Returns IRONAV_INVALID_ARGUMENT when the picture is not ready for decide mode.
int fill_decide_params(ironav_ctx* c, DecideParams& p, ironav_mbstate* d_states, ironav_mbcode* d_codes, void* y, int ys, void* cb, void* cr,
                       int cs);

}  // namespace ironav
