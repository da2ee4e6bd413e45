// residual.cuh — K6: the coding of inter macroblocks once decided (code_inter / code_inter_residual /
// code_luma8 / code_chroma, enc/frame.rs:1202-1305, 1856-1915): prediction, transform, quantisation,
// decimation and reconstruction, one warp per macroblock (every inter macroblock is independent).
//
// Lanes: the luma prediction takes a lane per 4x4 block (K2's pred4 with the partition's clamps), the
// chroma prediction 4 samples a lane (eighth-sample bilinear with clamped coordinates, chroma_mc
// h264/inter.rs:549-568). The 4x4 transform path takes a lane per 4x4 block (fdct4, quantisation, the
// decimation score, the 8x8 sums by shuffles, inverse transform and the reconstruction's 4x4); the 8x8 path
// takes 8 lanes per 8x8 block, a row then a column each, transposed through shared memory; chroma takes a
// lane per 4x4 block of Cb and Cr, the 2x2 DC transform by shuffles among a component's 4 lanes. Levels
// pass through shared memory across the shuffles (no 16-entry array live there), which holds the kernel
// to 128 registers: 4 blocks (16 warps) an SM.
#pragma once
#include "analyse.cuh"
#include "deblock.cuh"

namespace ironav {

struct CodeParams {
    AnalyseParams A;                  // planes (A.planes[r]: reference r's half-sample planes), sizes, source luma
    const uint8_t* ref_c[MAX_REFS];   // reference r's chroma: Cb then Cr, each cw x ch samples
    const uint8_t* src_c;             // the source's chroma: Cb then Cr, each cw x ch samples
    int cw, ch;                       // chroma plane size (8 * mb_w, 8 * mb_h)
    const ironav_interdec* decs;
    ironav_intercode* codes;
    uint8_t* rec[3];                  // reconstruction planes (byte addresses)
    int ys, cs;                       // their row strides in samples
    int qp;                           // QP_Y
    int bd;
    int nrefs;                        // references held (each with its chroma)
    unsigned* err;                    // 4: a decision names a reference, partitioning or sub-partitioning out of range
};

// enc/frame.rs:20-21, 33-40; h264/tables.rs:4278 (DEQUANT8_COEFF_INIT), h264/ps.rs:12 (ZIGZAG4),
// h264/tables.rs:4291 (ZIGZAG_DIRECT)
static __device__ __constant__ int c_q_mf[6][3] = {{13107, 5243, 8066}, {11916, 4660, 7490}, {10082, 4194, 6554},
                                                   {9362, 3647, 5825},  {8192, 3355, 5243}, {7282, 2893, 4559}};
static __device__ __constant__ int c_q_v[6][3] = {{10, 16, 13}, {11, 18, 14}, {13, 20, 16}, {14, 23, 18}, {16, 25, 20}, {18, 29, 23}};
static __device__ __constant__ int c_q_mf8[6][6] = {{13107, 11428, 20972, 12222, 16777, 15481}, {11916, 10826, 19174, 11058, 14980, 14290},
                                                    {10082, 8943, 15978, 9675, 12710, 11985},   {9362, 8228, 14913, 8931, 11984, 11259},
                                                    {8192, 7346, 13159, 7740, 10486, 9777},     {7282, 6428, 11570, 6830, 9118, 8640}};
static __device__ __constant__ int c_q_dq8[6][6] = {{20, 18, 32, 19, 25, 24}, {22, 19, 35, 21, 28, 26}, {26, 23, 42, 24, 33, 31},
                                                    {28, 25, 45, 26, 35, 33}, {32, 28, 51, 30, 40, 38}, {36, 32, 58, 34, 46, 43}};
// ZIGZAG4 as nibbles (entry k in bits 4k..4k+3): folds to a constant in an unrolled loop, so the
// coefficient arrays it indexes stay in registers
__device__ __forceinline__ constexpr int zz4_at(int k) { return (int)((0xFEB7ADC963258410ull >> (4 * k)) & 15); }
static __device__ __constant__ uint8_t c_zz8[64] = {0,  1,  8,  16, 9,  2,  3,  10, 17, 24, 32, 25, 18, 11, 4,  5,
                                                    12, 19, 26, 33, 40, 48, 41, 34, 27, 20, 13, 6,  7,  14, 21, 28,
                                                    35, 42, 49, 56, 57, 50, 43, 36, 29, 22, 15, 23, 30, 37, 44, 51,
                                                    58, 59, 52, 45, 38, 31, 39, 46, 53, 60, 61, 54, 47, 55, 62, 63};

__device__ __forceinline__ int q_class_d(int i) { return ((i & 1) == 0 && ((i >> 2) & 1) == 0) ? 0 : (((i & 1) && ((i >> 2) & 1)) ? 1 : 2); }
__device__ __forceinline__ int q_class8_d(int p) {
    const int i = p >> 3, j = p & 7;
    if ((i & 3) == 0 && (j & 3) == 0) return 0;
    if ((i & 1) && (j & 1)) return 1;
    if ((i & 3) == 2 && (j & 3) == 2) return 2;
    if (((i & 3) == 0 && (j & 1)) || ((i & 1) && (j & 3) == 0)) return 3;
    if (((i & 3) == 0 && (j & 3) == 2) || ((i & 3) == 2 && (j & 3) == 0)) return 4;
    return 5;
}
// quant, enc/frame.rs:134-141
__device__ __forceinline__ int q_quant_d(int c, int mf, int f, int qbits) {
    const int a = (int)(((long long)abs(c) * mf + f) >> qbits);
    return c < 0 ? -a : a;
}
// fdct4, enc/frame.rs:113-132
__device__ __forceinline__ void q_fdct4_d(const int (&d)[16], int (&o)[16]) {
    int t[16];
#pragma unroll
    for (int r = 0; r < 4; r++) {
        const int s03 = d[r * 4] + d[r * 4 + 3], d03 = d[r * 4] - d[r * 4 + 3], s12 = d[r * 4 + 1] + d[r * 4 + 2], d12 = d[r * 4 + 1] - d[r * 4 + 2];
        t[r * 4] = s03 + s12;
        t[r * 4 + 1] = 2 * d03 + d12;
        t[r * 4 + 2] = s03 - s12;
        t[r * 4 + 3] = d03 - 2 * d12;
    }
#pragma unroll
    for (int c = 0; c < 4; c++) {
        const int s03 = t[c] + t[12 + c], d03 = t[c] - t[12 + c], s12 = t[4 + c] + t[8 + c], d12 = t[4 + c] - t[8 + c];
        o[c] = s03 + s12;
        o[4 + c] = 2 * d03 + d12;
        o[8 + c] = s03 - s12;
        o[12 + c] = d03 - 2 * d12;
    }
}
// fdct8_1d, enc/frame.rs:46-54
__device__ __forceinline__ void q_fdct8_1d_d(const int (&d)[8], int (&o)[8]) {
    const int s07 = d[0] + d[7], s16 = d[1] + d[6], s25 = d[2] + d[5], s34 = d[3] + d[4];
    const int a0 = s07 + s34, a1 = s16 + s25, a2 = s07 - s34, a3 = s16 - s25;
    const int d07 = d[0] - d[7], d16 = d[1] - d[6], d25 = d[2] - d[5], d34 = d[3] - d[4];
    const int a4 = d16 + d25 + (d07 + (d07 >> 1));
    const int a5 = d07 - d34 - (d25 + (d25 >> 1));
    const int a6 = d07 + d34 - (d16 + (d16 >> 1));
    const int a7 = d16 - d25 + (d34 + (d34 >> 1));
    o[0] = a0 + a1;
    o[1] = a4 + (a7 >> 2);
    o[2] = a2 + (a3 >> 1);
    o[3] = a5 + (a6 >> 2);
    o[4] = a0 - a1;
    o[5] = a6 - (a5 >> 2);
    o[6] = (a2 >> 1) - a3;
    o[7] = (a4 >> 2) - a7;
}
// the inverse 8-point transform of h264/idct.rs:34-52 (two's-complement wrapping like the reference's)
__device__ __forceinline__ void q_row8_d(const int (&d)[8], int (&o)[8]) {
    const int a0 = d[0] + d[4], a4 = d[0] - d[4], a2 = (d[2] >> 1) - d[6], a6 = d[2] + (d[6] >> 1);
    const int b0 = a0 + a6, b2 = a4 + a2, b4 = a4 - a2, b6 = a0 - a6;
    const int a1 = d[5] - d[3] - d[7] - (d[7] >> 1);
    const int a3 = d[1] + d[7] - d[3] - (d[3] >> 1);
    const int a5 = d[7] - d[1] + d[5] + (d[5] >> 1);
    const int a7 = d[3] + d[5] + d[1] + (d[1] >> 1);
    const int b1 = a1 + (a7 >> 2), b7 = a7 - (a1 >> 2), b3 = a3 + (a5 >> 2), b5 = (a3 >> 2) - a5;
    o[0] = b0 + b7;
    o[1] = b2 + b5;
    o[2] = b4 + b3;
    o[3] = b6 + b1;
    o[4] = b6 - b1;
    o[5] = b4 - b3;
    o[6] = b2 - b5;
    o[7] = b0 - b7;
}
// idct4_add, h264/idct.rs:8-31, of raster coefficients c onto the prediction rows p (4 x 4), into out
__device__ __forceinline__ void q_idct4_d(const int (&c)[16], const int (&p)[16], int maxv, int (&out)[16]) {
    int t[16];
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int e0 = c[i * 4] + c[i * 4 + 2], e1 = c[i * 4] - c[i * 4 + 2];
        const int e2 = (c[i * 4 + 1] >> 1) - c[i * 4 + 3], e3 = c[i * 4 + 1] + (c[i * 4 + 3] >> 1);
        t[i * 4] = e0 + e3;
        t[i * 4 + 1] = e1 + e2;
        t[i * 4 + 2] = e1 - e2;
        t[i * 4 + 3] = e0 - e3;
    }
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const int g0 = t[j] + t[8 + j], g1 = t[j] - t[8 + j], g2 = (t[4 + j] >> 1) - t[12 + j], g3 = t[4 + j] + (t[12 + j] >> 1);
        const int h[4] = {g0 + g3, g1 + g2, g1 - g2, g0 - g3};
#pragma unroll
        for (int i = 0; i < 4; i++) out[i * 4 + j] = min(max(p[i * 4 + j] + ((h[i] + 32) >> 6), 0), maxv);
    }
}
// decimate_score over n levels in scan order (enc/frame.rs:2369-2440)
__device__ __forceinline__ int q_decimate_d(const int16_t* lv, int n) {
    int score = 0, i = n - 1;
    while (i >= 0 && lv[i] == 0) i--;
    while (i >= 0) {
        if (abs(lv[i]) > 1) return 9;
        i--;
        int run = 0;
        while (i >= 0 && lv[i] == 0) {
            i--;
            run++;
        }
        if (n == 16) score += run == 0 ? 3 : (run <= 2 ? 2 : (run <= 5 ? 1 : 0));
        else score += run <= 3 ? 3 : (run <= 11 ? 2 : (run <= 23 ? 1 : 0));
    }
    return score;
}

// Per-warp shared memory of the coding kernel.
struct CodeSmem {
    int pred[256];             // luma prediction, raster
    int cpred[2][64];          // chroma prediction
    int t8[4][8][9];           // 8x8 transform rows, transposed (padded)
    int co8[4][64];            // 8x8 dequantised coefficients (raster)
    int16_t lv8[4][64];        // 8x8 levels (scan order)
    int16_t lv4[16][16];       // 4x4 levels (scan order), luma
    int16_t cl[2][4][16];      // chroma AC levels
    uint16_t dec[40];          // the decision record (78 bytes)
};

// The rectangle (in 4x4 blocks) of rects(part, sub) holding 4x4 block (bx, by), its position in coding
// order and its reference index slot (rects / ref_of, enc/frame.rs:208-223).
__device__ __forceinline__ int4 rect_of(int part, const uint8_t* sub, int bx, int by, int* n_out, int* rslot) {
    if (part == 0) {
        *n_out = 0;
        *rslot = 0;
        return make_int4(0, 0, 4, 4);
    }
    if (part == 1) {
        *n_out = by >> 1;
        *rslot = by >> 1;
        return make_int4(0, (by >> 1) * 2, 4, 2);
    }
    if (part == 2) {
        *n_out = bx >> 1;
        *rslot = bx >> 1;
        return make_int4((bx >> 1) * 2, 0, 2, 4);
    }
    const int k = (by >> 1) * 2 + (bx >> 1), ox = (k & 1) * 2, oy = (k >> 1) * 2, lx = bx & 1, ly = by & 1;
    int n = 0;
    for (int q = 0; q < k; q++) n += sub[q] == 0 ? 1 : (sub[q] == 3 ? 4 : 2);
    const int s = sub[k];
    *rslot = k;
    if (s == 0) {
        *n_out = n;
        return make_int4(ox, oy, 2, 2);
    }
    if (s == 1) {
        *n_out = n + ly;
        return make_int4(ox, oy + ly, 2, 1);
    }
    if (s == 2) {
        *n_out = n + lx;
        return make_int4(ox + lx, oy, 1, 2);
    }
    *n_out = n + ly * 2 + lx;
    return make_int4(ox + lx, oy + ly, 1, 1);
}

// code_chroma, enc/frame.rs:1856-1915: both chroma components of the macroblock at (mbx, mby) against the
// prediction in S.cpred, into `out` and the reconstruction, a lane per 4x4 block of Cb (lanes 0-3) and Cr
// (4-7); the AC levels go to shared memory and come back after the DC transform's shuffles. intra: the
// intra rounding (f = 1/3) and no AC decimation. Returns the chroma part of the coded block pattern
// (bits 4-5), on every lane.
template <class T>
__device__ __forceinline__ uint32_t code_chroma_mb(const CodeParams& P, CodeSmem& S, int mbx, int mby, ironav_intercode* out, bool intra) {
    const int lane = threadIdx.x & 31;
    const int maxv = (1 << P.bd) - 1;
    int dc = 0, cscore = 0, anyac = 0;
    const int qpc = dbk_chroma_qp(P.qp, 0, P.bd) + 6 * (P.bd - 8), mc = qpc % 6;
    const int cc = (lane >> 2) & 1, blk = lane & 3, cbx = blk & 1, cby = blk >> 1;
    const T* SC = reinterpret_cast<const T*>(P.src_c) + (size_t)cc * P.cw * P.ch;
    if (lane < 8) {
        int d[16], c[16];
#pragma unroll
        for (int r = 0; r < 4; r++)
#pragma unroll
            for (int k = 0; k < 4; k++)
                d[r * 4 + k] = (int)SC[(size_t)(mby * 8 + cby * 4 + r) * P.cw + mbx * 8 + cbx * 4 + k] - S.cpred[cc][(cby * 4 + r) * 8 + cbx * 4 + k];
        q_fdct4_d(d, c);
        const int qbits = 15 + qpc / 6, f = (1 << qbits) / (intra ? 3 : 6);
#pragma unroll
        for (int k = 0; k < 16; k++) {
            const int pz = zz4_at(k);
            const int l = pz != 0 ? q_quant_d(c[pz], c_q_mf[mc][q_class_d(pz)], f, qbits) : 0;
            S.cl[cc][blk][k] = (int16_t)l;
            anyac |= l != 0;
        }
        dc = c[0];
        cscore = q_decimate_d(S.cl[cc][blk], 16);
    }
    // the DC transform over a component's 4 blocks (lanes 4cc..4cc+3)
    const int base = (lane & 4);
    const int d0 = __shfl_sync(FULL, dc, base), d1 = __shfl_sync(FULL, dc, base + 1), d2 = __shfl_sync(FULL, dc, base + 2),
              d3 = __shfl_sync(FULL, dc, base + 3);
    const int fdc = blk == 0 ? d0 + d1 + d2 + d3 : (blk == 1 ? d0 - d1 + d2 - d3 : (blk == 2 ? d0 + d1 - d2 - d3 : d0 - d1 - d2 + d3));
    const int qbits = 16 + qpc / 6, fr = (1 << qbits) / (intra ? 3 : 6);
    const int cdc = lane < 8 ? q_quant_d(fdc, c_q_mf[mc][0], fr, qbits) : 0;
    int acs = lane < 8 ? cscore : 0;
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) acs += __shfl_xor_sync(FULL, acs, off);
    const bool any_ac = (__ballot_sync(FULL, lane < 8 && anyac) != 0) && (intra || acs >= 7);
    const bool any_dc = __ballot_sync(FULL, lane < 8 && cdc != 0) != 0;
    const int cbpc = any_ac ? 2 : (any_dc ? 1 : 0);
    // the reconstruction: the DC levels' inverse 2x2 transform scaled, the AC as coded
    const int l0 = __shfl_sync(FULL, cdc, base), l1 = __shfl_sync(FULL, cdc, base + 1), l2 = __shfl_sync(FULL, cdc, base + 2),
              l3 = __shfl_sync(FULL, cdc, base + 3);
    const int fl = blk == 0 ? l0 + l1 + l2 + l3 : (blk == 1 ? l0 - l1 + l2 - l3 : (blk == 2 ? l0 + l1 - l2 - l3 : l0 - l1 - l2 + l3));
    if (lane < 8) {
        ironav_intercode& O = *out;
        const int sh = qpc / 6;
        int cco[16], cp[16], nz = 0, any = 0;
        uint32_t packed[8];
#pragma unroll
        for (int k = 0; k < 16; k++) {
            const int pz = zz4_at(k);
            const int l = any_ac ? S.cl[cc][blk][k] : 0;
            nz += l != 0;
            cco[pz] = (l * c_q_v[mc][q_class_d(pz)]) << sh;
            if (k & 1) packed[k >> 1] |= (uint32_t)(l & 0xffff) << 16;
            else packed[k >> 1] = (uint32_t)(l & 0xffff);
        }
        cco[0] = cbpc > 0 ? ((fl * (16 * c_q_v[mc][0])) << sh) >> 5 : 0;
#pragma unroll
        for (int k = 0; k < 16; k++) any |= cco[k];
        uint32_t* aw = reinterpret_cast<uint32_t*>(O.cac[cc][blk]);
#pragma unroll
        for (int k = 0; k < 8; k++) aw[k] = packed[k];
        O.cnnz[cc][blk] = (uint8_t)nz;
        O.cdc[cc][blk] = (int16_t)cdc;
#pragma unroll
        for (int r = 0; r < 4; r++)
#pragma unroll
            for (int k = 0; k < 4; k++) cp[r * 4 + k] = S.cpred[cc][(cby * 4 + r) * 8 + cbx * 4 + k];
        int recb[16];
        if (any) {
            q_idct4_d(cco, cp, maxv, recb);
        } else {
#pragma unroll
            for (int k = 0; k < 16; k++) recb[k] = cp[k];
        }
        T* RC = reinterpret_cast<T*>(P.rec[1 + cc]);
#pragma unroll
        for (int r = 0; r < 4; r++)
#pragma unroll
            for (int k = 0; k < 4; k++) RC[(size_t)(mby * 8 + cby * 4 + r) * P.cs + mbx * 8 + cbx * 4 + k] = (T)recb[r * 4 + k];
    }
    return (uint32_t)cbpc << 4;
}

// code_inter / code_inter_residual / code_luma8, enc/frame.rs:1202-1305: the macroblock whose decision
// (mode 1 P_Skip or 2 coded, validated) is in S.dec, into `out` (zeroed by the caller) and the
// reconstruction. Returns the coded block pattern, on every lane.
template <class T>
__device__ __forceinline__ uint32_t code_inter_mb(const CodeParams& P, CodeSmem& S, int mb, ironav_intercode* out) {
    const int lane = threadIdx.x & 31;
    const int maxv = (1 << P.bd) - 1;
    const int qp = P.qp + 6 * (P.bd - 8);
    const int mbx = mb % P.A.mb_w, mby = mb / P.A.mb_w, x0 = mbx * 16, y0 = mby * 16;
    const ironav_interdec& D = *reinterpret_cast<const ironav_interdec*>(S.dec);
    const int mode = D.mode;
    // luma prediction, a lane per 4x4 block
    if (lane < 16) {
        const int bx = lane & 3, by = lane >> 2;
        int n, rs;
        const int4 r = rect_of(D.part, D.sub, bx, by, &n, &rs);
        const int2 mv = make_int2(D.mvs[n][0], D.mvs[n][1]);
        uint32_t pr[4][sizeof(T)];
        pred4<T>(P.A, P.A.planes[D.refs[rs]], x0 + r.x * 4, y0 + r.y * 4, r.z * 4, r.w * 4, bx - r.x, by - r.y, mv, pr);
#pragma unroll
        for (int row = 0; row < 4; row++)
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const uint32_t wv = pr[row][(k * (int)sizeof(T)) >> 2];
                S.pred[(by * 4 + row) * 16 + bx * 4 + k] = (int)((wv >> ((k * 8 * (int)sizeof(T)) & 31)) & (uint32_t)maxv);
            }
    }
    // chroma prediction (chroma_mc from each partition's vector, in eighth samples), 4 samples a lane
    for (int i = lane; i < 128; i += 32) {
        const int cc = i >> 6, cy = (i >> 3) & 7, cx = i & 7;
        int n, rs;
        const int4 r = rect_of(D.part, D.sub, cx >> 1, cy >> 1, &n, &rs);
        (void)r;
        const int mx = D.mvs[n][0], my = D.mvs[n][1];
        const T* rc = reinterpret_cast<const T*>(P.ref_c[D.refs[rs]]) + (size_t)cc * P.cw * P.ch;
        const int fx = mx & 7, fy = my & 7;
        const int xs = mbx * 8 + cx + (mx >> 3), ysm = mby * 8 + cy + (my >> 3);
        const int xa = min(max(xs, 0), P.cw - 1), xb = min(max(xs + 1, 0), P.cw - 1);
        const int ya = min(max(ysm, 0), P.ch - 1), yb = min(max(ysm + 1, 0), P.ch - 1);
        const int A_ = rc[(size_t)ya * P.cw + xa], B_ = rc[(size_t)ya * P.cw + xb], C_ = rc[(size_t)yb * P.cw + xa], D_ = rc[(size_t)yb * P.cw + xb];
        S.cpred[cc][cy * 8 + cx] = ((8 - fx) * (8 - fy) * A_ + fx * (8 - fy) * B_ + (8 - fx) * fy * C_ + fx * fy * D_ + 32) >> 6;
    }
    __syncwarp();
    T* const RY = reinterpret_cast<T*>(P.rec[0]);
    const T* const SY = reinterpret_cast<const T*>(P.A.src);
    uint32_t cbp = 0;
    if (mode == 1) {
        // P_Skip: the prediction is the reconstruction
        for (int i = lane; i < 256; i += 32) RY[(size_t)(y0 + (i >> 4)) * P.ys + x0 + (i & 15)] = (T)S.pred[i];
    } else if (!D.t8) {
        // 4x4 transform: a lane per block; the levels go to shared memory and come back after the
        // decimation sums, so that no 16-entry array stays live across the shuffles
        int score = 0;
        const int bx = lane & 3, by = lane >> 2;
        if (lane < 16) {
            int d[16], c[16];
#pragma unroll
            for (int r = 0; r < 4; r++)
#pragma unroll
                for (int k = 0; k < 4; k++)
                    d[r * 4 + k] = (int)SY[(size_t)(y0 + by * 4 + r) * P.A.ls + x0 + bx * 4 + k] - S.pred[(by * 4 + r) * 16 + bx * 4 + k];
            q_fdct4_d(d, c);
            const int qbits = 15 + qp / 6, f = (1 << qbits) / 6, m = qp % 6;
#pragma unroll
            for (int k = 0; k < 16; k++) {
                const int pz = zz4_at(k);
                S.lv4[lane][k] = (int16_t)q_quant_d(c[pz], c_q_mf[m][q_class_d(pz)], f, qbits);
            }
            score = q_decimate_d(S.lv4[lane], 16);
        }
        // per 8x8 block: lanes (2i8x, 2i8y) quad sums; blocks b = by*4+bx, 8x8 index (by/2)*2 + bx/2
        const int i8 = ((lane >> 3) & 1) * 2 + ((lane & 3) >> 1);
        int s8 = 0, tot = 0;
#pragma unroll
        for (int q = 0; q < 4; q++) {
            int sq = 0;
#pragma unroll
            for (int b = 0; b < 16; b++) {
                const int v = __shfl_sync(FULL, score, b);
                if (((b >> 3) & 1) * 2 + ((b & 3) >> 1) == q) sq += v;
            }
            if (q == i8) s8 = sq;
            tot += sq;
        }
        if (lane < 16) {
            const bool drop = s8 < 4 || tot < 6;
            const int m = qp % 6, sh = qp / 6;
            int co[16], p[16], nz = 0;
            uint32_t packed[8];
#pragma unroll
            for (int k = 0; k < 16; k++) {
                const int pz = zz4_at(k);
                const int l = drop ? 0 : S.lv4[lane][k];
                nz += l != 0;
                co[pz] = (l * c_q_v[m][q_class_d(pz)]) << sh;
                if (k & 1) packed[k >> 1] |= (uint32_t)(l & 0xffff) << 16;
                else packed[k >> 1] = (uint32_t)(l & 0xffff);
            }
#pragma unroll
            for (int r = 0; r < 4; r++)
#pragma unroll
                for (int k = 0; k < 4; k++) p[r * 4 + k] = S.pred[(by * 4 + r) * 16 + bx * 4 + k];
            int recb[16];
            if (nz > 0) {
                q_idct4_d(co, p, maxv, recb);
            } else {
#pragma unroll
                for (int k = 0; k < 16; k++) recb[k] = p[k];
            }
#pragma unroll
            for (int r = 0; r < 4; r++)
#pragma unroll
                for (int k = 0; k < 4; k++) RY[(size_t)(y0 + by * 4 + r) * P.ys + x0 + bx * 4 + k] = (T)recb[r * 4 + k];
            ironav_intercode& O = *out;
            uint32_t* lw = reinterpret_cast<uint32_t*>(O.luma[lane]);
#pragma unroll
            for (int k = 0; k < 8; k++) lw[k] = packed[k];
            O.nnz[lane] = (uint8_t)nz;
            if (nz > 0) cbp |= 1u << ((by >> 1) * 2 + (bx >> 1));
        }
    } else {
        // 8x8 transform: 8 lanes per 8x8 block, a row then a column each
        const int b8 = lane >> 3, j = lane & 7, bx8 = (b8 & 1) * 8, by8 = (b8 >> 1) * 8;
        {
            int d[8], o[8];
#pragma unroll
            for (int k = 0; k < 8; k++)
                d[k] = (int)SY[(size_t)(y0 + by8 + j) * P.A.ls + x0 + bx8 + k] - S.pred[(by8 + j) * 16 + bx8 + k];
            q_fdct8_1d_d(d, o);
#pragma unroll
            for (int k = 0; k < 8; k++) S.t8[b8][j][k] = o[k];
        }
        __syncwarp();
        {
            int d[8], o[8];
#pragma unroll
            for (int k = 0; k < 8; k++) d[k] = S.t8[b8][k][j];
            q_fdct8_1d_d(d, o);
            __syncwarp();
#pragma unroll
            for (int k = 0; k < 8; k++) S.co8[b8][k * 8 + j] = o[k];  // raster (row k, column j)
        }
        __syncwarp();
        // quantise 8 scan positions a lane (quant8, enc/frame.rs:56-72)
        {
            const int m = qp % 6, qbits = 16 + qp / 6, f = (1 << qbits) / 6;
            int dq[8];
#pragma unroll
            for (int k = 0; k < 8; k++) {
                const int sk = j * 8 + k, pz = c_zz8[sk];
                const int l = q_quant_d(S.co8[b8][pz], c_q_mf8[m][q_class8_d(pz)], f, qbits);
                S.lv8[b8][sk] = (int16_t)l;
                int v = 0;
                if (l != 0) {
                    const int vv = l * 16 * c_q_dq8[m][q_class8_d(pz)];
                    v = qp >= 36 ? vv << (qp / 6 - 6) : (vv + (1 << (5 - qp / 6))) >> (6 - qp / 6);
                }
                dq[k] = v;
            }
            __syncwarp();
#pragma unroll
            for (int k = 0; k < 8; k++) S.co8[b8][c_zz8[j * 8 + k]] = dq[k];
        }
        __syncwarp();
        int score = 0;
        if (j == 0) score = q_decimate_d(S.lv8[b8], 64);
        score = __shfl_sync(FULL, score, b8 * 8);
        const int tot = __shfl_sync(FULL, score, 0) + __shfl_sync(FULL, score, 8) + __shfl_sync(FULL, score, 16) + __shfl_sync(FULL, score, 24);
        const bool drop = score < 4 || tot < 6;
        int nz = 0;
#pragma unroll
        for (int k = 0; k < 8; k++) nz += S.lv8[b8][j * 8 + k] != 0;
#pragma unroll
        for (int off = 1; off < 8; off <<= 1) nz += __shfl_xor_sync(FULL, nz, off);
        if (drop) nz = 0;
        // the reconstruction: rows of the inverse transform, then its columns onto the prediction
        const bool idct = !drop && nz > 0;
        if (idct) {
            int d[8], o[8];
#pragma unroll
            for (int k = 0; k < 8; k++) d[k] = S.co8[b8][j * 8 + k];
            q_row8_d(d, o);
#pragma unroll
            for (int k = 0; k < 8; k++) S.t8[b8][j][k] = o[k];
        }
        __syncwarp();
        {
            int o[8];
            if (idct) {
                int d[8];
#pragma unroll
                for (int k = 0; k < 8; k++) d[k] = S.t8[b8][k][j];
                q_row8_d(d, o);
            }
#pragma unroll
            for (int i = 0; i < 8; i++) {
                const int pv = S.pred[(by8 + i) * 16 + bx8 + j];
                RY[(size_t)(y0 + by8 + i) * P.ys + x0 + bx8 + j] = (T)(idct ? min(max(pv + ((o[i] + 32) >> 6), 0), maxv) : pv);
            }
        }
        ironav_intercode& O = *out;
        if (!drop) {
#pragma unroll
            for (int k = 0; k < 8; k++) O.luma8[b8][j * 8 + k] = S.lv8[b8][j * 8 + k];
        }
        if (j < 4 && !drop) O.nnz[((b8 >> 1) * 2 + (j >> 1)) * 4 + (b8 & 1) * 2 + (j & 1)] = (uint8_t)nz;
        if (j == 0 && nz > 0) cbp |= 1u << b8;
    }
    // the luma part of the coded block pattern, from every lane
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) cbp |= __shfl_xor_sync(FULL, cbp, off);
    // the luma part of the coded block pattern, from every lane
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) cbp |= __shfl_xor_sync(FULL, cbp, off);
    if (mode == 2) {
        cbp |= code_chroma_mb<T>(P, S, mbx, mby, out, false);
    } else {
        // P_Skip: the chroma prediction is the reconstruction
        for (int i = lane; i < 128; i += 32) {
            T* RC = reinterpret_cast<T*>(P.rec[1 + (i >> 6)]);
            RC[(size_t)(mby * 8 + ((i >> 3) & 7)) * P.cs + mbx * 8 + (i & 7)] = (T)S.cpred[i >> 6][i & 63];
        }
    }
    if (lane == 0 && mode == 2) {
        out->cbp = (uint8_t)cbp;
        out->t8x8 = (uint8_t)(D.t8 && (cbp & 15) != 0);
    }
    __syncwarp();
    return cbp;
}

template <class T>
__global__ void __launch_bounds__(128, 4) code_inter_kernel(const __grid_constant__ CodeParams P) {
    __shared__ CodeSmem smem[4];
    CodeSmem& S = smem[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const int nmb = P.A.mb_w * P.A.mb_h;
    for (int mb = blockIdx.x * 4 + (threadIdx.x >> 5); mb < nmb; mb += gridDim.x * 4) {
        // the decision (78 bytes: 2-byte aligned)
        const uint16_t* dp = reinterpret_cast<const uint16_t*>(reinterpret_cast<const uint8_t*>(P.decs) + (size_t)mb * sizeof(ironav_interdec));
        for (int k = lane; k < 39; k += 32) S.dec[k] = dp[k];
        __syncwarp();
        const ironav_interdec& D = *reinterpret_cast<const ironav_interdec*>(S.dec);
        const int mode = D.mode;
        // the output record starts from zero (and stays so for a macroblock that is not inter)
        uint32_t* outw = reinterpret_cast<uint32_t*>(&P.codes[mb]);
        for (int k = lane; k < (int)(sizeof(ironav_intercode) / 4); k += 32) outw[k] = 0;
        if (mode == 0) continue;
        // a decision that would read outside the tables: the macroblock is left alone, the call reports it
        bool bad = mode > 2 || D.part > 3;
        for (int k = 0; k < 4; k++) bad |= D.refs[k] >= P.nrefs || (D.part == 3 && D.sub[k] > 3);
        if (bad) {
            if (lane == 0) atomicOr(P.err, 4u);
            continue;
        }
        code_inter_mb<T>(P, S, mb, &P.codes[mb]);
    }
}

}  // namespace ironav
