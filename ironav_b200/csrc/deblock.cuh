// deblock.cuh — K4: the in-loop deblocking filter of a reconstructed picture (h264/deblock.rs), frame
// pictures, 4:2:0, 8-bit (uint8_t) or 10-bit (uint16_t) samples.
//
// The reference filters macroblocks in raster order (deblock_picture, deblock.rs:410-429); filtering a
// macroblock changes up to 3 samples on either side of its left and top edges, so macroblock (x, y) must
// see the final samples of (x - 1, y) and of (x + 1, y - 1) — the dependency deblock_picture_par keeps with
// its row wavefront (deblock.rs:583-605). Here one warp filters one macroblock row left to right, rows
// handed out by ticket, and before macroblock x it waits (bounded) until the row above has filtered
// macroblocks 0..x+1. Inside a macroblock the lanes take lines: 16 luma lines, 8 Cb and 8 Cr lines
// (rows for the vertical edges, then columns for the horizontal edges), on a staged tile of the
// macroblock with the 4 (luma) / 2 (chroma) samples left of and above it in shared memory. Samples shared
// between warps move through L2 only (ld.global.cg / st.global.cg) and are published with a release store
// of the row's progress.
#pragma once
#include "common.cuh"

namespace ironav {

constexpr int DBK_WARPS = 4;
constexpr unsigned DBK_ALL = 0xffffffffu;

// alpha' / beta' by indexA / indexB, tC0 by (indexA, bS 1..3) — Tables 8-16 and 8-17 of the standard as
// h264/tables.rs holds them — and the chroma QP for qPi >= 30 (h264/mb.rs:211).
static __device__ __constant__ uint8_t c_dbk_alpha[52] = {
    0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 4, 4, 5, 6, 7, 8, 9, 10, 12, 13,
    15, 17, 20, 22, 25, 28, 32, 36, 40, 45, 50, 56, 63, 71, 80, 90, 101, 113, 127, 144, 162, 182, 203, 226, 255, 255};
static __device__ __constant__ uint8_t c_dbk_beta[52] = {0, 0, 0, 0, 0, 0, 0, 0, 0,  0,  0,  0,  0,  0,  0,  0,  2,  2,
                                                        2, 3, 3, 3, 3, 4, 4, 4, 6,  6,  7,  7,  8,  8,  9,  9,  10, 10,
                                                        11, 11, 12, 12, 13, 13, 14, 14, 15, 15, 16, 16, 17, 17, 18, 18};
static __device__ __constant__ uint8_t c_dbk_tc0[52][3] = {
    {0, 0, 0},  {0, 0, 0},   {0, 0, 0},   {0, 0, 0},   {0, 0, 0},    {0, 0, 0},    {0, 0, 0},    {0, 0, 0},    {0, 0, 0},
    {0, 0, 0},  {0, 0, 0},   {0, 0, 0},   {0, 0, 0},   {0, 0, 0},    {0, 0, 0},    {0, 0, 0},    {0, 0, 0},    {0, 0, 1},
    {0, 0, 1},  {0, 0, 1},   {0, 0, 1},   {0, 1, 1},   {0, 1, 1},    {1, 1, 1},    {1, 1, 1},    {1, 1, 1},    {1, 1, 1},
    {1, 1, 2},  {1, 1, 2},   {1, 1, 2},   {1, 1, 2},   {1, 2, 3},    {1, 2, 3},    {2, 2, 3},    {2, 2, 4},    {2, 3, 4},
    {2, 3, 4},  {3, 3, 5},   {3, 4, 6},   {3, 4, 6},   {4, 5, 7},    {4, 5, 8},    {4, 6, 9},    {5, 7, 10},   {6, 8, 11},
    {6, 8, 13}, {7, 10, 14}, {8, 11, 16}, {9, 12, 18}, {10, 13, 20}, {11, 15, 23}, {13, 17, 25}};
static __device__ __constant__ uint8_t c_dbk_cqp[22] = {29, 30, 31, 32, 32, 33, 34, 34, 35, 35, 36,
                                                       36, 37, 37, 37, 38, 38, 38, 39, 39, 39, 39};

// One deblocking launch.
struct DbkParams {
    uint8_t* planes[3];               // Y, Cb, Cr (byte addresses; samples of the launch's type)
    int ys, cs;                       // row strides in samples
    const ironav_dbk_mb* mbs;
    const ironav_dbk_slice* slices;
    int nslices, mb_w, mb_h, bd;
    unsigned* progress;               // per macroblock row, luma then chroma: macroblocks done (zeroed before the launch)
    unsigned* ticket;                 // next row
    unsigned* err;                    // 1: a wait gave up; 4: a slice id beyond the table
    unsigned wait_limit;              // polls before a wait gives up
};


// chroma_qp, h264/mb.rs:214-221
__device__ __forceinline__ int dbk_chroma_qp(int qp, int off, int bd) {
    const int qpi = min(max(qp + off, -6 * (bd - 8)), 51);
    return qpi < 30 ? qpi : (int)c_dbk_cqp[qpi - 30];
}

// coded, deblock.rs:336-345
__device__ __forceinline__ bool dbk_coded(const ironav_dbk_mb& m, int bx, int by) {
    if (m.t8x8) {
        const int x0 = bx & 2, y0 = by & 2;
        return (m.nnz[y0 * 4 + x0] | m.nnz[y0 * 4 + x0 + 1] | m.nnz[(y0 + 1) * 4 + x0] | m.nnz[(y0 + 1) * 4 + x0 + 1]) != 0;
    }
    return m.nnz[by * 4 + bx] != 0;
}

// far, deblock.rs:347-350
__device__ __forceinline__ bool dbk_far(const int16_t* a, const int16_t* b) { return abs(a[0] - b[0]) >= 4 || abs(a[1] - b[1]) >= 4; }

// motion_differs, deblock.rs:352-383 (frame macroblocks: the vertical limit is 4 quarter samples)
static __device__ bool dbk_motion_differs(const ironav_dbk_mb& p, int pbx, int pby, const ironav_dbk_mb& q, int qbx, int qby) {
    const int pi = pby * 4 + pbx, qi = qby * 4 + qbx;
    const int p8 = (pby >> 1) * 2 + (pbx >> 1), q8 = (qby >> 1) * 2 + (qbx >> 1);
    const int pr0 = p.ref_id[0][p8], pr1 = p.ref_id[1][p8], qr0 = q.ref_id[0][q8], qr1 = q.ref_id[1][q8];
    const int16_t *pm0 = p.mv[0][pi], *pm1 = p.mv[1][pi], *qm0 = q.mv[0][qi], *qm1 = q.mv[1][qi];
    const int np = (pr0 >= 0) + (pr1 >= 0), nq = (qr0 >= 0) + (qr1 >= 0);
    if (np != nq) return true;
    if (np == 1) {
        const bool lp = pr0 < 0, lq = qr0 < 0;
        return (lp ? pr1 : pr0) != (lq ? qr1 : qr0) || dbk_far(lp ? pm1 : pm0, lq ? qm1 : qm0);
    }
    if (!((pr0 == qr0 && pr1 == qr1) || (pr0 == qr1 && pr1 == qr0))) return true;
    if (pr0 != pr1) {
        if (pr0 == qr0) return dbk_far(pm0, qm0) || dbk_far(pm1, qm1);
        return dbk_far(pm0, qm1) || dbk_far(pm1, qm0);
    }
    return (dbk_far(pm0, qm0) || dbk_far(pm1, qm1)) && (dbk_far(pm0, qm1) || dbk_far(pm1, qm0));
}

// filter_line, deblock.rs:279-333, on the staged line whose first sample past the edge is q[0] (step xs
// across the edge); the side of a keep macroblock (I_PCM / lossless) is left as it was (filter_edge,
// deblock.rs:251-272).
__device__ __forceinline__ void dbk_line(int* q, int xs, int b, int tc0, int alpha, int beta, bool chroma, int maxv, bool keep_p,
                                         bool keep_q) {
    const int p0 = q[-xs], q0 = q[0], p1 = q[-2 * xs], q1 = q[xs];
    if (abs(p0 - q0) >= alpha || abs(p1 - p0) >= beta || abs(q1 - q0) >= beta) return;
    if (chroma) {
        int np0, nq0;
        if (b < 4) {
            const int tc = tc0 + 1;
            const int delta = min(max((((q0 - p0) << 2) + (p1 - q1) + 4) >> 3, -tc), tc);
            np0 = min(max(p0 + delta, 0), maxv);
            nq0 = min(max(q0 - delta, 0), maxv);
        } else {
            np0 = (2 * p1 + p0 + q1 + 2) >> 2;
            nq0 = (2 * q1 + q0 + p1 + 2) >> 2;
        }
        if (!keep_p) q[-xs] = np0;
        if (!keep_q) q[0] = nq0;
        return;
    }
    const int p2 = q[-3 * xs], q2 = q[2 * xs];
    const int ap = abs(p2 - p0), aq = abs(q2 - q0);
    int np0 = p0, np1 = p1, np2 = p2, nq0 = q0, nq1 = q1, nq2 = q2;
    if (b < 4) {
        const int tc = tc0 + (ap < beta) + (aq < beta);
        const int delta = min(max((((q0 - p0) << 2) + (p1 - q1) + 4) >> 3, -tc), tc);
        np0 = min(max(p0 + delta, 0), maxv);
        nq0 = min(max(q0 - delta, 0), maxv);
        if (ap < beta) np1 = p1 + min(max((p2 + ((p0 + q0 + 1) >> 1) - (p1 << 1)) >> 1, -tc0), tc0);
        if (aq < beta) nq1 = q1 + min(max((q2 + ((p0 + q0 + 1) >> 1) - (q1 << 1)) >> 1, -tc0), tc0);
    } else {
        const bool small = abs(p0 - q0) < (alpha >> 2) + 2;
        if (ap < beta && small) {
            const int p3 = q[-4 * xs];
            np0 = (p2 + 2 * p1 + 2 * p0 + 2 * q0 + q1 + 4) >> 3;
            np1 = (p2 + p1 + p0 + q0 + 2) >> 2;
            np2 = (2 * p3 + 3 * p2 + p1 + p0 + q0 + 4) >> 3;
        } else {
            np0 = (2 * p1 + p0 + q1 + 2) >> 2;
        }
        if (aq < beta && small) {
            const int q3 = q[3 * xs];
            nq0 = (p1 + 2 * p0 + 2 * q0 + 2 * q1 + q2 + 4) >> 3;
            nq1 = (p0 + q0 + q1 + q2 + 2) >> 2;
            nq2 = (2 * q3 + 3 * q2 + q1 + q0 + p0 + 4) >> 3;
        } else {
            nq0 = (2 * q1 + q0 + p1 + 2) >> 2;
        }
    }
    if (!keep_p) {
        q[-xs] = np0;
        q[-2 * xs] = np1;
        q[-3 * xs] = np2;
    }
    if (!keep_q) {
        q[0] = nq0;
        q[xs] = nq1;
        q[2 * xs] = nq2;
    }
}

// The thresholds of one edge (deblock.rs:647-651, 680-683), packed alpha' | beta' << 8 | tC0(bS 1, 2, 3)
// << 13, 18, 23 (all before the bit-depth shift; beta' <= 18 and tC0 <= 25 fit 5 bits); 0 when alpha' or
// beta' is 0 (filter_edge leaves the edge alone, deblock.rs:233-235).
__device__ __forceinline__ uint32_t dbk_thresholds(int qpav, const ironav_dbk_slice& sp) {
    const int ia = min(max(qpav + sp.alpha_offset, 0), 51), ib = min(max(qpav + sp.beta_offset, 0), 51);
    const uint32_t a = c_dbk_alpha[ia], b = c_dbk_beta[ib];
    if (a == 0 || b == 0) return 0u;
    return a | b << 8 | (uint32_t)c_dbk_tc0[ia][0] << 13 | (uint32_t)c_dbk_tc0[ia][1] << 18 | (uint32_t)c_dbk_tc0[ia][2] << 23;
}

// What the filter of one macroblock needs besides its samples, worked out before the wavefront (it depends
// on the macroblock records only). An edge word is its thresholds (dbk_thresholds) | keep << 28 (bit 0:
// the p side is a keep macroblock, bit 1: the q side); 0 means the edge is not filtered at all.
struct DbkEdges {
    uint8_t bs[2][4][4];        // [dir][edge][segment]
    uint32_t luma[2][4];        // [dir][edge]
    uint32_t chroma[2][2][2];   // [comp][dir][edge / 2]
};
static_assert(sizeof(DbkEdges) == 96, "DbkEdges layout");

// Pass 1: the boundary strengths (strength, deblock.rs:391-408) and edge words of every macroblock
// (deblock_mb's decisions, deblock.rs:608-695), one warp per macroblock, all macroblocks independent.
// One macroblock's boundary strengths and edge words (pass 1): R holds 3 records of shared memory (the
// macroblock, its left and its top neighbour), Bs the strengths [dir][edge][segment].
__device__ __forceinline__ void dbk_edges_mb(const DbkParams& P, DbkEdges* __restrict__ out, int idx, ironav_dbk_mb* R,
                                             uint8_t (*Bs)[4][4]) {
    const int lane = threadIdx.x & 31;
    const int x = idx % P.mb_w, y = idx / P.mb_w;
    for (int k = lane; k < 3 * 48; k += 32) {
        const int which = k / 48, wd = k % 48;
        const int src = which == 0 ? idx : (which == 1 ? (x > 0 ? idx - 1 : idx) : (y > 0 ? idx - P.mb_w : idx));
        reinterpret_cast<uint32_t*>(&R[which])[wd] = __ldg(reinterpret_cast<const uint32_t*>(&P.mbs[src]) + wd);
    }
    __syncwarp();
    const ironav_dbk_mb& m = R[0];
    // the neighbours across the left and top edges; at the picture's edges the macroblock itself, whose
    // outer edges are then not filtered (deblock.rs:618-621)
    const ironav_dbk_mb& lm = R[1];
    const ironav_dbk_mb& tm = R[2];
    bool live = m.slice != 0;
    if (live && m.slice > P.nslices) {
        if (lane == 0) atomicOr(P.err, 4u);
        live = false;
    }
    ironav_dbk_slice sp = {};
    if (live) sp = P.slices[m.slice - 1];
    live = live && sp.disable_deblocking != 1;
    const bool left_ok = x > 0 && lm.slice != 0 && (sp.disable_deblocking == 0 || lm.slice == m.slice);
    const bool top_ok = y > 0 && tm.slice != 0 && (sp.disable_deblocking == 0 || tm.slice == m.slice);
    // inner edges of an inter macroblock moving as a whole with no coefficients are not filtered
    // (uniform_motion, deblock.rs:385-389, and deblock.rs:625)
    bool same = true;
    if (lane < 16) {
        same = m.nnz[lane] == 0 && m.mv[0][lane][0] == m.mv[0][0][0] && m.mv[0][lane][1] == m.mv[0][0][1] &&
               m.mv[1][lane][0] == m.mv[1][0][0] && m.mv[1][lane][1] == m.mv[1][0][1];
        if (lane < 4)
            same = same && m.ref_idx[0][lane] == m.ref_idx[0][0] && m.ref_idx[1][lane] == m.ref_idx[1][0] &&
                   m.ref_id[0][lane] == m.ref_id[0][0] && m.ref_id[1][lane] == m.ref_id[1][0];
    }
    const bool still = m.inter && __all_sync(DBK_ALL, same);
    // boundary strengths: lane = dir * 16 + edge * 4 + segment
    {
        const int dir = lane >> 4, e = (lane >> 2) & 3, i = lane & 3;
        const ironav_dbk_mb& o = e == 0 ? (dir == 0 ? lm : tm) : m;
        int b = 0;
        if (!(e > 0 && still)) {
            if (!m.inter || !o.inter) {
                b = e == 0 ? 4 : 3;
            } else {
                const int qx = dir == 0 ? e : i, qy = dir == 0 ? i : e;
                const int px = dir == 0 ? (e == 0 ? 3 : e - 1) : i, py = dir == 0 ? i : (e == 0 ? 3 : e - 1);
                b = (dbk_coded(m, qx, qy) || dbk_coded(o, px, py)) ? 2 : (dbk_motion_differs(o, px, py, m, qx, qy) ? 1 : 0);
            }
        }
        Bs[dir][e][i] = (uint8_t)b;
    }
    __syncwarp();
    DbkEdges& E = out[idx];
    if (lane < 8) reinterpret_cast<uint32_t*>(E.bs)[lane] = reinterpret_cast<const uint32_t*>(Bs)[lane];
    // edge words: lanes 0-7 luma (dir, edge), lanes 8-15 chroma (comp, dir, edge / 2)
    if (lane < 16) {
        const bool chroma = lane >= 8;
        const int dir = chroma ? ((lane - 8) >> 1) & 1 : lane >> 2;
        const int e = chroma ? ((lane - 8) & 1) * 2 : lane & 3;
        const int comp = (lane - 8) >> 2;
        const ironav_dbk_mb& o = e == 0 ? (dir == 0 ? lm : tm) : m;
        const bool any = *reinterpret_cast<const uint32_t*>(Bs[dir][e]) != 0;
        uint32_t wv = 0;
        if (live && any && !(e == 0 && !(dir == 0 ? left_ok : top_ok)) && !(!chroma && m.t8x8 && (e & 1))) {
            if (chroma) {
                const int off = sp.chroma_qp_offset[comp];
                wv = dbk_thresholds((dbk_chroma_qp(o.qp, off, P.bd) + dbk_chroma_qp(m.qp, off, P.bd) + 1) >> 1, sp);
            } else {
                wv = dbk_thresholds((o.qp + m.qp + 1) >> 1, sp);
            }
            if (wv) wv |= (uint32_t)((o.keep ? 1 : 0) | (m.keep ? 2 : 0)) << 28;
        }
        if (chroma) E.chroma[comp][dir][e >> 1] = wv;
        else E.luma[dir][e] = wv;
    }
    __syncwarp();
}

static __global__ void __launch_bounds__(DBK_WARPS * 32) deblock_edges_kernel(const __grid_constant__ DbkParams P, DbkEdges* __restrict__ out) {
    __shared__ ironav_dbk_mb rec[DBK_WARPS][3];
    __shared__ uint8_t bsm[DBK_WARPS][2][4][4];
    const int wid = threadIdx.x >> 5;
    const int nmb = P.mb_w * P.mb_h;
    for (int idx = blockIdx.x * DBK_WARPS + wid; idx < nmb; idx += gridDim.x * DBK_WARPS) dbk_edges_mb(P, out, idx, rec[wid], bsm[wid]);
}

// ---- pass 2: the samples, in the row wavefront ---------------------------------------------------------

// N samples of type T at p (aligned to their size, at most 16 bytes) into ints, through L2; and back.
template <class T, int N>
__device__ __forceinline__ void dbk_load(const T* p, int* v) {
    constexpr int NB = N * (int)sizeof(T);
    uint32_t w[NB >= 4 ? NB / 4 : 1];
    if constexpr (NB == 16) {
        const uint4 q = __ldcg(reinterpret_cast<const uint4*>(p));
        w[0] = q.x, w[1] = q.y, w[2] = q.z, w[3] = q.w;
    } else if constexpr (NB == 8) {
        const uint2 q = __ldcg(reinterpret_cast<const uint2*>(p));
        w[0] = q.x, w[1] = q.y;
    } else if constexpr (NB == 4) {
        w[0] = __ldcg(reinterpret_cast<const unsigned*>(p));
    } else {
        w[0] = __ldcg(reinterpret_cast<const unsigned short*>(p));
    }
#pragma unroll
    for (int k = 0; k < N; k++) v[k] = (int)((w[(k * (int)sizeof(T)) >> 2] >> ((k * 8 * (int)sizeof(T)) & 31)) & ((1u << (8 * sizeof(T))) - 1));
}
template <class T, int N>
__device__ __forceinline__ void dbk_store(T* p, const int* v) {
    constexpr int NB = N * (int)sizeof(T);
    uint32_t w[NB >= 4 ? NB / 4 : 1] = {};
#pragma unroll
    for (int k = 0; k < N; k++) w[(k * (int)sizeof(T)) >> 2] |= (uint32_t)v[k] << ((k * 8 * (int)sizeof(T)) & 31);
    if constexpr (NB == 16) __stcg(reinterpret_cast<uint4*>(p), make_uint4(w[0], w[1], w[2], w[3]));
    else if constexpr (NB == 8) __stcg(reinterpret_cast<uint2*>(p), make_uint2(w[0], w[1]));
    else if constexpr (NB == 4) __stcg(reinterpret_cast<unsigned*>(p), w[0]);
    else __stcg(reinterpret_cast<unsigned short*>(p), (unsigned short)w[0]);
}
// Up to 16 samples (two 16-byte pieces for 16 samples of 16 bits).
template <class T, int N>
__device__ __forceinline__ void dbk_load_row(const T* p, int* v) {
    if constexpr (N * sizeof(T) > 16) {
        dbk_load<T, N / 2>(p, v);
        dbk_load<T, N / 2>(p + N / 2, v + N / 2);
    } else {
        dbk_load<T, N>(p, v);
    }
}
template <class T, int N>
__device__ __forceinline__ void dbk_store_row(T* p, const int* v) {
    if constexpr (N * sizeof(T) > 16) {
        dbk_store<T, N / 2>(p, v);
        dbk_store<T, N / 2>(p + N / 2, v + N / 2);
    } else {
        dbk_store<T, N>(p, v);
    }
}

// Filters the edges across one line of NS samples (luma: 20 = 4 before the macroblock + 16; chroma: 10 =
// 2 + 8) in registers: luma edges at 4, 8, 12, 16; chroma edges at 2 and 6.
template <bool CHROMA, int NS>
__device__ __forceinline__ void dbk_filter_lines(int (&v)[NS], const uint32_t* words, const uint8_t (*bs)[4], int seg, int bd, int maxv) {
#pragma unroll
    for (int k = 0; k < (CHROMA ? 2 : 4); k++) {
        const uint32_t wv = words[k];
        const int e = CHROMA ? 2 * k : k;
        const int b = bs[e][seg];
        if (wv == 0 || b == 0) continue;
        const int alpha = (int)(wv & 0xff) << (bd - 8), beta = (int)((wv >> 8) & 0x1f) << (bd - 8);
        const int tc0 = b < 4 ? (int)((wv >> (8 + 5 * b)) & 0x1f) << (bd - 8) : 0;
        dbk_line(&v[CHROMA ? 2 + 4 * k : 4 + 4 * k], 1, b, tc0, alpha, beta, CHROMA, maxv, (wv >> 28) & 1, (wv >> 29) & 1);
    }
}

__device__ __forceinline__ unsigned ld_relaxed(const unsigned* p) {
    unsigned v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Waits until progress word `w` reaches `need`, at most P.wait_limit polls; false when it gave up or
// another warp already did (the error word is looked at every 64 polls). Relaxed polls, then one acquire
// fence: with the writer's release store they order the writer's samples before this warp's loads.
__device__ __forceinline__ bool dbk_wait(const DbkParams& P, const unsigned* w, unsigned need) {
    for (unsigned i = 0;; i++) {
        if (ld_relaxed(w) >= need) {
            asm volatile("fence.acq_rel.gpu;" ::: "memory");
            return true;
        }
        if ((i & 63) == 63) {
            if (ld_acquire(P.err) & 1u) return false;
            if (i >= P.wait_limit) {
                atomicOr(P.err, 1u);
                return false;
            }
        }
        if (i >= 16) __nanosleep(64);
    }
}

// Pass 2 for one macroblock row of one plane kind, left to right, by one warp. Luma: lanes 0-15 hold the
// macroblock's 16 rows (each with the 4 samples to its left); chroma: lanes 0-7 the Cb rows, 8-15 the Cr
// rows (each with 2 to the left); lanes 16-31 idle. The vertical edges are filtered in those registers,
// the horizontal ones on columns read back from a shared-memory tile that also holds the rows above (4
// luma / 2 chroma). The next macroblock's own samples and edge words are loaded while the current one
// waits and filters. The vertical edges come first and need nothing from the row above; they make the
// previous macroblock final (its last columns are the left edge's p side), so the warp stores those columns
// and publishes progress x + 1 (macroblocks 0..x-1 final) before it waits for the row above, loads the rows
// above and filters the horizontal edges.
template <class T, bool CHROMA>
__device__ __forceinline__ void dbk_row(const DbkParams& P, const DbkEdges* __restrict__ edges, int y, int (*L)[17],
                                        DbkEdges& E) {
    constexpr int W = CHROMA ? 8 : 16;   // samples of a macroblock row
    constexpr int LEFT = CHROMA ? 2 : 4; // samples kept to its left
    constexpr int H = CHROMA ? 2 : 4;    // rows above
    const int lane = threadIdx.x & 31;
    const bool active = lane < 16;
    const int comp = CHROMA ? lane >> 3 : 0, line = CHROMA ? lane & 7 : lane;
    T* const Pl = reinterpret_cast<T*>(P.planes[CHROMA ? 1 + comp : 0]);
    const int stride = CHROMA ? P.cs : P.ys;
    // the tile: luma rows y0-4..y0+15 in L[0..19]; chroma comp c rows yc-2..yc+7 in L[10c .. 10c+9]
    int (*Tl)[17] = CHROMA ? L + 10 * comp : L;
    const size_t lrow = (size_t)(y * (CHROMA ? 8 : 16) + line) * stride;
    const unsigned* above = P.progress + (CHROMA ? P.mb_h : 0) + (y - 1);
    unsigned* mine = P.progress + (CHROMA ? P.mb_h : 0) + y;
    const int maxv = (1 << P.bd) - 1;
    int lv[LEFT + W];
    int own[W];
    uint32_t ew = 0;
    auto prefetch = [&](int x) {
        if (active) dbk_load_row<T, W>(Pl + lrow + x * W, own);
        if (lane < 24) ew = __ldg(reinterpret_cast<const uint32_t*>(&edges[(size_t)y * P.mb_w + x]) + lane);
    };
    prefetch(0);
    for (int x = 0; x < P.mb_w; x++) {
        if (active) {
#pragma unroll
            for (int k = 0; k < W; k++) lv[LEFT + k] = own[k];
        }
        if (lane < 24) reinterpret_cast<uint32_t*>(&E)[lane] = ew;
        __syncwarp();
        // vertical edges, in registers: they touch this row of macroblocks only, so they need nothing
        // from the row above
        if (active) {
            const uint32_t* words = CHROMA ? E.chroma[comp][0] : E.luma[0];
            dbk_filter_lines<CHROMA, LEFT + W>(lv, words, E.bs[0], CHROMA ? line >> 1 : line >> 2, P.bd, maxv);
            // the previous macroblock's last columns are final now: store them and publish it
            if (x > 0) dbk_store<T, LEFT>(Pl + lrow + x * W - LEFT, lv);
        }
        __syncwarp();
        if (lane == 0) st_release(mine, (unsigned)(x + 1));  // the warp's stores, ordered by the barrier above
        // the next macroblock's samples and edge words (after the fence, which would wait for them)
        if (x + 1 < P.mb_w) prefetch(x + 1);
        // macroblocks 0..x+1 of the row above final (its last two macroblocks: the whole row, whose final
        // publish is mb_w + 1)
        const unsigned need = x + 2 < P.mb_w ? (unsigned)(x + 2) : (unsigned)P.mb_w + 1;
        if (y > 0 && !__all_sync(DBK_ALL, dbk_wait(P, above, need))) return;
        // the rows above, one lane each
        if (y > 0 && lane < 4) {
            const int cc = CHROMA ? lane >> 1 : 0, rr = CHROMA ? lane & 1 : lane;
            const T* src = reinterpret_cast<const T*>(P.planes[CHROMA ? 1 + cc : 0]) + (size_t)(y * (CHROMA ? 8 : 16) - H + rr) * stride + x * W;
            int r[W];
            dbk_load_row<T, W>(src, r);
            int (*dst)[17] = CHROMA ? L + 10 * cc : L;
#pragma unroll
            for (int k = 0; k < W; k++) dst[rr][k] = r[k];
        }
        if (active) {
#pragma unroll
            for (int k = 0; k < W; k++) Tl[H + line][k] = lv[LEFT + k];
        }
        __syncwarp();
        if (active) {
            // horizontal edges, a lane per column of the tile
            int cv[H + W];
#pragma unroll
            for (int k = 0; k < H + W; k++) cv[k] = Tl[k][line];
            const uint32_t* words = CHROMA ? E.chroma[comp][1] : E.luma[1];
            dbk_filter_lines<CHROMA, H + W>(cv, words, E.bs[1], CHROMA ? line >> 1 : line >> 2, P.bd, maxv);
#pragma unroll
            for (int k = 1; k < H + W; k++) Tl[k][line] = cv[k];
        }
        __syncwarp();
        if (active) {
#pragma unroll
            for (int k = 0; k < W; k++) lv[LEFT + k] = Tl[H + line][k];
            dbk_store_row<T, W>(Pl + lrow + x * W, &lv[LEFT]);
            if (y > 0 && line >= 1 && line < H) {
                int r[W];
#pragma unroll
                for (int k = 0; k < W; k++) r[k] = Tl[line][k];
                dbk_store_row<T, W>(Pl + (size_t)(y * (CHROMA ? 8 : 16) - H + line) * stride + x * W, r);
            }
            // this macroblock's last columns are the next one's left samples
#pragma unroll
            for (int k = 0; k < LEFT; k++) lv[k] = lv[W + k];
        }
        __syncwarp();
    }
    // the last macroblock's own rows were stored after the last publish: publish them too
    __syncwarp();
    if (lane == 0) st_release(mine, (unsigned)P.mb_w + 1);
}

// Pass 2: macroblock rows of the two plane kinds handed out by ticket (2y: luma row y, 2y + 1: chroma row y);
// a row waits only on the row above of its own kind, which holds a smaller ticket.
template <class T>
__global__ void __launch_bounds__(DBK_WARPS * 32) deblock_rows_kernel(const __grid_constant__ DbkParams P,
                                                                      const DbkEdges* __restrict__ edges) {
    __shared__ int Ls[DBK_WARPS][20][17];
    __shared__ DbkEdges Es[DBK_WARPS];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (;;) {
        unsigned t = 0;
        if (lane == 0) t = atomicAdd(P.ticket, 1u);
        t = __shfl_sync(DBK_ALL, t, 0);
        if (t >= 2u * (unsigned)P.mb_h) return;
        if (t & 1u) dbk_row<T, true>(P, edges, (int)(t >> 1), Ls[wid], Es[wid]);
        else dbk_row<T, false>(P, edges, (int)(t >> 1), Ls[wid], Es[wid]);
        if (ld_acquire(P.err) & 1u) return;
    }
}

// ---- many streams in one launch per pass (the batched form) ------------------------------------------

// One stream of a batched deblocking launch: its parameters (planes, records, slices, progress words, the
// batch's ticket and error words), its edge records, and its first macroblock in the launch's flat index.
struct DbkJob {
    DbkParams P;
    DbkEdges* edges;
    int mb0;
};

// Pass 1 for every stream: the flat macroblock index over the streams (stream by binary search on mb0).
static __global__ void __launch_bounds__(DBK_WARPS * 32) deblock_edges_batch_kernel(const DbkJob* __restrict__ jobs, int njobs, int total) {
    __shared__ ironav_dbk_mb rec[DBK_WARPS][3];
    __shared__ uint8_t bsm[DBK_WARPS][2][4][4];
    const int wid = threadIdx.x >> 5;
    for (int idx = blockIdx.x * DBK_WARPS + wid; idx < total; idx += gridDim.x * DBK_WARPS) {
        int lo = 0, hi = njobs - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (jobs[mid].mb0 <= idx) lo = mid;
            else hi = mid - 1;
        }
        const DbkJob& J = jobs[lo];
        dbk_edges_mb(J.P, J.edges, idx - J.mb0, rec[wid], bsm[wid]);
    }
}

// Pass 2 for every stream: ticket t is order[t] = stream << 20 | the stream's own row ticket (2y luma row y,
// 2y + 1 chroma row y), the streams' rows interleaved by their own tickets, so a row waits only on its own
// stream's row above, which holds a smaller ticket.
template <class T>
__global__ void __launch_bounds__(DBK_WARPS * 32) deblock_rows_batch_kernel(const DbkJob* __restrict__ jobs,
                                                                                   const uint32_t* __restrict__ order, unsigned ntickets,
                                                                                   unsigned* ticket, const unsigned* err) {
    __shared__ int Ls[DBK_WARPS][20][17];
    __shared__ DbkEdges Es[DBK_WARPS];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (;;) {
        unsigned t = 0;
        if (lane == 0) t = atomicAdd(ticket, 1u);
        t = __shfl_sync(DBK_ALL, t, 0);
        if (t >= ntickets) return;
        const uint32_t e = order[t];
        const DbkJob& J = jobs[e >> 20];
        const unsigned lt = e & 0xFFFFFu;
        if (lt & 1u) dbk_row<T, true>(J.P, J.edges, (int)(lt >> 1), Ls[wid], Es[wid]);
        else dbk_row<T, false>(J.P, J.edges, (int)(lt >> 1), Ls[wid], Es[wid]);
        if (ld_acquire(err) & 1u) return;
    }
}

}  // namespace ironav
