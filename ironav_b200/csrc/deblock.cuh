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
    unsigned* progress;               // per macroblock row: macroblocks filtered (zeroed before the launch)
    unsigned* ticket;                 // next row
    unsigned* err;                    // 1: a wait gave up; 4: a slice id beyond the table
    unsigned wait_limit;              // polls before a wait gives up
};

// Per-warp shared memory.
struct DbkWarp {
    int L[20][21];                    // luma rows y0-4..y0+15 (index +4), columns x0-4..x0+15 (index +4); odd stride
    int C[2][10][11];                 // Cb, Cr rows yc-2..yc+7, columns xc-2..xc+7
    ironav_dbk_mb mb[3];              // the macroblock, its left and its top neighbour
    uint8_t bs[2][4][4];              // boundary strengths [dir][edge][segment]
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
__device__ bool dbk_motion_differs(const ironav_dbk_mb& p, int pbx, int pby, const ironav_dbk_mb& q, int qbx, int qby) {
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

// The thresholds of one edge (deblock.rs:647-651, 680-683): alpha, beta, and indexA in .z; alpha == 0
// or beta == 0 means the edge is left alone (filter_edge, deblock.rs:233-235).
__device__ __forceinline__ int3 dbk_thresholds(int qpav, const ironav_dbk_slice& sp, int bd) {
    const int ia = min(max(qpav + sp.alpha_offset, 0), 51), ib = min(max(qpav + sp.beta_offset, 0), 51);
    return make_int3((int)c_dbk_alpha[ia] << (bd - 8), (int)c_dbk_beta[ib] << (bd - 8), ia);
}

// deblock_mb, deblock.rs:608-695, for macroblock (x, y) of a 4:2:0 frame picture, by one warp.
template <class T>
__device__ void dbk_mb(const DbkParams& __restrict__ P, DbkWarp& __restrict__ W, int x, int y) {
    const int lane = threadIdx.x & 31;
    const int idx = y * P.mb_w + x;
    // the three macroblock records (48 words each)
    for (int k = lane; k < 3 * 48; k += 32) {
        const int which = k / 48, wd = k % 48;
        const int src = which == 0 ? idx : (which == 1 ? (x > 0 ? idx - 1 : idx) : (y > 0 ? idx - P.mb_w : idx));
        reinterpret_cast<uint32_t*>(&W.mb[which])[wd] = __ldg(reinterpret_cast<const uint32_t*>(&P.mbs[src]) + wd);
    }
    __syncwarp();
    const ironav_dbk_mb& m = W.mb[0];
    if (m.slice == 0) return;
    if (m.slice > P.nslices) {
        if (lane == 0) atomicOr(P.err, 4u);
        return;
    }
    const ironav_dbk_slice sp = P.slices[m.slice - 1];
    if (sp.disable_deblocking == 1) return;
    // the neighbours across the left and top edges; at the picture's edges the macroblock itself, whose
    // outer edges are then not filtered (deblock.rs:618-621)
    const ironav_dbk_mb& lm = W.mb[1];
    const ironav_dbk_mb& tm = W.mb[2];
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
    // boundary strengths (strength, deblock.rs:391-408): lane = dir * 16 + edge * 4 + segment
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
        W.bs[dir][e][i] = (uint8_t)b;
    }
    // stage the macroblock's samples with 4 (luma) / 2 (chroma) samples to the left and above
    const T* Y = reinterpret_cast<const T*>(P.planes[0]);
    const int x0 = x * 16, y0 = y * 16, xc = x * 8, yc = y * 8;
    for (int t = lane; t < 400; t += 32) {
        const int rr = t / 20, cc = t % 20;
        if ((rr < 4 && (y == 0 || cc < 4)) || (cc < 4 && x == 0)) continue;
        W.L[rr][cc] = __ldcg(Y + (size_t)(y0 - 4 + rr) * P.ys + (x0 - 4 + cc));
    }
    for (int t = lane; t < 200; t += 32) {
        const int comp = t / 100, rr = (t % 100) / 10, cc = t % 10;
        if ((rr < 2 && (y == 0 || cc < 2)) || (cc < 2 && x == 0)) continue;
        const T* Cp = reinterpret_cast<const T*>(P.planes[1 + comp]);
        W.C[comp][rr][cc] = __ldcg(Cp + (size_t)(yc - 2 + rr) * P.cs + (xc - 2 + cc));
    }
    __syncwarp();
    const int maxv = (1 << P.bd) - 1;
    // dir 0: vertical edges, a lane per row; dir 1: horizontal edges, a lane per column
    for (int dir = 0; dir < 2; dir++) {
        const bool outer_ok = dir == 0 ? left_ok : top_ok;
        const ironav_dbk_mb& o0 = dir == 0 ? lm : tm;
        if (lane < 16) {
            const int line = lane;
            for (int e = 0; e < 4; e++) {
                if (e == 0 && !outer_ok) continue;
                if (m.t8x8 && (e & 1)) continue;
                const int b = W.bs[dir][e][line >> 2];
                if (b == 0) continue;
                const ironav_dbk_mb& o = e == 0 ? o0 : m;
                const int3 th = dbk_thresholds((o.qp + m.qp + 1) >> 1, sp, P.bd);
                if (th.x == 0 || th.y == 0) continue;
                const int tc0 = b < 4 ? (int)c_dbk_tc0[th.z][b - 1] << (P.bd - 8) : 0;
                int* q = dir == 0 ? &W.L[line + 4][4 * e + 4] : &W.L[4 * e + 4][line + 4];
                dbk_line(q, dir == 0 ? 1 : 21, b, tc0, th.x, th.y, false, maxv, o.keep, m.keep);
            }
        } else {
            const int comp = (lane - 16) >> 3, line = lane & 7;
            for (int e = 0; e < 4; e += 2) {
                if (e == 0 && !outer_ok) continue;
                const int b = W.bs[dir][e][line >> 1];
                if (b == 0) continue;
                const ironav_dbk_mb& o = e == 0 ? o0 : m;
                const int off = sp.chroma_qp_offset[comp];
                const int3 th = dbk_thresholds((dbk_chroma_qp(o.qp, off, P.bd) + dbk_chroma_qp(m.qp, off, P.bd) + 1) >> 1, sp, P.bd);
                if (th.x == 0 || th.y == 0) continue;
                const int tc0 = b < 4 ? (int)c_dbk_tc0[th.z][b - 1] << (P.bd - 8) : 0;
                int* q = dir == 0 ? &W.C[comp][line + 2][2 * e + 2] : &W.C[comp][2 * e + 2][line + 2];
                dbk_line(q, dir == 0 ? 1 : 11, b, tc0, th.x, th.y, true, maxv, o.keep, m.keep);
            }
        }
        __syncwarp();
    }
    // write back what the filter may have changed: the macroblock, 3 luma / 1 chroma samples to its left
    // and above
    T* Yw = reinterpret_cast<T*>(P.planes[0]);
    for (int t = lane; t < 400; t += 32) {
        const int rr = t / 20, cc = t % 20;
        if (rr == 0 || cc == 0 || (rr < 4 && (y == 0 || cc < 4)) || (cc < 4 && x == 0)) continue;
        __stcg(Yw + (size_t)(y0 - 4 + rr) * P.ys + (x0 - 4 + cc), (T)W.L[rr][cc]);
    }
    for (int t = lane; t < 200; t += 32) {
        const int comp = t / 100, rr = (t % 100) / 10, cc = t % 10;
        if (rr == 0 || cc == 0 || (rr < 2 && (y == 0 || cc < 2)) || (cc < 2 && x == 0)) continue;
        T* Cp = reinterpret_cast<T*>(P.planes[1 + comp]);
        __stcg(Cp + (size_t)(yc - 2 + rr) * P.cs + (xc - 2 + cc), (T)W.C[comp][rr][cc]);
    }
}

// Waits until row `row` has filtered `need` macroblocks, at most P.wait_limit polls; false when it gave up
// or another warp already did.
__device__ __forceinline__ bool dbk_wait(const DbkParams& P, int row, unsigned need) {
    for (unsigned i = 0;; i++) {
        if (ld_acquire(&P.progress[row]) >= need) return true;
        if (ld_acquire(P.err) & 1u) return false;
        if (i >= P.wait_limit) {
            atomicOr(P.err, 1u);
            return false;
        }
        __nanosleep(i < 64 ? 32 : 256);
    }
}

template <class T>
__global__ void __launch_bounds__(DBK_WARPS * 32) deblock_kernel(const __grid_constant__ DbkParams P) {
    __shared__ DbkWarp smem[DBK_WARPS];
    DbkWarp& W = smem[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    for (;;) {
        unsigned t = 0;
        if (lane == 0) t = atomicAdd(P.ticket, 1u);
        t = __shfl_sync(DBK_ALL, t, 0);
        if (t >= (unsigned)P.mb_h) return;
        const int y = (int)t;
        for (int x = 0; x < P.mb_w; x++) {
            if (y > 0 && !__all_sync(DBK_ALL, dbk_wait(P, y - 1, (unsigned)min(x + 2, P.mb_w)))) return;
            dbk_mb<T>(P, W, x, y);
            __threadfence();
            __syncwarp();
            if (lane == 0) st_release(&P.progress[y], (unsigned)(x + 1));
        }
    }
}

}  // namespace ironav
