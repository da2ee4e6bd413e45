// bpicture.cuh — K5: the searches of B macroblocks (decide_b, enc/frame.rs:1518-1572; best_b_parts
// 1626-1687; spatial direct, direct_mvs 1715-1747), replay mode, one warp per macroblock.
//
// Built from the P analysis's pieces: the per-list searches are motion_search on list l's reference planes
// (P.planes[l]) with the neighbour table of list l and reference index 0; the bi-predicted and direct
// costs are SATDs of averaged quarter-sample predictions (pred4 on both lists' planes, __vavgu4/2), lanes
// over 4x4 blocks. best_b_parts predicts every partition from the macroblock's own 16x16 predictors, so
// its searches depend on each other only through the early exits. The work counts follow the reference's
// evaluation order, with the bi-predicted and direct SATDs counted like the searches' ones.
#pragma once
#include "analyse.cuh"

namespace ironav {

// Per-warp shared memory of the B analysis: the P analysis's, plus list 1's neighbour table and the result
// being built.
template <class T>
struct WarpSmemB : WarpSmem<T> {
    Blk ext1[30];
    ironav_bresult bres;
};

// The neighbour tables of both lists (nb_motion, enc/frame.rs:522-538, on MbState.refs[l] / mvs / mvs1).
template <class T>
static __device__ void load_neighbours_b(const AnalyseParams& __restrict__ P, WarpSmemB<T>& __restrict__ S) {
    const int lane = threadIdx.x & 31;
    for (int k = lane; k < 60; k += 32) {
        const int l = k / 30, e_ = k % 30;
        const int ex = e_ % 6 - 1, ey = e_ / 6 - 1;
        Blk e = make_int4(0, 0, -1, 0);
        if (ey < 0 || ex < 0) {
            const int nx = S.mbx + (ex < 0 ? -1 : (ex >= 4 ? 1 : 0)), ny = S.mby + (ey < 0 ? -1 : 0);
            const int bx = ex < 0 ? 3 : (ex >= 4 ? 0 : ex), by = ey < 0 ? 3 : ey;
            if (nx >= 0 && nx < P.mb_w && ny >= P.band_start[S.mby] && ny < P.mb_h) {
                const ironav_mbstate_b* s = &P.bstates_in[(size_t)ny * P.mb_w + nx];
                e.w = 1;
                const int rf = s->refs[l][(by >> 1) * 2 + (bx >> 1)];
                if (s->inter && rf >= 0) {
                    e.x = s->mvs[l][by * 4 + bx][0];
                    e.y = s->mvs[l][by * 4 + bx][1];
                    e.z = rf;
                }
            }
        }
        (l == 0 ? S.ext : S.ext1)[e_] = e;
    }
    __syncwarp();
}

// SATD of the prediction of the partition at 4x4 block (bx, by), (4 << lgw) x (4 << lgh) samples, from list
// 0 with vector v0 (use bit 0), list 1 with v1 (bit 1), or both averaged ((a + b + 1) >> 1, b_pred
// enc/frame.rs:1766-1770 and decide_b's avg 1567); every lane gets the sum. Out of line: inlined at its five
// call sites it cost the kernel 6 % in instruction-cache misses.
template <class T>
static __device__ __noinline__ int mix_satd(const AnalyseParams& __restrict__ P, WarpSmemB<T>& __restrict__ S, int bx, int by, int lgw, int lgh, int2 v0,
                                               int2 v1, int use) {
    const int lane = threadIdx.x & 31;
    const int lg = lgw + lgh, w = 4 << lgw, h = 4 << lgh;
    const int x0 = S.mbx * 16 + bx * 4, y0 = S.mby * 16 + by * 4;
    int v = 0;
    if (lane < (1 << lg)) {
        const int bxx = lane & ((1 << lgw) - 1), byy = lane >> lgw;
        uint32_t pr[4][sizeof(T)];
        if (use & 1) pred4<T>(P, P.planes[0], x0, y0, w, h, bxx, byy, v0, pr);
        if (use & 2) {
            uint32_t p1[4][sizeof(T)];
            pred4<T>(P, P.planes[1], x0, y0, w, h, bxx, byy, v1, p1);
#pragma unroll
            for (int row = 0; row < 4; row++)
#pragma unroll
                for (int k = 0; k < (int)sizeof(T); k++)
                    pr[row][k] = (use & 1) ? (sizeof(T) == 1 ? __vavgu4(pr[row][k], p1[row][k]) : __vavgu2(pr[row][k], p1[row][k])) : p1[row][k];
        }
        v = score4<T>(S, bx + bxx, by + byy, pr, false);
    }
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) v += __shfl_xor_sync(FULL, v, off);
    return v;
}

__device__ __forceinline__ int minpos_d(int x, int y) { return (x >= 0 && y >= 0) ? min(x, y) : max(x, y); }
// the co-located vector scaled by picture distances (enc/frame.rs:1553-1554): i32 division, then i16
__device__ __forceinline__ int bscale_d(int v, int num, int den) { return (int)(int16_t)(v * num / den); }

// The search of one partition of best_b_parts (its `search` closure, enc/frame.rs:1631-1657): each list,
// both averaged, and for an 8x8 block its direct prediction (dv0 / dv1 with the direct lists duse). Returns
// (cost, direction, and the vectors packed as list 0 x | y << 16 in .z, list 1 in .w).
template <class T>
static __device__ int4 b_part_search(const AnalyseParams& __restrict__ P, WarpSmemB<T>& __restrict__ S, int bx, int by, int w4, int h4, int2 mvp0, int2 mvp1,
                                     const int2* ex0, const int2* ex1, int nex, bool direct, int2 dv0, int2 dv1, int duse) {
    const int lam = P.lambda;
    // the extra candidates of each list: the first two as registers, the rest (the halves' 3) by pointer
    const int4 m0 = motion_search<T, true>(P, S, S.ext, 0, 0, bx, by, w4, h4, mvp0.x, mvp0.y, ex0[0].x, ex0[0].y, nex > 1 ? ex0[1].x : 0,
                                  nex > 1 ? ex0[1].y : 0, min(nex, 2), nex > 2 ? ex0 + 2 : nullptr, max(nex - 2, 0));
    const int4 m1 = motion_search<T, true>(P, S, S.ext1, 0, 1, bx, by, w4, h4, mvp1.x, mvp1.y, ex1[0].x, ex1[0].y, nex > 1 ? ex1[1].x : 0,
                                  nex > 1 ? ex1[1].y : 0, min(nex, 2), nex > 2 ? ex1 + 2 : nullptr, max(nex - 2, 0));
    const int2 v0 = make_int2(m0.y, m0.z), v1 = make_int2(m1.y, m1.z);
    const int lgw = w4 == 4 ? 2 : (w4 == 2 ? 1 : 0), lgh = h4 == 4 ? 2 : (h4 == 2 ? 1 : 0);
    const int bi = mix_satd(P, S, bx, by, lgw, lgh, v0, v1, 3) +
                   lam * (mvd_bits_d(v0.x, v0.y, mvp0.x, mvp0.y) + mvd_bits_d(v1.x, v1.y, mvp1.x, mvp1.y) + 2);
    int cnt = w4 * h4 * 16;
    int bd, bc;
    if (bi < min(m0.x, m1.x)) {
        bd = 3;
        bc = bi;
    } else if (m0.x <= m1.x) {
        bd = 1;
        bc = m0.x;
    } else {
        bd = 2;
        bc = m1.x;
    }
    if (direct) {
        // sub_mb_type takes about one bin for direct and three for the others
        bc += lam * 3;
        const int d = mix_satd(P, S, bx, by, lgw, lgh, dv0, dv1, duse) + lam;
        cnt += w4 * h4 * 16;
        if (d < bc) {
            bd = 0;
            bc = d;
        }
    }
    if ((threadIdx.x & 31) == 0) S.satd_px += (uint32_t)cnt;
    return make_int4(bc, bd, (v0.x & 0xffff) | (v0.y << 16), (v1.x & 0xffff) | (v1.y << 16));
}

__device__ __forceinline__ int2 unpack_mv(int v) { return make_int2((int)(int16_t)(v & 0xffff), v >> 16); }

// best_b_parts, enc/frame.rs:1626-1687, into S.bres (part, bdir, pmv); false when no partitioning costs
// less than cost16.
template <class T>
static __device__ __noinline__ bool b_parts(const AnalyseParams& __restrict__ P, WarpSmemB<T>& __restrict__ S, int2 mv16a, int2 mv16b, int2 mvp0, int2 mvp1,
                                            int cost16, int4 dvs, int duse) {
    const int lane = threadIdx.x & 31;
    const int lam = P.lambda;
    // dvs: list 0's direct vector of each 8x8 block, packed (list 1's are read from S.bres)
    int dirs = 0;                 // 4 x 8 bits
    int pm0[4], pm1[4];           // packed vectors per 8x8 block
    int total = lam * 6;
    for (int k = 0; k < 4; k++) {
        const int bx = (k & 1) * 2, by = (k >> 1) * 2;
        const int2 dv0 = unpack_mv(k == 0 ? dvs.x : (k == 1 ? dvs.y : (k == 2 ? dvs.z : dvs.w)));
        const int2 dv1 = make_int2(S.bres.direct_mv[1][by * 4 + bx][0], S.bres.direct_mv[1][by * 4 + bx][1]);
        const int4 r = b_part_search(P, S, bx, by, 2, 2, mvp0, mvp1, &mv16a, &mv16b, 1, true, dv0, dv1, duse);
        dirs |= r.y << (8 * k);
        pm0[k] = r.z;
        pm1[k] = r.w;
        total += r.x;
        if (total >= cost16) return false;
    }
    int best_part = 3, best_dirs = dirs, best_total = total;
    int bm0[4] = {pm0[0], pm0[1], pm0[2], pm0[3]}, bm1[4] = {pm1[0], pm1[1], pm1[2], pm1[3]};
    // the halves take the four 8x8 vectors and the 16x16 one of their list as extra candidates
    int2 e0[5], e1[5];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        e0[k] = unpack_mv(pm0[k]);
        e1[k] = unpack_mv(pm1[k]);
    }
    e0[4] = mv16a;
    e1[4] = mv16b;
    for (int part = 1; part < 3; part++) {
        int pd = 0, q0[2] = {0, 0}, q1[2] = {0, 0};
        int pt = lam * 7;
        for (int k = 0; k < 2; k++) {
            const int bx = part == 2 ? 2 * k : 0, by = part == 1 ? 2 * k : 0, w4 = part == 1 ? 4 : 2, h4 = part == 1 ? 2 : 4;
            const int4 r = b_part_search(P, S, bx, by, w4, h4, mvp0, mvp1, e0, e1, 5, false, make_int2(0, 0), make_int2(0, 0), 0);
            pd |= r.y << (8 * k);
            q0[k] = r.z;
            q1[k] = r.w;
            pt += r.x;
            if (pt >= best_total) break;
        }
        if (pt < best_total) {
            best_part = part;
            best_dirs = pd;
            best_total = pt;
            bm0[0] = q0[0];
            bm0[1] = q0[1];
            bm0[2] = bm0[3] = 0;
            bm1[0] = q1[0];
            bm1[1] = q1[1];
            bm1[2] = bm1[3] = 0;
        }
    }
    if (lane == 0) {
        S.bres.part = (uint8_t)best_part;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            S.bres.bdir[k] = (uint8_t)((best_dirs >> (8 * k)) & 0xff);
            const int2 a = unpack_mv(bm0[k]), b = unpack_mv(bm1[k]);
            S.bres.pmv[0][k][0] = (int16_t)a.x;
            S.bres.pmv[0][k][1] = (int16_t)a.y;
            S.bres.pmv[1][k][0] = (int16_t)b.x;
            S.bres.pmv[1][k][1] = (int16_t)b.y;
        }
    }
    __syncwarp();
    return true;
}

// The searches of decide_b for the warp's macroblock (enc/frame.rs:1518-1572), into S.bres.
template <class T>
static __device__ void analyse_b(const AnalyseParams& __restrict__ P, WarpSmemB<T>& __restrict__ S) {
    const int lane = threadIdx.x & 31;
    const int lam = P.lambda;
    stage_source(P, S);
    if (lane < 50) reinterpret_cast<uint32_t*>(&S.bres)[lane] = 0;
    if (lane + 32 < 50) reinterpret_cast<uint32_t*>(&S.bres)[lane + 32] = 0;
    if (lane == 0) S.sad_px = S.satd_px = 0;
    __syncwarp();
    // spatial direct (direct_mvs, 1715-1747): per list the neighbours' least reference index
    int refs[2];
#pragma unroll
    for (int l = 0; l < 2; l++) {
        const Blk* e = l == 0 ? S.ext : S.ext1;
        const Blk a = nb(P, S, e, nullptr, -1, 0), b = nb(P, S, e, nullptr, 0, -1);
        Blk c = nb(P, S, e, nullptr, 4, -1);
        if (!c.w) c = nb(P, S, e, nullptr, -1, -1);
        refs[l] = minpos_d(a.z, minpos_d(b.z, c.z));
    }
    const int2 mvp0 = pred_mv(P, S, S.ext, nullptr, 0, 0, 4, 0, 0), mvp1 = pred_mv(P, S, S.ext1, nullptr, 0, 0, 4, 0, 0);
    const bool none = refs[0] < 0 && refs[1] < 0;
    const int duse = none ? 3 : ((refs[0] >= 0 ? 1 : 0) | (refs[1] >= 0 ? 2 : 0));
    // per 8x8 block (its corner 4x4 block stands for it, direct_8x8_inference_flag): the direct vectors,
    // zeroed where the co-located block of the list-1 picture (reference 0) barely moves
    const ironav_mbstate* col = P.bcol ? &P.bcol[S.mb] : nullptr;
    const bool col_inter = col && col->inter;
    if (lane < 16) {
        const int b = lane, cx = ((b % 4) >> 1) * 3, cy = ((b / 4) >> 1) * 3;
        bool zero = false;
        if (col_inter) {
            const int mx = col->mvs[cy * 4 + cx][0], my = col->mvs[cy * 4 + cx][1];
            zero = col->refs[(cy >> 1) * 2 + (cx >> 1)] == 0 && abs(mx) <= 1 && abs(my) <= 1;
        }
#pragma unroll
        for (int l = 0; l < 2; l++) {
            int2 v = make_int2(0, 0);
            if (!none && refs[l] >= 0 && !(zero && refs[l] == 0)) v = l == 0 ? mvp0 : mvp1;
            S.bres.direct_mv[l][b][0] = (int16_t)v.x;
            S.bres.direct_mv[l][b][1] = (int16_t)v.y;
        }
    }
    if (lane == 0) {
        S.bres.direct_use[0] = (uint8_t)(duse & 1);
        S.bres.direct_use[1] = (uint8_t)(duse >> 1);
    }
    __syncwarp();
    // 16x16 from either list or both (1549-1570); the co-located vector spans both lists' references,
    // split by the picture's distances from them
    int ce = 0, cx = 0, cy = 0;
    if (col_inter) {
        ce = 1;
        cx = col->mvs[5][0];
        cy = col->mvs[5][1];
    }
    const int tb = P.tb, td = P.td;
    const int4 s0 = motion_search<T, true>(P, S, S.ext, 0, 0, 0, 0, 4, 4, mvp0.x, mvp0.y, bscale_d(cx, tb, td), bscale_d(cy, tb, td), 0, 0, ce,
                                  (const int2*)nullptr, 0);
    const int2 v0 = make_int2(s0.y, s0.z);
    // list 1: the co-located vector (if any), then list 0's vector scaled
    const int e1x = bscale_d(v0.x, tb - td, tb), e1y = bscale_d(v0.y, tb - td, tb);
    const int4 s1 = col_inter ? motion_search<T, true>(P, S, S.ext1, 0, 1, 0, 0, 4, 4, mvp1.x, mvp1.y, bscale_d(cx, tb - td, td),
                                              bscale_d(cy, tb - td, td), e1x, e1y, 2, (const int2*)nullptr, 0)
                              : motion_search<T, true>(P, S, S.ext1, 0, 1, 0, 0, 4, 4, mvp1.x, mvp1.y, e1x, e1y, 0, 0, 1,
                                              (const int2*)nullptr, 0);
    const int2 v1 = make_int2(s1.y, s1.z);
    const int c0 = s0.x + lam * (mvd_bits_d(v0.x, v0.y, mvp0.x, mvp0.y) + 3);
    const int c1 = s1.x + lam * (mvd_bits_d(v1.x, v1.y, mvp1.x, mvp1.y) + 3);
    const int bi = mix_satd(P, S, 0, 0, 2, 2, v0, v1, 3) +
                   lam * (mvd_bits_d(v0.x, v0.y, mvp0.x, mvp0.y) + mvd_bits_d(v1.x, v1.y, mvp1.x, mvp1.y) + 5);
    if (lane == 0) {
        S.satd_px += 256;
        S.bres.dir16 = (uint8_t)(bi < min(c0, c1) ? 3 : (c0 <= c1 ? 1 : 2));
        S.bres.mv16[0][0] = (int16_t)v0.x;
        S.bres.mv16[0][1] = (int16_t)v0.y;
        S.bres.mv16[1][0] = (int16_t)v1.x;
        S.bres.mv16[1][1] = (int16_t)v1.y;
        S.bres.cost16[0] = c0;
        S.bres.cost16[1] = c1;
        S.bres.cost_bi = bi;
    }
    __syncwarp();
    // the smaller partitionings (best_b_parts): direct vectors of list 0 per 8x8 block, packed
    auto dv = [&](int k) {
        const int b = (k >> 1) * 8 + (k & 1) * 2;
        return (S.bres.direct_mv[0][b][0] & 0xffff) | ((int)S.bres.direct_mv[0][b][1] << 16);
    };
    const int4 dvs = make_int4(dv(0), dv(1), dv(2), dv(3));
    const bool parts = b_parts(P, S, v0, v1, mvp0, mvp1, min(bi, min(c0, c1)), dvs, duse);
    if (lane == 0) {
        S.bres.has_parts = parts ? 1 : 0;
        S.bres.sad_px = S.sad_px;
        S.bres.satd_px = S.satd_px;
    }
    __syncwarp();
}

// One warp per B macroblock, replay mode (every macroblock independent), persistent CTAs on tickets.
template <class T>
__global__ void __launch_bounds__(K2_WARPS * 32, K2_MIN_BLOCKS) analyse_b_kernel(const __grid_constant__ AnalyseParams P) {
    __shared__ WarpSmemB<T> smem[K2_WARPS];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    WarpSmemB<T>& S = smem[wid];
    for (;;) {
        unsigned t = 0;
        if (lane == 0) t = atomicAdd(P.ticket, 1u);
        t = __shfl_sync(FULL, t, 0);
        if (t >= (unsigned)P.nmb) break;
        const int mb = (int)t;
        if (lane == 0) {
            S.mb = mb;
            S.mbx = mb % P.mb_w;
            S.mby = mb / P.mb_w;
        }
        __syncwarp();
        load_neighbours_b(P, S);
        analyse_b(P, S);
        uint32_t* out = reinterpret_cast<uint32_t*>(&P.bresults[mb]);
        const uint32_t* res = reinterpret_cast<const uint32_t*>(&S.bres);
        out[lane] = res[lane];
        if (lane + 32 < 50) out[lane + 32] = res[lane + 32];
        __syncwarp();
    }
}

}  // namespace ironav
