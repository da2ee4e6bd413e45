// analyse_g8.cuh — K2 in replay mode with one macroblock per 8-lane group: four macroblocks a warp.
//
// Replay mode reads every macroblock's neighbours from the caller's final decisions, so all macroblocks of a
// picture are independent. The warp-per-macroblock kernel (analyse.cuh) spends most of its issue slots on the
// search's warp-uniform control (candidate bookkeeping, the diamond's move replay, loop tests), once per
// macroblock. Here each 8-lane group runs one macroblock's search as group-uniform scalar code — a direct
// statement of the reference's sequential search (enc/frame.rs:839-1019) — so every control instruction
// serves four macroblocks at once, and the lanes of a group share only the sample work:
//   - integer SAD: two candidate vectors per pass, four lanes each splitting the rows (sad2);
//   - a diamond round scores exactly the reference's points: left and right of the centre in one pass, then
//     up and down at the column the first two moves left in a second pass; when a move the search clamps
//     bent (or the centre lay outside the clamps) leaves the next point one not yet scored, it is scored on
//     its own;
//   - sub-sample SATD: the group's lanes over (vector, 4x4 block) tasks, per-vector sums by shared atomics.
// The four macroblocks of a warp are neighbours in a row and their searches mostly take the same paths; where
// they differ the hardware runs the paths one after another, so the group's shuffles and barriers name only
// the group's lanes.
#pragma once
#include "analyse.cuh"

namespace ironav {
namespace g8 {

constexpr int WARPS = 4;       // warps a CTA (8 and 16-lane groups)
constexpr int MIN_BLOCKS = 4;  // CTAs an SM the register budget must allow, at 128 registers a thread
// Warps a CTA for groups of GW lanes: the CTA's groups' shared memory stays within the 48 KB of static shared
// memory (16 groups of about 1.8 KB), and the CTAs an SM scale so that 16 warps an SM fit 128 registers.
__host__ __device__ constexpr int warps_for(int gw) { return gw == 4 ? 2 : WARPS; }

// Per-group shared memory; T is the sample type.
template <class T>
struct GroupSmem {
    uint32_t src[64 * sizeof(T)];  // the macroblock: 16 rows of 16 samples (4 * sizeof(T) words a row)
    Blk ext[30];                   // blocks around the macroblock: index (y + 1) * 6 + (x + 1)
    Blk st[16];                    // P_8x8: blocks decided so far (sub_search's `st`)
    Blk t[16];                     // trial blocks (sub_search's `t`, part_mvps's `cur`)
    Blk bt[16];                    // best trial
    int cost[16];                  // sub-sample sums of a batch
    int16_t best_mvs[16][2];       // best_inter_ref's running best, in coding order
    int16_t win_mvs[16][2];        // best over the references
    ironav_mbresult res;           // the result being assembled
};

// A group of GW lanes (8 or 16) analysing one macroblock: its lane index and mask.
template <int GW>
struct Grp {
    int gl;         // lane within the group
    unsigned mask;  // the group's lanes
};

template <int GW>
__device__ __forceinline__ Grp<GW> grp_of_lane() {
    const int lane = threadIdx.x & 31;
    return Grp<GW>{lane & (GW - 1), (GW == 32 ? 0xffffffffu : ((1u << GW) - 1u)) << (lane & (32 - GW))};
}

// The macroblock a group analyses and its work counts.
struct Mb {
    int mb, mbx, mby;
    uint32_t sad_px, satd_px;
};

// SAD of one row of w samples (w = 4, 8 or 16) at byte address G against source words sr: the reference's
// row read as aligned 32-bit words realigned with funnel shifts.
template <class T>
__device__ __forceinline__ int row_sad(const uint8_t* G, const uint32_t* sr, int w) {
    constexpr int B = sizeof(T);
    const uintptr_t a = reinterpret_cast<uintptr_t>(G);
    const uint32_t* q = reinterpret_cast<const uint32_t*>(a & ~uintptr_t(3));
    const unsigned sh = (unsigned)(a & 3) * 8u;
    const int nw = (w * B) >> 2;
    int sad = 0;
    uint32_t pv = __ldg(q);
#pragma unroll
    for (int k = 0; k < 4 * B; k++) {
        if (k < nw) {
            const uint32_t nx = __ldg(q + k + 1);
            const uint32_t v = __funnelshift_r(pv, nx, sh);
            sad += B == 1 ? __vsadu4(sr[k], v) : __vsadu2(sr[k], v);
            pv = nx;
        }
    }
    return sad;
}

// Integer SAD (sad_int, enc/frame.rs:662-671) of the w x h partition for two vectors at once: the first half
// of the group scores (ax, ay), the second (bx, by), the lanes of a half splitting the rows. g0: plane G at the partition's
// origin (bytes); src: the partition's first source word; sw: the plane stride in samples. Every lane of the
// group gets both sums.
template <class T, int GW>
__device__ __forceinline__ int2 sad2(const Grp<GW>& g, const uint8_t* __restrict__ g0, const uint32_t* __restrict__ src, int sw, int w, int h,
                                     int ax, int ay, int bx, int by) {
    constexpr int B = sizeof(T), H = GW / 2;  // lanes a vector
    const bool second = g.gl >= H;
    const int px = second ? bx : ax, py = second ? by : ay;
    const int r0 = g.gl & (H - 1);
    const uint8_t* G = g0 + (((py >> 2) + r0) * sw + (px >> 2)) * B;
    int s = 0;
    for (int row = r0; row < h; row += H, G += H * sw * B) s += row_sad<T>(G, src + row * 4 * B, w);
#pragma unroll
    for (int off = 1; off < H; off <<= 1) s += __shfl_xor_sync(g.mask, s, off, GW);
    const int o = __shfl_xor_sync(g.mask, s, H, GW);
    return second ? make_int2(o, s) : make_int2(s, o);
}

// The score of a 4x4 prediction against the source's 4x4 block (sbx, sby): SATD, or SAD when `sad`.
template <class T>
__device__ __forceinline__ int score4_src(const uint32_t* __restrict__ src, int sbx, int sby, const uint32_t (&pr)[4][sizeof(T)], bool sad) {
    constexpr int B = sizeof(T);
    uint32_t sr[4][B];
    const uint32_t* sp = &src[(sby * 16 + sbx) * B];
#pragma unroll
    for (int row = 0; row < 4; row++)
#pragma unroll
        for (int k = 0; k < B; k++) sr[row][k] = sp[row * 4 * B + k];
    int v = 0;
    if (sad) {
#pragma unroll
        for (int row = 0; row < 4; row++)
#pragma unroll
            for (int k = 0; k < B; k++) v += B == 1 ? __vsadu4(sr[row][k], pr[row][k]) : __vsadu2(sr[row][k], pr[row][k]);
    } else if constexpr (B == 1) {
        const uint32_t s1[4] = {sr[0][0], sr[1][0], sr[2][0], sr[3][0]}, p1[4] = {pr[0][0], pr[1][0], pr[2][0], pr[3][0]};
        v = satd4_packed(s1, p1);
    } else {
        v = satd4_packed16(sr, pr);
    }
    return v;
}

// Quarter-sample prediction of the partition at 4x4 block (bx, by) of (4 << lgw) x (4 << lgh) samples on the
// planes of reference r, scored by SATD (or SAD when `sad`) for the n vectors pt(0..n) (a group-uniform
// function of the index): the sums land in S.cost[0..n). The group's lanes take (vector, 4x4 block) tasks.
template <class T, int GW, class F>
__device__ __forceinline__ void pred_points(const AnalyseParams& __restrict__ P, GroupSmem<T>& __restrict__ S, const Grp<GW>& g, int mbx, int mby, int r,
                                            int bx, int by, int lgw, int lgh, F pt, int n, bool sad) {
    const int lg = lgw + lgh, total = n << lg, w = 4 << lgw, h = 4 << lgh;
#pragma unroll
    for (int k = 0; k < (9 + GW - 1) / GW; k++)
        if (g.gl + GW * k < n) S.cost[g.gl + GW * k] = 0;
    __syncwarp(g.mask);
    const int x0 = mbx * 16 + bx * 4, y0 = mby * 16 + by * 4;
    const uint8_t* base = P.planes[r];
    for (int t = g.gl; t < total; t += GW) {
        const int c = t >> lg, b = t & ((1 << lg) - 1), bxx = b & ((1 << lgw) - 1), byy = b >> lgw;
        uint32_t pr[4][sizeof(T)];
        pred4<T>(P, base, x0, y0, w, h, bxx, byy, pt(c), pr);
        atomicAdd(&S.cost[c], score4_src<T>(S.src, bx + bxx, by + byy, pr, sad));
    }
    __syncwarp(g.mask);
}

// nb_motion (enc/frame.rs:522-538) for the block at (x, y) relative to the macroblock: outside it from the
// neighbour table, inside it from the decided blocks `cur` (nullptr: none decided).
__device__ __forceinline__ Blk nb_g(const Blk* ext, const Blk* cur, int x, int y) {
    if (x >= 0 && x < 4 && y >= 0) return cur ? cur[y * 4 + x] : make_int4(0, 0, -1, 0);
    return ext[(y + 1) * 6 + (x + 1)];
}

// pred_mv, enc/frame.rs:543-570
__device__ __forceinline__ int2 pred_mv_g(const Blk* ext, const Blk* cur, int bx, int by, int w, int dir, int rf) {
    const Blk a = nb_g(ext, cur, bx - 1, by), b = nb_g(ext, cur, bx, by - 1);
    Blk c = nb_g(ext, cur, bx + w, by - 1);
    if (!c.w) c = nb_g(ext, cur, bx - 1, by - 1);
    if (dir == 1 && by == 0 && b.z == rf) return make_int2(b.x, b.y);
    if (dir == 1 && by != 0 && a.z == rf) return make_int2(a.x, a.y);
    if (dir == 2 && bx == 0 && a.z == rf) return make_int2(a.x, a.y);
    if (dir == 2 && bx != 0 && c.z == rf) return make_int2(c.x, c.y);
    if (!b.w && !c.w && a.w) return make_int2(a.x, a.y);
    const int ra = a.z == rf, rb = b.z == rf, rc = c.z == rf;
    if (ra + rb + rc == 1) {
        if (ra) return make_int2(a.x, a.y);
        if (rb) return make_int2(b.x, b.y);
        return make_int2(c.x, c.y);
    }
    return make_int2(median3_d(a.x, b.x, c.x), median3_d(a.y, b.y, c.y));
}

// One diamond round (enc/frame.rs:973-988) at `step` around (bxv, byv) of cost bc, scoring the reference's
// own points. Each of its four moves starts from the current best and clamps both coordinates: left and right
// of the centre are scored in one pass, up and down at the column the first two moves left in a second pass.
// When the left (up) move is taken, the right (down) point is taken from the new best: it is the point just
// beaten — whose cost cannot win — unless a clamp bent the move (or the centre lay outside the clamps, which
// the candidates' rounding allows at the +-2048 / +-512 limits), and then it is scored on its own. Returns
// whether the best moved.
template <class T, int GW>
__device__ __forceinline__ bool round_g(const AnalyseParams& __restrict__ P, const Grp<GW>& g, const uint8_t* g0, const uint32_t* src, int w, int h,
                                        int mvpx, int mvpy, int step, int cxlo, int cxhi, int cylo, int cyhi, int& bxv, int& byv, int& bc) {
    const int lam = P.lambda, sw = P.sw;
    auto clx = [&](int v) { return min(max(v, cxlo), cxhi); };
    auto cly = [&](int v) { return min(max(v, cylo), cyhi); };
    auto cost1 = [&](int x, int y) { return sad2<T, GW>(g, g0, src, sw, w, h, x, y, x, y).x + lam * mvd_bits_d(x, y, mvpx, mvpy); };
    bool moved = false;
    {
        const int cx0 = bxv, cy0 = byv, row = cly(cy0);
        const int lx = clx(cx0 - step), rx = clx(cx0 + step);
        const int2 s = sad2<T, GW>(g, g0, src, sw, w, h, lx, row, rx, row);
        const int cl = s.x + lam * mvd_bits_d(lx, row, mvpx, mvpy), cr = s.y + lam * mvd_bits_d(rx, row, mvpx, mvpy);
        if (cl < bc) {
            bxv = lx;
            byv = row;
            bc = cl;
            moved = true;
            const int nx = clx(lx + step);
            if (nx != cx0 || row != cy0) {
                const int c = cost1(nx, row);
                if (c < bc) {
                    bxv = nx;
                    bc = c;
                }
            }
        } else if (cr < bc) {
            bxv = rx;
            byv = row;
            bc = cr;
            moved = true;
        }
    }
    {
        const int bx1 = bxv, by1 = byv, col = clx(bx1);
        const int uy = cly(by1 - step), dy = cly(by1 + step);
        const int2 s = sad2<T, GW>(g, g0, src, sw, w, h, col, uy, col, dy);
        const int cu = s.x + lam * mvd_bits_d(col, uy, mvpx, mvpy), cd = s.y + lam * mvd_bits_d(col, dy, mvpx, mvpy);
        if (cu < bc) {
            bxv = col;
            byv = uy;
            bc = cu;
            moved = true;
            const int ny = cly(uy + step);
            if (col != bx1 || ny != by1) {
                const int c = cost1(col, ny);
                if (c < bc) {
                    byv = ny;
                    bc = c;
                }
            }
        } else if (cd < bc) {
            bxv = col;
            byv = dy;
            bc = cd;
            moved = true;
        }
    }
    return moved;
}

// motion_search, enc/frame.rs:949-1019 (list 0), for the partition at 4x4 block (bx, by) of w4 x h4 blocks:
// the candidates (the predictor, zero, the macroblock's left, top and top-right neighbours on this reference,
// then the extra vectors), the diamond, and the sub-sample refinement by SATD. Returns (cost without the
// vector's bits, mx, my).
template <class T, int GW>
__device__ __noinline__ int3 msearch(const AnalyseParams& __restrict__ P, GroupSmem<T>& __restrict__ S, const Grp<GW>& g, Mb& M, int r, int bx, int by,
                                     int w4, int h4, int mvpx, int mvpy, int e0x, int e0y, int e1x, int e1y, int nextra) {
    constexpr int B = sizeof(T);
    const int lam = P.lambda;
    const int x0 = M.mbx * 16 + bx * 4, y0 = M.mby * 16 + by * 4, w = w4 * 4, h = h4 * 4;
    const int cxlo = max(-(x0 + 24) * 4, -2048), cxhi = min((P.mb_w * 16 - x0 + 8) * 4, 2047);
    const int cylo = max(-(y0 + 24) * 4, -512), cyhi = min((P.mb_h * 16 - y0 + 8) * 4, 511);
    auto clx = [&](int v) { return min(max(v, cxlo), cxhi); };
    auto cly = [&](int v) { return min(max(v, cylo), cyhi); };
    auto intr = [](int v) { return (v + 2) & ~3; };
    const uint8_t* const g0 = P.planes[r] + ((y0 + PAD) * P.sw + x0 + PAD) * B;
    const uint32_t* const src = &S.src[(by * 16 + bx) * B];
    // candidates (958-964), in the reference's order; the first of least cost wins
    const Blk na = nb_g(S.ext, nullptr, -1, 0), nbb = nb_g(S.ext, nullptr, 0, -1), nc = nb_g(S.ext, nullptr, 4, -1);
    const bool va = na.w && na.z == r, vb = nbb.w && nbb.z == r, vc = nc.w && nc.z == r;
    int bxv = 0, byv = 0, bc = BIG;
    int ncand = 2;
    auto take = [&](bool valid, int x, int y, int sad) {
        if (!valid) return;
        const int c = sad + lam * mvd_bits_d(x, y, mvpx, mvpy);
        if (c < bc) {
            bxv = x;
            byv = y;
            bc = c;
        }
    };
    {
        const int px = intr(clx(mvpx)), py = intr(cly(mvpy));
        const int2 s = sad2<T, GW>(g, g0, src, P.sw, w, h, px, py, 0, 0);
        take(true, px, py, s.x);
        take(true, 0, 0, s.y);
    }
    {
        const int ax = intr(clx(na.x)), ay = intr(cly(na.y)), qx = intr(clx(nbb.x)), qy = intr(cly(nbb.y));
        if (va || vb) {
            const int2 s = sad2<T, GW>(g, g0, src, P.sw, w, h, va ? ax : 0, va ? ay : 0, vb ? qx : 0, vb ? qy : 0);
            take(va, ax, ay, s.x);
            take(vb, qx, qy, s.y);
            ncand += va + vb;
        }
    }
    {
        const int cx = intr(clx(nc.x)), cy = intr(cly(nc.y)), fx = intr(clx(e0x)), fy = intr(cly(e0y));
        const bool ve = nextra > 0;
        if (vc || ve) {
            const int2 s = sad2<T, GW>(g, g0, src, P.sw, w, h, vc ? cx : 0, vc ? cy : 0, ve ? fx : 0, ve ? fy : 0);
            take(vc, cx, cy, s.x);
            take(ve, fx, fy, s.y);
            ncand += vc + ve;
        }
    }
    if (nextra > 1) {
        const int fx = intr(clx(e1x)), fy = intr(cly(e1y));
        take(true, fx, fy, sad2<T, GW>(g, g0, src, P.sw, w, h, fx, fy, fx, fy).x);
        ncand++;
    }
    M.sad_px += (uint32_t)(ncand * w * h);
    // the diamond (973-988)
    const bool fast = P.fast != 0;
    const int nsteps = fast ? 2 : 3;
    int rounds = 0;
    for (int si = 0; si < nsteps; si++) {
        const int step = fast ? (si == 0 ? 8 : 4) : (16 >> si);
        const int iters = step == 4 ? 32 : 4;
        for (int it = 0; it < iters; it++) {
            rounds++;
            if (!round_g<T, GW>(P, g, g0, src, w, h, mvpx, mvpy, step, cxlo, cxhi, cylo, cyhi, bxv, byv, bc)) break;
        }
    }
    M.sad_px += (uint32_t)(4 * w * h * rounds);
    // live coding's early exit (990-992)
    if (fast && bc < (w * h) / 8 + lam) return make_int3(bc - lam * mvd_bits_d(bxv, byv, mvpx, mvpy), bxv, byv);
    const int lgw = w4 == 4 ? 2 : (w4 == 2 ? 1 : 0), lgh = h4 == 4 ? 2 : (h4 == 2 ? 1 : 0);
    // sub-sample refinement (994-1017): the centre, then the half-sample square in the reference's order
    // (-1,-1) (0,-1) (1,-1) (-1,0) (1,0) (-1,1) (0,1) (1,1), each clamped; the first of least cost wins
    {
        const int ccx = bxv, ccy = byv;
        auto sq = [&](int c) {
            if (c == 0) return make_int2(ccx, ccy);
            const int kk = c <= 4 ? c - 1 : c;
            return make_int2(clx(ccx + (kk % 3 - 1) * 2), cly(ccy + (kk / 3 - 1) * 2));
        };
        pred_points<T, GW>(P, S, g, M.mbx, M.mby, r, bx, by, lgw, lgh, sq, 9, false);
        bc = S.cost[0] + lam * mvd_bits_d(ccx, ccy, mvpx, mvpy);
        for (int c = 1; c < 9; c++) {
            const int2 q = sq(c);
            const int v = S.cost[c] + lam * mvd_bits_d(q.x, q.y, mvpx, mvpy);
            if (v < bc) {
                bc = v;
                bxv = q.x;
                byv = q.y;
            }
        }
        M.satd_px += (uint32_t)(9 * w * h);
        __syncwarp(g.mask);
    }
    if (!fast) {
        // the quarter-sample diamond around the new centre: (0,-1) (-1,0) (1,0) (0,1), clamped; the centre keeps ties
        const int ccx = bxv, ccy = byv;
        auto dm = [&](int c) {
            const int dx = c == 1 ? -1 : (c == 2 ? 1 : 0), dy = c == 0 ? -1 : (c == 3 ? 1 : 0);
            return make_int2(clx(ccx + dx), cly(ccy + dy));
        };
        pred_points<T, GW>(P, S, g, M.mbx, M.mby, r, bx, by, lgw, lgh, dm, 4, false);
        for (int c = 0; c < 4; c++) {
            const int2 q = dm(c);
            const int v = S.cost[c] + lam * mvd_bits_d(q.x, q.y, mvpx, mvpy);
            if (v < bc) {
                bc = v;
                bxv = q.x;
                byv = q.y;
            }
        }
        M.satd_px += (uint32_t)(4 * w * h);
        __syncwarp(g.mask);
    }
    return make_int3(bc - lam * mvd_bits_d(bxv, byv, mvpx, mvpy), bxv, byv);
}

// Block tables of a group (16 entries): the group's lanes take two entries each.
template <int GW>
__device__ __forceinline__ void blk_copy_g(const Grp<GW>& g, Blk* dst, const Blk* src) {
#pragma unroll
    for (int k = 0; k < 16 / GW; k++) dst[g.gl + GW * k] = src[g.gl + GW * k];
    __syncwarp(g.mask);
}
template <int GW>
__device__ __forceinline__ void blk_clear_g(const Grp<GW>& g, Blk* dst) {
#pragma unroll
    for (int k = 0; k < 16 / GW; k++) dst[g.gl + GW * k] = make_int4(0, 0, -1, 0);
    __syncwarp(g.mask);
}
// Marks the w x h blocks at (x, y) decided with vector (mx, my) on reference r.
template <int GW>
__device__ __forceinline__ void blk_paint_g(const Grp<GW>& g, Blk* dst, int x, int y, int w, int h, int mx, int my, int r) {
#pragma unroll
    for (int k = 0; k < 16 / GW; k++) {
        const int i = g.gl + GW * k, bx = i & 3, by = i >> 2;
        if (bx >= x && bx < x + w && by >= y && by < y + h) dst[i] = make_int4(mx, my, r, 1);
    }
    __syncwarp(g.mask);
}

// sub_search, enc/frame.rs:911-938, for 8x8 block k with the 16x16 vector (ex, ey) as extra candidate:
// returns (sub_mb_type, its cost) and leaves the block's vectors in S.st.
template <class T, int GW>
__device__ __noinline__ int2 sub_search_g(const AnalyseParams& __restrict__ P, GroupSmem<T>& __restrict__ S, const Grp<GW>& g, Mb& M, int r, int k,
                                          int ex, int ey) {
    const int lam = P.lambda;
    const int ox = (k & 1) * 2, oy = (k >> 1) * 2;
    const int ns = P.sub8 ? 4 : 1;
    int best_s = 0, best_cost = 0;
    for (int s = 0; s < ns; s++) {
        blk_copy_g(g, S.t, S.st);
        int cost = lam * (s == 0 ? 0 : 2);
        for (int q = 0; q < c_nsub[s]; q++) {
            const int x = ox + c_sub[s][q][0], y = oy + c_sub[s][q][1], w = c_sub[s][q][2], h = c_sub[s][q][3];
            const int2 p = pred_mv_g(S.ext, S.t, x, y, w, 0, r);
            const int3 ms = msearch<T, GW>(P, S, g, M, r, x, y, w, h, p.x, p.y, ex, ey, 0, 0, 1);
            cost += ms.x + lam * mvd_bits_d(ms.y, ms.z, p.x, p.y);
            blk_paint_g(g, S.t, x, y, w, h, ms.y, ms.z, r);
        }
        if (s == 0 || cost < best_cost) {
            best_s = s;
            best_cost = cost;
            if (ns > 1) blk_copy_g(g, S.bt, S.t);
        }
    }
    blk_copy_g(g, S.st, ns > 1 ? S.bt : S.t);
    return make_int2(best_s, best_cost);
}

// best_inter_ref, enc/frame.rs:852-905: returns (cost, part, sub (a byte per 8x8 block), cost16) and leaves the
// winner's vectors, in coding order, in S.best_mvs.
template <class T, int GW>
__device__ __noinline__ int4 best_inter_ref_g(const AnalyseParams& __restrict__ P, GroupSmem<T>& __restrict__ S, const Grp<GW>& g, Mb& M, int r) {
    const int lam = P.lambda;
    int rb = 0;
    if (P.nact == 2) rb = lam;  // ref_bits, enc/frame.rs:705-711
    else if (P.nact > 2) rb = lam * (2 * (31 - __clz(r + 1)) + 1);
    const int2 mvp = pred_mv_g(S.ext, nullptr, 0, 0, 4, 0, r);
    const ColMv col = P.col[M.mb];
    const int3 ms = msearch<T, GW>(P, S, g, M, r, 0, 0, 4, 4, mvp.x, mvp.y, col.mv[0], col.mv[1], 0, 0, col.valid ? 1 : 0);
    const int mx = ms.y, my = ms.z;
    int best_part = 0, best_cost = ms.x + lam * (mvd_bits_d(mx, my, mvp.x, mvp.y) + 1) + rb;
    const int cost16 = best_cost;
    uint32_t sub_out = 0;
    const uint32_t mv16 = (uint32_t)(uint16_t)mx | ((uint32_t)(uint16_t)my << 16);
#pragma unroll
    for (int k = 0; k < 16 / GW; k++) *reinterpret_cast<uint32_t*>(&S.best_mvs[g.gl + GW * k][0]) = mv16;
    __syncwarp(g.mask);
    if (P.fast) return make_int4(best_cost, 0, 0, cost16);
    // P_8x8 (868-876)
    blk_clear_g(g, S.st);
    uint32_t sub = 0;
    int cost8 = lam * 9;
    for (int k = 0; k < 4; k++) {
        const int2 ss = sub_search_g<T, GW>(P, S, g, M, r, k, mx, my);
        sub |= (uint32_t)ss.x << (8 * k);
        cost8 += ss.y + rb;
        if (cost8 >= best_cost) break;
    }
    if (cost8 < best_cost) {
        // v8: the vectors of rects(3, sub) in coding order (882-885)
        if (g.gl == 0) {
            int n = 0;
            for (int k = 0; k < 4; k++) {
                const int s = (sub >> (8 * k)) & 0xff;
                for (int q = 0; q < c_nsub[s]; q++) {
                    const int x = (k & 1) * 2 + c_sub[s][q][0], y = (k >> 1) * 2 + c_sub[s][q][1];
                    S.best_mvs[n][0] = (int16_t)S.st[y * 4 + x].x;
                    S.best_mvs[n][1] = (int16_t)S.st[y * 4 + x].y;
                    n++;
                }
            }
            for (; n < 16; n++) S.best_mvs[n][0] = S.best_mvs[n][1] = 0;
        }
        __syncwarp(g.mask);
        best_part = 3;
        best_cost = cost8;
        sub_out = sub;
        // 16x8 and 8x16 (886-903), with the 8x8 blocks' vectors as candidates
        for (int part = 1; part < 3; part++) {
            int pc = lam * 3;
            int m0x = 0, m0y = 0, m1x = 0, m1y = 0;
            bool complete = true;
            for (int k = 0; k < 2; k++) {
                // part_mvps (579-594): partition k's predictor given the vectors before it
                if (k == 1) {
                    blk_clear_g(g, S.t);
                    blk_paint_g(g, S.t, c_parts[part][0][0], c_parts[part][0][1], c_parts[part][0][2], c_parts[part][0][3], m0x, m0y, r);
                }
                const int x = c_parts[part][k][0], y = c_parts[part][k][1], w = c_parts[part][k][2], h = c_parts[part][k][3];
                const int2 p = pred_mv_g(S.ext, k == 0 ? nullptr : S.t, x, y, w, part, r);
                const int i0 = part == 1 ? 2 * k : k, i1 = part == 1 ? 2 * k + 1 : k + 2;
                const Blk a0 = S.st[(i0 / 2) * 8 + (i0 % 2) * 2], a1 = S.st[(i1 / 2) * 8 + (i1 % 2) * 2];
                const int3 m = msearch<T, GW>(P, S, g, M, r, x, y, w, h, p.x, p.y, a0.x, a0.y, a1.x, a1.y, 2);
                if (k == 0) {
                    m0x = m.y;
                    m0y = m.z;
                } else {
                    m1x = m.y;
                    m1y = m.z;
                }
                pc += m.x + lam * mvd_bits_d(m.y, m.z, p.x, p.y) + rb;
                if (pc >= best_cost) {
                    complete = false;
                    break;
                }
            }
            if (complete && pc < best_cost) {
                best_part = part;
                best_cost = pc;
                sub_out = 0;
#pragma unroll
                for (int k = 0; k < 16 / GW; k++) {
                    const int i = g.gl + GW * k;
                    uint32_t v = 0;
                    if (i == 0) v = (uint32_t)(uint16_t)m0x | ((uint32_t)(uint16_t)m0y << 16);
                    else if (i == 1) v = (uint32_t)(uint16_t)m1x | ((uint32_t)(uint16_t)m1y << 16);
                    *reinterpret_cast<uint32_t*>(&S.best_mvs[i][0]) = v;
                }
                __syncwarp(g.mask);
            }
        }
    }
    return make_int4(best_cost, best_part, (int)sub_out, cost16);
}

// The macroblock's source rows into the group's shared memory (16 rows of 16 * sizeof(T) bytes, as 128-bit
// loads) and the table of its neighbours' blocks from the caller's final decisions (load_neighbours).
template <class T, int GW>
__device__ __forceinline__ void stage_g(const AnalyseParams& __restrict__ P, GroupSmem<T>& __restrict__ S, const Grp<GW>& g, const Mb& M,
                                        const ironav_mbstate* __restrict__ states) {
    constexpr int B = sizeof(T);
#pragma unroll
    for (int k = 0; k < 16 * B / GW; k++) {
        const int i = g.gl + GW * k, row = i / B, part = i % B;
        const uint4 v = *reinterpret_cast<const uint4*>(P.src + ((size_t)(M.mby * 16 + row) * P.ls + M.mbx * 16) * B + part * 16);
        *reinterpret_cast<uint4*>(&S.src[i * 4]) = v;
    }
#pragma unroll
    for (int k = 0; k < (30 + GW - 1) / GW; k++) {
        const int i = g.gl + GW * k;
        if (i < 30) {
            const int ex = i % 6 - 1, ey = i / 6 - 1;
            Blk e = make_int4(0, 0, -1, 0);
            if (ey < 0 || ex < 0) {
                const int nx = M.mbx + (ex < 0 ? -1 : (ex >= 4 ? 1 : 0)), ny = M.mby + (ey < 0 ? -1 : 0);
                const int bx = ex < 0 ? 3 : (ex >= 4 ? 0 : ex), by = ey < 0 ? 3 : ey;
                // macroblocks of earlier slices are not available (enc/frame.rs:509-515)
                if (nx >= 0 && nx < P.mb_w && ny >= P.band_start[M.mby] && ny < P.mb_h) {
                    const ironav_mbstate* st = &states[(size_t)ny * P.mb_w + nx];
                    e.w = 1;
                    const int rf = st->refs[(by >> 1) * 2 + (bx >> 1)];
                    if (st->inter && rf >= 0) {
                        const uint32_t mv = *reinterpret_cast<const uint32_t*>(&st->mvs[by * 4 + bx][0]);
                        e.x = (int)(int16_t)(mv & 0xffffu);
                        e.y = (int)(int16_t)(mv >> 16);
                        e.z = rf;
                    }
                }
            }
            S.ext[i] = e;
        }
    }
    __syncwarp(g.mask);
}

// One macroblock (enc/frame.rs:722-729 and best_inter, 839-849): the P_Skip vector and SAD, then every
// reference's best_inter_ref, the cheapest (first on ties) winning; the result record. Replay mode reads the
// neighbours from the caller's decisions; AUTO (auto mode) reads them from the decisions already published,
// stops at the P_Skip test when its SAD is under the threshold, and writes the macroblock's own decision
// (its MbState, finish_mb, enc/frame.rs:2281-2321) for the macroblocks after it.
template <class T, int GW, bool AUTO = false>
__device__ __forceinline__ void analyse_mb_g(const AnalyseParams& __restrict__ P, GroupSmem<T>& __restrict__ S, const Grp<GW>& g, Mb& M) {
    stage_g<T, GW>(P, S, g, M, AUTO ? P.states_out : P.states_in);
    // P_Skip (skip_mv, enc/frame.rs:597-603; the SAD of its prediction, 722-729)
    int2 sv = make_int2(0, 0);
    {
        const Blk a = nb_g(S.ext, nullptr, -1, 0), b = nb_g(S.ext, nullptr, 0, -1);
        if (!(!a.w || !b.w || (a.z == 0 && a.x == 0 && a.y == 0) || (b.z == 0 && b.x == 0 && b.y == 0)))
            sv = pred_mv_g(S.ext, nullptr, 0, 0, 4, 0, 0);
    }
    pred_points<T, GW>(P, S, g, M.mbx, M.mby, 0, 0, 0, 2, 2, [&](int) { return sv; }, 1, true);
    const int skip_sad = S.cost[0];
    M.sad_px += 256;
    __syncwarp(g.mask);
    const bool skip = AUTO && skip_sad < P.skip_thresh;
    int part = 0, cost = 0, cost16 = 0, bestr = 0;
    uint32_t sub = 0;
    for (int r = 0; r < (skip ? 0 : P.nact); r++) {
        const int4 bi = best_inter_ref_g<T, GW>(P, S, g, M, r);
        if (r == 0 || bi.x < cost) {
            cost = bi.x;
            part = bi.y;
            sub = (uint32_t)bi.z;
            cost16 = bi.w;
            bestr = r;
#pragma unroll
            for (int k = 0; k < 16 / GW; k++)
                *reinterpret_cast<uint32_t*>(&S.win_mvs[g.gl + GW * k][0]) = *reinterpret_cast<const uint32_t*>(&S.best_mvs[g.gl + GW * k][0]);
            __syncwarp(g.mask);
        }
    }
    ironav_mbresult& R = S.res;
    if (g.gl == 0) {
        R.skip_mv[0] = (int16_t)sv.x;
        R.skip_mv[1] = (int16_t)sv.y;
        R.skip_sad = skip_sad;
        R.part = (uint8_t)part;
        for (int i = 0; i < 4; i++) {
            R.refs[i] = (uint8_t)bestr;
            R.sub[i] = (uint8_t)((sub >> (8 * i)) & 0xff);
        }
        R.flags = skip ? IRONAV_RESULT_SKIP : IRONAV_RESULT_INTER;
        R.pad[0] = R.pad[1] = 0;
        R.cost = cost;
        R.cost16 = cost16;
        R.sad_px = M.sad_px;
        R.satd_px = M.satd_px;
        R.pad2 = 0;
    }
#pragma unroll
    for (int k = 0; k < 16 / GW; k++)
        *reinterpret_cast<uint32_t*>(&R.mvs[g.gl + GW * k][0]) = skip ? 0u : *reinterpret_cast<const uint32_t*>(&S.win_mvs[g.gl + GW * k][0]);
    __syncwarp(g.mask);
    if constexpr (AUTO) {
        // the decision's MbState: the vector of the rectangle of rects(part, sub) holding each 4x4 block, the
        // reference of each 8x8 block
        uint32_t* so = reinterpret_cast<uint32_t*>(&P.states_out[M.mb]);
#pragma unroll
        for (int k = 0; k < 16 / GW; k++) {
            const int i = g.gl + GW * k, bx = i & 3, by = i >> 2;
            uint32_t mv = (uint32_t)(uint16_t)sv.x | ((uint32_t)(uint16_t)sv.y << 16);
            if (!skip) {
                int idx = 0;
                if (part == 1) idx = by >> 1;
                else if (part == 2) idx = bx >> 1;
                else if (part == 3) {
                    const int kk = (by >> 1) * 2 + (bx >> 1);
                    int n = 0;
                    for (int q = 0; q < kk; q++) n += c_nsub[(sub >> (8 * q)) & 0xff];
                    const int s8 = (sub >> (8 * kk)) & 0xff, lx = bx & 1, ly = by & 1;
                    idx = n + (s8 == 0 ? 0 : (s8 == 1 ? ly : (s8 == 2 ? lx : ly * 2 + lx)));
                }
                mv = *reinterpret_cast<const uint32_t*>(&S.win_mvs[idx][0]);
            }
            so[2 + i] = mv;
        }
        if (g.gl == 0) {
            const uint32_t rf = (uint32_t)(uint8_t)(int8_t)(skip ? 0 : bestr);
            so[0] = 1u | (rf << 8) | (rf << 16) | (rf << 24);  // inter, refs[0..2]
            so[1] = rf;                                         // refs[3], pad
        }
    }
    uint32_t* out = reinterpret_cast<uint32_t*>(&P.results[M.mb]);
    const uint32_t* in = reinterpret_cast<const uint32_t*>(&R);
#pragma unroll
    for (int k = 0; k < (26 + GW - 1) / GW; k++)
        if (g.gl + GW * k < 26) out[g.gl + GW * k] = in[g.gl + GW * k];
    __syncwarp(g.mask);
}

// K2 in replay mode: a warp takes 32 / GW tickets at a time, one macroblock per group of GW lanes.
template <class T, int GW>
__global__ void __launch_bounds__(warps_for(GW) * 32, MIN_BLOCKS * WARPS / warps_for(GW)) analyse_replay_g8_kernel(const __grid_constant__ AnalyseParams P) {
    constexpr int MBS = 32 / GW;  // macroblocks a warp
    __shared__ GroupSmem<T> smem[warps_for(GW) * MBS];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const Grp<GW> g = grp_of_lane<GW>();
    GroupSmem<T>& S = smem[wid * MBS + lane / GW];
    for (;;) {
        unsigned t = 0;
        if (lane == 0) t = atomicAdd(P.ticket, (unsigned)MBS);
        t = __shfl_sync(FULL, t, 0);
        if (t >= (unsigned)P.nmb) break;
        const unsigned mt = t + (unsigned)(lane / GW);
        if (mt < (unsigned)P.nmb) {
            Mb M;
            M.mb = P.order ? P.order[mt] : (int)mt;
            M.mbx = M.mb % P.mb_w;
            M.mby = M.mb / P.mb_w;
            M.sad_px = M.satd_px = 0;
            analyse_mb_g<T, GW>(P, S, g, M);
        }
        __syncwarp();
    }
}

// Every stream's auto-mode analysis in one launch with one macroblock per 8-lane group (the batched form's
// group variant): a warp takes four tickets of the merged wavefront order; each group looks its stream up in
// the table, waits (bounded) until its left and top-right neighbours are published, analyses its macroblock and
// publishes it. A group may wait on another group of its own warp (tickets of one block can follow each other
// in a stream's wavefront); no barrier of the whole warp sits between a group's wait and its publication, so the
// waiting group never holds the other back.
template <class T>
__global__ void __launch_bounds__(WARPS * 32, MIN_BLOCKS) analyse_batch_g8_kernel(const AnalyseParams* __restrict__ table,
                                                                                  const uint32_t* __restrict__ order, unsigned ntickets,
                                                                                  unsigned* ticket, const unsigned* err) {
    __shared__ GroupSmem<T> smem[WARPS * 4];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const Grp<8> g = grp_of_lane<8>();
    GroupSmem<T>& S = smem[wid * 4 + (lane >> 3)];
    for (;;) {
        unsigned t = 0;
        if (lane == 0) t = atomicAdd(ticket, 4u);
        t = __shfl_sync(FULL, t, 0);
        if (t >= ntickets || ld_acquire(err) != 0) break;
        const unsigned mt = t + (unsigned)(lane >> 3);
        if (mt < ntickets) {
            const uint32_t e = order[mt];
            const AnalyseParams& P = table[e >> 20];
            Mb M;
            M.mb = (int)(e & 0xFFFFFu);
            M.mbx = M.mb % P.mb_w;
            M.mby = M.mb / P.mb_w;
            M.sad_px = M.satd_px = 0;
            const int start = P.band_start[M.mby];
            bool ok = true;
            if (M.mbx > 0) ok = wait_published(P, M.mb - 1);
            if (ok && M.mby > start) ok = wait_published(P, (M.mbx + 1 < P.mb_w) ? M.mb - P.mb_w + 1 : M.mb - P.mb_w);
            ok = __all_sync(g.mask, ok);
            if (ok) {
                analyse_mb_g<T, 8, true>(P, S, g, M);
                __threadfence();
                __syncwarp(g.mask);
                if (g.gl == 0) st_release(&P.flags[M.mb], P.epoch);
            }
        }
        __syncwarp();
    }
}

}  // namespace g8
}  // namespace ironav
