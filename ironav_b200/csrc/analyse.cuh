// analyse.cuh — K2: P-macroblock inter analysis (P_Skip vector + SAD, best_inter with its motion
// searches), one warp per macroblock.
//
// The reference's analysis of a macroblock (enc/frame.rs:722-729, 839-1019) is a sequential,
// data-dependent search. Here every lane of a warp runs the same control flow (all decisions are
// warp-uniform) and the sample work of each step is spread over the lanes:
//   - integer SAD: a batch of up to 8 candidate vectors at once, lanes split over (candidate,
//     8-sample row chunk); reference rows read as aligned 32-bit words and realigned with funnel
//     shifts, compared with __vsadu4; per-candidate sums by xor shuffles;
//   - sub-sample SATD: a batch of up to 9 vectors, lanes split over (vector, 4x4 block); the
//     quarter-sample prediction is __vavgu4 of two half-sample planes; 4x4 Hadamard in registers;
//   - the diamond's greedy rounds are resolved exactly: the 4 points around the round's centre are
//     scored as one batch, then the reference's order of moves (left, right, up, down, each from the
//     current best, strict '<') is replayed against a small table of scored points; a point the
//     table lacks (the y-phase after an x move, or a clamp at the search bounds) is scored on demand.
// The result is the same vector, cost, partition and evaluation count as the sequential code.
//
// Replay mode reads each macroblock's neighbours from the caller's final decisions, so every
// macroblock is independent. Auto mode decides each macroblock with the analysis policy and publishes
// its decision; a macroblock first waits (bounded) until its left and top-right neighbours are
// published, in tickets handed out in wavefront order so a waiting warp only ever waits on warps that
// hold smaller tickets and are already running.
#pragma once
#include "common.cuh"

namespace ironav {

constexpr int K2_WARPS = 4;  // warps per CTA; each warp works alone
constexpr unsigned FULL = 0xffffffffu;

// MIX, enc/subpel.rs:26-38, packed per [fy][fx]: pa | ax<<2 | ay<<3 | pb<<4 | bx<<6 | by<<7
static __constant__ uint8_t c_mix[16] = {
    0x00, 0x10, 0x11, 0x14,
    0x20, 0x21, 0x31, 0x61,
    0x22, 0x32, 0x33, 0x63,
    0x28, 0x92, 0x93, 0x96,
};

struct Rect4 {
    int x, y, w, h;
};

static __device__ __constant__ int8_t c_parts[4][4][4] = {
    {{0, 0, 4, 4}}, {{0, 0, 4, 2}, {0, 2, 4, 2}}, {{0, 0, 2, 4}, {2, 0, 2, 4}}, {{0, 0, 2, 2}, {2, 0, 2, 2}, {0, 2, 2, 2}, {2, 2, 2, 2}}};
static __device__ __constant__ int8_t c_sub[4][4][4] = {
    {{0, 0, 2, 2}}, {{0, 0, 2, 1}, {0, 1, 2, 1}}, {{0, 0, 1, 2}, {1, 0, 1, 2}}, {{0, 0, 1, 1}, {1, 0, 1, 1}, {0, 1, 1, 1}, {1, 1, 1, 1}}};
static __device__ __constant__ int8_t c_nsub[4] = {1, 2, 2, 4};

// Vector state of the 4x4 blocks of the macroblock being analysed (nb_motion's cur/cref/done).
struct BlkState {
    int16_t mv[16][2];
    int8_t ref[16];
    uint32_t done;
};

// Per-warp shared memory.
struct WarpSmem {
    uint32_t src[64];          // current macroblock, 16 rows x 4 words
    ironav_mbstate nb[4];      // neighbours: 0 left (A), 1 top (B), 2 top-right (C), 3 top-left (D)
    int nb_avail[4];
    int2 cand[16];             // the batch being scored
    int cost[16];
    uint32_t ckey[12];         // scored points of the current diamond round
    int cval[12];
    BlkState st;               // P_8x8 blocks decided so far (sub_search's `st`)
    BlkState t;                // trial state (sub_search's `t`, part_mvps's `cur`)
    BlkState bt;               // best trial
    int16_t best_mvs[16][2];   // best_inter_ref's running best, in coding order
    int16_t win_mvs[16][2];    // best over the references
    int16_t half_mvs[16][2];   // 16x8 / 8x16 vectors being searched
    ironav_mbresult res;
    ironav_mbstate out;
};

__device__ __forceinline__ int ue_bits_d(unsigned v) { return 2 * (32 - __clz(v + 1)) - 1; }  // enc/bitw.rs:81-83
__device__ __forceinline__ int se_bits_d(int v) {                                             // enc/bitw.rs:86-89
    return ue_bits_d(v > 0 ? 2u * (unsigned)v - 1u : (unsigned)(-2 * v));
}
__device__ __forceinline__ int mvd_bits_d(int mx, int my, int px, int py) { return se_bits_d(mx - px) + se_bits_d(my - py); }
__device__ __forceinline__ int median3_d(int a, int b, int c) { return min(max(a, b), max(min(a, b), c)); }

// 4 bytes at any address, as aligned 32-bit loads and a funnel shift.
__device__ __forceinline__ uint32_t ldu32(const uint8_t* p) {
    uintptr_t a = reinterpret_cast<uintptr_t>(p);
    const uint32_t* q = reinterpret_cast<const uint32_t*>(a & ~uintptr_t(3));
    return __funnelshift_r(__ldg(q), __ldg(q + 1), (unsigned)(a & 3) * 8u);
}

__device__ __forceinline__ int satd4_d(const int d[16]) {  // satd4, enc/frame.rs:144-161
    int t[16];
#pragma unroll
    for (int r = 0; r < 4; r++) {
        int a = d[r * 4], b = d[r * 4 + 1], c = d[r * 4 + 2], e = d[r * 4 + 3];
        int s0 = a + b, s1 = c + e, d0 = a - b, d1 = c - e;
        t[r * 4] = s0 + s1;
        t[r * 4 + 1] = s0 - s1;
        t[r * 4 + 2] = d0 - d1;
        t[r * 4 + 3] = d0 + d1;
    }
    int sum = 0;
#pragma unroll
    for (int c = 0; c < 4; c++) {
        int a = t[c], b = t[4 + c], cc = t[8 + c], e = t[12 + c];
        int s0 = a + b, s1 = cc + e, d0 = a - b, d1 = cc - e;
        sum += abs(s0 + s1) + abs(s0 - s1) + abs(d0 - d1) + abs(d0 + d1);
    }
    return sum >> 1;
}

struct Nb {
    int avail, ref, mx, my;
};

class MbWarp {
  public:
    const AnalyseParams& P;
    WarpSmem& S;
    const int lane;
    int mbx, mby, mb;
    uint32_t sad_px, satd_px;

    __device__ MbWarp(const AnalyseParams& p, WarpSmem& s, int l) : P(p), S(s), lane(l) {}

    // ---- neighbours (nb_state / nb_motion, enc/frame.rs:509-538) ----------------------------------

    __device__ void load_neighbours(const ironav_mbstate* states) {
        const int start = P.band_start[mby];
        const int nx[4] = {mbx - 1, mbx, mbx + 1, mbx - 1}, ny[4] = {mby, mby - 1, mby - 1, mby - 1};
        // 4 states x 18 words
        for (int i = lane; i < 4 * 18; i += 32) {
            int k = i / 18, wd = i % 18;
            bool ok = nx[k] >= 0 && ny[k] >= start && nx[k] < P.mb_w && ny[k] < P.mb_h;
            uint32_t v = 0;
            if (ok) v = reinterpret_cast<const uint32_t*>(&states[(size_t)ny[k] * P.mb_w + nx[k]])[wd];
            reinterpret_cast<uint32_t*>(&S.nb[k])[wd] = v;
            if (wd == 0) S.nb_avail[k] = ok;
        }
        __syncwarp();
    }

    // (x, y) in 4x4 blocks relative to the macroblock; inside it, `cur` holds the decided blocks.
    __device__ Nb nb_motion(const BlkState* cur, int x, int y) const {
        Nb r = {0, -1, 0, 0};
        int k, bx, by;
        if (x < 0 && y < 0) { k = 3; bx = 3; by = 3; }
        else if (x < 0) { k = 0; bx = 3; by = y; }
        else if (x >= 4 && y < 0) { k = 2; bx = 0; by = 3; }
        else if (x >= 4) return r;
        else if (y < 0) { k = 1; bx = x; by = 3; }
        else {
            int b = y * 4 + x;
            if (cur && ((cur->done >> b) & 1)) {
                r.avail = 1;
                r.ref = cur->ref[b];
                r.mx = cur->mv[b][0];
                r.my = cur->mv[b][1];
            }
            return r;
        }
        if (!S.nb_avail[k]) return r;
        r.avail = 1;
        const ironav_mbstate& s = S.nb[k];
        int rf = s.refs[(by / 2) * 2 + bx / 2];
        if (s.inter && rf >= 0) {
            r.ref = rf;
            r.mx = s.mvs[by * 4 + bx][0];
            r.my = s.mvs[by * 4 + bx][1];
        }
        return r;
    }

    // pred_mv, enc/frame.rs:543-570
    __device__ __noinline__ void pred_mv(const BlkState* cur, int bx, int by, int w, int dir, int rf, int& ox, int& oy) const {
        Nb a = nb_motion(cur, bx - 1, by);
        Nb b = nb_motion(cur, bx, by - 1);
        Nb c = nb_motion(cur, bx + w, by - 1);
        if (!c.avail) c = nb_motion(cur, bx - 1, by - 1);
        if (dir == 1 && by == 0 && b.ref == rf) { ox = b.mx; oy = b.my; return; }
        if (dir == 1 && by != 0 && a.ref == rf) { ox = a.mx; oy = a.my; return; }
        if (dir == 2 && bx == 0 && a.ref == rf) { ox = a.mx; oy = a.my; return; }
        if (dir == 2 && bx != 0 && c.ref == rf) { ox = c.mx; oy = c.my; return; }
        if (!b.avail && !c.avail && a.avail) { ox = a.mx; oy = a.my; return; }
        int ra = a.ref == rf, rb = b.ref == rf, rc = c.ref == rf;
        if (ra + rb + rc == 1) {
            if (ra) { ox = a.mx; oy = a.my; }
            else if (rb) { ox = b.mx; oy = b.my; }
            else { ox = c.mx; oy = c.my; }
            return;
        }
        ox = median3_d(a.mx, b.mx, c.mx);
        oy = median3_d(a.my, b.my, c.my);
    }

    // skip_mv, enc/frame.rs:597-603
    __device__ void skip_mv(int& ox, int& oy) const {
        Nb a = nb_motion(nullptr, -1, 0), b = nb_motion(nullptr, 0, -1);
        if (!a.avail || !b.avail || (a.ref == 0 && a.mx == 0 && a.my == 0) || (b.ref == 0 && b.mx == 0 && b.my == 0)) {
            ox = oy = 0;
            return;
        }
        pred_mv(nullptr, 0, 0, 4, 0, 0, ox, oy);
    }

    // ---- scoring -------------------------------------------------------------------------------------

    // Integer SAD (sad_int, enc/frame.rs:662-671) + lambda * mvd_bits of S.cand[0..n) -> S.cost.
    __device__ __noinline__ void sad_batch(int r, int bx, int by, int w, int h, int n, int mvpx, int mvpy) {
        const int cb = n <= 1 ? 0 : (n <= 2 ? 1 : (n <= 4 ? 2 : 3));
        const int c = lane & ((1 << cb) - 1), rg = lane >> cb, nrg = 32 >> cb;
        const int cpr = w >= 16 ? 2 : 1;           // 8-sample chunks per row (4-sample rows when w == 4)
        const int ntask = h * cpr;
        const int x0 = mbx * 16 + bx * 4, y0 = mby * 16 + by * 4;
        int sad = 0;
        int2 mv = make_int2(0, 0);
        if (c < n) {
            mv = S.cand[c];
            const uint8_t* G = P.planes[r] + (long long)(y0 + (mv.y >> 2) + PAD) * P.sw + (x0 + (mv.x >> 2) + PAD);
            for (int i = rg; i < ntask; i += nrg) {
                const int row = cpr == 2 ? (i >> 1) : i, cc = cpr == 2 ? (i & 1) : 0;
                const uint8_t* p = G + (long long)row * P.sw + cc * 8;
                uintptr_t a = reinterpret_cast<uintptr_t>(p);
                const uint32_t* q = reinterpret_cast<const uint32_t*>(a & ~uintptr_t(3));
                const unsigned sh = (unsigned)(a & 3) * 8u;
                const uint32_t* s = &S.src[(by * 4 + row) * 4 + bx + cc * 2];
                uint32_t w0 = __ldg(q), w1 = __ldg(q + 1);
                sad += __vsadu4(s[0], __funnelshift_r(w0, w1, sh));
                if (w >= 8) {
                    uint32_t w2 = __ldg(q + 2);
                    sad += __vsadu4(s[1], __funnelshift_r(w1, w2, sh));
                }
            }
        }
#pragma unroll
        for (int off = 16; off >= 1; off >>= 1)
            if (off >= (1 << cb)) sad += __shfl_xor_sync(FULL, sad, off);
        if (rg == 0 && c < n) S.cost[c] = sad + P.lambda * mvd_bits_d(mv.x, mv.y, mvpx, mvpy);
        __syncwarp();
    }

    // Quarter-sample prediction (HalfPel::predict, enc/subpel.rs:122-145) scored by SATD (satd,
    // enc/frame.rs:641-659) + lambda * mvd_bits, or by SAD when `sad` (the P_Skip test), for
    // S.cand[0..n) -> S.cost.
    __device__ __noinline__ void pred_batch(int r, int bx, int by, int w, int h, int n, int mvpx, int mvpy, bool sad) {
        const int nbw = w >> 2, nblk = nbw * (h >> 2), total = n * nblk;
        if (lane < n) S.cost[lane] = 0;
        __syncwarp();
        const int x0 = mbx * 16 + bx * 4, y0 = mby * 16 + by * 4;
        const uint8_t* base = P.planes[r];
        for (int t = lane; t < total; t += 32) {
            const int c = t / nblk, b = t - c * nblk, bxx = b % nbw, byy = b / nbw;
            const int2 mv = S.cand[c];
            const int ix = min(max(x0 + (mv.x >> 2), -w - 3), P.pw + 1);
            const int iy = min(max(y0 + (mv.y >> 2), -h - 3), P.ph + 1);
            const unsigned m = c_mix[(mv.y & 3) * 4 + (mv.x & 3)];
            const int pa = m & 3, ax = (m >> 2) & 1, ay = (m >> 3) & 1, pb = (m >> 4) & 3, bbx = (m >> 6) & 1, bby = (m >> 7) & 1;
            const bool same = (m & 0xf) == (m >> 4);
            const long long ox = ix + PAD + bxx * 4, oy = iy + PAD + byy * 4;
            const uint8_t* A = base + pa * P.psize + (oy + ay) * P.sw + ox + ax;
            const uint8_t* B = base + pb * P.psize + (oy + bby) * P.sw + ox + bbx;
            const uint32_t* s = &S.src[(by * 4 + byy * 4) * 4 + bx + bxx];
            int v;
            if (sad) {
                v = 0;
#pragma unroll
                for (int row = 0; row < 4; row++) {
                    uint32_t wa = ldu32(A + row * P.sw);
                    uint32_t wp = same ? wa : __vavgu4(wa, ldu32(B + row * P.sw));
                    v += __vsadu4(s[row * 4], wp);
                }
            } else {
                int d[16];
#pragma unroll
                for (int row = 0; row < 4; row++) {
                    uint32_t wa = ldu32(A + row * P.sw);
                    uint32_t wp = same ? wa : __vavgu4(wa, ldu32(B + row * P.sw));
                    uint32_t ws = s[row * 4];
#pragma unroll
                    for (int k = 0; k < 4; k++) d[row * 4 + k] = (int)((ws >> (8 * k)) & 255u) - (int)((wp >> (8 * k)) & 255u);
                }
                v = satd4_d(d);
            }
            atomicAdd(&S.cost[c], v);
        }
        __syncwarp();
        if (lane < n && !sad) S.cost[lane] += P.lambda * mvd_bits_d(S.cand[lane].x, S.cand[lane].y, mvpx, mvpy);
        __syncwarp();
    }

    // ---- motion_search, enc/frame.rs:949-1019 --------------------------------------------------------

    __device__ __noinline__ int motion_search(int r, Rect4 pr, int mvpx, int mvpy, const int2* extra, int nextra, int& ox, int& oy) {
        const int lam = P.lambda;
        const int x0 = mbx * 16 + pr.x * 4, y0 = mby * 16 + pr.y * 4, w = pr.w * 4, h = pr.h * 4;
        const int cxlo = max(-(x0 + 24) * 4, -2048), cxhi = min((P.mb_w * 16 - x0 + 8) * 4, 2047);
        const int cylo = max(-(y0 + 24) * 4, -512), cyhi = min((P.mb_h * 16 - y0 + 8) * 4, 511);
        auto clx = [&](int v) { return min(max(v, cxlo), cxhi); };
        auto cly = [&](int v) { return min(max(v, cylo), cyhi); };
        auto intr = [](int v) { return (v + 2) & ~3; };
        // candidates (958-964)
        int n = 0;
        int2 cands[8];
        cands[n++] = make_int2(intr(clx(mvpx)), intr(cly(mvpy)));
        cands[n++] = make_int2(0, 0);
        {
            Nb a = nb_motion(nullptr, -1, 0), b = nb_motion(nullptr, 0, -1), c = nb_motion(nullptr, 4, -1);
            if (a.avail && a.ref == r) cands[n++] = make_int2(intr(clx(a.mx)), intr(cly(a.my)));
            if (b.avail && b.ref == r) cands[n++] = make_int2(intr(clx(b.mx)), intr(cly(b.my)));
            if (c.avail && c.ref == r) cands[n++] = make_int2(intr(clx(c.mx)), intr(cly(c.my)));
        }
        for (int k = 0; k < nextra; k++) cands[n++] = make_int2(intr(clx(extra[k].x)), intr(cly(extra[k].y)));
        if (lane < 8) {
            int2 v = cands[0];
#pragma unroll
            for (int k = 1; k < 8; k++)
                if (lane == k) v = cands[k];
            S.cand[lane] = v;
        }
        __syncwarp();
        sad_batch(r, pr.x, pr.y, w, h, n, mvpx, mvpy);
        sad_px += (uint32_t)(n * w * h);
        int bx = 0, by = 0, bc = 0x7fffffff;
        for (int k = 0; k < n; k++) {
            int cost = S.cost[k];
            if (cost < bc) {
                bx = cands[k].x;
                by = cands[k].y;
                bc = cost;
            }
        }
        // diamond (973-988)
        const int nsteps = P.fast ? 2 : 3;
        for (int si = 0; si < nsteps; si++) {
            const int step = P.fast ? (si == 0 ? 8 : 4) : (16 >> si);
            const int iters = step == 4 ? 32 : 4;
            for (int it = 0; it < iters; it++) {
                // score the 4 points around the round's centre as one batch
                const int cx = bx, cy = by;
                if (lane < 4) {
                    int2 v;
                    if (lane == 0) v = make_int2(clx(cx - step), cy);
                    else if (lane == 1) v = make_int2(clx(cx + step), cy);
                    else if (lane == 2) v = make_int2(cx, cly(cy - step));
                    else v = make_int2(cx, cly(cy + step));
                    S.cand[lane] = v;
                }
                __syncwarp();
                sad_batch(r, pr.x, pr.y, w, h, 4, mvpx, mvpy);
                int nk = 0;
                auto key = [](int x, int y) { return ((uint32_t)x & 0xffffu) | ((uint32_t)y << 16); };
                // the table of scored points (uniform writes: every lane stores the same value)
                S.ckey[nk] = key(cx, cy);
                S.cval[nk] = bc;
                nk++;
                for (int k = 0; k < 4; k++) {
                    int2 v = S.cand[k];
                    S.ckey[nk] = key(v.x, v.y);
                    S.cval[nk] = S.cost[k];
                    nk++;
                }
                __syncwarp();
                auto lookup = [&](int x, int y, int& cost) {
                    uint32_t kk = key(x, y);
                    for (int i = 0; i < nk; i++)
                        if (S.ckey[i] == kk) {
                            cost = S.cval[i];
                            return true;
                        }
                    return false;
                };
                auto score = [&](int x, int y) {
                    int cost;
                    if (lookup(x, y, cost)) return cost;
                    if (lane == 0) S.cand[0] = make_int2(x, y);
                    __syncwarp();
                    sad_batch(r, pr.x, pr.y, w, h, 1, mvpx, mvpy);
                    cost = S.cost[0];
                    if (nk < 12) {
                        S.ckey[nk] = key(x, y);
                        S.cval[nk] = cost;
                        nk++;
                    }
                    __syncwarp();
                    return cost;
                };
                bool moved = false;
                // (-step, 0) then (step, 0) from the current best
                {
                    int px = clx(bx - step), py = by;
                    int cost = score(px, py);
                    if (cost < bc) { bx = px; by = py; bc = cost; moved = true; }
                    px = clx(bx + step);
                    py = by;
                    cost = score(px, py);
                    if (cost < bc) { bx = px; by = py; bc = cost; moved = true; }
                }
                // after an x move the y-phase points are new: score both as one batch
                if (bx != cx) {
                    int2 e0 = make_int2(bx, cly(by - step)), e1 = make_int2(bx, cly(by + step));
                    int tmp;
                    bool h0 = lookup(e0.x, e0.y, tmp), h1 = lookup(e1.x, e1.y, tmp);
                    if (!h0 || !h1) {
                        int m = 0;
                        if (!h0) { if (lane == 0) S.cand[m] = e0; m++; }
                        if (!h1) { if (lane == 0) S.cand[m] = e1; m++; }
                        __syncwarp();
                        sad_batch(r, pr.x, pr.y, w, h, m, mvpx, mvpy);
                        int q = 0;
                        if (!h0) { S.ckey[nk] = key(e0.x, e0.y); S.cval[nk] = S.cost[q++]; nk++; }
                        if (!h1) { S.ckey[nk] = key(e1.x, e1.y); S.cval[nk] = S.cost[q++]; nk++; }
                        __syncwarp();
                    }
                }
                {
                    int px = bx, py = cly(by - step);
                    int cost = score(px, py);
                    if (cost < bc) { bx = px; by = py; bc = cost; moved = true; }
                    px = bx;
                    py = cly(by + step);
                    cost = score(px, py);
                    if (cost < bc) { bx = px; by = py; bc = cost; moved = true; }
                }
                sad_px += (uint32_t)(4 * w * h);
                if (!moved) break;
            }
        }
        // live coding's early exit (990-992)
        if (P.fast && bc < (w * h) / 8 + lam) {
            ox = bx;
            oy = by;
            return bc - lam * mvd_bits_d(bx, by, mvpx, mvpy);
        }
        // sub-sample refinement (994-1017): the centre and the 8 half samples around it, as one batch
        {
            const int sq[8][2] = {{-1, -1}, {0, -1}, {1, -1}, {-1, 0}, {1, 0}, {-1, 1}, {0, 1}, {1, 1}};
            if (lane < 9) {
                int2 v = make_int2(bx, by);
#pragma unroll
                for (int k = 0; k < 8; k++)
                    if (lane == k + 1) v = make_int2(clx(bx + sq[k][0] * 2), cly(by + sq[k][1] * 2));
                S.cand[lane] = v;
            }
            __syncwarp();
            pred_batch(r, pr.x, pr.y, w, h, 9, mvpx, mvpy, false);
            satd_px += (uint32_t)(9 * w * h);
            bc = S.cost[0];
            for (int k = 1; k < 9; k++) {
                int cost = S.cost[k];
                if (cost < bc) {
                    bx = S.cand[k].x;
                    by = S.cand[k].y;
                    bc = cost;
                }
            }
        }
        if (!P.fast) {
            const int dm[4][2] = {{0, -1}, {-1, 0}, {1, 0}, {0, 1}};
            if (lane < 4) {
                int2 v = make_int2(0, 0);
#pragma unroll
                for (int k = 0; k < 4; k++)
                    if (lane == k) v = make_int2(clx(bx + dm[k][0]), cly(by + dm[k][1]));
                S.cand[lane] = v;
            }
            __syncwarp();
            pred_batch(r, pr.x, pr.y, w, h, 4, mvpx, mvpy, false);
            satd_px += (uint32_t)(4 * w * h);
            int nbx = bx, nby = by;
            for (int k = 0; k < 4; k++) {
                int cost = S.cost[k];
                if (cost < bc) {
                    nbx = S.cand[k].x;
                    nby = S.cand[k].y;
                    bc = cost;
                }
            }
            bx = nbx;
            by = nby;
        }
        __syncwarp();
        ox = bx;
        oy = by;
        return bc - lam * mvd_bits_d(bx, by, mvpx, mvpy);
    }

    // ---- partition decision ----------------------------------------------------------------------------

    __device__ void blk_clear(BlkState& b) {
        if (lane < 16) {
            b.mv[lane][0] = 0;
            b.mv[lane][1] = 0;
            b.ref[lane] = 0;
        }
        if (lane == 0) b.done = 0;
        __syncwarp();
    }
    __device__ void blk_copy(BlkState& d, const BlkState& s) {
        if (lane < 16) {
            d.mv[lane][0] = s.mv[lane][0];
            d.mv[lane][1] = s.mv[lane][1];
            d.ref[lane] = s.ref[lane];
        }
        if (lane == 0) d.done = s.done;
        __syncwarp();
    }
    // Marks rectangle (x, y, w, h) of `b` as decided with vector m and reference rf.
    __device__ void blk_paint(BlkState& b, Rect4 rr, int mx, int my, int rf) {
        if (lane < 16) {
            int bx = lane & 3, by = lane >> 2;
            if (bx >= rr.x && bx < rr.x + rr.w && by >= rr.y && by < rr.y + rr.h) {
                b.mv[lane][0] = (int16_t)mx;
                b.mv[lane][1] = (int16_t)my;
                b.ref[lane] = (int8_t)rf;
            }
        }
        __syncwarp();
        uint32_t bits = 0;
        for (int yy = rr.y; yy < rr.y + rr.h; yy++)
            for (int xx = rr.x; xx < rr.x + rr.w; xx++) bits |= 1u << (yy * 4 + xx);
        if (lane == 0) b.done |= bits;
        __syncwarp();
    }

    // sub_search, enc/frame.rs:911-938: returns sub_mb_type, cost in `cost`; leaves the block in S.st.
    __device__ __noinline__ int sub_search(int r, int k, int ex, int ey, int& cost_out) {
        const int lam = P.lambda;
        const int ox = (k & 1) * 2, oy = (k >> 1) * 2;
        const int ns = P.sub8 ? 4 : 1;
        int best_s = 0, best_cost = 0;
        for (int s = 0; s < ns; s++) {
            blk_copy(S.t, S.st);
            int cost = lam * (s == 0 ? 0 : 2);
            for (int q = 0; q < c_nsub[s]; q++) {
                Rect4 rr = {ox + c_sub[s][q][0], oy + c_sub[s][q][1], c_sub[s][q][2], c_sub[s][q][3]};
                int px, py, mx, my;
                pred_mv(&S.t, rr.x, rr.y, rr.w, 0, r, px, py);
                int2 extra = make_int2(ex, ey);
                int c = motion_search(r, rr, px, py, &extra, 1, mx, my);
                cost += c + lam * mvd_bits_d(mx, my, px, py);
                blk_paint(S.t, rr, mx, my, r);
            }
            if (s == 0 || cost < best_cost) {
                best_s = s;
                best_cost = cost;
                if (ns > 1) blk_copy(S.bt, S.t);
            }
        }
        blk_copy(S.st, ns > 1 ? S.bt : S.t);
        cost_out = best_cost;
        return best_s;
    }

    // best_inter_ref, enc/frame.rs:852-905. Leaves the winner's vectors in S.best_mvs.
    __device__ int best_inter_ref(int r, int& part_out, uint8_t sub_out[4], int& cost16) {
        const int lam = P.lambda;
        int rb = 0;
        if (P.nact == 2) rb = lam;  // ref_bits, enc/frame.rs:705-711
        else if (P.nact > 2) rb = lam * (2 * (31 - __clz(r + 1)) + 1);
        int mvpx, mvpy;
        pred_mv(nullptr, 0, 0, 4, 0, r, mvpx, mvpy);
        const ColMv col = P.col[mb];
        int2 colv = make_int2(col.mv[0], col.mv[1]);
        int mx, my;
        Rect4 whole = {0, 0, 4, 4};
        int c = motion_search(r, whole, mvpx, mvpy, &colv, col.valid ? 1 : 0, mx, my);
        int best_part = 0, best_cost = c + lam * (mvd_bits_d(mx, my, mvpx, mvpy) + 1) + rb;
        cost16 = best_cost;
        if (lane < 16) {
            S.best_mvs[lane][0] = (int16_t)mx;
            S.best_mvs[lane][1] = (int16_t)my;
        }
        __syncwarp();
        uint8_t sub[4] = {0, 0, 0, 0};
        for (int i = 0; i < 4; i++) sub_out[i] = 0;
        if (P.fast) {
            part_out = 0;
            return best_cost;
        }
        // P_8x8 (868-876)
        blk_clear(S.st);
        int cost8 = lam * 9;
        for (int k = 0; k < 4; k++) {
            int ck;
            sub[k] = (uint8_t)sub_search(r, k, mx, my, ck);
            cost8 += ck + rb;
            if (cost8 >= best_cost) break;
        }
        if (cost8 < best_cost) {
            // v8: the vectors of rects(3, sub) in coding order (882-885)
            if (lane == 0) {
                int n = 0;
                for (int k = 0; k < 4; k++)
                    for (int q = 0; q < c_nsub[sub[k]]; q++) {
                        int x = (k & 1) * 2 + c_sub[sub[k]][q][0], y = (k >> 1) * 2 + c_sub[sub[k]][q][1];
                        S.best_mvs[n][0] = S.st.mv[y * 4 + x][0];
                        S.best_mvs[n][1] = S.st.mv[y * 4 + x][1];
                        n++;
                    }
                for (; n < 16; n++) S.best_mvs[n][0] = S.best_mvs[n][1] = 0;
            }
            __syncwarp();
            best_part = 3;
            best_cost = cost8;
            for (int i = 0; i < 4; i++) sub_out[i] = sub[i];
            // 16x8 and 8x16 halves searched from the 8x8 vectors they cover (886-902)
            for (int part = 1; part < 3; part++) {
                int pc = lam * 3;
                int hv[2][2] = {{0, 0}, {0, 0}};
                for (int k = 0; k < 2; k++) {
                    // part_mvps(...)[k]: the halves before k are decided
                    blk_clear(S.t);
                    if (k == 1) {
                        Rect4 r0 = {c_parts[part][0][0], c_parts[part][0][1], c_parts[part][0][2], c_parts[part][0][3]};
                        blk_paint(S.t, r0, hv[0][0], hv[0][1], r);
                    }
                    Rect4 rk = {c_parts[part][k][0], c_parts[part][k][1], c_parts[part][k][2], c_parts[part][k][3]};
                    int px, py;
                    pred_mv(&S.t, rk.x, rk.y, rk.w, part, r, px, py);
                    int i0 = part == 1 ? 2 * k : k, i1 = part == 1 ? 2 * k + 1 : k + 2;
                    int2 cands[2];
                    int b0 = (i0 / 2) * 8 + (i0 % 2) * 2, b1 = (i1 / 2) * 8 + (i1 % 2) * 2;
                    cands[0] = make_int2(S.st.mv[b0][0], S.st.mv[b0][1]);
                    cands[1] = make_int2(S.st.mv[b1][0], S.st.mv[b1][1]);
                    int m0, m1;
                    int cc = motion_search(r, rk, px, py, cands, 2, m0, m1);
                    hv[k][0] = m0;
                    hv[k][1] = m1;
                    pc += cc + lam * mvd_bits_d(m0, m1, px, py) + rb;
                    if (pc >= best_cost) break;
                }
                if (pc < best_cost) {
                    best_part = part;
                    best_cost = pc;
                    for (int i = 0; i < 4; i++) sub_out[i] = 0;
                    if (lane < 16) {
                        int v0 = lane < 2 ? hv[lane][0] : 0, v1 = lane < 2 ? hv[lane][1] : 0;
                        S.best_mvs[lane][0] = (int16_t)v0;
                        S.best_mvs[lane][1] = (int16_t)v1;
                    }
                    __syncwarp();
                }
            }
        }
        part_out = best_part;
        return best_cost;
    }

    // ---- one macroblock --------------------------------------------------------------------------------

    __device__ void analyse(bool auto_policy) {
        // the current macroblock: 16 rows of 16 bytes, as 128-bit loads
        if (lane < 16) {
            const uint4 v = *reinterpret_cast<const uint4*>(P.src + (size_t)(mby * 16 + lane) * P.ls + mbx * 16);
            S.src[lane * 4 + 0] = v.x;
            S.src[lane * 4 + 1] = v.y;
            S.src[lane * 4 + 2] = v.z;
            S.src[lane * 4 + 3] = v.w;
        }
        if (lane < 26) reinterpret_cast<uint32_t*>(&S.res)[lane] = 0;
        __syncwarp();
        sad_px = satd_px = 0;
        // P_Skip (enc/frame.rs:722-729)
        int sx, sy;
        skip_mv(sx, sy);
        if (lane == 0) S.cand[0] = make_int2(sx, sy);
        __syncwarp();
        pred_batch(0, 0, 0, 16, 16, 1, 0, 0, true);
        const int skip_sad = S.cost[0];
        sad_px += 256;
        const bool skip = auto_policy && skip_sad < P.skip_thresh;
        int part = 0, cost = 0, cost16 = 0, bestr = 0;
        uint8_t sub[4] = {0, 0, 0, 0};
        if (!skip) {
            // best_inter, enc/frame.rs:839-849: every reference, the cheapest (first on ties) wins
            for (int r = 0; r < P.nact; r++) {
                int p, c16;
                uint8_t sb[4];
                int c = best_inter_ref(r, p, sb, c16);
                if (r == 0 || c < cost) {
                    part = p;
                    cost = c;
                    cost16 = c16;
                    bestr = r;
                    for (int i = 0; i < 4; i++) sub[i] = sb[i];
                    if (lane < 16) {
                        S.win_mvs[lane][0] = S.best_mvs[lane][0];
                        S.win_mvs[lane][1] = S.best_mvs[lane][1];
                    }
                    __syncwarp();
                }
            }
        }
        // the result
        if (lane == 0) {
            ironav_mbresult& R = S.res;
            R.skip_mv[0] = (int16_t)sx;
            R.skip_mv[1] = (int16_t)sy;
            R.skip_sad = skip_sad;
            R.flags = skip ? IRONAV_RESULT_SKIP : IRONAV_RESULT_INTER;
            if (!skip) {
                R.part = (uint8_t)part;
                for (int i = 0; i < 4; i++) {
                    R.refs[i] = (uint8_t)bestr;
                    R.sub[i] = sub[i];
                }
                R.cost = cost;
                R.cost16 = cost16;
            }
            R.sad_px = sad_px;
            R.satd_px = satd_px;
        }
        __syncwarp();
        if (lane < 16 && !skip) {
            S.res.mvs[lane][0] = S.win_mvs[lane][0];
            S.res.mvs[lane][1] = S.win_mvs[lane][1];
        }
        __syncwarp();
        if (lane < 26) reinterpret_cast<uint32_t*>(&P.results[mb])[lane] = reinterpret_cast<const uint32_t*>(&S.res)[lane];
        if (auto_policy) {
            // the decision's MbState (finish_mb, enc/frame.rs:2281-2321)
            if (lane < 16) {
                int bx = lane & 3, by = lane >> 2, mx = sx, my = sy;
                if (!skip) {
                    // the rectangle of rects(part, sub) holding this block, in coding order
                    int idx = 0;
                    if (part == 1) idx = by >> 1;
                    else if (part == 2) idx = bx >> 1;
                    else if (part == 3) {
                        int k = (by >> 1) * 2 + (bx >> 1), n = 0;
                        for (int q = 0; q < k; q++) n += c_nsub[sub[q]];
                        int s = sub[k], lx = bx & 1, ly = by & 1;
                        int within = s == 0 ? 0 : (s == 1 ? ly : (s == 2 ? lx : ly * 2 + lx));
                        idx = n + within;
                    }
                    mx = S.win_mvs[idx][0];
                    my = S.win_mvs[idx][1];
                }
                S.out.mvs[lane][0] = (int16_t)mx;
                S.out.mvs[lane][1] = (int16_t)my;
            }
            if (lane == 0) {
                S.out.inter = 1;
                for (int i = 0; i < 4; i++) S.out.refs[i] = (int8_t)(skip ? 0 : bestr);
                S.out.pad[0] = S.out.pad[1] = S.out.pad[2] = 0;
            }
            __syncwarp();
            if (lane < 18) reinterpret_cast<uint32_t*>(&P.states_out[mb])[lane] = reinterpret_cast<const uint32_t*>(&S.out)[lane];
        }
        __syncwarp();
    }
};

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(unsigned* p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Waits until macroblock `m`'s decision is published, at most P.wait_limit polls. Returns false when
// it gave up or another warp already did (the launch is then abandoned and the host reports a timeout).
static __device__ bool wait_published(const AnalyseParams& P, int m) {
    for (unsigned i = 0;; i++) {
        if (ld_acquire(&P.flags[m]) == P.epoch) return true;
        if (ld_acquire(P.err) != 0) return false;
        if (i >= P.wait_limit) {
            atomicOr(P.err, 1u);
            return false;
        }
        __nanosleep(i < 64 ? 32 : 256);
    }
}

template <bool AUTO>
__global__ void __launch_bounds__(K2_WARPS * 32) analyse_kernel(const AnalyseParams P) {
    __shared__ WarpSmem smem[K2_WARPS];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    MbWarp W(P, smem[wid], lane);
    for (;;) {
        unsigned t = 0;
        if (lane == 0) t = atomicAdd(P.ticket, 1u);
        t = __shfl_sync(FULL, t, 0);
        if (t >= (unsigned)P.nmb) break;
        const int mb = P.order ? P.order[t] : (int)t;
        W.mb = mb;
        W.mbx = mb % P.mb_w;
        W.mby = mb / P.mb_w;
        if (AUTO) {
            // the left and top-right (top at the right edge) neighbours; their own waits cover the rest
            const int start = P.band_start[W.mby];
            bool ok = true;
            if (W.mbx > 0) ok = wait_published(P, mb - 1);
            if (ok && W.mby > start) ok = wait_published(P, (W.mbx + 1 < P.mb_w) ? mb - P.mb_w + 1 : mb - P.mb_w);
            ok = __all_sync(FULL, ok);
            if (!ok) break;
            W.load_neighbours(P.states_out);
        } else {
            W.load_neighbours(P.states_in);
        }
        W.analyse(AUTO);
        if (AUTO) {
            __threadfence();
            __syncwarp();
            if (lane == 0 && mb != P.withhold) st_release(&P.flags[mb], P.epoch);
        }
    }
}

}  // namespace ironav
