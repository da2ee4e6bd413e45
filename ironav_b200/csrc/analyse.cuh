// analyse.cuh — K2: P-macroblock inter analysis (P_Skip vector + SAD, best_inter with its motion
// searches), one warp per macroblock.
//
// The reference's analysis of a macroblock (enc/frame.rs:722-729, 839-1019) is a sequential,
// data-dependent search. Here every lane of a warp follows the same control flow (all decisions are
// warp-uniform) while the sample work of each step is spread over the lanes, and the warp-uniform
// bookkeeping is kept small:
//   - integer SAD: 8 candidate vectors per batch, lane group c = lane & 7 scores candidate c (each lane
//     works out its own candidate), its 4 lanes split the rows; reference rows are read as aligned
//     32-bit words realigned with funnel shifts and compared with __vsadu4; sums by 2 xor shuffles;
//   - the diamond's greedy rounds (each move relative to the current best, strict '<', enc/frame.rs:
//     973-988) are resolved exactly: one batch scores the whole 3x3 square of the round's step around
//     the centre, which holds every point the four sequential moves can visit, and the moves are then
//     replayed in registers; a point the square lacks (only when a move was bent by the search clamps)
//     is scored on demand;
//   - the neighbours' blocks that the predictors read (nb_motion, enc/frame.rs:522-538) are gathered
//     once per macroblock into a 6x5 table of 4x4 blocks around the macroblock, so pred_mv and the
//     neighbour candidates are table lookups;
//   - sub-sample SATD: lanes over (vector, 4x4 block); the quarter-sample prediction is __vavgu4 of two
//     half-sample planes; per-vector sums by shared-memory atomics.
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

constexpr int K2_WARPS = 4;       // warps per CTA; each warp works alone
constexpr int K2_MIN_BLOCKS = 4;  // CTAs per SM the register budget must allow (128 registers a thread)
constexpr unsigned FULL = 0xffffffffu;
constexpr int BIG = 0x7fffffff;

// MIX, enc/subpel.rs:26-38: per [fy][fx] the byte pa | ax<<2 | ay<<3 | pb<<4 | bx<<6 | by<<7 (planes G=0,
// b=1, h=2, j=3), four entries per 32-bit word so a lane picks its entry from registers (no constant-memory
// reads that would serialise when the lanes' vectors differ).
__device__ __forceinline__ unsigned mix_entry(int fx, int fy) {
    const unsigned w = fy == 0 ? 0x14111000u : (fy == 1 ? 0x61312120u : (fy == 2 ? 0x63333222u : 0x96939228u));
    return (w >> (8 * fx)) & 0xffu;
}

// PARTS and SUB, enc/frame.rs:182,204: (x, y, w, h) in 4x4 blocks
static __device__ __constant__ int8_t c_parts[4][4][4] = {
    {{0, 0, 4, 4}}, {{0, 0, 4, 2}, {0, 2, 4, 2}}, {{0, 0, 2, 4}, {2, 0, 2, 4}}, {{0, 0, 2, 2}, {2, 0, 2, 2}, {0, 2, 2, 2}, {2, 2, 2, 2}}};
static __device__ __constant__ int8_t c_sub[4][4][4] = {
    {{0, 0, 2, 2}}, {{0, 0, 2, 1}, {0, 1, 2, 1}}, {{0, 0, 1, 2}, {1, 0, 1, 2}}, {{0, 0, 1, 1}, {1, 0, 1, 1}, {0, 1, 1, 1}, {1, 1, 1, 1}}};
static __device__ __constant__ int8_t c_nsub[4] = {1, 2, 2, 4};

// A 4x4 block's list-0 motion as the predictors see it: (mx, my, ref (-1 none), available).
using Blk = int4;

// Per-warp shared memory; T is the sample type (uint8_t for 8-bit pictures, uint16_t for 10-bit).
template <class T>
struct WarpSmem {
    uint32_t src[64 * sizeof(T)];  // current macroblock, 16 rows of 16 samples (4 * sizeof(T) words each)
    Blk ext[30];              // blocks around the macroblock: index (y + 1) * 6 + (x + 1), x in -1..4, y in -1..3
    Blk st[16];               // P_8x8: blocks decided so far (sub_search's `st`)
    Blk t[16];                // trial blocks (sub_search's `t`, part_mvps's `cur`)
    Blk bt[16];               // best trial
    int2 cand[16];            // the sub-sample batch's vectors
    int cost[16];             // sub-sample batch sums (and a clamped round's square)
    int16_t best_mvs[16][2];  // best_inter_ref's running best, in coding order
    int16_t win_mvs[16][2];   // best over the references
    ironav_mbresult res;
    ironav_mbstate out;
    int mb, mbx, mby;         // the macroblock being analysed
    uint32_t sad_px, satd_px; // its work counts
};

__device__ __forceinline__ int ue_bits_d(unsigned v) { return 2 * (32 - __clz(v + 1)) - 1; }  // enc/bitw.rs:81-83
__device__ __forceinline__ int se_bits_d(int v) {                                             // enc/bitw.rs:86-89
    return ue_bits_d(v > 0 ? 2u * (unsigned)v - 1u : (unsigned)(-2 * v));
}
__device__ __forceinline__ int mvd_bits_d(int mx, int my, int px, int py) { return se_bits_d(mx - px) + se_bits_d(my - py); }
__device__ __forceinline__ int median3_d(int a, int b, int c) { return min(max(a, b), max(min(a, b), c)); }

// dp4a with unsigned bytes in a and signed bytes in b: c + sum of a_k * b_k.
__device__ __forceinline__ int dp4a_us(uint32_t a, uint32_t b, int c) {
    int d;
    asm("dp4a.u32.s32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
    return d;
}

// satd4, enc/frame.rs:144-161, of the 4x4 block with source rows s[r] and prediction rows p[r] (4 packed
// bytes each). The row transform is the 4-point Hadamard of each row's differences, H(s - p) = Hs - Hp,
// taken straight from the packed bytes with dp4a (rows (1,1,1,1), (1,1,-1,-1), (1,-1,-1,1), (1,-1,1,-1):
// the reference's outputs in its order); the column transform's last stage is folded, |a+b| + |a-b| =
// 2 max(|a|, |b|), so (sum of the 16 magnitudes) >> 1 is the sum over the 8 last-stage pairs of max(|a|, |b|).
__device__ __forceinline__ int satd4_packed(const uint32_t s[4], const uint32_t p[4]) {
    const uint32_t H[4] = {0x01010101u, 0xFFFF0101u, 0x01FFFF01u, 0xFF01FF01u};
    const uint32_t NH[4] = {0xFFFFFFFFu, 0x0101FFFFu, 0xFF0101FFu, 0x01FF01FFu};
    int t[4][4];
#pragma unroll
    for (int r = 0; r < 4; r++)
#pragma unroll
        for (int j = 0; j < 4; j++) t[r][j] = dp4a_us(p[r], NH[j], dp4a_us(s[r], H[j], 0));
    int sum = 0;
#pragma unroll
    for (int c = 0; c < 4; c++) {
        const int a = t[0][c], b = t[1][c], cc = t[2][c], e = t[3][c];
        const int s0 = a + b, s1 = cc + e, d0 = a - b, d1 = cc - e;
        sum += max(abs(s0), abs(s1)) + max(abs(d0), abs(d1));
    }
    return sum;
}

// Two-way dot products of the unsigned 16-bit halves of a with the signed bytes 0-1 (lo) or 2-3 (hi) of b.
__device__ __forceinline__ int dp2a_lo_us(uint32_t a, uint32_t b, int c) {
    int d;
    asm("dp2a.lo.u32.s32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
    return d;
}
__device__ __forceinline__ int dp2a_hi_us(uint32_t a, uint32_t b, int c) {
    int d;
    asm("dp2a.hi.u32.s32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
    return d;
}

// satd4 of a 4x4 block of 16-bit samples: rows s[r][0..1] and p[r][0..1] hold 2 samples per word. The same
// transform as satd4_packed, the row Hadamard taken with dp2a over the two words of each row.
__device__ __forceinline__ int satd4_packed16(const uint32_t s[4][2], const uint32_t p[4][2]) {
    const uint32_t H[4] = {0x01010101u, 0xFFFF0101u, 0x01FFFF01u, 0xFF01FF01u};
    const uint32_t NH[4] = {0xFFFFFFFFu, 0x0101FFFFu, 0xFF0101FFu, 0x01FF01FFu};
    int t[4][4];
#pragma unroll
    for (int r = 0; r < 4; r++)
#pragma unroll
        for (int j = 0; j < 4; j++)
            t[r][j] = dp2a_hi_us(p[r][1], NH[j], dp2a_lo_us(p[r][0], NH[j], dp2a_hi_us(s[r][1], H[j], dp2a_lo_us(s[r][0], H[j], 0))));
    int sum = 0;
#pragma unroll
    for (int c = 0; c < 4; c++) {
        const int a = t[0][c], b = t[1][c], cc = t[2][c], e = t[3][c];
        const int s0 = a + b, s1 = cc + e, d0 = a - b, d1 = cc - e;
        sum += max(abs(s0), abs(s1)) + max(abs(d0), abs(d1));
    }
    return sum;
}

// ---- neighbours (nb_state / nb_motion, enc/frame.rs:509-538) ----------------------------------

// Fills the table of blocks around the macroblock: left column (x = -1), top row (y = -1), top-right
// (4, -1), top-left (-1, -1); (4, y >= 0) is never available; inside slots are unused.
template <class T>
static __device__ void load_neighbours(const AnalyseParams& __restrict__ P, WarpSmem<T>& __restrict__ S, const ironav_mbstate* states) {
    const int lane = threadIdx.x & 31;
    if (lane < 30) {
        const int ex = lane % 6 - 1, ey = lane / 6 - 1;
        Blk e = make_int4(0, 0, -1, 0);
        if (ey < 0 || ex < 0) {
            const int nx = S.mbx + (ex < 0 ? -1 : (ex >= 4 ? 1 : 0)), ny = S.mby + (ey < 0 ? -1 : 0);
            const int bx = ex < 0 ? 3 : (ex >= 4 ? 0 : ex), by = ey < 0 ? 3 : ey;
            // macroblocks of earlier slices are not available (enc/frame.rs:509-515)
            if (nx >= 0 && nx < P.mb_w && ny >= P.band_start[S.mby] && ny < P.mb_h) {
                const ironav_mbstate* s = &states[(size_t)ny * P.mb_w + nx];
                e.w = 1;
                const int rf = s->refs[(by >> 1) * 2 + (bx >> 1)];
                if (s->inter && rf >= 0) {
                    const uint32_t mv = *reinterpret_cast<const uint32_t*>(&s->mvs[by * 4 + bx][0]);
                    e.x = (int)(int16_t)(mv & 0xffffu);
                    e.y = (int)(int16_t)(mv >> 16);
                    e.z = rf;
                }
            }
        }
        S.ext[lane] = e;
    }
    __syncwarp();
}

// nb_motion for the block at (x, y) relative to the macroblock, from the neighbour table `ext` of one list;
// inside the macroblock, `cur` holds the decided blocks (nullptr: none decided).
template <class T>
static __device__ __forceinline__ Blk nb(const AnalyseParams& __restrict__ P, WarpSmem<T>& __restrict__ S, const Blk* ext, const Blk* cur, int x, int y) {
    if (x >= 0 && x < 4 && y >= 0) return cur ? cur[y * 4 + x] : make_int4(0, 0, -1, 0);
    return ext[(y + 1) * 6 + (x + 1)];
}

// pred_mv, enc/frame.rs:543-570
template <class T>
static __device__ __forceinline__ int2 pred_mv(const AnalyseParams& __restrict__ P, WarpSmem<T>& __restrict__ S, const Blk* ext, const Blk* cur, int bx, int by, int w,
                                               int dir, int rf) {
    const Blk a = nb(P, S, ext, cur, bx - 1, by), b = nb(P, S, ext, cur, bx, by - 1);
    Blk c = nb(P, S, ext, cur, bx + w, by - 1);
    if (!c.w) c = nb(P, S, ext, cur, bx - 1, by - 1);
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

// skip_mv, enc/frame.rs:597-603
template <class T>
static __device__ int2 skip_mv(const AnalyseParams& __restrict__ P, WarpSmem<T>& __restrict__ S) {
    const Blk a = nb(P, S, S.ext, nullptr, -1, 0), b = nb(P, S, S.ext, nullptr, 0, -1);
    if (!a.w || !b.w || (a.z == 0 && a.x == 0 && a.y == 0) || (b.z == 0 && b.x == 0 && b.y == 0)) return make_int2(0, 0);
    return pred_mv(P, S, S.ext, nullptr, 0, 0, 4, 0, 0);
}

// ---- scoring -------------------------------------------------------------------------------------

// Integer SAD (sad_int, enc/frame.rs:662-671) of the partition at this lane's candidate (px, py): g0 is the
// reference plane G at the partition's origin (a byte address), src the partition's first source word, w x h
// its size, sw the plane stride in samples. The lanes of a group (same lane & 7) share a candidate and split
// its rows; every lane of the group gets the sum. Rows are read as aligned 32-bit words realigned with funnel
// shifts: 4 samples a word compared with __vsadu4 (8-bit), 2 with __vsadu2 (16-bit).
template <class T>
static __device__ __forceinline__ int sad_lane(const uint8_t* __restrict__ g0, const uint32_t* __restrict__ src, int sw, int w,
                                               int h, int px, int py, bool valid) {
    constexpr int B = sizeof(T);
    const int lane = threadIdx.x & 31;
    int sad = 0;
    if (!valid) px = py = 0;  // scored at a position always inside the planes, and discarded: no divergent branch
    {
        const int row0 = lane >> 3;
        const uint8_t* G = g0 + (((py >> 2) + row0) * sw + (px >> 2)) * B;
        const int step4 = 4 * sw * B;
        for (int row = row0; row < h; row += 4, G += step4) {
            const uintptr_t a = reinterpret_cast<uintptr_t>(G);
            const uint32_t* q = reinterpret_cast<const uint32_t*>(a & ~uintptr_t(3));
            const unsigned sh = (unsigned)(a & 3) * 8u;
            const uint32_t* sr = src + row * 4 * B;
            if constexpr (B == 1) {
                const uint32_t w0 = __ldg(q), w1 = __ldg(q + 1);
                sad += __vsadu4(sr[0], __funnelshift_r(w0, w1, sh));
                if (w >= 8) {
                    const uint32_t w2 = __ldg(q + 2);
                    sad += __vsadu4(sr[1], __funnelshift_r(w1, w2, sh));
                    if (w == 16) {
                        const uint32_t w3 = __ldg(q + 3), w4 = __ldg(q + 4);
                        sad += __vsadu4(sr[2], __funnelshift_r(w2, w3, sh)) + __vsadu4(sr[3], __funnelshift_r(w3, w4, sh));
                    }
                }
            } else {
                const uint32_t w0 = __ldg(q), w1 = __ldg(q + 1), w2 = __ldg(q + 2);
                sad += __vsadu2(sr[0], __funnelshift_r(w0, w1, sh)) + __vsadu2(sr[1], __funnelshift_r(w1, w2, sh));
                if (w >= 8) {
                    const uint32_t w3 = __ldg(q + 3), w4 = __ldg(q + 4);
                    sad += __vsadu2(sr[2], __funnelshift_r(w2, w3, sh)) + __vsadu2(sr[3], __funnelshift_r(w3, w4, sh));
                    if (w == 16) {
                        uint32_t pv = w4;
#pragma unroll
                        for (int k = 4; k < 8; k++) {
                            const uint32_t nx = __ldg(q + k + 1);
                            sad += __vsadu2(sr[k], __funnelshift_r(pv, nx, sh));
                            pv = nx;
                        }
                    }
                }
            }
        }
    }
    sad += __shfl_xor_sync(FULL, sad, 8);
    sad += __shfl_xor_sync(FULL, sad, 16);
    return sad;
}

// The quarter-sample prediction (HalfPel::predict, enc/subpel.rs:122-145) of the 4x4 block (bxx, byy), in
// 4x4 blocks, of the w x h partition at picture sample (x0, y0), from the half-sample planes at `base`:
// 4 rows of sizeof(T) words (4 samples a row).
template <class T>
__device__ __forceinline__ void pred4(const AnalyseParams& __restrict__ P, const uint8_t* base, int x0, int y0, int w, int h, int bxx, int byy, int2 mv,
                                      uint32_t (&pr)[4][sizeof(T)]) {
    constexpr int B = sizeof(T);
    const int sw = P.sw, psize = (int)P.psize;
    const int ix = min(max(x0 + (mv.x >> 2), -w - 3), P.pw + 1) + PAD + bxx * 4;
    const int iy = min(max(y0 + (mv.y >> 2), -h - 3), P.ph + 1) + PAD + byy * 4;
    const unsigned m = mix_entry(mv.x & 3, mv.y & 3);
    const int pa = m & 3, ax = (m >> 2) & 1, ay = (m >> 3) & 1, pb = (m >> 4) & 3, bbx = (m >> 6) & 1, bby = (m >> 7) & 1;
    const bool same = (m & 0xf) == (m >> 4);
    // every row of a plane block has the same alignment (sw is a multiple of 16); a row of 4 samples is
    // B words, read as B + 1 aligned words
    const uintptr_t ua = reinterpret_cast<uintptr_t>(base + (unsigned)(pa * psize + (iy + ay) * sw + ix + ax) * B);
    const uint32_t* qa = reinterpret_cast<const uint32_t*>(ua & ~uintptr_t(3));
    const unsigned sha = (unsigned)(ua & 3) * 8u;
    const int swq = (sw * B) >> 2;
#pragma unroll
    for (int row = 0; row < 4; row++) {
        uint32_t pv = __ldg(qa + row * swq);
#pragma unroll
        for (int k = 0; k < B; k++) {
            const uint32_t nx = __ldg(qa + row * swq + k + 1);
            pr[row][k] = __funnelshift_r(pv, nx, sha);
            pv = nx;
        }
    }
    if (!same) {
        const uintptr_t ub = reinterpret_cast<uintptr_t>(base + (unsigned)(pb * psize + (iy + bby) * sw + ix + bbx) * B);
        const uint32_t* qb = reinterpret_cast<const uint32_t*>(ub & ~uintptr_t(3));
        const unsigned shb = (unsigned)(ub & 3) * 8u;
#pragma unroll
        for (int row = 0; row < 4; row++) {
            uint32_t pv = __ldg(qb + row * swq);
#pragma unroll
            for (int k = 0; k < B; k++) {
                const uint32_t nx = __ldg(qb + row * swq + k + 1);
                const uint32_t o = __funnelshift_r(pv, nx, shb);
                pr[row][k] = B == 1 ? __vavgu4(pr[row][k], o) : __vavgu2(pr[row][k], o);
                pv = nx;
            }
        }
    }
}

// The score of prediction rows pr against the source's 4x4 block (sbx, sby) of the macroblock: SATD
// (satd, enc/frame.rs:641-659), or SAD when `sad`.
template <class T>
__device__ __forceinline__ int score4(const WarpSmem<T>& __restrict__ S, int sbx, int sby, const uint32_t (&pr)[4][sizeof(T)], bool sad) {
    constexpr int B = sizeof(T);
    uint32_t sr[4][B];
    const uint32_t* sp = &S.src[(sby * 16 + sbx) * B];
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

// Quarter-sample prediction of the partition at 4x4 block (bx, by), (4 << lgw) x (4 << lgh) samples, scored
// by SATD, or by SAD when `sad` (the P_Skip test), for the n vectors S.cand[0..n) on the planes of
// reference r; the sums land in S.cost[0..n). Lanes over (vector, 4x4 block).
template <class T>
static __device__ __forceinline__ void pred_batch(const AnalyseParams& __restrict__ P, WarpSmem<T>& __restrict__ S, int r, int bx, int by, int lgw, int lgh, int n, bool sad) {
    const int lane = threadIdx.x & 31;
    const int lg = lgw + lgh, total = n << lg, w = 4 << lgw, h = 4 << lgh;
    if (lane < n) S.cost[lane] = 0;
    __syncwarp();
    const int x0 = S.mbx * 16 + bx * 4, y0 = S.mby * 16 + by * 4;
    const uint8_t* base = P.planes[r];
    for (int t = lane; t < total; t += 32) {
        const int c = t >> lg, b = t & ((1 << lg) - 1), bxx = b & ((1 << lgw) - 1), byy = b >> lgw;
        uint32_t pr[4][sizeof(T)];
        pred4<T>(P, base, x0, y0, w, h, bxx, byy, S.cand[c], pr);
        atomicAdd(&S.cost[c], score4<T>(S, bx + bxx, by + byy, pr, sad));
    }
    __syncwarp();
}

// ---- motion_search, enc/frame.rs:949-1019 --------------------------------------------------------

// One diamond round whose moves were bent by the search clamps (or whose centre lies outside them): the
// reference's four moves replayed against the scored 3x3 square (S.cost[0..9), centre at 4), scoring on demand
// the points it lacks.
// Returns whether the best moved.
template <class T>
static __device__ __noinline__ int4 round_clamped(const AnalyseParams& __restrict__ P, WarpSmem<T>& __restrict__ S, int r, int bx, int by, int w, int h, int mvpx, int mvpy, int step, int cxlo,
                                           int cxhi, int cylo, int cyhi, int bxv, int byv, int bc) {
    const int lane = threadIdx.x & 31;
    const int cx = bxv, cy = byv;
    const int X0 = min(max(cx - step, cxlo), cxhi), X2 = min(max(cx + step, cxlo), cxhi);
    const int Y0 = min(max(cy - step, cylo), cyhi), Y2 = min(max(cy + step, cylo), cyhi);
    bool moved = false;
    for (int d = 0; d < 4; d++) {
        // each move clamps both coordinates of the current best (the unmoved one matters when the centre lies
        // outside the clamps, as a rounded candidate at the +-2048 / +-512 limits can)
        int nx = min(max(bxv, cxlo), cxhi), ny = min(max(byv, cylo), cyhi);
        if (d == 0) nx = min(max(bxv - step, cxlo), cxhi);
        else if (d == 1) nx = min(max(bxv + step, cxlo), cxhi);
        else if (d == 2) ny = min(max(byv - step, cylo), cyhi);
        else ny = min(max(byv + step, cylo), cyhi);
        const int ix = nx == X0 ? 0 : (nx == cx ? 1 : (nx == X2 ? 2 : -1));
        const int iy = ny == Y0 ? 0 : (ny == cy ? 1 : (ny == Y2 ? 2 : -1));
        int v;
        if (ix >= 0 && iy >= 0) {
            v = S.cost[iy * 3 + ix];
        } else {
            const uint8_t* g0 = P.planes[r] + ((S.mby * 16 + by * 4 + PAD) * P.sw + S.mbx * 16 + bx * 4 + PAD) * (int)sizeof(T);
            const int s1 = sad_lane<T>(g0, &S.src[(by * 16 + bx) * (int)sizeof(T)], P.sw, w, h, nx, ny, (lane & 7) == 0);
            v = __shfl_sync(FULL, s1, 0) + P.lambda * mvd_bits_d(nx, ny, mvpx, mvpy);
        }
        if (v < bc) {
            bxv = nx;
            byv = ny;
            bc = v;
            moved = true;
        }
    }
    return make_int4(moved, bxv, byv, bc);
}

// Out-of-line copies of sad_lane and pred_batch for the B-picture form of motion_search (MORE): the B
// kernel's code is large enough that its copies of them inlined at every call cost it instruction-cache
// misses (0.725 -> 0.662 ms per 1080p B picture out of line); the P kernels keep them inlined.
template <class T>
static __device__ __noinline__ int sad_lane_ni(const uint8_t* __restrict__ g0, const uint32_t* __restrict__ src, int sw, int w, int h, int px,
                                              int py, bool valid) {
    return sad_lane<T>(g0, src, sw, w, h, px, py, valid);
}
template <class T>
static __device__ __noinline__ void pred_batch_ni(const AnalyseParams& __restrict__ P, WarpSmem<T>& __restrict__ S, int r, int bx, int by, int lgw,
                                                 int lgh, int n) {
    pred_batch<T>(P, S, r, bx, by, lgw, lgh, n, false);
}

// One round of the diamond (enc/frame.rs:973-988) at `step` around (bxv, byv) of cost bc: the 3x3 square of the
// step is scored in one batch (lane group g -> square position k = g < 4 ? g : g + 1), then the reference's four
// moves are replayed in order (left, else right; then up from that column, else down). Returns whether the
// centre moved; (bxv, byv, bc) become the new centre. g0 and src0 as for sad_lane, sw the plane stride.
template <class T, bool MORE>
static __device__ __forceinline__ bool diamond_round(const AnalyseParams& __restrict__ P, WarpSmem<T>& __restrict__ S, int r, int bx, int by, int w,
                                                     int h, int mvpx, int mvpy, int step, int cxlo, int cxhi, int cylo, int cyhi,
                                                     const uint8_t* __restrict__ g0, const uint32_t* __restrict__ src0, int sw, int& bxv,
                                                     int& byv, int& bc) {
    const int lane = threadIdx.x & 31, g = lane & 7;
    const int lam = P.lambda;
    const int k = g < 4 ? g : g + 1, kx = k % 3, ky = k / 3;
    auto clx = [&](int v) { return min(max(v, cxlo), cxhi); };
    auto cly = [&](int v) { return min(max(v, cylo), cyhi); };
    const int cx = bxv, cy = byv, c0 = bc;
    const int X0 = clx(cx - step), X2 = clx(cx + step), Y0 = cly(cy - step), Y2 = cly(cy + step);
    const int qx = kx == 0 ? X0 : (kx == 1 ? cx : X2), qy = ky == 0 ? Y0 : (ky == 1 ? cy : Y2);
    const int sc = (MORE ? sad_lane_ni<T>(g0, src0, sw, w, h, qx, qy, true) : sad_lane<T>(g0, src0, sw, w, h, qx, qy, true)) + lam * mvd_bits_d(qx, qy, mvpx, mvpy);
    bool moved;
    if (X0 == cx - step && X2 == cx + step && Y0 == cy - step && Y2 == cy + step) {
        // no clamp: left, else right; then up from that column, else down
        const int sL = __shfl_sync(FULL, sc, 3), sR = __shfl_sync(FULL, sc, 4);
        int col = 1, b1 = c0;
        if (sL < c0) {
            col = 0;
            b1 = sL;
        } else if (sR < c0) {
            col = 2;
            b1 = sR;
        }
        const int sU = __shfl_sync(FULL, sc, col), sD = __shfl_sync(FULL, sc, 5 + col);
        int row = 1, b2 = b1;
        if (sU < b1) {
            row = 0;
            b2 = sU;
        } else if (sD < b1) {
            row = 2;
            b2 = sD;
        }
        bxv = col == 0 ? X0 : (col == 1 ? cx : X2);
        byv = row == 0 ? Y0 : (row == 1 ? cy : Y2);
        bc = b2;
        moved = col != 1 || row != 1;
    } else {
        if (lane < 8) S.cost[k] = sc;
        if (lane == 0) S.cost[4] = c0;
        __syncwarp();
        const int4 rc = round_clamped(P, S, r, bx, by, w, h, mvpx, mvpy, step, cxlo, cxhi, cylo, cyhi, bxv, byv, bc);
        moved = rc.x != 0;
        bxv = rc.y;
        byv = rc.z;
        bc = rc.w;
        __syncwarp();
    }
    return moved;
}

// Returns the best vector in (ox, oy) and its cost without the vector's bits. The search runs on the
// half-sample planes P.planes[r]; the neighbour candidates come from the table `ext` of the list searched
// and count when their reference index is rsel. (e0x, e0y) and (e1x, e1y) are the first extra candidates
// (nextra of them), more[0..nmore) the ones after them (B-picture partitions; at most 9; compiled in only
// when MORE).
template <class T, bool MORE>
static __device__ __noinline__ int4 motion_search(const AnalyseParams& __restrict__ P, WarpSmem<T>& __restrict__ S, const Blk* ext, int rsel, int r, int bx, int by,
                                                  int w4, int h4, int mvpx, int mvpy, int e0x, int e0y, int e1x, int e1y, int nextra,
                                                  const int2* more, int nmore) {
    const int lane = threadIdx.x & 31;
    const int lam = P.lambda;
    const int x0 = S.mbx * 16 + bx * 4, y0 = S.mby * 16 + by * 4, w = w4 * 4, h = h4 * 4;
    const int cxlo = max(-(x0 + 24) * 4, -2048), cxhi = min((P.mb_w * 16 - x0 + 8) * 4, 2047);
    const int cylo = max(-(y0 + 24) * 4, -512), cyhi = min((P.mb_h * 16 - y0 + 8) * 4, 511);
    auto clx = [&](int v) { return min(max(v, cxlo), cxhi); };
    auto cly = [&](int v) { return min(max(v, cylo), cyhi); };
    auto intr = [](int v) { return (v + 2) & ~3; };
    const int g = lane & 7;
    // candidates (958-964): lane group g scores candidate g; absent ones are skipped in order
    int px = 0, py = 0;
    bool valid = true;
    if (g == 0) {
        px = intr(clx(mvpx));
        py = intr(cly(mvpy));
    } else if (g >= 2 && g <= 4) {
        // P pictures: the list-0 table and the searched reference (the arguments are those)
        const Blk* E = MORE ? ext : S.ext;
        const int rs = MORE ? rsel : r;
        const Blk n = g == 2 ? nb(P, S, E, nullptr, -1, 0) : (g == 3 ? nb(P, S, E, nullptr, 0, -1) : nb(P, S, E, nullptr, 4, -1));
        valid = n.w && n.z == rs;
        px = intr(clx(n.x));
        py = intr(cly(n.y));
    } else if (g == 5) {
        valid = nextra > 0;
        px = intr(clx(e0x));
        py = intr(cly(e0y));
    } else if (g == 6) {
        valid = nextra > 1;
        px = intr(clx(e1x));
        py = intr(cly(e1y));
    } else if (g == 7) {
        valid = MORE && nmore > 0;
        if (MORE && valid) {
            px = intr(clx(more[0].x));
            py = intr(cly(more[0].y));
        }
    }
    const int sw = P.sw;
    const uint8_t* const g0 = P.planes[r] + ((y0 + PAD) * sw + x0 + PAD) * (int)sizeof(T);
    const uint32_t* const src0 = &S.src[(by * 16 + bx) * (int)sizeof(T)];
    int cost = MORE ? sad_lane_ni<T>(g0, src0, sw, w, h, px, py, valid) : sad_lane<T>(g0, src0, sw, w, h, px, py, valid);
    cost = valid ? cost + lam * mvd_bits_d(px, py, mvpx, mvpy) : BIG;
    const unsigned vmask = __ballot_sync(FULL, valid) & 0xffu;
    if (lane == 0) S.sad_px += (uint32_t)(__popc(vmask) * w * h);
    // the first candidate of least cost: min over (cost, position in the list)
    unsigned long long key = ((unsigned long long)(unsigned)cost << 4) | (unsigned)g;
    if (MORE && nmore > 1) {
        // the candidates after the eighth (list positions 8..15): a second batch
        const bool v2 = g + 1 < nmore;
        int qx = 0, qy = 0;
        if (v2) {
            qx = intr(clx(more[g + 1].x));
            qy = intr(cly(more[g + 1].y));
        }
        int c2 = sad_lane_ni<T>(g0, src0, sw, w, h, qx, qy, v2);
        c2 = v2 ? c2 + lam * mvd_bits_d(qx, qy, mvpx, mvpy) : BIG;
        const unsigned vm2 = __ballot_sync(FULL, v2) & 0xffu;
        if (lane == 0) S.sad_px += (uint32_t)(__popc(vm2) * w * h);
        key = min(key, ((unsigned long long)(unsigned)c2 << 4) | (unsigned)(8 + g));
        // the lane keeps the vector of whichever of its two candidates its key now names
        px = (key & 15u) >= 8 ? qx : px;
        py = (key & 15u) >= 8 ? qy : py;
    }
#pragma unroll
    for (int off = 1; off < 8; off <<= 1) key = min(key, __shfl_xor_sync(FULL, key, off));
    const int win = (int)(key & 7u);  // the lane group holding the winning candidate
    int bc = (int)(key >> 4);
    int bxv = __shfl_sync(FULL, px, win), byv = __shfl_sync(FULL, py, win);
    // the diamond (973-988): each round scores the 3x3 square of its step around the centre in one
    // batch (group g -> square position k = g < 4 ? g : g + 1), then replays the four moves in order
    const bool fast = P.fast != 0;
    const int nsteps = fast ? 2 : 3;
    int rounds = 0;  // the reference evaluates four moves a round (counted once, after the diamond)
    for (int si = 0; si < nsteps; si++) {
        const int step = fast ? (si == 0 ? 8 : 4) : (16 >> si);
        const int iters = step == 4 ? 32 : 4;
        for (int it = 0; it < iters; it++) {
            rounds++;
            if (!diamond_round<T, MORE>(P, S, r, bx, by, w, h, mvpx, mvpy, step, cxlo, cxhi, cylo, cyhi, g0, src0, sw, bxv, byv, bc)) break;
        }
    }
    if (lane == 0) S.sad_px += (uint32_t)(4 * w * h * rounds);
    // live coding's early exit (990-992)
    if (P.fast && bc < (w * h) / 8 + lam) return make_int4(bc - lam * mvd_bits_d(bxv, byv, mvpx, mvpy), bxv, byv, 0);
    const int lgw = w4 == 4 ? 2 : (w4 == 2 ? 1 : 0), lgh = h4 == 4 ? 2 : (h4 == 2 ? 1 : 0);
    // sub-sample refinement (994-1017): the centre and the 8 half samples around it in one batch,
    // square (-1,-1) (0,-1) (1,-1) (-1,0) (1,0) (-1,1) (0,1) (1,1) in order
    if (lane < 9) {
        int2 q = make_int2(bxv, byv);
        if (lane > 0) {
            const int kk = lane <= 4 ? lane - 1 : lane;
            q = make_int2(clx(bxv + (kk % 3 - 1) * 2), cly(byv + (kk / 3 - 1) * 2));
        }
        S.cand[lane] = q;
    }
    __syncwarp();
    if constexpr (MORE) pred_batch_ni<T>(P, S, r, bx, by, lgw, lgh, 9);
    else pred_batch(P, S, r, bx, by, lgw, lgh, 9, false);
    // the first of least cost in the square's order (strict <, centre first): min over (cost, position);
    // costs are SATD + lambda * bits, far below 2^27
    {
        unsigned key = 0xffffffffu;
        if (lane < 9) key = ((unsigned)(S.cost[lane] + lam * mvd_bits_d(S.cand[lane].x, S.cand[lane].y, mvpx, mvpy)) << 4) | (unsigned)lane;
#pragma unroll
        for (int off = 16; off >= 1; off >>= 1) key = min(key, __shfl_xor_sync(FULL, key, off));
        const int c = (int)(key & 15u);
        bc = (int)(key >> 4);
        bxv = S.cand[c].x;
        byv = S.cand[c].y;
    }
    if (lane == 0) S.satd_px += (uint32_t)(9 * w * h);
    __syncwarp();
    if (!P.fast) {
        // the 4 quarter samples around the new centre: (0,-1) (-1,0) (1,0) (0,1)
        if (lane < 4) {
            const int dx = lane == 1 ? -1 : (lane == 2 ? 1 : 0), dy = lane == 0 ? -1 : (lane == 3 ? 1 : 0);
            S.cand[lane] = make_int2(clx(bxv + dx), cly(byv + dy));
        }
        __syncwarp();
        if constexpr (MORE) pred_batch_ni<T>(P, S, r, bx, by, lgw, lgh, 4);
    else pred_batch(P, S, r, bx, by, lgw, lgh, 4, false);
        // the centre keeps ties (key position 0), then the four in order
        {
            unsigned key = (unsigned)bc << 4;
            if (lane < 4) key = ((unsigned)(S.cost[lane] + lam * mvd_bits_d(S.cand[lane].x, S.cand[lane].y, mvpx, mvpy)) << 4) | (unsigned)(lane + 1);
#pragma unroll
            for (int off = 16; off >= 1; off >>= 1) key = min(key, __shfl_xor_sync(FULL, key, off));
            const int c = (int)(key & 15u);
            bc = (int)(key >> 4);
            if (c > 0) {
                bxv = S.cand[c - 1].x;
                byv = S.cand[c - 1].y;
            }
        }
        if (lane == 0) S.satd_px += (uint32_t)(4 * w * h);
        __syncwarp();
    }
    return make_int4(bc - lam * mvd_bits_d(bxv, byv, mvpx, mvpy), bxv, byv, 0);
}

// ---- partition decision ----------------------------------------------------------------------------

template <class T>
static __device__ __forceinline__ void blk_clear(const AnalyseParams& __restrict__ P, WarpSmem<T>& __restrict__ S, Blk* b) {
    const int lane = threadIdx.x & 31;
    if (lane < 16) b[lane] = make_int4(0, 0, -1, 0);
    __syncwarp();
}
template <class T>
static __device__ __forceinline__ void blk_copy(const AnalyseParams& __restrict__ P, WarpSmem<T>& __restrict__ S, Blk* d, const Blk* s) {
    const int lane = threadIdx.x & 31;
    if (lane < 16) d[lane] = s[lane];
    __syncwarp();
}
// Marks rectangle (x, y, w, h) of `b` as decided with vector (mx, my) and reference rf.
template <class T>
static __device__ __forceinline__ void blk_paint(const AnalyseParams& __restrict__ P, WarpSmem<T>& __restrict__ S, Blk* b, int x, int y, int w, int h, int mx, int my, int rf) {
    const int lane = threadIdx.x & 31;
    if (lane < 16) {
        const int bx = lane & 3, by = lane >> 2;
        if (bx >= x && bx < x + w && by >= y && by < y + h) b[lane] = make_int4(mx, my, rf, 1);
    }
    __syncwarp();
}

// sub_search, enc/frame.rs:911-938: returns sub_mb_type, its cost in cost_out; leaves the 8x8
// block's vectors in S.st.
template <class T>
static __device__ __noinline__ int2 sub_search(const AnalyseParams& __restrict__ P, WarpSmem<T>& __restrict__ S, int r, int k, int ex, int ey) {
    const int lam = P.lambda;
    const int ox = (k & 1) * 2, oy = (k >> 1) * 2;
    const int ns = P.sub8 ? 4 : 1;
    int best_s = 0, best_cost = 0;
    for (int s = 0; s < ns; s++) {
        blk_copy(P, S, S.t, S.st);
        int cost = lam * (s == 0 ? 0 : 2);
        for (int q = 0; q < c_nsub[s]; q++) {
            const int x = ox + c_sub[s][q][0], y = oy + c_sub[s][q][1], w = c_sub[s][q][2], h = c_sub[s][q][3];
            const int2 p = pred_mv(P, S, S.ext, S.t, x, y, w, 0, r);
            const int4 ms = motion_search<T, false>(P, S, S.ext, r, r, x, y, w, h, p.x, p.y, ex, ey, 0, 0, 1, nullptr, 0);
            const int c = ms.x, mx = ms.y, my = ms.z;
            cost += c + lam * mvd_bits_d(mx, my, p.x, p.y);
            blk_paint(P, S, S.t, x, y, w, h, mx, my, r);
        }
        if (s == 0 || cost < best_cost) {
            best_s = s;
            best_cost = cost;
            if (ns > 1) blk_copy(P, S, S.bt, S.t);
        }
    }
    blk_copy(P, S, S.st, ns > 1 ? S.bt : S.t);
    return make_int2(best_s, best_cost);
}

// best_inter_ref, enc/frame.rs:852-905. Leaves the winner's vectors in S.best_mvs.
template <class T>
static __device__ __noinline__ int4 best_inter_ref(const AnalyseParams& __restrict__ P, WarpSmem<T>& __restrict__ S, int r) {
    const int lane = threadIdx.x & 31;
    const int lam = P.lambda;
    int rb = 0;
    if (P.nact == 2) rb = lam;  // ref_bits, enc/frame.rs:705-711
    else if (P.nact > 2) rb = lam * (2 * (31 - __clz(r + 1)) + 1);
    const int2 mvp = pred_mv(P, S, S.ext, nullptr, 0, 0, 4, 0, r);
    const ColMv col = P.col[S.mb];
    const int4 ms = motion_search<T, false>(P, S, S.ext, r, r, 0, 0, 4, 4, mvp.x, mvp.y, col.mv[0], col.mv[1], 0, 0, col.valid ? 1 : 0, nullptr, 0);
    const int c = ms.x, mx = ms.y, my = ms.z;
    int best_part = 0, best_cost = c + lam * (mvd_bits_d(mx, my, mvp.x, mvp.y) + 1) + rb;
    const int cost16 = best_cost;
    uint32_t sub_out = 0;
    if (lane < 16) {
        S.best_mvs[lane][0] = (int16_t)mx;
        S.best_mvs[lane][1] = (int16_t)my;
    }
    __syncwarp();
    if (P.fast) return make_int4(best_cost, 0, 0, cost16);
    // P_8x8 (868-876)
    blk_clear(P, S, S.st);
    uint32_t sub = 0;
    int cost8 = lam * 9;
    for (int k = 0; k < 4; k++) {
        const int2 ss = sub_search(P, S, r, k, mx, my);
        const int ck = ss.y;
        sub |= (uint32_t)ss.x << (8 * k);
        cost8 += ck + rb;
        if (cost8 >= best_cost) break;
    }
    if (cost8 < best_cost) {
        // v8: the vectors of rects(3, sub) in coding order (882-885)
        if (lane == 0) {
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
        __syncwarp();
        best_part = 3;
        best_cost = cost8;
        sub_out = sub;
        // 16x8 and 8x16 halves searched from the 8x8 vectors they cover (886-902)
        for (int part = 1; part < 3; part++) {
            int pc = lam * 3;
            int h0x = 0, h0y = 0, h1x = 0, h1y = 0;
            for (int k = 0; k < 2; k++) {
                // part_mvps(...)[k]: the halves before k are decided
                blk_clear(P, S, S.t);
                if (k == 1)
                    blk_paint(P, S, S.t, c_parts[part][0][0], c_parts[part][0][1], c_parts[part][0][2], c_parts[part][0][3], h0x, h0y, r);
                const int x = c_parts[part][k][0], y = c_parts[part][k][1], w = c_parts[part][k][2], h = c_parts[part][k][3];
                const int2 p = pred_mv(P, S, S.ext, S.t, x, y, w, part, r);
                const int i0 = part == 1 ? 2 * k : k, i1 = part == 1 ? 2 * k + 1 : k + 2;
                const Blk a0 = S.st[(i0 / 2) * 8 + (i0 % 2) * 2], a1 = S.st[(i1 / 2) * 8 + (i1 % 2) * 2];
                const int4 ms = motion_search<T, false>(P, S, S.ext, r, r, x, y, w, h, p.x, p.y, a0.x, a0.y, a1.x, a1.y, 2, nullptr, 0);
                const int cc = ms.x, m0 = ms.y, m1 = ms.z;
                if (k == 0) {
                    h0x = m0;
                    h0y = m1;
                } else {
                    h1x = m0;
                    h1y = m1;
                }
                pc += cc + lam * mvd_bits_d(m0, m1, p.x, p.y) + rb;
                if (pc >= best_cost) break;
            }
            if (pc < best_cost) {
                best_part = part;
                best_cost = pc;
                sub_out = 0;
                if (lane < 16) {
                    S.best_mvs[lane][0] = (int16_t)(lane == 0 ? h0x : (lane == 1 ? h1x : 0));
                    S.best_mvs[lane][1] = (int16_t)(lane == 0 ? h0y : (lane == 1 ? h1y : 0));
                }
                __syncwarp();
            }
        }
    }
    return make_int4(best_cost, best_part, (int)sub_out, cost16);
}

// ---- the learned form's judge ------------------------------------------------------------------------

// The 16x16 partitioning of reference r judged from the learned proposer's candidates instead of searched:
// the exact integer cost (SAD + lambda * the vector's bits, as the plain search scores it) of every integer
// vector within +-2 samples of each of the 4 proposals (100 points, eight a batch, the search's clamps), the
// plain search's small diamond (step 1 sample) from the best of them, then its sub-sample refinement (the
// half-sample square and the quarter-sample diamond by SATD). Falls back (returns x = -1) when the proposed partitioning is not P_Skip or 16x16, or when
// the best proposal costs more than the predictor's own start (the plain search's first candidate) plus the
// margin. Otherwise returns best_inter_ref's result for a 16x16 choice.
template <class T>
static __device__ __noinline__ int4 learned_inter(const AnalyseParams& __restrict__ P, WarpSmem<T>& __restrict__ S, int r) {
    const int lane = threadIdx.x & 31, g = lane & 7;
    const int lam = P.lambda;
    if (P.learned_cls[S.mb] >= 2) {
        if (lane == 0) atomicAdd(&P.learned_stats[1], 1u);
        return make_int4(-1, 0, 0, 0);
    }
    int rb = 0;
    if (P.nact == 2) rb = lam;
    else if (P.nact > 2) rb = lam * (2 * (31 - __clz(r + 1)) + 1);
    const int2 mvp = pred_mv(P, S, S.ext, nullptr, 0, 0, 4, 0, r);
    const int x0 = S.mbx * 16, y0 = S.mby * 16;
    const int cxlo = max(-(x0 + 24) * 4, -2048), cxhi = min((P.mb_w * 16 - x0 + 8) * 4, 2047);
    const int cylo = max(-(y0 + 24) * 4, -512), cyhi = min((P.mb_h * 16 - y0 + 8) * 4, 511);
    auto clx = [&](int v) { return min(max(v, cxlo), cxhi); };
    auto cly = [&](int v) { return min(max(v, cylo), cyhi); };
    auto intr = [](int v) { return (v + 2) & ~3; };
    const int16_t* cand = P.learned + (size_t)S.mb * 8;
    const int sw = P.sw;
    const uint8_t* const g0 = P.planes[r] + ((y0 + PAD) * sw + x0 + PAD) * (int)sizeof(T);
    const uint32_t* const src0 = &S.src[0];
    unsigned best = 0xffffffffu, start = 0xffffffffu;
    for (int b = 0; b < 13; b++) {
        const int i = b * 8 + g;  // 0..99: proposal i / 25, offset i % 25; 100: the predictor start
        const bool valid = i <= 100;
        int px = intr(clx(mvp.x)), py = intr(cly(mvp.y));
        if (i < 100) {
            const int k = i / 25, d = i % 25;
            px = clx(intr(clx(cand[2 * k])) + 4 * (d % 5 - 2));
            py = cly(intr(cly(cand[2 * k + 1])) + 4 * (d / 5 - 2));
        }
        const int sad = sad_lane<T>(g0, src0, sw, 16, 16, px, py, valid);
        const unsigned cost = (unsigned)(sad + lam * mvd_bits_d(px, py, mvp.x, mvp.y));
        unsigned kp = (valid && i < 100) ? ((cost << 7) | (unsigned)i) : 0xffffffffu;
        unsigned ks = (i == 100) ? cost : 0xffffffffu;
#pragma unroll
        for (int off = 1; off < 8; off <<= 1) {
            kp = min(kp, __shfl_xor_sync(FULL, kp, off));
            ks = min(ks, __shfl_xor_sync(FULL, ks, off));
        }
        best = min(best, kp);
        start = min(start, ks);
    }
    if (lane == 0) S.sad_px += 101u * 256u;
    if ((int)(best >> 7) > (int)start + P.learned_margin) {
        if (lane == 0) atomicAdd(&P.learned_stats[2], 1u);
        return make_int4(-1, 0, 0, 0);
    }
    const int bi = (int)(best & 127u), k = bi / 25, d = bi % 25;
    int bxv = clx(intr(clx(cand[2 * k])) + 4 * (d % 5 - 2)), byv = cly(intr(cly(cand[2 * k + 1])) + 4 * (d / 5 - 2));
    int bc = (int)(best >> 7);
    // the plain search's small diamond (step 4, at most 32 rounds) from the best of the windows
    {
        int rounds = 0;
        for (int it = 0; it < 32; it++) {
            rounds++;
            if (!diamond_round<T, false>(P, S, r, 0, 0, 16, 16, mvp.x, mvp.y, 4, cxlo, cxhi, cylo, cyhi, g0, src0, sw, bxv, byv, bc)) break;
        }
        if (lane == 0) S.sad_px += (uint32_t)(4 * 256 * rounds);
    }
    // the plain search's sub-sample refinement (motion_search, enc/frame.rs:994-1017)
    if (lane < 9) {
        int2 q = make_int2(bxv, byv);
        if (lane > 0) {
            const int kk = lane <= 4 ? lane - 1 : lane;
            q = make_int2(clx(bxv + (kk % 3 - 1) * 2), cly(byv + (kk / 3 - 1) * 2));
        }
        S.cand[lane] = q;
    }
    __syncwarp();
    pred_batch(P, S, r, 0, 0, 2, 2, 9, false);
    {
        unsigned key = 0xffffffffu;
        if (lane < 9) key = ((unsigned)(S.cost[lane] + lam * mvd_bits_d(S.cand[lane].x, S.cand[lane].y, mvp.x, mvp.y)) << 4) | (unsigned)lane;
#pragma unroll
        for (int off = 16; off >= 1; off >>= 1) key = min(key, __shfl_xor_sync(FULL, key, off));
        const int c = (int)(key & 15u);
        bc = (int)(key >> 4);
        bxv = S.cand[c].x;
        byv = S.cand[c].y;
    }
    __syncwarp();
    if (!P.fast) {
        if (lane < 4) {
            const int dx = lane == 1 ? -1 : (lane == 2 ? 1 : 0), dy = lane == 0 ? -1 : (lane == 3 ? 1 : 0);
            S.cand[lane] = make_int2(clx(bxv + dx), cly(byv + dy));
        }
        __syncwarp();
        pred_batch(P, S, r, 0, 0, 2, 2, 4, false);
        unsigned key = (unsigned)bc << 4;
        if (lane < 4) key = ((unsigned)(S.cost[lane] + lam * mvd_bits_d(S.cand[lane].x, S.cand[lane].y, mvp.x, mvp.y)) << 4) | (unsigned)(lane + 1);
#pragma unroll
        for (int off = 16; off >= 1; off >>= 1) key = min(key, __shfl_xor_sync(FULL, key, off));
        const int c = (int)(key & 15u);
        bc = (int)(key >> 4);
        if (c > 0) {
            bxv = S.cand[c - 1].x;
            byv = S.cand[c - 1].y;
        }
        __syncwarp();
    }
    if (lane == 0) S.satd_px += (P.fast ? 9u : 13u) * 256u;
    // bc holds SATD + lambda * bits; the 16x16 cost of best_inter_ref (855-858) adds the mb_type bit and ref_bits
    const int cost16 = bc + lam + rb;
    if (lane < 16) {
        S.best_mvs[lane][0] = (int16_t)bxv;
        S.best_mvs[lane][1] = (int16_t)byv;
    }
    if (lane == 0) atomicAdd(&P.learned_stats[0], 1u);
    __syncwarp();
    return make_int4(cost16, 0, 0, cost16);
}

// best_inter_ref, or the learned form's judge on the newest reference when proposals are given.
template <class T>
static __device__ __forceinline__ int4 best_inter_or_learned(const AnalyseParams& __restrict__ P, WarpSmem<T>& __restrict__ S, int r) {
    if (P.learned != nullptr && r == 0) {
        const int4 li = learned_inter(P, S, r);
        if (li.x >= 0) return li;
    }
    return best_inter_ref(P, S, r);
}

// ---- one macroblock --------------------------------------------------------------------------------

// The current macroblock into shared memory: 16 rows of 16 samples, as 128-bit loads (sizeof(T) per row).
template <class T>
static __device__ __forceinline__ void stage_source(const AnalyseParams& __restrict__ P, WarpSmem<T>& __restrict__ S) {
    const int lane = threadIdx.x & 31;
    constexpr int B = sizeof(T);
    if (lane < 16 * B) {
        const int row = lane / B, part = lane % B;
        const uint4 v = *reinterpret_cast<const uint4*>(P.src + ((size_t)(S.mby * 16 + row) * P.ls + S.mbx * 16) * B + part * 16);
        S.src[lane * 4 + 0] = v.x;
        S.src[lane * 4 + 1] = v.y;
        S.src[lane * 4 + 2] = v.z;
        S.src[lane * 4 + 3] = v.w;
    }
}

template <class T>
static __device__ void analyse(const AnalyseParams& __restrict__ P, WarpSmem<T>& __restrict__ S, bool auto_policy) {
    const int lane = threadIdx.x & 31;
    stage_source(P, S);
    if (lane < 26) reinterpret_cast<uint32_t*>(&S.res)[lane] = 0;
    __syncwarp();
    if (lane == 0) S.sad_px = S.satd_px = 0;
    // P_Skip (enc/frame.rs:722-729)
    const int2 sv = skip_mv(P, S);
    if (lane == 0) S.cand[0] = sv;
    __syncwarp();
    pred_batch(P, S, 0, 0, 0, 2, 2, 1, true);
    const int skip_sad = S.cost[0];
    __syncwarp();
    if (lane == 0) S.sad_px += 256;
    const bool skip = auto_policy && skip_sad < P.skip_thresh;
    int part = 0, cost = 0, cost16 = 0, bestr = 0;
    uint32_t sub = 0;
    if (!skip) {
        // best_inter, enc/frame.rs:839-849: every reference, the cheapest (first on ties) wins
        for (int r = 0; r < P.nact; r++) {
            const int4 bi = best_inter_or_learned(P, S, r);
            const int c = bi.x, p = bi.y, c16 = bi.w;
            const uint32_t sb = (uint32_t)bi.z;
            if (r == 0 || c < cost) {
                part = p;
                cost = c;
                cost16 = c16;
                bestr = r;
                sub = sb;
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
        R.skip_mv[0] = (int16_t)sv.x;
        R.skip_mv[1] = (int16_t)sv.y;
        R.skip_sad = skip_sad;
        R.flags = skip ? IRONAV_RESULT_SKIP : IRONAV_RESULT_INTER;
        if (!skip) {
            R.part = (uint8_t)part;
            for (int i = 0; i < 4; i++) {
                R.refs[i] = (uint8_t)bestr;
                R.sub[i] = (uint8_t)((sub >> (8 * i)) & 0xff);
            }
            R.cost = cost;
            R.cost16 = cost16;
        }
        R.sad_px = S.sad_px;
        R.satd_px = S.satd_px;
    }
    __syncwarp();
    if (lane < 16 && !skip) {
        S.res.mvs[lane][0] = S.win_mvs[lane][0];
        S.res.mvs[lane][1] = S.win_mvs[lane][1];
    }
    __syncwarp();
    if (lane < 26) reinterpret_cast<uint32_t*>(&P.results[S.mb])[lane] = reinterpret_cast<const uint32_t*>(&S.res)[lane];
    if (auto_policy) {
        // the decision's MbState (finish_mb, enc/frame.rs:2281-2321)
        if (lane < 16) {
            const int bx = lane & 3, by = lane >> 2;
            int mx = sv.x, my = sv.y;
            if (!skip) {
                // the rectangle of rects(part, sub) holding this block, in coding order
                int idx = 0;
                if (part == 1) idx = by >> 1;
                else if (part == 2) idx = bx >> 1;
                else if (part == 3) {
                    const int k = (by >> 1) * 2 + (bx >> 1);
                    int n = 0;
                    for (int q = 0; q < k; q++) n += c_nsub[(sub >> (8 * q)) & 0xff];
                    const int s = (sub >> (8 * k)) & 0xff, lx = bx & 1, ly = by & 1;
                    idx = n + (s == 0 ? 0 : (s == 1 ? ly : (s == 2 ? lx : ly * 2 + lx)));
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
        if (lane < 18) reinterpret_cast<uint32_t*>(&P.states_out[S.mb])[lane] = reinterpret_cast<const uint32_t*>(&S.out)[lane];
    }
    __syncwarp();
}


// Waits until macroblock `m`'s decision is published, at most P.wait_limit polls. Returns false when
// it gave up or another warp already did (the launch is then abandoned and the host reports a timeout).
// Polls are relaxed loads and one fence.acq_rel follows the flag (the acquire pattern of the PTX memory
// model): an acquire load per poll would order, and cost, every poll of every waiting warp.
static __device__ bool wait_published(const AnalyseParams& P, int m) {
    for (unsigned i = 0;; i++) {
        unsigned f, e;
        asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(f) : "l"(&P.flags[m]) : "memory");
        if (f == P.epoch) {
            asm volatile("fence.acq_rel.gpu;" ::: "memory");
            return true;
        }
        asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(e) : "l"(P.err) : "memory");
        if (e != 0) return false;
        if (i >= P.wait_limit) {
            atomicOr(P.err, 1u);
            return false;
        }
        __nanosleep(i < 64 ? 32 : 256);
    }
}

enum : int { MODE_REPLAY = 0, MODE_AUTO = 1, MODE_INLOOP = 2 };

__device__ __forceinline__ unsigned ld_acquire_sys(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.sys.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_sys(unsigned* p, unsigned v) {
    asm volatile("st.release.sys.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long globaltimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// In-loop mode: waits until the caller has committed macroblock m's final decision, for at most
// P.wait_ns of wall time (the caller's own mode decision sits between two macroblocks). Backs off to
// microsecond sleeps: the flag lives in host memory, so every poll crosses the bus.
static __device__ bool wait_committed(const AnalyseParams& P, int m) {
    const unsigned long long t0 = globaltimer();
    for (unsigned i = 0;; i++) {
        if (ld_acquire_sys(&P.commit_flags[m]) == P.epoch) return true;
        if (ld_acquire(P.err) != 0) return false;
        if ((i & 15) == 15 && globaltimer() - t0 > P.wait_ns) {
            atomicOr(P.err, 1u);
            return false;
        }
        __nanosleep(i < 32 ? 256 : 4000);
    }
}

// The neighbours of an in-loop macroblock from the caller's committed decisions (host memory: read
// around the caches, after the acquire of their flags).
template <class T>
static __device__ void load_committed(const AnalyseParams& __restrict__ P, WarpSmem<T>& __restrict__ S) {
    const int lane = threadIdx.x & 31;
    if (lane < 30) {
        const int ex = lane % 6 - 1, ey = lane / 6 - 1;
        Blk e = make_int4(0, 0, -1, 0);
        if (ey < 0 || ex < 0) {
            const int nx = S.mbx + (ex < 0 ? -1 : (ex >= 4 ? 1 : 0)), ny = S.mby + (ey < 0 ? -1 : 0);
            const int bx = ex < 0 ? 3 : (ex >= 4 ? 0 : ex), by = ey < 0 ? 3 : ey;
            if (nx >= 0 && nx < P.mb_w && ny >= P.band_start[S.mby] && ny < P.mb_h) {
                const uint32_t* w = reinterpret_cast<const uint32_t*>(&P.committed[(size_t)ny * P.mb_w + nx]);
                const uint32_t w0 = __ldcv(w), w1 = __ldcv(w + 1);  // inter, refs[0..2] | refs[3], pad
                const uint32_t mv = __ldcv(w + 2 + by * 4 + bx);
                const int inter = w0 & 0xff;
                const int rsel = (by >> 1) * 2 + (bx >> 1);
                const int rf = (int)(int8_t)(rsel < 3 ? (w0 >> (8 * (rsel + 1))) & 0xff : w1 & 0xff);
                e.w = 1;
                if (inter && rf >= 0) {
                    e.x = (int)(int16_t)(mv & 0xffffu);
                    e.y = (int)(int16_t)(mv >> 16);
                    e.z = rf;
                }
            }
        }
        S.ext[lane] = e;
    }
    __syncwarp();
}

template <int MODE, class T>
__global__ void __launch_bounds__(K2_WARPS * 32, K2_MIN_BLOCKS) analyse_kernel(const __grid_constant__ AnalyseParams P) {
    __shared__ WarpSmem<T> smem[K2_WARPS];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    WarpSmem<T>& S = smem[wid];
    for (;;) {
        unsigned t = 0;
        if (lane == 0) t = atomicAdd(P.ticket, 1u);
        t = __shfl_sync(FULL, t, 0);
        if (t >= (unsigned)P.nmb) break;
        const int mb = P.order ? P.order[t] : (int)t;
        const int mbx = mb % P.mb_w, mby = mb / P.mb_w;
        if (lane == 0) {
            S.mb = mb;
            S.mbx = mbx;
            S.mby = mby;
        }
        __syncwarp();
        if (MODE == MODE_REPLAY) {
            load_neighbours(P, S, P.states_in);
        } else {
            // the left and top-right (top at the right edge) neighbours; their own waits cover the rest
            const int start = P.band_start[mby];
            const int m1 = mb - 1, m2 = (mbx + 1 < P.mb_w) ? mb - P.mb_w + 1 : mb - P.mb_w;
            bool ok = true;
            if (MODE == MODE_AUTO) {
                if (mbx > 0) ok = wait_published(P, m1);
                if (ok && mby > start) ok = wait_published(P, m2);
            } else {
                if (mbx > 0) ok = wait_committed(P, m1);
                if (ok && mby > start) ok = wait_committed(P, m2);
            }
            ok = __all_sync(FULL, ok);
            if (!ok) break;
            if (MODE == MODE_AUTO) load_neighbours(P, S, P.states_out);
            else load_committed(P, S);
        }
        analyse(P, S, MODE == MODE_AUTO);
        if (MODE == MODE_AUTO) {
            __threadfence();
            __syncwarp();
            if (lane == 0 && mb != P.withhold) st_release(&P.flags[mb], P.epoch);
        } else if (MODE == MODE_INLOOP) {
            // the result is in host memory: make it visible there before its flag
            __threadfence_system();
            __syncwarp();
            if (lane == 0) st_release_sys(&P.done_flags[mb], P.epoch);
        }
    }
}

}  // namespace ironav
