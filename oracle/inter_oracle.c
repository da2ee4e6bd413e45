/*
 * inter_oracle.c — CPU restatement of IronAV's H.264 P-picture inter-analysis stage.
 *
 * TEST INFRASTRUCTURE ONLY. This file is the parity checker and the timed CPU baseline. It is never
 * part of the product path: only the tests, the smoke check and the benchmark's CPU-baseline leg load
 * the library built from it (liboracle: oracle/_build/libironav_inter_cpu.so).
 *
 * The reference is Rust (nervosys/IronAV 0.1.10, crate ironav-codec) and no Rust toolchain exists
 * here, so this is a line-by-line restatement in C of the functions listed below, each citing the file
 * and lines it follows (paths relative to crates/ironav-codec/src/h264/):
 *   HalfPel::build / predict / rows ........ enc/subpel.rs:21-151
 *   luma_mc_ref (decoder's per-sample form)  inter.rs:466-546   (only to pin predict, as enc/subpel.rs:160-194 does)
 *   satd4, lambda, mvd_bits, median ........ enc/frame.rs:144-175
 *   se_bits / ue_bits ...................... enc/bitw.rs:81-89
 *   PARTS, SUB, rects, spread, paint ....... enc/frame.rs:182-236
 *   nb_state, nb_motion, pred_mv, mv_pred,
 *   part_mvps, skip_mv ..................... enc/frame.rs:509-603
 *   satd, sad_int, luma_pred, ref_bits ..... enc/frame.rs:641-711
 *   P_Skip SAD ............................. enc/frame.rs:722-729
 *   best_inter, best_inter_ref, sub_search,
 *   col_mv, motion_search .................. enc/frame.rs:839-1019
 *   slice bands ............................ enc/mod.rs:192,603
 *   source padding ......................... enc/mod.rs:481-529
 * and beyond the stage, the encoder around it (decide mode, the bitstream), among them the High profile
 * with CABAC (the reference encoder's default):
 *   CabacWriter, CabacCost, write_block .... enc/cabac.rs:10-250
 *   mb_bins / write_mb_cabac, mvd_bins ..... enc/frame.rs:2020-2279,2393-2414
 *   decide_rd, rd_cost, ssd_mb, save/restore enc/frame.rs:1406-1513
 *   code_i8, filter_8x8_edges, predict_nxn(8)  enc/frame.rs:1307-1388; intra.rs:30-158
 *   sps / pps (Main, High), cabac_init_idc . enc/mod.rs:296-400,566-600
 * whose streams FFmpeg decodes to the oracle's reconstruction (tests/test_cabac.py), and whose arithmetic
 * coder reads back through a decoder of the standard on the reference's own coder test.
 *
 * Pinning. The interpolation (planes + predict) is pinned by the reference's own known-answer test,
 * predict == the decoder's interpolation over the same grid of blocks and vectors (enc/subpel.rs:160-194,
 * restated in tests/test_oracle.py against luma_mc_ref below), and the Exp-Golomb bit counts by the
 * code lengths of enc/bitw.rs:110-135. The motion search and partition decision have no golden
 * vectors in the reference (no test pins MVs, costs or partitions): for them parity is UNPINNED beyond
 * this restatement, which follows the Rust statement by statement (strict '<' with first-wins order,
 * the same clamps, the same early breaks).
 *
 * Samples are kept as uint16 like the reference, so the 10-bit planes of the known-answer test run
 * through the same code.
 */
#include "../include/ironav_inter.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define PAD 48 /* enc/subpel.rs:7 */

/* ---------------------------------------------------------------------------------------------------
 * HalfPel (enc/subpel.rs)
 * ------------------------------------------------------------------------------------------------- */

typedef struct halfpel {
    int stride, pw, ph, sh;
    uint16_t* planes[4]; /* G, b, h, j */
} halfpel;

static int tap6(int a, int b, int c, int d, int e, int f) { return a - 5 * b + 20 * c + 20 * d - 5 * e + f; } /* subpel.rs:21-23 */

static int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
static int mini(int a, int b) { return a < b ? a : b; }
static int maxi(int a, int b) { return a > b ? a : b; }

/* HalfPel::build, enc/subpel.rs:57-115 (single-threaded; the threaded form gives the same planes). */
static void halfpel_build(halfpel* hp, const uint16_t* luma, int pw, int ph, int bd) {
    int maxv = (1 << bd) - 1;
    int sw = pw + 2 * PAD, sh = ph + 2 * PAD;
    size_t n = (size_t)sw * sh;
    hp->stride = sw;
    hp->pw = pw;
    hp->ph = ph;
    hp->sh = sh;
    for (int k = 0; k < 4; k++) hp->planes[k] = (uint16_t*)calloc(n, sizeof(uint16_t));
    int32_t* b1 = (int32_t*)calloc(n, sizeof(int32_t));
    uint16_t *g = hp->planes[0], *b = hp->planes[1], *h = hp->planes[2], *j = hp->planes[3];
    /* round1: integer samples with the edges repeated, and the horizontal half samples (subpel.rs:71-85) */
    for (int y = 0; y < sh; y++) {
        int sy = mini(y >= PAD ? y - PAD : 0, ph - 1);
        uint16_t* gr = g + (size_t)y * sw;
        for (int x = 0; x < sw; x++) gr[x] = luma[(size_t)sy * pw + mini(x >= PAD ? x - PAD : 0, pw - 1)];
        for (int x = 2; x < sw - 3; x++) {
            int v = tap6(gr[x - 2], gr[x - 1], gr[x], gr[x + 1], gr[x + 2], gr[x + 3]);
            b1[(size_t)y * sw + x] = v;
            b[(size_t)y * sw + x] = (uint16_t)clampi((v + 16) >> 5, 0, maxv);
        }
    }
    /* round2: vertical half samples from G and diagonal ones from the unrounded sums (subpel.rs:93-108) */
    for (int y = 2; y < sh - 3; y++) {
        for (int x = 0; x < sw; x++) {
#define G_(yy) ((int)g[(size_t)(yy) * sw + x])
#define B1_(yy) (b1[(size_t)(yy) * sw + x])
            int v = tap6(G_(y - 2), G_(y - 1), G_(y), G_(y + 1), G_(y + 2), G_(y + 3));
            h[(size_t)y * sw + x] = (uint16_t)clampi((v + 16) >> 5, 0, maxv);
            v = tap6(B1_(y - 2), B1_(y - 1), B1_(y), B1_(y + 1), B1_(y + 2), B1_(y + 3));
            j[(size_t)y * sw + x] = (uint16_t)clampi((v + 512) >> 10, 0, maxv);
#undef G_
#undef B1_
        }
    }
    free(b1);
}

static void halfpel_free(halfpel* hp) {
    for (int k = 0; k < 4; k++) {
        free(hp->planes[k]);
        hp->planes[k] = NULL;
    }
}

/* MIX, enc/subpel.rs:26-38: [fy][fx] -> (plane a, dx, dy, plane b, dx, dy) with G=0, B=1, H=2, J=3. */
static const unsigned char MIX[4][4][6] = {
    {{0, 0, 0, 0, 0, 0}, {0, 0, 0, 1, 0, 0}, {1, 0, 0, 1, 0, 0}, {0, 1, 0, 1, 0, 0}},
    {{0, 0, 0, 2, 0, 0}, {1, 0, 0, 2, 0, 0}, {1, 0, 0, 3, 0, 0}, {1, 0, 0, 2, 1, 0}},
    {{2, 0, 0, 2, 0, 0}, {2, 0, 0, 3, 0, 0}, {3, 0, 0, 3, 0, 0}, {3, 0, 0, 2, 1, 0}},
    {{0, 0, 1, 2, 0, 0}, {2, 0, 0, 1, 0, 1}, {3, 0, 0, 1, 0, 1}, {2, 1, 0, 1, 0, 1}},
};

static size_t hp_offset(const halfpel* hp, int x, int y) { return (size_t)(y + PAD) * hp->stride + (size_t)(x + PAD); } /* subpel.rs:117-119 */

/* HalfPel::predict, enc/subpel.rs:122-145. */
static void halfpel_predict(const halfpel* hp, int x, int y, int mvx, int mvy, int w, int h, uint16_t* out) {
    int fx = mvx & 3, fy = mvy & 3;
    int ix = clampi(x + (mvx >> 2), -w - 3, hp->pw + 1);
    int iy = clampi(y + (mvy >> 2), -h - 3, hp->ph + 1);
    const unsigned char* m = MIX[fy][fx];
    int s = hp->stride;
    const uint16_t* a = hp->planes[m[0]] + hp_offset(hp, ix + m[1], iy + m[2]);
    if (m[0] == m[3] && m[1] == m[4] && m[2] == m[5]) {
        for (int r = 0; r < h; r++)
            for (int c = 0; c < w; c++) out[r * w + c] = a[r * s + c];
    } else {
        const uint16_t* b = hp->planes[m[3]] + hp_offset(hp, ix + m[4], iy + m[5]);
        for (int r = 0; r < h; r++)
            for (int c = 0; c < w; c++) out[r * w + c] = (uint16_t)(((unsigned)a[r * s + c] + b[r * s + c] + 1) >> 1);
    }
}

/* ---------------------------------------------------------------------------------------------------
 * luma_mc_ref, h264/inter.rs:466-546: the decoder's per-sample interpolation (8.4.2.2.1), restated to
 * pin HalfPel::predict as the reference's test enc/subpel.rs:160-194 does.
 * ------------------------------------------------------------------------------------------------- */

static int clip1(int v, int maxv) { return clampi(v, 0, maxv); } /* inter.rs:3-5 */

void oracle_luma_mc_ref(const uint16_t* refp, int stride, int pw, int ph, int x, int y, int mx, int my, int w, int h,
                        uint16_t* out, int maxv) {
    int fx = mx & 3, fy = my & 3;
    int x0 = x + (mx >> 2), y0 = y + (my >> 2);
    if (fx == 0 && fy == 0) {
        for (int r = 0; r < h; r++) {
            int yy = clampi(y0 + r, 0, ph - 1);
            for (int c = 0; c < w; c++) out[r * w + c] = refp[(size_t)yy * stride + clampi(x0 + c, 0, pw - 1)];
        }
        return; /* the in-picture fast path of inter.rs:470-475 reads the same samples */
    }
    /* window of (w+5) x (h+5) samples from 2 left of and 2 above the block, edges repeated (inter.rs:489-506) */
    int ww = w + 5, wh = h + 5;
    int win[21 * 21];
    for (int r = 0; r < wh; r++) {
        int yy = clampi(y0 - 2 + r, 0, ph - 1);
        for (int c = 0; c < ww; c++) win[r * ww + c] = refp[(size_t)yy * stride + clampi(x0 - 2 + c, 0, pw - 1)];
    }
#define GW(c, r) (win[((r) + 2) * ww + (c) + 2])
    /* unrounded horizontal sums at (window column c, window row rr) (inter.rs:509-520) */
    int b1[21 * 21];
    memset(b1, 0, sizeof(b1));
    for (int rr = 0; rr < wh; rr++)
        for (int c = 0; c < w; c++) {
            const int* t = &win[rr * ww + c];
            b1[rr * ww + c] = tap6(t[0], t[1], t[2], t[3], t[4], t[5]);
        }
#define BH(c, r) (clip1((b1[((r) + 2) * ww + (c)] + 16) >> 5, maxv))
#define HV(c, r) (clip1((tap6(win[(r)*ww + (c) + 2], win[((r) + 1) * ww + (c) + 2], win[((r) + 2) * ww + (c) + 2],       \
                              win[((r) + 3) * ww + (c) + 2], win[((r) + 4) * ww + (c) + 2], win[((r) + 5) * ww + (c) + 2]) + \
                         16) >> 5,                                                                                        \
                        maxv))
#define JJ(c, r) (clip1((tap6(b1[(r)*ww + (c)], b1[((r) + 1) * ww + (c)], b1[((r) + 2) * ww + (c)],                       \
                              b1[((r) + 3) * ww + (c)], b1[((r) + 4) * ww + (c)], b1[((r) + 5) * ww + (c)]) + 512) >> 10, \
                        maxv))
    for (int r = 0; r < h; r++) {
        for (int c = 0; c < w; c++) {
            int v;
            switch (fy * 4 + fx) { /* (fx, fy) cases of inter.rs:529-545 */
            case 0 * 4 + 1: v = (GW(c, r) + BH(c, r) + 1) >> 1; break;
            case 0 * 4 + 2: v = BH(c, r); break;
            case 0 * 4 + 3: v = (GW(c + 1, r) + BH(c, r) + 1) >> 1; break;
            case 1 * 4 + 0: v = (GW(c, r) + HV(c, r) + 1) >> 1; break;
            case 2 * 4 + 0: v = HV(c, r); break;
            case 3 * 4 + 0: v = (GW(c, r + 1) + HV(c, r) + 1) >> 1; break;
            case 1 * 4 + 1: v = (BH(c, r) + HV(c, r) + 1) >> 1; break;
            case 1 * 4 + 3: v = (BH(c, r) + HV(c + 1, r) + 1) >> 1; break;
            case 3 * 4 + 1: v = (HV(c, r) + BH(c, r + 1) + 1) >> 1; break;
            case 3 * 4 + 3: v = (HV(c + 1, r) + BH(c, r + 1) + 1) >> 1; break;
            case 1 * 4 + 2: v = (BH(c, r) + JJ(c, r) + 1) >> 1; break;
            case 3 * 4 + 2: v = (JJ(c, r) + BH(c, r + 1) + 1) >> 1; break;
            case 2 * 4 + 1: v = (HV(c, r) + JJ(c, r) + 1) >> 1; break;
            case 2 * 4 + 3: v = (JJ(c, r) + HV(c + 1, r) + 1) >> 1; break;
            default: v = JJ(c, r); break;
            }
            out[r * w + c] = (uint16_t)v;
        }
    }
#undef GW
#undef BH
#undef HV
#undef JJ
}

/* ---------------------------------------------------------------------------------------------------
 * Costs and bit counts
 * ------------------------------------------------------------------------------------------------- */

/* satd4, enc/frame.rs:144-161 */
static int satd4(const int d[16]) {
    int t[16];
    for (int r = 0; r < 4; r++) {
        int a = d[r * 4], b = d[r * 4 + 1], c = d[r * 4 + 2], e = d[r * 4 + 3];
        int s0 = a + b, s1 = c + e, d0 = a - b, d1 = c - e;
        t[r * 4] = s0 + s1;
        t[r * 4 + 1] = s0 - s1;
        t[r * 4 + 2] = d0 - d1;
        t[r * 4 + 3] = d0 + d1;
    }
    int sum = 0;
    for (int c = 0; c < 4; c++) {
        int a = t[c], b = t[4 + c], cc = t[8 + c], e = t[12 + c];
        int s0 = a + b, s1 = cc + e, d0 = a - b, d1 = cc - e;
        sum += abs(s0 + s1) + abs(s0 - s1) + abs(d0 - d1) + abs(d0 + d1);
    }
    return sum >> 1;
}

/* ue_bits / se_bits, enc/bitw.rs:81-89 */
int ironav_ue_bits(unsigned v) {
    unsigned x = v + 1;
    int len = 32 - __builtin_clz(x);
    return 2 * len - 1;
}
int ironav_se_bits(int v) {
    unsigned u = v > 0 ? 2u * (unsigned)v - 1u : (unsigned)(-2 * (long long)v);
    return ironav_ue_bits(u);
}

/* lambda, enc/frame.rs:164-166 */
int ironav_lambda(int qp) {
    int l = (int)round(pow(2.0, ((double)qp - 12.0) / 6.0));
    return l < 1 ? 1 : l;
}

/* The P_Skip test `(sad as f64) < 256.0 * 0.625 * step` with step = 2^(qp'/6), enc/frame.rs:730,742,
 * as an integer bound: sad < ceil(x) for every integer sad. */
int ironav_skip_threshold(int qpp) {
    double x = 256.0 * 0.625 * pow(2.0, (double)qpp / 6.0);
    return (int)ceil(x);
}

/* mvd_bits, enc/frame.rs:169-171 */
static int mvd_bits(int mx, int my, int px, int py) { return ironav_se_bits(mx - px) + ironav_se_bits(my - py); }

/* median, enc/frame.rs:173-175 */
static int median3(int a, int b, int c) { return mini(maxi(a, b), maxi(mini(a, b), c)); }

const char* ironav_version(void) { return "cpu-oracle (C restatement of ironav-codec 0.1.10 h264::enc inter analysis)"; }

/* ---------------------------------------------------------------------------------------------------
 * Partition geometry, enc/frame.rs:182-236
 * ------------------------------------------------------------------------------------------------- */

typedef struct { int x, y, w, h; } rect4;

static const rect4 PARTS_[4][4] = {
    {{0, 0, 4, 4}}, {{0, 0, 4, 2}, {0, 2, 4, 2}}, {{0, 0, 2, 4}, {2, 0, 2, 4}}, {{0, 0, 2, 2}, {2, 0, 2, 2}, {0, 2, 2, 2}, {2, 2, 2, 2}}};
static const int NPARTS[4] = {1, 2, 2, 4};
static const rect4 SUB_[4][4] = {
    {{0, 0, 2, 2}}, {{0, 0, 2, 1}, {0, 1, 2, 1}}, {{0, 0, 1, 2}, {1, 0, 1, 2}}, {{0, 0, 1, 1}, {1, 0, 1, 1}, {0, 1, 1, 1}, {1, 1, 1, 1}}};
static const int NSUB[4] = {1, 2, 2, 4};

/* rects, enc/frame.rs:208-213: returns the count */
static int rects(int part, const uint8_t sub[4], rect4 out[16]) {
    if (part != 3) {
        for (int k = 0; k < NPARTS[part]; k++) out[k] = PARTS_[part][k];
        return NPARTS[part];
    }
    int n = 0;
    for (int k = 0; k < 4; k++)
        for (int s = 0; s < NSUB[sub[k]]; s++) {
            rect4 r = SUB_[sub[k]][s];
            r.x += (k & 1) * 2;
            r.y += (k >> 1) * 2;
            out[n++] = r;
        }
    return n;
}

/* ref_of (enc/frame.rs:217-223) is not needed: a P macroblock's partitions all use the reference
 * best_inter_ref searches (refs = [r; 4], enc/frame.rs:854). */

/* ---------------------------------------------------------------------------------------------------
 * One picture's analysis (FrameCoder, enc/frame.rs:337-1019, the parts the stage covers)
 * ------------------------------------------------------------------------------------------------- */

typedef struct colmv { int16_t mv[2]; uint8_t valid; } colmv;

typedef struct refpic {
    halfpel hp;
    colmv* col;         /* per macroblock: mvs[5] when the macroblock was inter (col_mv, enc/frame.rs:944-947) */
    uint16_t* chroma[2]; /* Cb, Cr of the reconstruction (8*mb_w x 8*mb_h), when attached */
} refpic;

struct ironav_ctx {
    int width, height, bd, mb_w, mb_h, pw, ph, max_refs, nslices;
    int* band_start; /* per macroblock row: first row of its slice band */
    uint16_t* src;   /* padded source, pw x ph */
    refpic* refs;    /* newest first */
    int nrefs;
    /* picture parameters */
    int qpp, lambda, skip_thresh, nact, fast, sub8;
    int intra_pic; /* the picture parameters are an IDR picture's (ironav_begin_i_picture) */
    int cabac, t8; /* entropy coding: CABAC, and transform_8x8_mode_flag with it (ironav_set_entropy) */
    int threads;
    void* inloop; /* in-loop mode state */
    /* B picture parameters */
    int b_ref[2];           /* held references used as list 0 and list 1 */
    ironav_mbstate* b_col;  /* the list-1 picture's decisions, or NULL */
    int b_tb, b_td, b_set;
    uint16_t* src_c[2]; /* the source's chroma, padded to 8*mb_w x 8*mb_h */
    /* the learned form's proposals (ironav_set_learned; host pointers here) */
    const int16_t* learned;
    const uint8_t* learned_cls;
    int learned_margin;
    unsigned* learned_stats;
};

typedef struct fc {
    const struct ironav_ctx* c;
    const ironav_mbstate* states;    /* final states of the whole picture (P pictures) */
    const ironav_mbstate_b* bstates; /* B pictures: final states with both lists (NULL for P pictures) */
    int list;                        /* B pictures: the list the neighbour lookups and searches use */
    const halfpel* bhp;              /* B pictures: that list's reference picture */
} fc;

/* nb_state, enc/frame.rs:509-515: the index of the neighbour's state, or -1 when it is not available */
static long nb_index(const fc* f, int mbx, int mby, int cur_mby) {
    const struct ironav_ctx* c = f->c;
    int start = c->band_start[cur_mby];
    if (mbx < 0 || mby < start || mbx >= c->mb_w || mby >= c->mb_h) return -1;
    return (long)mby * c->mb_w + mbx;
}

typedef struct nbm { int avail, ref, mv[2]; } nbm;

/* nb_motion, enc/frame.rs:522-538 (list 0; P slices never set the high `done` bits) */
static nbm nb_motion(const fc* f, int mbx, int mby, const int16_t cur[16][2], const int8_t cref[16], uint32_t done, int x, int y) {
    nbm r = {0, -1, {0, 0}};
    int dx, dy, bx, by;
    if (x < 0 && y < 0) { dx = -1; dy = -1; bx = 3; by = 3; }
    else if (x < 0) { dx = -1; dy = 0; bx = 3; by = y; }
    else if (x >= 4 && y < 0) { dx = 1; dy = -1; bx = 0; by = 3; }
    else if (x >= 4) return r;
    else if (y < 0) { dx = 0; dy = -1; bx = x; by = 3; }
    else {
        int b = y * 4 + x;
        if ((done >> b) & 1) {
            r.avail = 1;
            if ((done >> (16 + b)) & 1) return r; /* (-1, [0, 0]) */
            r.ref = cref[b];
            r.mv[0] = cur[b][0];
            r.mv[1] = cur[b][1];
        }
        return r;
    }
    long i = nb_index(f, mbx + dx, mby + dy, mby);
    if (i < 0) return r;
    r.avail = 1;
    if (f->bstates) {
        /* a B picture's neighbour, in list f->list (MbState.refs[l], mvs / mvs1) */
        const ironav_mbstate_b* sb = &f->bstates[i];
        int rf = sb->refs[f->list][(by / 2) * 2 + bx / 2];
        if (sb->inter && rf >= 0) {
            r.ref = rf;
            r.mv[0] = sb->mvs[f->list][by * 4 + bx][0];
            r.mv[1] = sb->mvs[f->list][by * 4 + bx][1];
        }
        return r;
    }
    const ironav_mbstate* s = &f->states[i];
    int rf = s->refs[(by / 2) * 2 + bx / 2];
    if (s->inter && rf >= 0) {
        r.ref = rf;
        r.mv[0] = s->mvs[by * 4 + bx][0];
        r.mv[1] = s->mvs[by * 4 + bx][1];
    }
    return r;
}

/* pred_mv, enc/frame.rs:543-570 */
static void pred_mv(const fc* f, int mbx, int mby, const int16_t cur[16][2], const int8_t cref[16], uint32_t done, int bx, int by,
                    int w, int dir, int rf, int out[2]) {
    nbm a = nb_motion(f, mbx, mby, cur, cref, done, bx - 1, by);
    nbm b = nb_motion(f, mbx, mby, cur, cref, done, bx, by - 1);
    nbm c = nb_motion(f, mbx, mby, cur, cref, done, bx + w, by - 1);
    if (!c.avail) c = nb_motion(f, mbx, mby, cur, cref, done, bx - 1, by - 1);
    /* r(n) = n.map_or(-1, ref) — an unavailable neighbour has ref -1 and vector 0 */
    const nbm* pick = NULL;
    if (dir == 1 && by == 0 && b.ref == rf) pick = &b;
    else if (dir == 1 && by != 0 && a.ref == rf) pick = &a;
    else if (dir == 2 && bx == 0 && a.ref == rf) pick = &a;
    else if (dir == 2 && bx != 0 && c.ref == rf) pick = &c;
    if (pick) { out[0] = pick->mv[0]; out[1] = pick->mv[1]; return; }
    if (!b.avail && !c.avail && a.avail) { out[0] = a.mv[0]; out[1] = a.mv[1]; return; }
    int ra = a.ref == rf, rb = b.ref == rf, rc = c.ref == rf;
    if (ra + rb + rc == 1) {
        const nbm* p = ra ? &a : (rb ? &b : &c);
        out[0] = p->mv[0];
        out[1] = p->mv[1];
        return;
    }
    out[0] = median3(a.mv[0], b.mv[0], c.mv[0]);
    out[1] = median3(a.mv[1], b.mv[1], c.mv[1]);
}

static const int16_t ZERO_MVS[16][2];
static const int8_t NO_REF[16];

/* mv_pred, enc/frame.rs:573-575 */
static void mv_pred(const fc* f, int mbx, int mby, int rf, int out[2]) { pred_mv(f, mbx, mby, ZERO_MVS, NO_REF, 0, 0, 0, 4, 0, rf, out); }

/* part_mvps, enc/frame.rs:579-594: the predictor of partition k of `part` given mvs of those before */
static void part_mvp(const fc* f, int mbx, int mby, int part, const int16_t mvs[16][2], int rf, int want, int out[2]) {
    int16_t cur[16][2];
    int8_t cref[16];
    uint32_t done = 0;
    memset(cur, 0, sizeof(cur));
    memset(cref, 0, sizeof(cref));
    static const uint8_t nosub[4] = {0, 0, 0, 0};
    rect4 rs[16];
    int n = rects(part, nosub, rs);
    int dir = part == 1 ? 1 : (part == 2 ? 2 : 0);
    for (int k = 0; k < n; k++) {
        rect4 r = rs[k];
        if (k == want) {
            pred_mv(f, mbx, mby, cur, cref, done, r.x, r.y, r.w, dir, rf, out);
            return;
        }
        for (int by = r.y; by < r.y + r.h; by++)
            for (int bx = r.x; bx < r.x + r.w; bx++) {
                cur[by * 4 + bx][0] = mvs[k][0];
                cur[by * 4 + bx][1] = mvs[k][1];
                cref[by * 4 + bx] = (int8_t)rf;
                done |= 1u << (by * 4 + bx);
            }
    }
}

/* skip_mv, enc/frame.rs:597-603 */
static void skip_mv(const fc* f, int mbx, int mby, int out[2]) {
    nbm a = nb_motion(f, mbx, mby, ZERO_MVS, NO_REF, 0, -1, 0);
    nbm b = nb_motion(f, mbx, mby, ZERO_MVS, NO_REF, 0, 0, -1);
    if (!a.avail || !b.avail || (a.ref == 0 && a.mv[0] == 0 && a.mv[1] == 0) || (b.ref == 0 && b.mv[0] == 0 && b.mv[1] == 0)) {
        out[0] = out[1] = 0;
        return;
    }
    mv_pred(f, mbx, mby, 0, out);
}

/* satd, enc/frame.rs:641-659 (luma) */
static int satd_blk(const fc* f, int x, int y, int w, int h, const uint16_t* pred) {
    int s = f->c->pw;
    const uint16_t* src = f->c->src;
    int total = 0;
    for (int by = 0; by < h; by += 4)
        for (int bx = 0; bx < w; bx += 4) {
            int d[16];
            for (int r = 0; r < 4; r++)
                for (int c = 0; c < 4; c++) d[r * 4 + c] = (int)src[(size_t)(y + by + r) * s + x + bx + c] - (int)pred[(by + r) * w + bx + c];
            total += satd4(d);
        }
    return total;
}

/* sad_int, enc/frame.rs:662-671 with HalfPel::rows, enc/subpel.rs:148-151 */
static int sad_int(const fc* f, int r, int x, int y, int w, int h, int mvx, int mvy) {
    const halfpel* hp = f->bhp ? f->bhp : &f->c->refs[r].hp;
    const uint16_t* g = hp->planes[0] + hp_offset(hp, x + (mvx >> 2), y + (mvy >> 2));
    const uint16_t* src = f->c->src + (size_t)y * f->c->pw + x;
    int sad = 0;
    for (int rr = 0; rr < h; rr++)
        for (int c = 0; c < w; c++) sad += abs((int)src[(size_t)rr * f->c->pw + c] - (int)g[(size_t)rr * hp->stride + c]);
    return sad;
}

/* ref_bits, enc/frame.rs:705-711 */
static int ref_bits(const fc* f, int r) {
    int n = f->c->nact;
    if (n <= 1) return 0;
    if (n == 2) return 1;
    unsigned v = (unsigned)r + 1;
    return 2 * (31 - __builtin_clz(v)) + 1;
}

typedef struct counters { uint32_t sad_px, satd_px; } counters;

/* motion_search, enc/frame.rs:949-1019 (list 0). Returns the cost without the vector's bits. */
static int motion_search(const fc* f, counters* cnt, int r, int mbx, int mby, rect4 pr, const int mvp[2], const int (*extra)[2],
                         int nextra, int out[2]) {
    const struct ironav_ctx* c = f->c;
    int lam = c->lambda;
    int x0 = mbx * 16 + pr.x * 4, y0 = mby * 16 + pr.y * 4, w = pr.w * 4, h = pr.h * 4;
    int lo_x = -(x0 + 24) * 4, hi_x = (c->mb_w * 16 - x0 + 8) * 4;
    int lo_y = -(y0 + 24) * 4, hi_y = (c->mb_h * 16 - y0 + 8) * 4;
    int cxlo = maxi(lo_x, -2048), cxhi = mini(hi_x, 2047), cylo = maxi(lo_y, -512), cyhi = mini(hi_y, 511);
#define CLX(v) clampi((v), cxlo, cxhi)
#define CLY(v) clampi((v), cylo, cyhi)
#define INTR(v) (((v) + 2) & ~3)
#define COST_INT(mx, my) (cnt->sad_px += (uint32_t)(w * h), sad_int(f, r, x0, y0, w, h, (mx), (my)) + lam * mvd_bits((mx), (my), mvp[0], mvp[1]))
    int cands[16][2];
    int nc = 0;
    cands[nc][0] = INTR(CLX(mvp[0]));
    cands[nc][1] = INTR(CLY(mvp[1]));
    nc++;
    cands[nc][0] = 0;
    cands[nc][1] = 0;
    nc++;
    static const int NB[3][2] = {{-1, 0}, {0, -1}, {4, -1}};
    for (int k = 0; k < 3; k++) {
        nbm n = nb_motion(f, mbx, mby, ZERO_MVS, NO_REF, 0, NB[k][0], NB[k][1]);
        if (n.avail && n.ref == r) {
            cands[nc][0] = INTR(CLX(n.mv[0]));
            cands[nc][1] = INTR(CLY(n.mv[1]));
            nc++;
        }
    }
    for (int k = 0; k < nextra; k++) {
        cands[nc][0] = INTR(CLX(extra[k][0]));
        cands[nc][1] = INTR(CLY(extra[k][1]));
        nc++;
    }
    int bx = 0, by = 0, bc = 0x7fffffff;
    for (int k = 0; k < nc; k++) {
        int cost = COST_INT(cands[k][0], cands[k][1]);
        if (cost < bc) {
            bx = cands[k][0];
            by = cands[k][1];
            bc = cost;
        }
    }
    /* large diamond steps, then the small diamond (enc/frame.rs:973-988) */
    static const int STEPS[3] = {16, 8, 4}, STEPS_FAST[2] = {8, 4};
    const int* steps = c->fast ? STEPS_FAST : STEPS;
    int nsteps = c->fast ? 2 : 3;
    for (int si = 0; si < nsteps; si++) {
        int step = steps[si];
        int iters = step == 4 ? 32 : 4;
        for (int it = 0; it < iters; it++) {
            int moved = 0;
            const int D[4][2] = {{-step, 0}, {step, 0}, {0, -step}, {0, step}};
            for (int d = 0; d < 4; d++) {
                int cx = CLX(bx + D[d][0]), cy = CLY(by + D[d][1]);
                int cost = COST_INT(cx, cy);
                if (cost < bc) {
                    bx = cx;
                    by = cy;
                    bc = cost;
                    moved = 1;
                }
            }
            if (!moved) break;
        }
    }
    /* live coding stops at the integer vector when it is already as good as the reference gets (990-992) */
    if (c->fast && bc < (w * h) / 8 + lam) {
        out[0] = bx;
        out[1] = by;
        return bc - lam * mvd_bits(bx, by, mvp[0], mvp[1]);
    }
    /* sub-sample refinement by SATD (994-1017) */
    uint16_t pred[256];
    const halfpel* hp = f->bhp ? f->bhp : &c->refs[r].hp;
#define COST_SUB(mx, my)                                                                                   \
    (cnt->satd_px += (uint32_t)(w * h), halfpel_predict(hp, x0, y0, (mx), (my), w, h, pred),              \
     satd_blk(f, x0, y0, w, h, pred) + lam * mvd_bits((mx), (my), mvp[0], mvp[1]))
    bc = COST_SUB(bx, by);
    static const int SQUARE[8][2] = {{-1, -1}, {0, -1}, {1, -1}, {-1, 0}, {1, 0}, {-1, 1}, {0, 1}, {1, 1}};
    static const int DIAMOND[4][2] = {{0, -1}, {-1, 0}, {1, 0}, {0, 1}};
    for (int stage = 0; stage < 2; stage++) {
        if (c->fast && stage == 1) break;
        int step = stage == 0 ? 2 : 1;
        const int(*pts)[2] = stage == 0 ? SQUARE : DIAMOND;
        int npts = stage == 0 ? 8 : 4;
        int ccx = bx, ccy = by;
        for (int k = 0; k < npts; k++) {
            int cx = CLX(ccx + pts[k][0] * step), cy = CLY(ccy + pts[k][1] * step);
            int cost = COST_SUB(cx, cy);
            if (cost < bc) {
                bx = cx;
                by = cy;
                bc = cost;
            }
        }
    }
    out[0] = bx;
    out[1] = by;
    return bc - lam * mvd_bits(bx, by, mvp[0], mvp[1]);
#undef CLX
#undef CLY
#undef INTR
#undef COST_INT
#undef COST_SUB
}

typedef struct sub_st { int16_t mv[16][2]; int8_t ref[16]; uint32_t done; } sub_st;

/* sub_search, enc/frame.rs:911-938 */
static int sub_search(const fc* f, counters* cnt, int mbx, int mby, int r, int k, const int extra[2], sub_st* st, int* cost_out) {
    int lam = f->c->lambda;
    int ox = (k & 1) * 2, oy = (k >> 1) * 2;
    int have = 0, best_s = 0, best_cost = 0;
    sub_st best_t;
    int ns = f->c->sub8 ? 4 : 1;
    for (int s = 0; s < ns; s++) {
        sub_st t = *st;
        int cost = lam * (s == 0 ? 0 : 2);
        for (int q = 0; q < NSUB[s]; q++) {
            rect4 rr = SUB_[s][q];
            rr.x += ox;
            rr.y += oy;
            int mvp[2], m[2];
            pred_mv(f, mbx, mby, (const int16_t(*)[2])t.mv, t.ref, t.done, rr.x, rr.y, rr.w, 0, r, mvp);
            int ex[1][2] = {{extra[0], extra[1]}};
            int cst = motion_search(f, cnt, r, mbx, mby, rr, mvp, (const int(*)[2])ex, 1, m);
            cost += cst + lam * mvd_bits(m[0], m[1], mvp[0], mvp[1]);
            for (int by = rr.y; by < rr.y + rr.h; by++)
                for (int bx = rr.x; bx < rr.x + rr.w; bx++) {
                    t.mv[by * 4 + bx][0] = (int16_t)m[0];
                    t.mv[by * 4 + bx][1] = (int16_t)m[1];
                    t.ref[by * 4 + bx] = (int8_t)r;
                    t.done |= 1u << (by * 4 + bx);
                }
        }
        if (!have || cost < best_cost) {
            have = 1;
            best_s = s;
            best_cost = cost;
            best_t = t;
        }
    }
    *st = best_t;
    *cost_out = best_cost;
    return best_s;
}

typedef struct inter_res { int part; int16_t mvs[16][2]; uint8_t sub[4]; int cost; int cost16; } inter_res;

/* best_inter_ref, enc/frame.rs:852-905 */
static void best_inter_ref(const fc* f, counters* cnt, int mbx, int mby, int r, inter_res* best) {
    const struct ironav_ctx* c = f->c;
    int lam = c->lambda;
    int rb = lam * ref_bits(f, r);
    int mvp[2];
    mv_pred(f, mbx, mby, r, mvp);
    /* col_mv of the newest reference (self.refp), enc/frame.rs:857,944-947 */
    const colmv* col = &c->refs[0].col[(size_t)mby * c->mb_w + mbx];
    int colv[1][2] = {{col->mv[0], col->mv[1]}};
    int mv[2];
    int cost = motion_search(f, cnt, r, mbx, mby, PARTS_[0][0], mvp, (const int(*)[2])colv, col->valid ? 1 : 0, mv);
    memset(best, 0, sizeof(*best));
    best->part = 0;
    for (int i = 0; i < 16; i++) {
        best->mvs[i][0] = (int16_t)mv[0];
        best->mvs[i][1] = (int16_t)mv[1];
    }
    best->cost = cost + lam * (mvd_bits(mv[0], mv[1], mvp[0], mvp[1]) + 1) + rb;
    best->cost16 = best->cost;
    if (c->fast) return;
    /* P_8x8 (868-876) */
    sub_st st;
    memset(&st, 0, sizeof(st));
    uint8_t sub[4] = {0, 0, 0, 0};
    int cost8 = lam * 9;
    for (int k = 0; k < 4; k++) {
        int ck;
        sub[k] = (uint8_t)sub_search(f, cnt, mbx, mby, r, k, mv, &st, &ck);
        cost8 += ck + rb;
        if (cost8 >= best->cost) break;
    }
#define AT8(b) (st.mv[((b) / 2) * 8 + ((b) % 2) * 2])
    if (cost8 < best->cost) {
        rect4 rs[16];
        int n = rects(3, sub, rs);
        int16_t v8[16][2];
        memset(v8, 0, sizeof(v8));
        for (int q = 0; q < n; q++) {
            v8[q][0] = st.mv[rs[q].y * 4 + rs[q].x][0];
            v8[q][1] = st.mv[rs[q].y * 4 + rs[q].x][1];
        }
        best->part = 3;
        memcpy(best->mvs, v8, sizeof(v8));
        memcpy(best->sub, sub, 4);
        best->cost = cost8;
        for (int part = 1; part < 3; part++) {
            int16_t mvs[16][2];
            memset(mvs, 0, sizeof(mvs));
            int pc = lam * 3;
            for (int k = 0; k < 2; k++) {
                int p[2];
                part_mvp(f, mbx, mby, part, (const int16_t(*)[2])mvs, r, k, p);
                int cands[2][2];
                int i0 = part == 1 ? 2 * k : k, i1 = part == 1 ? 2 * k + 1 : k + 2;
                cands[0][0] = AT8(i0)[0];
                cands[0][1] = AT8(i0)[1];
                cands[1][0] = AT8(i1)[0];
                cands[1][1] = AT8(i1)[1];
                int m[2];
                int cc = motion_search(f, cnt, r, mbx, mby, PARTS_[part][k], p, (const int(*)[2])cands, 2, m);
                mvs[k][0] = (int16_t)m[0];
                mvs[k][1] = (int16_t)m[1];
                pc += cc + lam * mvd_bits(m[0], m[1], p[0], p[1]) + rb;
                if (pc >= best->cost) break;
            }
            if (pc < best->cost) {
                best->part = part;
                memcpy(best->mvs, mvs, sizeof(mvs));
                memset(best->sub, 0, 4);
                best->cost = pc;
            }
        }
    }
#undef AT8
}

/* The learned form's judge (no counterpart in the reference): the 16x16 partitioning of the newest reference
 * from the proposals instead of the search. Every integer vector within +-2 samples of each of the 4 proposals
 * (rounded to the integer grid and clamped as motion_search clamps its candidates) is scored by SAD + lambda *
 * bits, the first of least cost in proposal-major, row-major order wins; then motion_search's small diamond
 * (step 4, at most 32 rounds) and its sub-sample refinement (994-1017). Returns 0 (the caller searches) when the proposed class is not P_Skip or 16x16, or when
 * the winner costs more than the predictor's own start plus the margin; counters as ironav_set_learned states. */
static int learned_inter(const fc* f, counters* cnt, int mbx, int mby, inter_res* best) {
    const struct ironav_ctx* c = f->c;
    const int r = 0, lam = c->lambda, mb = mby * c->mb_w + mbx;
    if (c->learned_cls[mb] >= 2) {
        __atomic_fetch_add(&c->learned_stats[1], 1u, __ATOMIC_RELAXED);
        return 0;
    }
    int mvp[2];
    mv_pred(f, mbx, mby, r, mvp);
    const int x0 = mbx * 16, y0 = mby * 16, w = 16, h = 16;
    const int cxlo = maxi(-(x0 + 24) * 4, -2048), cxhi = mini((c->mb_w * 16 - x0 + 8) * 4, 2047);
    const int cylo = maxi(-(y0 + 24) * 4, -512), cyhi = mini((c->mb_h * 16 - y0 + 8) * 4, 511);
#define CLX(v) clampi((v), cxlo, cxhi)
#define CLY(v) clampi((v), cylo, cyhi)
#define INTR(v) (((v) + 2) & ~3)
#define COST_INT(mx, my) (sad_int(f, r, x0, y0, w, h, (mx), (my)) + lam * mvd_bits((mx), (my), mvp[0], mvp[1]))
    const int16_t* cand = c->learned + (size_t)mb * 8;
    int bx = 0, by = 0, bc = 0x7fffffff;
    for (int i = 0; i < 100; i++) {
        const int k = i / 25, d = i % 25;
        const int px = CLX(INTR(CLX(cand[2 * k])) + 4 * (d % 5 - 2)), py = CLY(INTR(CLY(cand[2 * k + 1])) + 4 * (d / 5 - 2));
        const int cost = COST_INT(px, py);
        if (cost < bc) {
            bx = px;
            by = py;
            bc = cost;
        }
    }
    const int start = COST_INT(INTR(CLX(mvp[0])), INTR(CLY(mvp[1])));
    cnt->sad_px += 101u * 256u;
    if (bc > start + c->learned_margin) {
        __atomic_fetch_add(&c->learned_stats[2], 1u, __ATOMIC_RELAXED);
        return 0;
    }
    /* motion_search's small diamond (973-988, step 4) from the best of the windows */
    for (int it = 0; it < 32; it++) {
        int moved = 0;
        const int D[4][2] = {{-4, 0}, {4, 0}, {0, -4}, {0, 4}};
        for (int dd = 0; dd < 4; dd++) {
            const int qx = CLX(bx + D[dd][0]), qy = CLY(by + D[dd][1]);
            const int cost = COST_INT(qx, qy);
            if (cost < bc) {
                bx = qx;
                by = qy;
                bc = cost;
                moved = 1;
            }
        }
        cnt->sad_px += 4u * 256u;
        if (!moved) break;
    }
    uint16_t pred[256];
    const halfpel* hp = &c->refs[r].hp;
#define COST_SUB(mx, my)                                                                                   \
    (cnt->satd_px += (uint32_t)(w * h), halfpel_predict(hp, x0, y0, (mx), (my), w, h, pred),              \
     satd_blk(f, x0, y0, w, h, pred) + lam * mvd_bits((mx), (my), mvp[0], mvp[1]))
    bc = COST_SUB(bx, by);
    static const int SQUARE[8][2] = {{-1, -1}, {0, -1}, {1, -1}, {-1, 0}, {1, 0}, {-1, 1}, {0, 1}, {1, 1}};
    static const int DIAMOND[4][2] = {{0, -1}, {-1, 0}, {1, 0}, {0, 1}};
    for (int stage = 0; stage < 2; stage++) {
        if (c->fast && stage == 1) break;
        const int step = stage == 0 ? 2 : 1;
        const int(*pts)[2] = stage == 0 ? SQUARE : DIAMOND;
        const int npts = stage == 0 ? 8 : 4;
        const int ccx = bx, ccy = by;
        for (int k = 0; k < npts; k++) {
            const int qx = CLX(ccx + pts[k][0] * step), qy = CLY(ccy + pts[k][1] * step);
            const int cost = COST_SUB(qx, qy);
            if (cost < bc) {
                bx = qx;
                by = qy;
                bc = cost;
            }
        }
    }
#undef CLX
#undef CLY
#undef INTR
#undef COST_INT
#undef COST_SUB
    memset(best, 0, sizeof(*best));
    best->part = 0;
    for (int i = 0; i < 16; i++) {
        best->mvs[i][0] = (int16_t)bx;
        best->mvs[i][1] = (int16_t)by;
    }
    /* the 16x16 cost of best_inter_ref (855-858): the vector's bits, the mb_type bit and ref_bits */
    best->cost = bc + lam + lam * ref_bits(f, r);
    best->cost16 = best->cost;
    __atomic_fetch_add(&c->learned_stats[0], 1u, __ATOMIC_RELAXED);
    return 1;
}

/* best_inter, enc/frame.rs:839-849 (the newest reference judged from the proposals when they are set) */
static void best_inter(const fc* f, counters* cnt, int mbx, int mby, ironav_mbresult* out) {
    inter_res best, cur;
    int have = 0, bestr = 0;
    for (int r = 0; r < f->c->nact; r++) {
        if (!(r == 0 && f->c->learned && learned_inter(f, cnt, mbx, mby, &cur))) best_inter_ref(f, cnt, mbx, mby, r, &cur);
        if (!have || cur.cost < best.cost) {
            best = cur;
            bestr = r;
            have = 1;
        }
    }
    out->part = (uint8_t)best.part;
    for (int k = 0; k < 4; k++) {
        out->refs[k] = (uint8_t)bestr;
        out->sub[k] = best.sub[k];
    }
    memcpy(out->mvs, best.mvs, sizeof(best.mvs));
    out->cost = best.cost;
    out->cost16 = best.cost16;
    out->flags |= IRONAV_RESULT_INTER;
}

/* The P_Skip vector and SAD of code_mb, enc/frame.rs:722-729 */
static void skip_test(const fc* f, counters* cnt, int mbx, int mby, ironav_mbresult* out) {
    int sv[2];
    skip_mv(f, mbx, mby, sv);
    uint16_t pred[256];
    halfpel_predict(&f->c->refs[0].hp, mbx * 16, mby * 16, sv[0], sv[1], 16, 16, pred);
    const uint16_t* src = f->c->src + (size_t)mby * 16 * f->c->pw + mbx * 16;
    int sad = 0;
    for (int i = 0; i < 256; i++) sad += abs((int)src[(size_t)(i / 16) * f->c->pw + i % 16] - (int)pred[i]);
    cnt->sad_px += 256;
    out->skip_mv[0] = (int16_t)sv[0];
    out->skip_mv[1] = (int16_t)sv[1];
    out->skip_sad = sad;
}

/* The MbState a decided macroblock leaves (finish_mb, enc/frame.rs:2281-2321): a P macroblock's
 * vectors painted over its partitions and the reference index of each 8x8 block. */
static void state_from_result(const ironav_mbresult* r, int skip, ironav_mbstate* s) {
    memset(s, 0, sizeof(*s));
    s->inter = 1;
    if (skip) {
        for (int i = 0; i < 16; i++) {
            s->mvs[i][0] = r->skip_mv[0];
            s->mvs[i][1] = r->skip_mv[1];
        }
        for (int k = 0; k < 4; k++) s->refs[k] = 0;
        return;
    }
    rect4 rs[16];
    int n = rects(r->part, r->sub, rs);
    for (int q = 0; q < n; q++)
        for (int by = rs[q].y; by < rs[q].y + rs[q].h; by++)
            for (int bx = rs[q].x; bx < rs[q].x + rs[q].w; bx++) {
                s->mvs[by * 4 + bx][0] = r->mvs[q][0];
                s->mvs[by * 4 + bx][1] = r->mvs[q][1];
            }
    /* spread(part, refs) then the 8x8 block's first 4x4 block (2298-2300) */
    for (int b8 = 0; b8 < 4; b8++) {
        int blk = (b8 / 2) * 8 + (b8 % 2) * 2, bx = blk % 4, by = blk / 4, k = 0;
        if (r->part == 1) k = by >= 2;
        else if (r->part == 2) k = bx >= 2;
        else if (r->part == 3) k = (by / 2) * 2 + bx / 2;
        s->refs[b8] = (int8_t)r->refs[k];
    }
}

static void analyse_mb(const fc* f, int mbx, int mby, int auto_policy, ironav_mbresult* out, ironav_mbstate* state_out) {
    counters cnt = {0, 0};
    memset(out, 0, sizeof(*out));
    skip_test(f, &cnt, mbx, mby, out);
    int skip = auto_policy && out->skip_sad < f->c->skip_thresh;
    if (skip) out->flags |= IRONAV_RESULT_SKIP;
    else best_inter(f, &cnt, mbx, mby, out);
    out->sad_px = cnt.sad_px;
    out->satd_px = cnt.satd_px;
    if (state_out) state_from_result(out, skip, state_out);
}

/* ---------------------------------------------------------------------------------------------------
 * The C ABI on the CPU
 * ------------------------------------------------------------------------------------------------- */

static void refpic_free(refpic* r) {
    halfpel_free(&r->hp);
    free(r->col);
    r->col = NULL;
    free(r->chroma[0]);
    free(r->chroma[1]);
    r->chroma[0] = r->chroma[1] = NULL;
}

int ironav_ctx_create(ironav_ctx** out, int width, int height, int bd, int max_refs, int nslices, const int* band_rows) {
    if (!out) return IRONAV_INVALID_ARGUMENT;
    *out = NULL;
    /* 8-bit (Yuv420p) or 10-bit (Yuv420p10) pictures, enc/mod.rs:140-143 */
    if (width <= 0 || height <= 0 || (width & 1) || (height & 1) || (bd != 8 && bd != 10)) return IRONAV_INVALID_ARGUMENT;
    int mb_w = (width + 15) / 16, mb_h = (height + 15) / 16;
    if (mb_w > 1024 || mb_h > 1024 || max_refs < 1 || max_refs > 16 || nslices < 1 || nslices > mb_h) return IRONAV_INVALID_ARGUMENT;
    if (band_rows) {
        if (band_rows[0] != 0 || band_rows[nslices] != mb_h) return IRONAV_INVALID_ARGUMENT;
        for (int i = 0; i < nslices; i++)
            if (band_rows[i + 1] <= band_rows[i]) return IRONAV_INVALID_ARGUMENT;
    }
    struct ironav_ctx* c = (struct ironav_ctx*)calloc(1, sizeof(*c));
    c->width = width;
    c->height = height;
    c->bd = bd;
    c->mb_w = mb_w;
    c->mb_h = mb_h;
    c->pw = mb_w * 16;
    c->ph = mb_h * 16;
    c->max_refs = max_refs;
    c->nslices = nslices;
    c->band_start = (int*)calloc((size_t)mb_h, sizeof(int));
    for (int i = 0; i < nslices; i++) {
        int a = band_rows ? band_rows[i] : i * mb_h / nslices, b = band_rows ? band_rows[i + 1] : (i + 1) * mb_h / nslices;
        for (int r = a; r < b; r++) c->band_start[r] = a;
    }
    c->src = (uint16_t*)calloc((size_t)c->pw * c->ph, sizeof(uint16_t));
    c->refs = (refpic*)calloc((size_t)max_refs, sizeof(refpic));
    c->threads = 1;
    *out = c;
    return IRONAV_OK;
}

int ironav_ctx_destroy(ironav_ctx* c) {
    if (!c) return IRONAV_INVALID_ARGUMENT;
    for (int i = 0; i < c->nrefs; i++) refpic_free(&c->refs[i]);
    free(c->refs);
    free(c->src);
    free(c->band_start);
    free(c->b_col);
    free(c->src_c[0]);
    free(c->src_c[1]);
    if (c->inloop) free(((ironav_mbstate**)c->inloop)[0]);
    free(c->inloop);
    free(c);
    return IRONAV_OK;
}

int ironav_ctx_dims(const ironav_ctx* c, int* mb_w, int* mb_h, int* sw, int* sh) {
    if (!c) return IRONAV_INVALID_ARGUMENT;
    if (mb_w) *mb_w = c->mb_w;
    if (mb_h) *mb_h = c->mb_h;
    if (sw) *sw = c->pw + 2 * PAD;
    if (sh) *sh = c->ph + 2 * PAD;
    return IRONAV_OK;
}

int ironav_ctx_set_stream(ironav_ctx* c, void* s) {
    (void)s;
    return c ? IRONAV_OK : IRONAV_INVALID_ARGUMENT;
}

/* Edge-repeated padding to whole macroblocks, H264Encoder::source, enc/mod.rs:502-519. y holds uint8_t
 * samples (8-bit contexts) or uint16_t samples (bd > 8), rows `stride` samples apart. */
static int sample_bytes(const struct ironav_ctx* c) { return c->bd > 8 ? 2 : 1; }

static void pad_plane(const void* y, int bytes, int stride, int w, int h, int pw, int ph, uint16_t* out) {
    for (int r = 0; r < ph; r++) {
        size_t row = (size_t)mini(r, h - 1) * stride;
        uint16_t* o = out + (size_t)r * pw;
        if (bytes == 2)
            for (int x = 0; x < w; x++) o[x] = ((const uint16_t*)y)[row + x];
        else
            for (int x = 0; x < w; x++) o[x] = ((const uint8_t*)y)[row + x];
        for (int x = w; x < pw; x++) o[x] = o[w - 1];
    }
}

int ironav_set_source(ironav_ctx* c, const void* y, int stride) {
    if (!c || !y || stride < c->width) return IRONAV_INVALID_ARGUMENT;
    pad_plane(y, sample_bytes(c), stride, c->width, c->height, c->pw, c->ph, c->src);
    return IRONAV_OK;
}

int ironav_push_reference(ironav_ctx* c, const void* y, int stride, int w, int h, const ironav_mbstate* col) {
    if (!c || !y) return IRONAV_INVALID_ARGUMENT;
    if (!((w == c->width && h == c->height) || (w == c->pw && h == c->ph)) || stride < w) return IRONAV_INVALID_ARGUMENT;
    if (c->nrefs == c->max_refs) {
        refpic_free(&c->refs[c->max_refs - 1]);
        c->nrefs--;
    }
    memmove(&c->refs[1], &c->refs[0], sizeof(refpic) * (size_t)c->nrefs);
    refpic* r = &c->refs[0];
    memset(r, 0, sizeof(*r));
    uint16_t* luma = (uint16_t*)malloc(sizeof(uint16_t) * (size_t)c->pw * c->ph);
    pad_plane(y, sample_bytes(c), stride, w, h, c->pw, c->ph, luma);
    halfpel_build(&r->hp, luma, c->pw, c->ph, c->bd);
    free(luma);
    size_t nmb = (size_t)c->mb_w * c->mb_h;
    r->col = (colmv*)calloc(nmb, sizeof(colmv));
    if (col)
        for (size_t i = 0; i < nmb; i++)
            if (col[i].inter) {
                r->col[i].valid = 1;
                r->col[i].mv[0] = col[i].mvs[5][0];
                r->col[i].mv[1] = col[i].mvs[5][1];
            }
    c->nrefs++;
    return IRONAV_OK;
}

int ironav_clear_references(ironav_ctx* c) {
    if (!c) return IRONAV_INVALID_ARGUMENT;
    for (int i = 0; i < c->nrefs; i++) refpic_free(&c->refs[i]);
    c->nrefs = 0;
    return IRONAV_OK;
}

int ironav_get_planes(ironav_ctx* c, int idx, void* out) {
    if (!c || !out || idx < 0 || idx >= c->nrefs) return IRONAV_INVALID_ARGUMENT;
    size_t n = (size_t)c->refs[idx].hp.stride * c->refs[idx].hp.sh;
    for (int k = 0; k < 4; k++)
        for (size_t i = 0; i < n; i++) {
            if (c->bd > 8) ((uint16_t*)out)[k * n + i] = c->refs[idx].hp.planes[k][i];
            else ((uint8_t*)out)[k * n + i] = (uint8_t)c->refs[idx].hp.planes[k][i];
        }
    return IRONAV_OK;
}

int ironav_begin_p_picture(ironav_ctx* c, int qpp, int lambda, int skip_thresh, int nact, int fast, int sub8) {
    if (!c || lambda < 1 || nact < 1 || nact > c->nrefs || qpp < 0 || qpp > 63) return IRONAV_INVALID_ARGUMENT;
    c->qpp = qpp;
    c->lambda = lambda;
    c->skip_thresh = skip_thresh;
    c->intra_pic = 0;
    c->nact = nact;
    c->fast = fast ? 1 : 0;
    c->sub8 = sub8 ? 1 : 0;
    return IRONAV_OK;
}

/* Threads for the replay mode's all-core run (oracle only; not part of the header). */
int oracle_set_threads(ironav_ctx* c, int n) {
    if (!c || n < 1) return IRONAV_INVALID_ARGUMENT;
    c->threads = n;
    return IRONAV_OK;
}

int ironav_analyse_picture_replay(ironav_ctx* c, const ironav_mbstate* states, ironav_mbresult* out) {
    if (!c || !states || !out || c->nact < 1) return IRONAV_INVALID_ARGUMENT;
    fc f = {c, states, NULL, 0, NULL};
    long n = (long)c->mb_w * c->mb_h;
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 16) num_threads(c->threads)
#endif
    for (long i = 0; i < n; i++) analyse_mb(&f, (int)(i % c->mb_w), (int)(i / c->mb_w), 0, &out[i], NULL);
    return IRONAV_OK;
}

/* Replay over a subset of macroblocks (indices), for bounded CPU-baseline samples. */
int oracle_analyse_replay_subset(ironav_ctx* c, const ironav_mbstate* states, const int* idx, int count, ironav_mbresult* out) {
    if (!c || !states || !out || !idx || c->nact < 1) return IRONAV_INVALID_ARGUMENT;
    fc f = {c, states, NULL, 0, NULL};
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 16) num_threads(c->threads)
#endif
    for (int i = 0; i < count; i++) analyse_mb(&f, idx[i] % c->mb_w, idx[i] / c->mb_w, 0, &out[i], NULL);
    return IRONAV_OK;
}

/* Auto mode: each slice band in raster order (FrameCoder::encode, enc/frame.rs:467-478), bands in
 * parallel when threads > 1 (enc/mod.rs:620-628); the decision is the analysis policy. */
int ironav_analyse_picture_auto(ironav_ctx* c, ironav_mbstate* states, ironav_mbresult* out) {
    if (!c || !states || !out || c->nact < 1) return IRONAV_INVALID_ARGUMENT;
    memset(states, 0, sizeof(ironav_mbstate) * (size_t)c->mb_w * c->mb_h);
    fc f = {c, states, NULL, 0, NULL};
    int nb = 0;
    int starts[1025];
    for (int r = 0; r < c->mb_h; r++)
        if (c->band_start[r] == r) starts[nb++] = r;
    starts[nb] = c->mb_h;
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 1) num_threads(c->threads)
#endif
    for (int b = 0; b < nb; b++)
        for (int mby = starts[b]; mby < starts[b + 1]; mby++)
            for (int mbx = 0; mbx < c->mb_w; mbx++) {
                size_t i = (size_t)mby * c->mb_w + mbx;
                analyse_mb(&f, mbx, mby, 1, &out[i], &states[i]);
            }
    return IRONAV_OK;
}

int ironav_set_source_device(ironav_ctx* c, const void* d, int s) { (void)c; (void)d; (void)s; return IRONAV_HARDWARE_UNAVAILABLE; }
int ironav_push_reference_device(ironav_ctx* c, const void* d, int s, int w, int h, const ironav_mbstate* col) {
    (void)c; (void)d; (void)s; (void)w; (void)h; (void)col;
    return IRONAV_HARDWARE_UNAVAILABLE;
}
int ironav_analyse_picture_replay_device(ironav_ctx* c, const ironav_mbstate* s, ironav_mbresult* o) { (void)c; (void)s; (void)o; return IRONAV_HARDWARE_UNAVAILABLE; }
int ironav_analyse_picture_auto_device(ironav_ctx* c, ironav_mbstate* s, ironav_mbresult* o) { (void)c; (void)s; (void)o; return IRONAV_HARDWARE_UNAVAILABLE; }
int ironav_ctx_sync(ironav_ctx* c) { return c ? IRONAV_OK : IRONAV_INVALID_ARGUMENT; }

/* ---------------------------------------------------------------------------------------------------
 * 16-bit entry points for the interpolation known-answer test (8- and 10-bit)
 * ------------------------------------------------------------------------------------------------- */

typedef struct oracle_halfpel { halfpel hp; } oracle_halfpel;

oracle_halfpel* oracle_halfpel_new(const uint16_t* luma, int pw, int ph, int bd) {
    oracle_halfpel* o = (oracle_halfpel*)calloc(1, sizeof(*o));
    halfpel_build(&o->hp, luma, pw, ph, bd);
    return o;
}
void oracle_halfpel_free(oracle_halfpel* o) {
    if (!o) return;
    halfpel_free(&o->hp);
    free(o);
}
void oracle_halfpel_predict(const oracle_halfpel* o, int x, int y, int mvx, int mvy, int w, int h, uint16_t* out) {
    halfpel_predict(&o->hp, x, y, mvx, mvy, w, h, out);
}
/* Copies plane k (sw x sh samples). */
void oracle_halfpel_plane(const oracle_halfpel* o, int k, uint16_t* out) {
    memcpy(out, o->hp.planes[k], sizeof(uint16_t) * (size_t)o->hp.stride * o->hp.sh);
}
int oracle_satd4(const int* d) { return satd4(d); }

/* Device-memory entry point of the CUDA library; the CPU library has no device memory. */
int ironav_analyse_auto_noalloc(const uint8_t* d_src, int src_stride, const uint8_t* d_ref, int ref_stride, int ref_w, int ref_h,
                                const ironav_mbstate* d_col, int width, int height, int nslices, int qp_prime, int lambda,
                                int skip_thresh, int fast, int sub8, uint8_t* d_planes, ironav_mbstate* d_states,
                                ironav_mbresult* d_results, void* stream) {
    return IRONAV_HARDWARE_UNAVAILABLE;
}

/* In-loop mode on the CPU: a macroblock is analysed when its result is asked for, against the decisions
 * committed so far (the caller's order guarantees its neighbours are among them). */
typedef struct inloop_state { ironav_mbstate* committed; int active; } inloop_state;
static inloop_state* inloop_of(ironav_ctx* c) { return (inloop_state*)c->inloop; }

int ironav_inloop_begin(ironav_ctx* c, int order) {
    if (!c || c->nact < 1 || (order != IRONAV_INLOOP_RASTER && order != IRONAV_INLOOP_BANDS)) return IRONAV_INVALID_ARGUMENT;
    if (!c->inloop) c->inloop = calloc(1, sizeof(inloop_state));
    inloop_state* s = inloop_of(c);
    if (s->active) return IRONAV_INVALID_INPUT;
    free(s->committed);
    s->committed = (ironav_mbstate*)calloc((size_t)c->mb_w * c->mb_h, sizeof(ironav_mbstate));
    s->active = 1;
    return IRONAV_OK;
}

int ironav_inloop_result(ironav_ctx* c, int mb, ironav_mbresult* out, int timeout_ms) {
    (void)timeout_ms;
    if (!c || !out || !c->inloop || !inloop_of(c)->active || mb < 0 || mb >= c->mb_w * c->mb_h) return IRONAV_INVALID_ARGUMENT;
    fc f = {c, inloop_of(c)->committed, NULL, 0, NULL};
    analyse_mb(&f, mb % c->mb_w, mb / c->mb_w, 0, out, NULL);
    return IRONAV_OK;
}

int ironav_inloop_commit(ironav_ctx* c, int mb, const ironav_mbstate* st) {
    if (!c || !st || !c->inloop || !inloop_of(c)->active || mb < 0 || mb >= c->mb_w * c->mb_h) return IRONAV_INVALID_ARGUMENT;
    inloop_of(c)->committed[mb] = *st;
    return IRONAV_OK;
}

int ironav_inloop_end(ironav_ctx* c) {
    if (!c || !c->inloop || !inloop_of(c)->active) return IRONAV_INVALID_ARGUMENT;
    inloop_of(c)->active = 0;
    return IRONAV_OK;
}

int ironav_inloop_set_wait(ironav_ctx* c, int ms) { return (c && ms > 0) ? IRONAV_OK : IRONAV_INVALID_ARGUMENT; }

/* The batched form is a device form (device pointers); the CPU library has none. */
int ironav_batch_create(ironav_batch** out, ironav_ctx* const* ctxs, int n) { (void)out; (void)ctxs; (void)n; return IRONAV_HARDWARE_UNAVAILABLE; }
int ironav_batch_destroy(ironav_batch* b) { (void)b; return IRONAV_INVALID_ARGUMENT; }
int ironav_batch_step(ironav_batch* b, const void* const* s, const void* const* r, const ironav_mbstate* const* c,
                      ironav_mbstate* const* st, ironav_mbresult* const* res) {
    (void)b; (void)s; (void)r; (void)c; (void)st; (void)res;
    return IRONAV_HARDWARE_UNAVAILABLE;
}
int ironav_batch_sync(ironav_batch* b) { (void)b; return IRONAV_INVALID_ARGUMENT; }
int ironav_batch_set_tuning(ironav_batch* b, const ironav_batch_tuning* t) { (void)b; (void)t; return IRONAV_INVALID_ARGUMENT; }
int ironav_batch_get_tuning(const ironav_batch* b, ironav_batch_tuning* t) { (void)b; (void)t; return IRONAV_INVALID_ARGUMENT; }
int ironav_batch_autotune(ironav_batch* b, const void* const* s, const void* const* r, const ironav_mbstate* const* c, ironav_mbstate* const* st,
                          ironav_mbresult* const* res, int reps, ironav_batch_tuning* best, ironav_batch_tuning* all, int cap, int* n_all) {
    (void)b; (void)s; (void)r; (void)c; (void)st; (void)res; (void)reps; (void)best; (void)all; (void)cap; (void)n_all;
    return IRONAV_INVALID_ARGUMENT;
}
int ironav_batch_decide(ironav_batch* b, ironav_mbstate* const* s, ironav_mbcode* const* c, void* const* y, const int* ys, void* const* cb,
                        void* const* cr, const int* cs) {
    (void)b; (void)s; (void)c; (void)y; (void)ys; (void)cb; (void)cr; (void)cs;
    return IRONAV_INVALID_ARGUMENT;
}

/* ---------------------------------------------------------------------------------------------------
 * Scene-cut measure: LowRes::new (codec/change.rs:16-24) on the padded source as H264Encoder::low_res
 * takes it (enc/mod.rs:689-693), and change_threads (codec/change.rs:56-90; single-threaded: the
 * threaded form gives the same totals).
 * ------------------------------------------------------------------------------------------------- */

static void lowres_of(const uint16_t* src, int pw, int lw, int lh, int32_t* out) {
    for (int i = 0; i < lw * lh; i++) {
        int x0 = i % lw * 4, y0 = i / lw * 4, sum = 0;
        for (int k = 0; k < 16; k++) sum += src[(size_t)(y0 + k / 4) * pw + x0 + k % 4];
        out[i] = sum >> 4;
    }
}

static void change_of(const int32_t* prev, const int32_t* cur, int lw, int lh, int64_t* inter_out, int64_t* intra_out) {
    int64_t inter = 0, intra = 0;
    for (int by = 0; by + 7 < lh; by += 8)
        for (int bx = 0; bx + 7 < lw; bx += 8) {
#define AT(x, y) cur[(size_t)(by + (y)) * lw + bx + (x)]
            int sum = 0;
            for (int k = 0; k < 64; k++) sum += AT(k % 8, k / 8);
            int mean = sum / 64;
            for (int k = 0; k < 64; k++) intra += abs(AT(k % 8, k / 8) - mean);
            int64_t best = INT64_MAX;
            for (int dy = -4; dy <= 4; dy++)
                for (int dx = -4; dx <= 4; dx++) {
                    int ox = bx + dx, oy = by + dy;
                    if (ox < 0 || oy < 0 || ox + 8 > lw || oy + 8 > lh) continue;
                    int64_t sad = 0;
                    for (int k = 0; k < 64; k++) sad += abs(AT(k % 8, k / 8) - prev[(size_t)(oy + k / 8) * lw + ox + k % 8]);
                    if (sad < best) best = sad;
                }
            inter += best;
#undef AT
        }
    *inter_out = inter;
    *intra_out = intra;
}

int ironav_scene_change(ironav_ctx* c, const void* prev_y, const void* cur_y, int stride, int64_t* out) {
    if (!c || !prev_y || !cur_y || !out || stride < c->width) return IRONAV_INVALID_ARGUMENT;
    int lw = c->mb_w * 4, lh = c->mb_h * 4;
    uint16_t* a = (uint16_t*)malloc(sizeof(uint16_t) * (size_t)c->pw * c->ph);
    uint16_t* b = (uint16_t*)malloc(sizeof(uint16_t) * (size_t)c->pw * c->ph);
    int32_t* la = (int32_t*)malloc(sizeof(int32_t) * (size_t)lw * lh);
    int32_t* lb = (int32_t*)malloc(sizeof(int32_t) * (size_t)lw * lh);
    pad_plane(prev_y, sample_bytes(c), stride, c->width, c->height, c->pw, c->ph, a);
    pad_plane(cur_y, sample_bytes(c), stride, c->width, c->height, c->pw, c->ph, b);
    lowres_of(a, c->pw, lw, lh, la);
    lowres_of(b, c->pw, lw, lh, lb);
    change_of(la, lb, lw, lh, &out[0], &out[1]);
    free(a);
    free(b);
    free(la);
    free(lb);
    return IRONAV_OK;
}

int ironav_scene_change_device(ironav_ctx* c, const void* d_prev, const void* d_cur, int stride, int64_t* out) {
    (void)c; (void)d_prev; (void)d_cur; (void)stride; (void)out;
    return IRONAV_HARDWARE_UNAVAILABLE;
}

/* ---------------------------------------------------------------------------------------------------
 * Deblocking of the reconstruction (h264/deblock.rs): frame pictures, 4:2:0, macroblocks in raster
 * order (deblock_picture / deblock_rows, deblock.rs:410-429), on 16-bit planes of 16*mb_w x 16*mb_h
 * luma and 8*mb_w x 8*mb_h chroma (rows 16*mb_w and 8*mb_w apart, as Picture::planes).
 * ------------------------------------------------------------------------------------------------- */

/* alpha', beta' (indexA / indexB) and tC0 (indexA, bS 1..3) of the standard's Tables 8-16 and 8-17, as
 * h264/tables.rs holds them (ALPHA, BETA, TC0), and the chroma QP mapping for qPi >= 30 (mb.rs:211). */
static const uint8_t DBK_ALPHA[52] = {0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,   0,   0,   0,   4,   4,
                                      5,  6,  7,  8,  9,  10, 12, 13, 15, 17, 20, 22, 25,  28,  32,  36,  40,  45,
                                      50, 56, 63, 71, 80, 90, 101, 113, 127, 144, 162, 182, 203, 226, 255, 255};
static const uint8_t DBK_BETA[52] = {0, 0, 0, 0, 0, 0, 0, 0, 0,  0,  0,  0,  0,  0,  0,  0,  2,  2,  2,  3,  3,  3,  3,  4,  4,  4,
                                     6, 6, 7, 7, 8, 8, 9, 9, 10, 10, 11, 11, 12, 12, 13, 13, 14, 14, 15, 15, 16, 16, 17, 17, 18, 18};
static const uint8_t DBK_TC0[52][3] = {
    {0, 0, 0},  {0, 0, 0},   {0, 0, 0},   {0, 0, 0},   {0, 0, 0},   {0, 0, 0},    {0, 0, 0},    {0, 0, 0},    {0, 0, 0},
    {0, 0, 0},  {0, 0, 0},   {0, 0, 0},   {0, 0, 0},   {0, 0, 0},   {0, 0, 0},    {0, 0, 0},    {0, 0, 0},    {0, 0, 1},
    {0, 0, 1},  {0, 0, 1},   {0, 0, 1},   {0, 1, 1},   {0, 1, 1},   {1, 1, 1},    {1, 1, 1},    {1, 1, 1},    {1, 1, 1},
    {1, 1, 2},  {1, 1, 2},   {1, 1, 2},   {1, 1, 2},   {1, 2, 3},   {1, 2, 3},    {2, 2, 3},    {2, 2, 4},    {2, 3, 4},
    {2, 3, 4},  {3, 3, 5},   {3, 4, 6},   {3, 4, 6},   {4, 5, 7},   {4, 5, 8},    {4, 6, 9},    {5, 7, 10},   {6, 8, 11},
    {6, 8, 13}, {7, 10, 14}, {8, 11, 16}, {9, 12, 18}, {10, 13, 20}, {11, 15, 23}, {13, 17, 25}};
static const uint8_t DBK_CHROMA_QP[22] = {29, 30, 31, 32, 32, 33, 34, 34, 35, 35, 36, 36, 37, 37, 37, 38, 38, 38, 39, 39, 39, 39};

/* chroma_qp, mb.rs:214-221 */
static int dbk_chroma_qp(int qp, int off, int bd) {
    int qpi = clampi(qp + off, -6 * (bd - 8), 51);
    return qpi < 30 ? qpi : DBK_CHROMA_QP[qpi - 30];
}

static uint16_t dbk_clip1(int v, int bd) { return (uint16_t)clampi(v, 0, (1 << bd) - 1); } /* deblock.rs:13-15 */

/* filter_line, deblock.rs:279-333: the line through q (first sample past the edge), step xs across it */
static void dbk_filter_line(uint16_t* pl, long q, long xs, int b, int tc0, int alpha, int beta, int chroma, int bd) {
    int p0 = pl[q - xs], q0 = pl[q], p1 = pl[q - 2 * xs], q1 = pl[q + xs];
    if (abs(p0 - q0) >= alpha || abs(p1 - p0) >= beta || abs(q1 - q0) >= beta) return;
    if (chroma) {
        if (b < 4) {
            int tc = tc0 + 1;
            int delta = clampi((((q0 - p0) << 2) + (p1 - q1) + 4) >> 3, -tc, tc);
            pl[q - xs] = dbk_clip1(p0 + delta, bd);
            pl[q] = dbk_clip1(q0 - delta, bd);
        } else {
            pl[q - xs] = (uint16_t)((2 * p1 + p0 + q1 + 2) >> 2);
            pl[q] = (uint16_t)((2 * q1 + q0 + p1 + 2) >> 2);
        }
        return;
    }
    int p2 = pl[q - 3 * xs], q2 = pl[q + 2 * xs];
    int ap = abs(p2 - p0), aq = abs(q2 - q0);
    if (b < 4) {
        int tc = tc0 + (ap < beta) + (aq < beta);
        int delta = clampi((((q0 - p0) << 2) + (p1 - q1) + 4) >> 3, -tc, tc);
        pl[q - xs] = dbk_clip1(p0 + delta, bd);
        pl[q] = dbk_clip1(q0 - delta, bd);
        if (ap < beta) pl[q - 2 * xs] = (uint16_t)(p1 + clampi((p2 + ((p0 + q0 + 1) >> 1) - (p1 << 1)) >> 1, -tc0, tc0));
        if (aq < beta) pl[q + xs] = (uint16_t)(q1 + clampi((q2 + ((p0 + q0 + 1) >> 1) - (q1 << 1)) >> 1, -tc0, tc0));
    } else {
        int small = abs(p0 - q0) < (alpha >> 2) + 2;
        if (ap < beta && small) {
            int p3 = pl[q - 4 * xs];
            pl[q - xs] = (uint16_t)((p2 + 2 * p1 + 2 * p0 + 2 * q0 + q1 + 4) >> 3);
            pl[q - 2 * xs] = (uint16_t)((p2 + p1 + p0 + q0 + 2) >> 2);
            pl[q - 3 * xs] = (uint16_t)((2 * p3 + 3 * p2 + p1 + p0 + q0 + 4) >> 3);
        } else {
            pl[q - xs] = (uint16_t)((2 * p1 + p0 + q1 + 2) >> 2);
        }
        if (aq < beta && small) {
            int q3 = pl[q + 3 * xs];
            pl[q] = (uint16_t)((p1 + 2 * p0 + 2 * q0 + 2 * q1 + q2 + 4) >> 3);
            pl[q + xs] = (uint16_t)((p0 + q0 + q1 + q2 + 2) >> 2);
            pl[q + 2 * xs] = (uint16_t)((2 * q3 + 3 * q2 + q1 + q0 + p0 + 4) >> 3);
        } else {
            pl[q] = (uint16_t)((2 * q1 + q0 + p1 + 2) >> 2);
        }
    }
}

/* filter_edge, deblock.rs:232-276: four segments of per_bs lines, one strength each; the samples of a
 * keep (I_PCM / lossless) side are put back after each line */
static void dbk_filter_edge(uint16_t* pl, long pos, long xs, long ys, int per_bs, const uint8_t bs[4], int alpha, int beta, int ia,
                            int chroma, int bd, int keep_p, int keep_q) {
    if (alpha == 0 || beta == 0) return;
    int n = chroma ? 1 : 3;
    for (int s = 0; s < 4; s++) {
        int b = bs[s];
        if (b == 0) continue;
        int tc0 = b < 4 ? DBK_TC0[ia][b - 1] << (bd - 8) : 0;
        for (int k = s * per_bs; k < (s + 1) * per_bs; k++) {
            long q = pos + k * ys;
            uint16_t sp[3], sq[3];
            for (int i = 0; i < n; i++) {
                sp[i] = pl[q - (i + 1) * xs];
                sq[i] = pl[q + i * xs];
            }
            dbk_filter_line(pl, q, xs, b, tc0, alpha, beta, chroma, bd);
            for (int i = 0; i < n; i++) {
                if (keep_p) pl[q - (i + 1) * xs] = sp[i];
                if (keep_q) pl[q + i * xs] = sq[i];
            }
        }
    }
}

/* coded, deblock.rs:336-345 */
static int dbk_coded(const ironav_dbk_mb* m, int bx, int by) {
    if (m->t8x8) {
        int x0 = bx & 2, y0 = by & 2;
        return m->nnz[y0 * 4 + x0] || m->nnz[y0 * 4 + x0 + 1] || m->nnz[(y0 + 1) * 4 + x0] || m->nnz[(y0 + 1) * 4 + x0 + 1];
    }
    return m->nnz[by * 4 + bx] > 0;
}

/* far, deblock.rs:347-350 */
static int dbk_far(const int16_t* a, const int16_t* b, int mvy) { return abs(a[0] - b[0]) >= 4 || abs(a[1] - b[1]) >= mvy; }

/* motion_differs, deblock.rs:352-383 */
static int dbk_motion_differs(const ironav_dbk_mb* p, int pbx, int pby, const ironav_dbk_mb* q, int qbx, int qby, int mvy) {
    int pi = pby * 4 + pbx, qi = qby * 4 + qbx;
    int p8 = (pby >> 1) * 2 + (pbx >> 1), q8 = (qby >> 1) * 2 + (qbx >> 1);
    int32_t pr[2] = {p->ref_id[0][p8], p->ref_id[1][p8]}, qr[2] = {q->ref_id[0][q8], q->ref_id[1][q8]};
    const int16_t *pm[2] = {p->mv[0][pi], p->mv[1][pi]}, *qm[2] = {q->mv[0][qi], q->mv[1][qi]};
    int np = (pr[0] >= 0) + (pr[1] >= 0), nq = (qr[0] >= 0) + (qr[1] >= 0);
    if (np != nq) return 1;
    if (np == 1) {
        int lp = pr[0] >= 0 ? 0 : 1, lq = qr[0] >= 0 ? 0 : 1;
        return pr[lp] != qr[lq] || dbk_far(pm[lp], qm[lq], mvy);
    }
    if (!((pr[0] == qr[0] && pr[1] == qr[1]) || (pr[0] == qr[1] && pr[1] == qr[0]))) return 1;
    if (pr[0] != pr[1]) {
        if (pr[0] == qr[0]) return dbk_far(pm[0], qm[0], mvy) || dbk_far(pm[1], qm[1], mvy);
        return dbk_far(pm[0], qm[1], mvy) || dbk_far(pm[1], qm[0], mvy);
    }
    return (dbk_far(pm[0], qm[0], mvy) || dbk_far(pm[1], qm[1], mvy)) && (dbk_far(pm[0], qm[1], mvy) || dbk_far(pm[1], qm[0], mvy));
}

/* uniform_motion, deblock.rs:385-389 */
static int dbk_uniform(const ironav_dbk_mb* m) {
    for (int l = 0; l < 2; l++) {
        for (int k = 0; k < 4; k++)
            if (m->ref_idx[l][k] != m->ref_idx[l][0] || m->ref_id[l][k] != m->ref_id[l][0]) return 0;
        for (int k = 0; k < 16; k++)
            if (m->mv[l][k][0] != m->mv[l][0][0] || m->mv[l][k][1] != m->mv[l][0][1]) return 0;
    }
    return 1;
}

/* strength, deblock.rs:391-408 */
static void dbk_strength(const ironav_dbk_mb* m, const ironav_dbk_mb* other, int dir, int e, int mvy, uint8_t out[4]) {
    int mb_edge = e == 0;
    if (!m->inter || !other->inter) {
        for (int i = 0; i < 4; i++) out[i] = mb_edge ? 4 : 3;
        return;
    }
    for (int i = 0; i < 4; i++) {
        int qx, qy, px, py;
        if (dir == 0) {
            qx = e; qy = i; px = mb_edge ? 3 : e - 1; py = i;
        } else {
            qx = i; qy = e; px = i; py = mb_edge ? 3 : e - 1;
        }
        if (dbk_coded(m, qx, qy) || dbk_coded(other, px, py)) out[i] = 2;
        else out[i] = dbk_motion_differs(other, px, py, m, qx, qy, mvy) ? 1 : 0;
    }
}

/* deblock_mb, deblock.rs:608-695, for 4:2:0 (chroma 8 rows a macroblock). Returns nonzero for a slice id
 * beyond the table. */
static int dbk_mb(uint16_t* planes[3], const ironav_dbk_mb* mbs, const ironav_dbk_slice* slices, int nslices, int mb_w, int bd,
                  int mbx, int mby) {
    int w = mb_w, ls = w * 16, cs = w * 8, idx = mby * w + mbx;
    const ironav_dbk_mb* m = &mbs[idx];
    if (m->slice == 0) return 0;
    if (m->slice > nslices) return 1;
    const ironav_dbk_slice* sp = &slices[m->slice - 1];
    if (sp->disable_deblocking == 1) return 0;
#define USABLE(o) ((o)->slice != 0 && (sp->disable_deblocking == 0 || (o)->slice == m->slice))
    int left_ok = mbx > 0 && USABLE(&mbs[idx - 1]);
    int top_ok = mby > 0 && USABLE(&mbs[idx - w]);
#undef USABLE
    const ironav_dbk_mb* edge_mb[2] = {mbx > 0 ? &mbs[idx - 1] : m, mby > 0 ? &mbs[idx - w] : m};
    uint8_t bs[2][4][4];
    memset(bs, 0, sizeof(bs));
    int still = m->inter && dbk_uniform(m);
    for (int k = 0; k < 16 && still; k++)
        if (m->nnz[k]) still = 0;
    for (int dir = 0; dir < 2; dir++)
        for (int e = 0; e < 4; e++) {
            if (e > 0 && still) continue;
            dbk_strength(m, e == 0 ? edge_mb[dir] : m, dir, e, 4, bs[dir][e]);
        }
#define ALL0(v) ((v)[0] == 0 && (v)[1] == 0 && (v)[2] == 0 && (v)[3] == 0)
    /* luma */
    for (int dir = 0; dir < 2; dir++)
        for (int e = 0; e < 4; e++) {
            if (e == 0 && !(dir == 0 ? left_ok : top_ok)) continue;
            if ((m->t8x8 && (e & 1)) || ALL0(bs[dir][e])) continue;
            const ironav_dbk_mb* other = e == 0 ? edge_mb[dir] : m;
            int qpav = (other->qp + m->qp + 1) >> 1;
            int ia = clampi(qpav + sp->alpha_offset, 0, 51), ib = clampi(qpav + sp->beta_offset, 0, 51);
            int alpha = DBK_ALPHA[ia] << (bd - 8), beta = DBK_BETA[ib] << (bd - 8);
            long x0 = mbx * 16, y0 = mby * 16;
            if (dir == 0)
                dbk_filter_edge(planes[0], y0 * ls + x0 + e * 4, 1, ls, 4, bs[dir][e], alpha, beta, ia, 0, bd, other->keep, m->keep);
            else
                dbk_filter_edge(planes[0], (y0 + e * 4) * ls + x0, ls, 1, 4, bs[dir][e], alpha, beta, ia, 0, bd, other->keep, m->keep);
        }
    /* chroma: vertical edges at 0 and 4, horizontal edges at rows 0 and 4, each with the strength of the
     * luma edge it lines up with */
    for (int comp = 0; comp < 2; comp++) {
        int off = sp->chroma_qp_offset[comp];
        for (int dir = 0; dir < 2; dir++)
            for (int e = 0; e < 4; e += 2) {
                if ((e == 0 && !(dir == 0 ? left_ok : top_ok)) || ALL0(bs[dir][e])) continue;
                const ironav_dbk_mb* other = e == 0 ? edge_mb[dir] : m;
                int qpav = (dbk_chroma_qp(other->qp, off, bd) + dbk_chroma_qp(m->qp, off, bd) + 1) >> 1;
                int ia = clampi(qpav + sp->alpha_offset, 0, 51), ib = clampi(qpav + sp->beta_offset, 0, 51);
                int alpha = DBK_ALPHA[ia] << (bd - 8), beta = DBK_BETA[ib] << (bd - 8);
                long x0 = mbx * 8, y0 = mby * 8;
                if (dir == 0)
                    dbk_filter_edge(planes[1 + comp], y0 * cs + x0 + e * 2, 1, cs, 2, bs[dir][e], alpha, beta, ia, 1, bd, other->keep, m->keep);
                else
                    dbk_filter_edge(planes[1 + comp], (y0 + e * 2) * cs + x0, cs, 1, 2, bs[dir][e], alpha, beta, ia, 1, bd, other->keep, m->keep);
            }
    }
#undef ALL0
    return 0;
}

static void dbk_copy_in(uint16_t* dst, const void* src, int bytes, int stride, int w, int h) {
    for (int r = 0; r < h; r++)
        for (int x = 0; x < w; x++)
            dst[(size_t)r * w + x] = bytes == 2 ? ((const uint16_t*)src)[(size_t)r * stride + x] : ((const uint8_t*)src)[(size_t)r * stride + x];
}

static void dbk_copy_out(void* dst, const uint16_t* src, int bytes, int stride, int w, int h) {
    for (int r = 0; r < h; r++)
        for (int x = 0; x < w; x++) {
            if (bytes == 2) ((uint16_t*)dst)[(size_t)r * stride + x] = src[(size_t)r * w + x];
            else ((uint8_t*)dst)[(size_t)r * stride + x] = (uint8_t)src[(size_t)r * w + x];
        }
}

int ironav_deblock_picture(ironav_ctx* c, void* y, int y_stride, void* cb, void* cr, int c_stride, const ironav_dbk_mb* mbs,
                           const ironav_dbk_slice* slices, int nslices) {
    if (!c || !y || !cb || !cr || !mbs || !slices || nslices < 1 || nslices > 65535 || y_stride < c->pw || c_stride < c->pw / 2)
        return IRONAV_INVALID_ARGUMENT;
    int pw = c->pw, ph = c->ph, B = sample_bytes(c);
    uint16_t* planes[3];
    planes[0] = (uint16_t*)malloc(sizeof(uint16_t) * (size_t)pw * ph);
    planes[1] = (uint16_t*)malloc(sizeof(uint16_t) * (size_t)pw * ph / 4);
    planes[2] = (uint16_t*)malloc(sizeof(uint16_t) * (size_t)pw * ph / 4);
    dbk_copy_in(planes[0], y, B, y_stride, pw, ph);
    dbk_copy_in(planes[1], cb, B, c_stride, pw / 2, ph / 2);
    dbk_copy_in(planes[2], cr, B, c_stride, pw / 2, ph / 2);
    int bad = 0;
    for (int mby = 0; mby < c->mb_h; mby++)
        for (int mbx = 0; mbx < c->mb_w; mbx++) bad |= dbk_mb(planes, mbs, slices, nslices, c->mb_w, c->bd, mbx, mby);
    dbk_copy_out(y, planes[0], B, y_stride, pw, ph);
    dbk_copy_out(cb, planes[1], B, c_stride, pw / 2, ph / 2);
    dbk_copy_out(cr, planes[2], B, c_stride, pw / 2, ph / 2);
    for (int k = 0; k < 3; k++) free(planes[k]);
    return bad ? IRONAV_INVALID_INPUT : IRONAV_OK;
}

int ironav_deblock_picture_device(ironav_ctx* c, void* d_y, int y_stride, void* d_cb, void* d_cr, int c_stride, const ironav_dbk_mb* d_mbs,
                                  const ironav_dbk_slice* slices, int nslices) {
    (void)c; (void)d_y; (void)y_stride; (void)d_cb; (void)d_cr; (void)c_stride; (void)d_mbs; (void)slices; (void)nslices;
    return IRONAV_HARDWARE_UNAVAILABLE;
}

/* The deblocking tables as the oracle holds them (tests only): alpha[52], beta[52], tc0[52][3] (bS 1..3),
 * chroma_qp[22]. */
int oracle_dbk_tables(uint8_t* alpha, uint8_t* beta, uint8_t* tc0, uint8_t* cqp) {
    memcpy(alpha, DBK_ALPHA, 52);
    memcpy(beta, DBK_BETA, 52);
    memcpy(tc0, DBK_TC0, 52 * 3);
    memcpy(cqp, DBK_CHROMA_QP, 22);
    return 0;
}

/* ---------------------------------------------------------------------------------------------------
 * B pictures: the searches of decide_b (enc/frame.rs:1518-1572), best_b_parts (1626-1687) and spatial
 * direct (direct_mvs, 1715-1747), for replay mode. One reference picture per list, reference index 0.
 * ------------------------------------------------------------------------------------------------- */

/* the co-located vector scaled by picture distances, enc/frame.rs:1553-1554 (i32 division, toward zero) */
static int bscale(int v, int num, int den) { return (int16_t)(v * num / den); }

/* minpos of direct_mvs: the smaller of two reference indices that are both present, else the present one */
static int minpos(int x, int y) { return (x >= 0 && y >= 0) ? mini(x, y) : maxi(x, y); }

/* direct_mvs, enc/frame.rs:1715-1747 */
static void b_direct(const fc fl[2], int mbx, int mby, const ironav_mbstate* col, int16_t d[2][16][2], uint8_t use[2]) {
    int refs[2];
    for (int l = 0; l < 2; l++) {
        nbm a = nb_motion(&fl[l], mbx, mby, ZERO_MVS, NO_REF, 0, -1, 0);
        nbm b = nb_motion(&fl[l], mbx, mby, ZERO_MVS, NO_REF, 0, 0, -1);
        nbm c = nb_motion(&fl[l], mbx, mby, ZERO_MVS, NO_REF, 0, 4, -1);
        if (!c.avail) c = nb_motion(&fl[l], mbx, mby, ZERO_MVS, NO_REF, 0, -1, -1);
        refs[l] = minpos(a.ref, minpos(b.ref, c.ref)); /* an unavailable neighbour has ref -1 */
    }
    memset(d, 0, sizeof(int16_t) * 2 * 16 * 2);
    if (refs[0] < 0 && refs[1] < 0) {
        use[0] = use[1] = 1;
        return;
    }
    for (int l = 0; l < 2; l++) {
        if (refs[l] < 0) continue;
        int mv[2];
        mv_pred(&fl[l], mbx, mby, 0, mv);
        for (int b = 0; b < 16; b++) {
            d[l][b][0] = (int16_t)mv[0];
            d[l][b][1] = (int16_t)mv[1];
        }
    }
    if (col && col->inter) {
        for (int b = 0; b < 16; b++) {
            /* the corner 4x4 block of each 8x8 block stands for it (direct_8x8_inference_flag) */
            int cx = ((b % 4) >> 1) * 3, cy = ((b / 4) >> 1) * 3;
            const int16_t* m = col->mvs[cy * 4 + cx];
            if (col->refs[(cy >> 1) * 2 + (cx >> 1)] == 0 && abs(m[0]) <= 1 && abs(m[1]) <= 1)
                for (int l = 0; l < 2; l++)
                    if (refs[l] == 0) d[l][b][0] = d[l][b][1] = 0;
        }
    }
    use[0] = refs[0] >= 0;
    use[1] = refs[1] >= 0;
}

/* the search of one partition of best_b_parts (its `search` closure, enc/frame.rs:1631-1657): each list,
 * both averaged, and (8x8 blocks) direct prediction; returns the direction, its cost, and the vectors */
static int b_part_search(const fc fl[2], counters* cnt, int mbx, int mby, rect4 pr, const int mvps[2][2], const int (*extra[2])[2],
                         const int nextra[2], int direct, const uint16_t dpred[256], int mv[2][2], int* dir_out) {
    int lam = fl[0].c->lambda;
    int x0 = mbx * 16 + pr.x * 4, y0 = mby * 16 + pr.y * 4, pw = pr.w * 4, ph = pr.h * 4;
    int cost[2];
    uint16_t preds[2][128];
    for (int l = 0; l < 2; l++) {
        cost[l] = motion_search(&fl[l], cnt, 0, mbx, mby, pr, mvps[l], extra[l], nextra[l], mv[l]);
        halfpel_predict(fl[l].bhp, x0, y0, mv[l][0], mv[l][1], pw, ph, preds[l]);
    }
    uint16_t avg[128];
    for (int i = 0; i < pw * ph; i++) avg[i] = (uint16_t)((preds[0][i] + preds[1][i] + 1) >> 1);
    cnt->satd_px += (uint32_t)(pw * ph);
    int bi = satd_blk(&fl[0], x0, y0, pw, ph, avg) + lam * (mvd_bits(mv[0][0], mv[0][1], mvps[0][0], mvps[0][1]) +
                                                           mvd_bits(mv[1][0], mv[1][1], mvps[1][0], mvps[1][1]) + 2);
    int bd, bc;
    if (bi < mini(cost[0], cost[1])) { bd = 3; bc = bi; }
    else if (cost[0] <= cost[1]) { bd = 1; bc = cost[0]; }
    else { bd = 2; bc = cost[1]; }
    if (direct) {
        /* sub_mb_type takes about one bin for direct and three for the others */
        bc += lam * 3;
        uint16_t sub[128];
        for (int i = 0; i < pw * ph; i++) sub[i] = dpred[(pr.y * 4 + i / pw) * 16 + pr.x * 4 + i % pw];
        cnt->satd_px += (uint32_t)(pw * ph);
        int dc = satd_blk(&fl[0], x0, y0, pw, ph, sub) + lam;
        if (dc < bc) { bd = 0; bc = dc; }
    }
    *dir_out = bd;
    return bc;
}

/* best_b_parts, enc/frame.rs:1626-1687: returns 0 when no partitioning costs less than cost16 */
static int b_parts(const fc fl[2], counters* cnt, int mbx, int mby, const int mvs16[2][2], const int mvps[2][2], int cost16,
                   const uint16_t dpred[256], ironav_bresult* out) {
    int lam = fl[0].c->lambda;
    int dirs[4] = {0, 0, 0, 0}, pmv[2][4][2];
    memset(pmv, 0, sizeof(pmv));
    int total = lam * 6;
    for (int k = 0; k < 4; k++) {
        int ex[2][1][2] = {{{mvs16[0][0], mvs16[0][1]}}, {{mvs16[1][0], mvs16[1][1]}}};
        const int (*extra[2])[2] = {ex[0], ex[1]};
        const int nex[2] = {1, 1};
        int mv[2][2], d;
        total += b_part_search(fl, cnt, mbx, mby, PARTS_[3][k], mvps, extra, nex, 1, dpred, mv, &d);
        dirs[k] = d;
        for (int l = 0; l < 2; l++) {
            pmv[l][k][0] = mv[l][0];
            pmv[l][k][1] = mv[l][1];
        }
        if (total >= cost16) return 0;
    }
    int best_part = 3, best_dirs[4], best_mv[2][4][2], best_total = total;
    memcpy(best_dirs, dirs, sizeof(dirs));
    memcpy(best_mv, pmv, sizeof(pmv));
    for (int part = 1; part < 3; part++) {
        int pd[4] = {0, 0, 0, 0}, pm[2][4][2], pt = lam * 7;
        memset(pm, 0, sizeof(pm));
        int ex[2][5][2];
        for (int l = 0; l < 2; l++) {
            for (int k = 0; k < 4; k++) {
                ex[l][k][0] = pmv[l][k][0];
                ex[l][k][1] = pmv[l][k][1];
            }
            ex[l][4][0] = mvs16[l][0];
            ex[l][4][1] = mvs16[l][1];
        }
        const int (*extra[2])[2] = {ex[0], ex[1]};
        const int nex[2] = {5, 5};
        for (int k = 0; k < NPARTS[part]; k++) {
            int mv[2][2], d;
            pt += b_part_search(fl, cnt, mbx, mby, PARTS_[part][k], mvps, extra, nex, 0, dpred, mv, &d);
            pd[k] = d;
            for (int l = 0; l < 2; l++) {
                pm[l][k][0] = mv[l][0];
                pm[l][k][1] = mv[l][1];
            }
            if (pt >= best_total) break;
        }
        if (pt < best_total) {
            best_part = part;
            memcpy(best_dirs, pd, sizeof(pd));
            memcpy(best_mv, pm, sizeof(pm));
            best_total = pt;
        }
    }
    out->part = (uint8_t)best_part;
    for (int k = 0; k < 4; k++) {
        out->bdir[k] = (uint8_t)best_dirs[k];
        for (int l = 0; l < 2; l++) {
            out->pmv[l][k][0] = (int16_t)best_mv[l][k][0];
            out->pmv[l][k][1] = (int16_t)best_mv[l][k][1];
        }
    }
    return 1;
}

/* The searches of decide_b for macroblock (mbx, mby), enc/frame.rs:1518-1572. */
static void analyse_b_mb(const struct ironav_ctx* c, const ironav_mbstate_b* states, int mbx, int mby, ironav_bresult* out) {
    fc fl[2];
    for (int l = 0; l < 2; l++) {
        fl[l].c = c;
        fl[l].states = NULL;
        fl[l].bstates = states;
        fl[l].list = l;
        fl[l].bhp = &c->refs[c->b_ref[l]].hp;
    }
    counters cnt = {0, 0};
    memset(out, 0, sizeof(*out));
    int lam = c->lambda;
    size_t idx = (size_t)mby * c->mb_w + mbx;
    const ironav_mbstate* col = c->b_col ? &c->b_col[idx] : NULL;
    /* spatial direct and its luma prediction (b_pred with the direct vectors, 1749-1781) */
    int16_t direct[2][16][2];
    uint8_t duse[2];
    b_direct(fl, mbx, mby, col, direct, duse);
    memcpy(out->direct_mv, direct, sizeof(direct));
    out->direct_use[0] = duse[0];
    out->direct_use[1] = duse[1];
    int x0 = mbx * 16, y0 = mby * 16;
    uint16_t dpred[256];
    for (int i8 = 0; i8 < 4; i8++) {
        int bx = (i8 & 1) * 8, by = (i8 >> 1) * 8;
        uint16_t lp[2][64];
        memset(lp, 0, sizeof(lp));
        for (int l = 0; l < 2; l++)
            if (duse[l]) {
                const int16_t* v = direct[l][(by / 4) * 4 + bx / 4];
                halfpel_predict(fl[l].bhp, x0 + bx, y0 + by, v[0], v[1], 8, 8, lp[l]);
            }
        for (int k = 0; k < 64; k++) {
            int a = lp[0][k], b = lp[1][k];
            dpred[(by + k / 8) * 16 + bx + k % 8] = (uint16_t)(duse[0] && duse[1] ? (a + b + 1) >> 1 : (duse[0] ? a : b));
        }
    }
    /* 16x16 from either list or both */
    int mvps[2][2], mvs[2][2], costs[2];
    for (int l = 0; l < 2; l++) mv_pred(&fl[l], mbx, mby, 0, mvps[l]);
    int tb = c->b_tb, td = c->b_td;
    uint16_t preds[2][256];
    for (int l = 0; l < 2; l++) {
        int extra[2][2], n = 0;
        if (col && col->inter) {
            extra[n][0] = l == 0 ? bscale(col->mvs[5][0], tb, td) : bscale(col->mvs[5][0], tb - td, td);
            extra[n][1] = l == 0 ? bscale(col->mvs[5][1], tb, td) : bscale(col->mvs[5][1], tb - td, td);
            n++;
        }
        if (l == 1) {
            extra[n][0] = bscale(mvs[0][0], tb - td, tb);
            extra[n][1] = bscale(mvs[0][1], tb - td, tb);
            n++;
        }
        int cst = motion_search(&fl[l], &cnt, 0, mbx, mby, PARTS_[0][0], mvps[l], (const int(*)[2])extra, n, mvs[l]);
        costs[l] = cst + lam * (mvd_bits(mvs[l][0], mvs[l][1], mvps[l][0], mvps[l][1]) + 3);
        halfpel_predict(fl[l].bhp, x0, y0, mvs[l][0], mvs[l][1], 16, 16, preds[l]);
    }
    uint16_t avg[256];
    for (int i = 0; i < 256; i++) avg[i] = (uint16_t)((preds[0][i] + preds[1][i] + 1) >> 1);
    cnt.satd_px += 256;
    int bi = satd_blk(&fl[0], x0, y0, 16, 16, avg) +
             lam * (mvd_bits(mvs[0][0], mvs[0][1], mvps[0][0], mvps[0][1]) + mvd_bits(mvs[1][0], mvs[1][1], mvps[1][0], mvps[1][1]) + 5);
    out->dir16 = (uint8_t)(bi < mini(costs[0], costs[1]) ? 3 : (costs[0] <= costs[1] ? 1 : 2));
    for (int l = 0; l < 2; l++) {
        out->mv16[l][0] = (int16_t)mvs[l][0];
        out->mv16[l][1] = (int16_t)mvs[l][1];
        out->cost16[l] = costs[l];
    }
    out->cost_bi = bi;
    out->has_parts = (uint8_t)b_parts(fl, &cnt, mbx, mby, (const int(*)[2])mvs, (const int(*)[2])mvps, mini(bi, mini(costs[0], costs[1])),
                                      dpred, out);
    out->sad_px = cnt.sad_px;
    out->satd_px = cnt.satd_px;
}

static int b_params_ok(struct ironav_ctx* c, int qpp, int lambda, int l0, int l1, int tb, int td) {
    return c && lambda >= 1 && qpp >= 0 && qpp <= 63 && l0 >= 0 && l0 < c->nrefs && l1 >= 0 && l1 < c->nrefs && tb != 0 && td != 0;
}

int ironav_begin_b_picture(ironav_ctx* c, int qpp, int lambda, int ref_l0, int ref_l1, const ironav_mbstate* col, int tb, int td, int fast) {
    if (!b_params_ok(c, qpp, lambda, ref_l0, ref_l1, tb, td)) return IRONAV_INVALID_ARGUMENT;
    c->qpp = qpp;
    c->lambda = lambda;
    c->fast = fast ? 1 : 0;
    c->b_ref[0] = ref_l0;
    c->b_ref[1] = ref_l1;
    c->b_tb = tb;
    c->b_td = td;
    free(c->b_col);
    c->b_col = NULL;
    if (col) {
        size_t n = (size_t)c->mb_w * c->mb_h;
        c->b_col = (ironav_mbstate*)malloc(sizeof(ironav_mbstate) * n);
        memcpy(c->b_col, col, sizeof(ironav_mbstate) * n);
    }
    c->b_set = 1;
    return IRONAV_OK;
}

int ironav_begin_b_picture_device(ironav_ctx* c, int qpp, int lambda, int ref_l0, int ref_l1, const ironav_mbstate* d_col, int tb, int td,
                                  int fast) {
    (void)c; (void)qpp; (void)lambda; (void)ref_l0; (void)ref_l1; (void)d_col; (void)tb; (void)td; (void)fast;
    return IRONAV_HARDWARE_UNAVAILABLE;
}

int ironav_analyse_b_replay(ironav_ctx* c, const ironav_mbstate_b* states, ironav_bresult* out) {
    if (!c || !states || !out || !c->b_set || c->b_ref[0] >= c->nrefs || c->b_ref[1] >= c->nrefs) return IRONAV_INVALID_ARGUMENT;
    long n = (long)c->mb_w * c->mb_h;
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 16) num_threads(c->threads)
#endif
    for (long i = 0; i < n; i++) analyse_b_mb(c, states, (int)(i % c->mb_w), (int)(i / c->mb_w), &out[i]);
    return IRONAV_OK;
}

int ironav_analyse_b_replay_device(ironav_ctx* c, const ironav_mbstate_b* s, ironav_bresult* o) {
    (void)c; (void)s; (void)o;
    return IRONAV_HARDWARE_UNAVAILABLE;
}

/* ---------------------------------------------------------------------------------------------------
 * Inter residual coding and reconstruction: code_inter, code_inter_residual, code_luma8, code_chroma
 * (enc/frame.rs:1202-1305, 1856-1915) with quant_block (1025-1046), quant8 (56-72), fdct4 / fdct8
 * (46-54, 79-98), decimate_score(8) (2369-2440), chroma_mc (h264/inter.rs:549-568) and idct4_add /
 * idct8_add (h264/idct.rs:8-76).
 * ------------------------------------------------------------------------------------------------- */

/* quantisation multipliers / dequantisation scales by QP % 6 and class (enc/frame.rs:20-21), the 8x8
 * transform's (MF8 enc/frame.rs:33-40; DEQUANT8_COEFF_INIT h264/tables.rs:4278), the scans (ZIGZAG4
 * h264/ps.rs:12, ZIGZAG_DIRECT h264/tables.rs:4291) */
static const int Q_MF[6][3] = {{13107, 5243, 8066}, {11916, 4660, 7490}, {10082, 4194, 6554},
                               {9362, 3647, 5825},  {8192, 3355, 5243}, {7282, 2893, 4559}};
static const int Q_V[6][3] = {{10, 16, 13}, {11, 18, 14}, {13, 20, 16}, {14, 23, 18}, {16, 25, 20}, {18, 29, 23}};
static const int Q_MF8[6][6] = {{13107, 11428, 20972, 12222, 16777, 15481}, {11916, 10826, 19174, 11058, 14980, 14290},
                                {10082, 8943, 15978, 9675, 12710, 11985},   {9362, 8228, 14913, 8931, 11984, 11259},
                                {8192, 7346, 13159, 7740, 10486, 9777},     {7282, 6428, 11570, 6830, 9118, 8640}};
static const int Q_DQ8[6][6] = {{20, 18, 32, 19, 25, 24}, {22, 19, 35, 21, 28, 26}, {26, 23, 42, 24, 33, 31},
                                {28, 25, 45, 26, 35, 33}, {32, 28, 51, 30, 40, 38}, {36, 32, 58, 34, 46, 43}};
static const int ZZ4[16] = {0, 1, 4, 8, 5, 2, 3, 6, 9, 12, 13, 10, 7, 11, 14, 15};
static const int ZZ8[64] = {0,  1,  8,  16, 9,  2,  3,  10, 17, 24, 32, 25, 18, 11, 4,  5,  12, 19, 26, 33, 40, 48,
                            41, 34, 27, 20, 13, 6,  7,  14, 21, 28, 35, 42, 49, 56, 57, 50, 43, 36, 29, 22, 15, 23,
                            30, 37, 44, 51, 58, 59, 52, 45, 38, 31, 39, 46, 53, 60, 61, 54, 47, 55, 62, 63};

static int q_class(int i) { return ((i & 1) == 0 && ((i >> 2) & 1) == 0) ? 0 : (((i & 1) == 1 && ((i >> 2) & 1) == 1) ? 1 : 2); }
static int q_class8(int p) {
    int i = p / 8, j = p % 8;
    if (i % 4 == 0 && j % 4 == 0) return 0;
    if (i % 2 == 1 && j % 2 == 1) return 1;
    if (i % 4 == 2 && j % 4 == 2) return 2;
    if ((i % 4 == 0 && j % 2 == 1) || (i % 2 == 1 && j % 4 == 0)) return 3;
    if ((i % 4 == 0 && j % 4 == 2) || (i % 4 == 2 && j % 4 == 0)) return 4;
    return 5;
}

static void q_fdct4(const int d[16], int o[16]) {
    int t[16];
    for (int r = 0; r < 4; r++) {
        const int* a = d + r * 4;
        int s03 = a[0] + a[3], d03 = a[0] - a[3], s12 = a[1] + a[2], d12 = a[1] - a[2];
        t[r * 4] = s03 + s12;
        t[r * 4 + 1] = 2 * d03 + d12;
        t[r * 4 + 2] = s03 - s12;
        t[r * 4 + 3] = d03 - 2 * d12;
    }
    for (int c = 0; c < 4; c++) {
        int s03 = t[c] + t[12 + c], d03 = t[c] - t[12 + c], s12 = t[4 + c] + t[8 + c], d12 = t[4 + c] - t[8 + c];
        o[c] = s03 + s12;
        o[4 + c] = 2 * d03 + d12;
        o[8 + c] = s03 - s12;
        o[12 + c] = d03 - 2 * d12;
    }
}

static void q_fdct8_1d(const int d[8], int o[8]) {
    int s07 = d[0] + d[7], s16 = d[1] + d[6], s25 = d[2] + d[5], s34 = d[3] + d[4];
    int a0 = s07 + s34, a1 = s16 + s25, a2 = s07 - s34, a3 = s16 - s25;
    int d07 = d[0] - d[7], d16 = d[1] - d[6], d25 = d[2] - d[5], d34 = d[3] - d[4];
    int a4 = d16 + d25 + (d07 + (d07 >> 1));
    int a5 = d07 - d34 - (d25 + (d25 >> 1));
    int a6 = d07 + d34 - (d16 + (d16 >> 1));
    int a7 = d16 - d25 + (d34 + (d34 >> 1));
    o[0] = a0 + a1;
    o[1] = a4 + (a7 >> 2);
    o[2] = a2 + (a3 >> 1);
    o[3] = a5 + (a6 >> 2);
    o[4] = a0 - a1;
    o[5] = a6 - (a5 >> 2);
    o[6] = (a2 >> 1) - a3;
    o[7] = (a4 >> 2) - a7;
}

static void q_fdct8(const int d[64], int o[64]) {
    int t[64], v[8], w[8];
    for (int r = 0; r < 8; r++) q_fdct8_1d(d + r * 8, t + r * 8);
    for (int c = 0; c < 8; c++) {
        for (int r = 0; r < 8; r++) v[r] = t[r * 8 + c];
        q_fdct8_1d(v, w);
        for (int r = 0; r < 8; r++) o[r * 8 + c] = w[r];
    }
}

/* quant, enc/frame.rs:134-141 */
static int q_quant(int c, int mf, int f, int qbits) {
    int a = (int)(((int64_t)(c < 0 ? -(int64_t)c : c) * mf + f) >> qbits);
    return c < 0 ? -a : a;
}

/* quant_block, enc/frame.rs:1025-1046 */
static void q_block(const int src[16], const int pred[16], int qp, int intra, int skip_dc, int lv[16], int co[16], int* dc) {
    int d[16], c[16];
    for (int k = 0; k < 16; k++) d[k] = src[k] - pred[k];
    q_fdct4(d, c);
    int qbits = 15 + qp / 6, f = (1 << qbits) / (intra ? 3 : 6), m = qp % 6;
    memset(lv, 0, sizeof(int) * 16);
    memset(co, 0, sizeof(int) * 16);
    for (int k = 0; k < 16; k++) {
        int p = ZZ4[k];
        if (skip_dc && p == 0) continue;
        int l = q_quant(c[p], Q_MF[m][q_class(p)], f, qbits);
        lv[k] = l;
        co[p] = (l * Q_V[m][q_class(p)]) << (qp / 6);
    }
    *dc = c[0];
}

/* quant8, enc/frame.rs:56-72 */
static void q_block8(const int src[64], const int pred[64], int qp, int intra, int lv[64], int co[64]) {
    int d[64], c[64];
    for (int k = 0; k < 64; k++) d[k] = src[k] - pred[k];
    q_fdct8(d, c);
    int m = qp % 6, qbits = 16 + qp / 6, f = (1 << qbits) / (intra ? 3 : 6);
    memset(lv, 0, sizeof(int) * 64);
    memset(co, 0, sizeof(int) * 64);
    for (int k = 0; k < 64; k++) {
        int p = ZZ8[k];
        int l = q_quant(c[p], Q_MF8[m][q_class8(p)], f, qbits);
        lv[k] = l;
        if (l != 0) {
            int v = l * 16 * Q_DQ8[m][q_class8(p)];
            co[p] = qp >= 36 ? v << (qp / 6 - 6) : (v + (1 << (5 - qp / 6))) >> (6 - qp / 6);
        }
    }
}

/* idct4_add / idct8_add, h264/idct.rs:8-76 (wrapping 32-bit arithmetic) */
static void q_idct4_add(const int c[16], uint16_t* dst, int stride, int maxv) {
    int32_t t[16];
    for (int i = 0; i < 4; i++) {
        const int* d = c + i * 4;
        int32_t e0 = (int32_t)((uint32_t)d[0] + (uint32_t)d[2]), e1 = (int32_t)((uint32_t)d[0] - (uint32_t)d[2]);
        int32_t e2 = (int32_t)((uint32_t)(d[1] >> 1) - (uint32_t)d[3]), e3 = (int32_t)((uint32_t)d[1] + (uint32_t)(d[3] >> 1));
        t[i * 4] = (int32_t)((uint32_t)e0 + (uint32_t)e3);
        t[i * 4 + 1] = (int32_t)((uint32_t)e1 + (uint32_t)e2);
        t[i * 4 + 2] = (int32_t)((uint32_t)e1 - (uint32_t)e2);
        t[i * 4 + 3] = (int32_t)((uint32_t)e0 - (uint32_t)e3);
    }
    for (int j = 0; j < 4; j++) {
        int32_t g0 = (int32_t)((uint32_t)t[j] + (uint32_t)t[8 + j]), g1 = (int32_t)((uint32_t)t[j] - (uint32_t)t[8 + j]);
        int32_t g2 = (int32_t)((uint32_t)(t[4 + j] >> 1) - (uint32_t)t[12 + j]), g3 = (int32_t)((uint32_t)t[4 + j] + (uint32_t)(t[12 + j] >> 1));
        int32_t h[4] = {(int32_t)((uint32_t)g0 + (uint32_t)g3), (int32_t)((uint32_t)g1 + (uint32_t)g2), (int32_t)((uint32_t)g1 - (uint32_t)g2),
                        (int32_t)((uint32_t)g0 - (uint32_t)g3)};
        for (int i = 0; i < 4; i++) {
            uint16_t* p = dst + (size_t)i * stride + j;
            *p = (uint16_t)clampi(*p + ((int32_t)((uint32_t)h[i] + 32u) >> 6), 0, maxv);
        }
    }
}

static void q_row8(const int32_t d[8], int32_t o[8]) {
#define W(x) ((uint32_t)(x))
    int32_t a0 = (int32_t)(W(d[0]) + W(d[4])), a4 = (int32_t)(W(d[0]) - W(d[4]));
    int32_t a2 = (int32_t)(W(d[2] >> 1) - W(d[6])), a6 = (int32_t)(W(d[2]) + W(d[6] >> 1));
    int32_t b0 = (int32_t)(W(a0) + W(a6)), b2 = (int32_t)(W(a4) + W(a2)), b4 = (int32_t)(W(a4) - W(a2)), b6 = (int32_t)(W(a0) - W(a6));
    int32_t a1 = (int32_t)(W(d[5]) - W(d[3]) - W(d[7]) - W(d[7] >> 1));
    int32_t a3 = (int32_t)(W(d[1]) + W(d[7]) - W(d[3]) - W(d[3] >> 1));
    int32_t a5 = (int32_t)(W(d[7]) - W(d[1]) + W(d[5]) + W(d[5] >> 1));
    int32_t a7 = (int32_t)(W(d[3]) + W(d[5]) + W(d[1]) + W(d[1] >> 1));
    int32_t b1 = (int32_t)(W(a1) + W(a7 >> 2)), b7 = (int32_t)(W(a7) - W(a1 >> 2));
    int32_t b3 = (int32_t)(W(a3) + W(a5 >> 2)), b5 = (int32_t)(W(a3 >> 2) - W(a5));
    o[0] = (int32_t)(W(b0) + W(b7));
    o[1] = (int32_t)(W(b2) + W(b5));
    o[2] = (int32_t)(W(b4) + W(b3));
    o[3] = (int32_t)(W(b6) + W(b1));
    o[4] = (int32_t)(W(b6) - W(b1));
    o[5] = (int32_t)(W(b4) - W(b3));
    o[6] = (int32_t)(W(b2) - W(b5));
    o[7] = (int32_t)(W(b0) - W(b7));
#undef W
}

static void q_idct8_add(const int c[64], uint16_t* dst, int stride, int maxv) {
    int32_t t[64], d[8], h[8];
    for (int i = 0; i < 8; i++) q_row8(c + i * 8, t + i * 8);
    for (int j = 0; j < 8; j++) {
        for (int i = 0; i < 8; i++) d[i] = t[i * 8 + j];
        q_row8(d, h);
        for (int i = 0; i < 8; i++) {
            uint16_t* p = dst + (size_t)i * stride + j;
            *p = (uint16_t)clampi(*p + ((int32_t)((uint32_t)h[i] + 32u) >> 6), 0, maxv);
        }
    }
}

/* decimate_score / decimate_score8, enc/frame.rs:2369-2440 */
static int q_decimate(const int* lv, int n) {
    static const int RUN4[16] = {3, 2, 2, 1, 1, 1, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    static const int RUN8[25] = {3, 3, 3, 3, 2, 2, 2, 2, 2, 2, 2, 2, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 0};
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
        score += n == 16 ? RUN4[mini(run, 15)] : RUN8[mini(run, 24)];
    }
    return score;
}

/* Test hooks: the residual's building blocks, called one at a time by the reference's own unit tests of
 * them (enc/frame.rs:2442-2492, restated in tests/test_residual.py). */
int oracle_decimate(const int* lv, int n) { return q_decimate(lv, n); }
void oracle_fdct4(const int* d, int* o) { q_fdct4(d, o); }
int oracle_quant(int c, int mf, int f, int qbits) { return q_quant(c, mf, f, qbits); }
void oracle_idct4_add(const int* c, uint16_t* dst, int stride, int maxv) { q_idct4_add(c, dst, stride, maxv); }
void oracle_quant8(const int* src, const int* pred, int qp, int intra, int* lv, int* co) { q_block8(src, pred, qp, intra, lv, co); }
void oracle_idct8_add(const int* c, uint16_t* dst, int stride, int maxv) { q_idct8_add(c, dst, stride, maxv); }

/* chroma_mc, h264/inter.rs:549-568: eighth-sample bilinear, coordinates clamped to the plane */
static void q_chroma_mc(const uint16_t* refp, int pw, int ph, int x, int y, int mx, int my, int w, int h, uint16_t* out) {
    int fx = mx & 7, fy = my & 7, x0 = x + (mx >> 3), y0 = y + (my >> 3);
    int wa = (8 - fx) * (8 - fy), wb = fx * (8 - fy), wc = (8 - fx) * fy, wd = fx * fy;
#define AT(c, r) ((int)refp[(size_t)clampi(y0 + (r), 0, ph - 1) * pw + clampi(x0 + (c), 0, pw - 1)])
    for (int r = 0; r < h; r++)
        for (int c = 0; c < w; c++) out[r * w + c] = (uint16_t)((wa * AT(c, r) + wb * AT(c + 1, r) + wc * AT(c, r + 1) + wd * AT(c + 1, r + 1) + 32) >> 6);
#undef AT
}

/* inter_pred, enc/frame.rs:1783-1804 */
static void q_inter_pred(const struct ironav_ctx* c, int mbx, int mby, const ironav_interdec* d, uint16_t pred[256], uint16_t cpred[2][64]) {
    rect4 rs[16];
    int n = rects(d->part, d->sub, rs);
    int cw = c->mb_w * 8, ch = c->mb_h * 8;
    uint16_t tmp[256];
    for (int k = 0; k < n; k++) {
        rect4 r = rs[k];
        int ri = d->part == 3 ? (r.y / 2) * 2 + r.x / 2 : k;
        const refpic* rp = &c->refs[d->refs[ri]];
        int mx = d->mvs[k][0], my = d->mvs[k][1];
        halfpel_predict(&rp->hp, mbx * 16 + r.x * 4, mby * 16 + r.y * 4, mx, my, r.w * 4, r.h * 4, tmp);
        for (int row = 0; row < r.h * 4; row++)
            for (int col = 0; col < r.w * 4; col++) pred[(r.y * 4 + row) * 16 + r.x * 4 + col] = tmp[row * r.w * 4 + col];
        for (int cc = 0; cc < 2; cc++) {
            q_chroma_mc(rp->chroma[cc], cw, ch, mbx * 8 + r.x * 2, mby * 8 + r.y * 2, mx, my, r.w * 2, r.h * 2, tmp);
            for (int row = 0; row < r.h * 2; row++)
                for (int col = 0; col < r.w * 2; col++) cpred[cc][(r.y * 2 + row) * 8 + r.x * 2 + col] = tmp[row * r.w * 2 + col];
        }
    }
}

/* code_chroma, enc/frame.rs:1856-1915 (intra: the intra rounding and no AC decimation) */
static void q_code_chroma(const struct ironav_ctx* c, int mbx, int mby, int qp_y, const uint16_t cpred[2][64], ironav_intercode* out,
                          uint16_t* const rec_c[2], int cs, int intra) {
    int x0 = mbx * 8, y0 = mby * 8, scs = c->mb_w * 8;
    int qoff = 6 * (c->bd - 8), maxv = (1 << c->bd) - 1;
    int qp = dbk_chroma_qp(qp_y, 0, c->bd) + qoff, m = qp % 6;
    int lv[2][4][16], cos[2][4][16], cdc[2][4];
    int any_dc = 0, any_ac = 0;
    for (int cc = 0; cc < 2; cc++) {
        int dcs[4];
        for (int blk = 0; blk < 4; blk++) {
            int bx = blk & 1, by = blk >> 1, s[16], pr[16];
            for (int r = 0; r < 4; r++)
                for (int k = 0; k < 4; k++) {
                    s[r * 4 + k] = c->src_c[cc][(size_t)(y0 + by * 4 + r) * scs + x0 + bx * 4 + k];
                    pr[r * 4 + k] = cpred[cc][(by * 4 + r) * 8 + bx * 4 + k];
                }
            q_block(s, pr, qp, intra, 1, lv[cc][blk], cos[cc][blk], &dcs[blk]);
            for (int k = 0; k < 16; k++)
                if (lv[cc][blk][k]) any_ac = 1;
        }
        int f[4] = {dcs[0] + dcs[1] + dcs[2] + dcs[3], dcs[0] - dcs[1] + dcs[2] - dcs[3], dcs[0] + dcs[1] - dcs[2] - dcs[3],
                    dcs[0] - dcs[1] - dcs[2] + dcs[3]};
        int qbits = 16 + qp / 6, fr = (1 << qbits) / (intra ? 3 : 6);
        for (int k = 0; k < 4; k++) {
            cdc[cc][k] = q_quant(f[k], Q_MF[m][0], fr, qbits);
            if (cdc[cc][k]) any_dc = 1;
        }
    }
    /* a lone small AC level is not worth signalling chroma AC for */
    int ac_score = 0;
    for (int cc = 0; cc < 2; cc++)
        for (int blk = 0; blk < 4; blk++) ac_score += q_decimate(lv[cc][blk], 16);
    if (!intra && ac_score < 7) any_ac = 0;
    if (!any_ac) {
        memset(lv, 0, sizeof(lv));
        memset(cos, 0, sizeof(cos));
    }
    int cbpc = any_ac ? 2 : (any_dc ? 1 : 0);
    out->cbp |= (uint8_t)(cbpc << 4);
    int lsd = 16 * Q_V[m][0];
    for (int cc = 0; cc < 2; cc++) {
        const int* l = cdc[cc];
        int f[4] = {l[0] + l[1] + l[2] + l[3], l[0] - l[1] + l[2] - l[3], l[0] + l[1] - l[2] - l[3], l[0] - l[1] - l[2] + l[3]};
        for (int y = 0; y < 8; y++)
            for (int x = 0; x < 8; x++) rec_c[cc][(size_t)(y0 + y) * cs + x0 + x] = cpred[cc][y * 8 + x];
        for (int blk = 0; blk < 4; blk++) {
            int co[16];
            memcpy(co, cos[cc][blk], sizeof(co));
            co[0] = cbpc > 0 ? ((f[blk] * lsd) << (qp / 6)) >> 5 : 0;
            int nz = 0, any = 0;
            for (int k = 0; k < 16; k++) {
                out->cac[cc][blk][k] = (int16_t)lv[cc][blk][k];
                if (lv[cc][blk][k]) nz++;
                if (co[k]) any = 1;
            }
            out->cnnz[cc][blk] = (uint8_t)nz;
            if (any) q_idct4_add(co, rec_c[cc] + (size_t)(y0 + (blk >> 1) * 4) * cs + x0 + (blk & 1) * 4, cs, maxv);
        }
        for (int k = 0; k < 4; k++) out->cdc[cc][k] = (int16_t)cdc[cc][k];
    }
}

/* code_inter_residual / code_luma8, enc/frame.rs:1217-1305, of one macroblock into the reconstruction */
static void q_code_inter(const struct ironav_ctx* c, int mbx, int mby, int qp_y, const ironav_interdec* d, ironav_intercode* out,
                         uint16_t* const rec[3], int ys, int cs) {
    memset(out, 0, sizeof(*out));
    uint16_t pred[256], cpred[2][64];
    q_inter_pred(c, mbx, mby, d, pred, cpred);
    int x0 = mbx * 16, y0 = mby * 16, sls = c->pw, maxv = (1 << c->bd) - 1;
    int qp = qp_y + 6 * (c->bd - 8);
    if (d->mode == 1) {
        /* P_Skip: the prediction is the reconstruction */
        for (int y = 0; y < 16; y++)
            for (int x = 0; x < 16; x++) rec[0][(size_t)(y0 + y) * ys + x0 + x] = pred[y * 16 + x];
        for (int cc = 0; cc < 2; cc++)
            for (int y = 0; y < 8; y++)
                for (int x = 0; x < 8; x++) rec[1 + cc][(size_t)(mby * 8 + y) * cs + mbx * 8 + x] = cpred[cc][y * 8 + x];
        return;
    }
    for (int y = 0; y < 16; y++)
        for (int x = 0; x < 16; x++) rec[0][(size_t)(y0 + y) * ys + x0 + x] = pred[y * 16 + x];
    if (d->t8) {
        int lv[4][64], cos[4][64], score[4];
        for (int i8 = 0; i8 < 4; i8++) {
            int bx = (i8 & 1) * 8, by = (i8 >> 1) * 8, s[64], pr[64];
            for (int k = 0; k < 64; k++) {
                s[k] = c->src[(size_t)(y0 + by + k / 8) * sls + x0 + bx + k % 8];
                pr[k] = pred[(by + k / 8) * 16 + bx + k % 8];
            }
            q_block8(s, pr, qp, 0, lv[i8], cos[i8]);
            score[i8] = q_decimate(lv[i8], 64);
        }
        int total = score[0] + score[1] + score[2] + score[3];
        for (int i8 = 0; i8 < 4; i8++) {
            if (score[i8] < 4 || total < 6) continue; /* levels dropped (out stays zero) */
            int n = 0;
            for (int k = 0; k < 64; k++) {
                out->luma8[i8][k] = (int16_t)lv[i8][k];
                if (lv[i8][k]) n++;
            }
            if (n > 0) {
                q_idct8_add(cos[i8], rec[0] + (size_t)(y0 + (i8 >> 1) * 8) * ys + x0 + (i8 & 1) * 8, ys, maxv);
                out->cbp |= (uint8_t)(1 << i8);
            }
            for (int j = 0; j < 4; j++) out->nnz[((i8 >> 1) * 2 + (j >> 1)) * 4 + (i8 & 1) * 2 + (j & 1)] = (uint8_t)n;
        }
        out->t8x8 = (out->cbp & 15) != 0;
    } else {
        int lv[16][16], cos[16][16], score[4] = {0, 0, 0, 0};
        for (int b = 0; b < 16; b++) {
            int bx = b % 4, by = b / 4, s[16], pr[16], dc;
            for (int r = 0; r < 4; r++)
                for (int k = 0; k < 4; k++) {
                    s[r * 4 + k] = c->src[(size_t)(y0 + by * 4 + r) * sls + x0 + bx * 4 + k];
                    pr[r * 4 + k] = pred[(by * 4 + r) * 16 + bx * 4 + k];
                }
            q_block(s, pr, qp, 0, 0, lv[b], cos[b], &dc);
            score[(by / 2) * 2 + bx / 2] += q_decimate(lv[b], 16);
        }
        /* drop 8x8 blocks (and whole macroblocks) whose few small levels cost more than they give */
        int total = score[0] + score[1] + score[2] + score[3];
        for (int i8 = 0; i8 < 4; i8++)
            if (score[i8] < 4 || total < 6)
                for (int dy = 0; dy < 2; dy++)
                    for (int dx = 0; dx < 2; dx++) {
                        int b = ((i8 >> 1) * 2 + dy) * 4 + (i8 & 1) * 2 + dx;
                        memset(lv[b], 0, sizeof(lv[b]));
                        memset(cos[b], 0, sizeof(cos[b]));
                    }
        for (int b = 0; b < 16; b++) {
            int n = 0;
            for (int k = 0; k < 16; k++) {
                out->luma[b][k] = (int16_t)lv[b][k];
                if (lv[b][k]) n++;
            }
            out->nnz[b] = (uint8_t)n;
            if (n > 0) {
                int bx = b % 4, by = b / 4;
                q_idct4_add(cos[b], rec[0] + (size_t)(y0 + by * 4) * ys + x0 + bx * 4, ys, maxv);
                out->cbp |= (uint8_t)(1 << ((by / 2) * 2 + bx / 2));
            }
        }
    }
    q_code_chroma(c, mbx, mby, qp_y, cpred, out, rec + 1, cs, 0);
}

int ironav_set_source_chroma(ironav_ctx* c, const void* cb, const void* cr, int stride) {
    if (!c || !cb || !cr || stride < c->width / 2) return IRONAV_INVALID_ARGUMENT;
    int cw = c->mb_w * 8, ch = c->mb_h * 8;
    for (int k = 0; k < 2; k++) {
        if (!c->src_c[k]) c->src_c[k] = (uint16_t*)malloc(sizeof(uint16_t) * (size_t)cw * ch);
        pad_plane(k ? cr : cb, sample_bytes(c), stride, c->width / 2, c->height / 2, cw, ch, c->src_c[k]);
    }
    return IRONAV_OK;
}

int ironav_push_reference_chroma(ironav_ctx* c, const void* cb, const void* cr, int stride, int w, int h) {
    if (!c || !cb || !cr || c->nrefs < 1) return IRONAV_INVALID_ARGUMENT;
    int cw = c->mb_w * 8, ch = c->mb_h * 8;
    if (!((w == c->width / 2 && h == c->height / 2) || (w == cw && h == ch)) || stride < w) return IRONAV_INVALID_ARGUMENT;
    refpic* r = &c->refs[0];
    for (int k = 0; k < 2; k++) {
        if (!r->chroma[k]) r->chroma[k] = (uint16_t*)malloc(sizeof(uint16_t) * (size_t)cw * ch);
        pad_plane(k ? cr : cb, sample_bytes(c), stride, w, h, cw, ch, r->chroma[k]);
    }
    return IRONAV_OK;
}

int ironav_code_inter_picture(ironav_ctx* c, int qp, const ironav_interdec* decs, ironav_intercode* codes, void* rec_y, int ys, void* rec_cb,
                              void* rec_cr, int cs) {
    if (!c || !decs || !codes || !rec_y || !rec_cb || !rec_cr || ys < c->pw || cs < c->pw / 2 || qp < -6 * (c->bd - 8) || qp > 51 || !c->src_c[0])
        return IRONAV_INVALID_ARGUMENT;
    long n = (long)c->mb_w * c->mb_h;
    for (long i = 0; i < n; i++) {
        const ironav_interdec* d = &decs[i];
        if (d->mode == 0) continue;
        if (d->mode > 2 || d->part > 3) return IRONAV_INVALID_INPUT;
        for (int k = 0; k < 4; k++)
            if (d->refs[k] >= c->nrefs || !c->refs[d->refs[k]].chroma[0] || d->sub[k] > 3) return IRONAV_INVALID_INPUT;
    }
    int B = sample_bytes(c), cw = c->mb_w * 8, ch = c->mb_h * 8;
    uint16_t* rec[3];
    rec[0] = (uint16_t*)malloc(sizeof(uint16_t) * (size_t)c->pw * c->ph);
    rec[1] = (uint16_t*)malloc(sizeof(uint16_t) * (size_t)cw * ch);
    rec[2] = (uint16_t*)malloc(sizeof(uint16_t) * (size_t)cw * ch);
    dbk_copy_in(rec[0], rec_y, B, ys, c->pw, c->ph);
    dbk_copy_in(rec[1], rec_cb, B, cs, cw, ch);
    dbk_copy_in(rec[2], rec_cr, B, cs, cw, ch);
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 16) num_threads(c->threads)
#endif
    for (long i = 0; i < n; i++) {
        if (decs[i].mode == 0) {
            memset(&codes[i], 0, sizeof(codes[i]));
            continue;
        }
        q_code_inter(c, (int)(i % c->mb_w), (int)(i / c->mb_w), qp, &decs[i], &codes[i], rec, c->pw, cw);
    }
    dbk_copy_out(rec_y, rec[0], B, ys, c->pw, c->ph);
    dbk_copy_out(rec_cb, rec[1], B, cs, cw, ch);
    dbk_copy_out(rec_cr, rec[2], B, cs, cw, ch);
    for (int k = 0; k < 3; k++) free(rec[k]);
    return IRONAV_OK;
}

int ironav_code_inter_picture_device(ironav_ctx* c, int qp, const ironav_interdec* d, ironav_intercode* o, void* y, int ys, void* cb, void* cr,
                                     int cs) {
    (void)c; (void)qp; (void)d; (void)o; (void)y; (void)ys; (void)cb; (void)cr; (void)cs;
    return IRONAV_HARDWARE_UNAVAILABLE;
}


/* ---------------------------------------------------------------------------------------------------
 * The P macroblock decision (decide mode): code_mb without CABAC, enc/frame.rs:715-790
 * ------------------------------------------------------------------------------------------------- */

enum { KIND_I4 = 1, KIND_I8 = 2, KIND_I16 = 3, KIND_INTER = 5 }; /* Kind, h264/mb.rs:21-30 */

/* MbState::i4, enc/frame.rs:2309: Intra4x4 and Intra8x8 macroblocks give their prediction modes */
static int kind_nxn(int kind) { return kind == KIND_I4 || kind == KIND_I8; }

/* Edges, h264/intra.rs:17-26 (a 4x4 block: 8 samples above, 4 to the left) */
typedef struct i_edges { int top[8], left[4], topleft, have_top, have_left, have_topleft; } i_edges;

/* predict_nxn for n = 4, h264/intra.rs:30-128 (ITU-T H.264 8.3.1.2) */
static void i_pred4(int mode, const i_edges* e, int bd, int out[16]) {
#define T(i) ((i) < 0 ? e->topleft : e->top[(i)])
#define L(j) ((j) < 0 ? e->topleft : e->left[(j)])
    for (int y = 0; y < 4; y++)
        for (int x = 0; x < 4; x++) {
            int v;
            switch (mode) {
            case 0: v = T(x); break;
            case 1: v = L(y); break;
            case 2: {
                int st = T(0) + T(1) + T(2) + T(3), sl = L(0) + L(1) + L(2) + L(3);
                if (e->have_top && e->have_left) v = (st + sl + 4) >> 3;
                else if (e->have_left) v = (sl + 2) >> 2;
                else if (e->have_top) v = (st + 2) >> 2;
                else v = 1 << (bd - 1);
                break;
            }
            case 3: v = (x == 3 && y == 3) ? (T(6) + 3 * T(7) + 2) >> 2 : (T(x + y) + 2 * T(x + y + 1) + T(x + y + 2) + 2) >> 2; break;
            case 4:
                if (x > y) v = (T(x - y - 2) + 2 * T(x - y - 1) + T(x - y) + 2) >> 2;
                else if (x < y) v = (L(y - x - 2) + 2 * L(y - x - 1) + L(y - x) + 2) >> 2;
                else v = (T(0) + 2 * e->topleft + L(0) + 2) >> 2;
                break;
            case 5: {
                int z = 2 * x - y, i = x - (y >> 1);
                if (z >= 0 && (z & 1) == 0) v = (T(i - 1) + T(i) + 1) >> 1;
                else if (z >= 0) v = (T(i - 2) + 2 * T(i - 1) + T(i) + 2) >> 2;
                else if (z == -1) v = (L(0) + 2 * e->topleft + T(0) + 2) >> 2;
                else v = (L(y - 2 * x - 1) + 2 * L(y - 2 * x - 2) + L(y - 2 * x - 3) + 2) >> 2;
                break;
            }
            case 6: {
                int z = 2 * y - x, j = y - (x >> 1);
                if (z >= 0 && (z & 1) == 0) v = (L(j - 1) + L(j) + 1) >> 1;
                else if (z >= 0) v = (L(j - 2) + 2 * L(j - 1) + L(j) + 2) >> 2;
                else if (z == -1) v = (L(0) + 2 * e->topleft + T(0) + 2) >> 2;
                else v = (T(x - 2 * y - 1) + 2 * T(x - 2 * y - 2) + T(x - 2 * y - 3) + 2) >> 2;
                break;
            }
            case 7: {
                int i = x + (y >> 1);
                v = (y & 1) == 0 ? (T(i) + T(i + 1) + 1) >> 1 : (T(i) + 2 * T(i + 1) + T(i + 2) + 2) >> 2;
                break;
            }
            default: {
                int z = x + 2 * y, j = y + (x >> 1);
                if (z > 5) v = L(3);
                else if (z == 5) v = (L(2) + 3 * L(3) + 2) >> 2;
                else if ((z & 1) == 0) v = (L(j) + L(j + 1) + 1) >> 1;
                else v = (L(j) + 2 * L(j + 1) + L(j + 2) + 2) >> 2;
                break;
            }
            }
            out[y * 4 + x] = v;
        }
#undef T
#undef L
}

/* predict_16x16, h264/intra.rs:161-209 (8.3.3) */
static void i_pred16(int mode, const int top[16], const int left[16], int tl, int ht, int hl, int bd, int out[256]) {
    if (mode == 0 || mode == 1) {
        for (int i = 0; i < 256; i++) out[i] = mode == 0 ? top[i % 16] : left[i / 16];
    } else if (mode == 2) {
        int st = 0, sl = 0, v;
        for (int i = 0; i < 16; i++) st += top[i], sl += left[i];
        if (ht && hl) v = (st + sl + 16) >> 5;
        else if (hl) v = (sl + 8) >> 4;
        else if (ht) v = (st + 8) >> 4;
        else v = 1 << (bd - 1);
        for (int i = 0; i < 256; i++) out[i] = v;
    } else {
        int h = 0, v = 0;
        for (int k = 0; k < 8; k++) {
            h += (k + 1) * (top[8 + k] - (6 - k < 0 ? tl : top[6 - k]));
            v += (k + 1) * (left[8 + k] - (6 - k < 0 ? tl : left[6 - k]));
        }
        int a = 16 * (left[15] + top[15]), b = (5 * h + 32) >> 6, c = (5 * v + 32) >> 6, maxv = (1 << bd) - 1;
        for (int y = 0; y < 16; y++)
            for (int x = 0; x < 16; x++) out[y * 16 + x] = clampi((a + b * (x - 7) + c * (y - 7) + 16) >> 5, 0, maxv);
    }
}

/* predict_chroma for an 8x8 component, h264/intra.rs:212-287 (8.3.4); mode 0 DC, 1 horizontal, 2 vertical, 3 plane */
static void i_pred_chroma(int mode, const int top[8], const int left[8], int tl, int ht, int hl, int bd, int out[64]) {
    if (mode == 0) {
        for (int by = 0; by < 2; by++)
            for (int bx = 0; bx < 2; bx++) {
                int st = top[bx * 4] + top[bx * 4 + 1] + top[bx * 4 + 2] + top[bx * 4 + 3];
                int sl = left[by * 4] + left[by * 4 + 1] + left[by * 4 + 2] + left[by * 4 + 3];
                int v, mid = 1 << (bd - 1);
                if (bx == by) v = (ht && hl) ? (st + sl + 4) >> 3 : (hl ? (sl + 2) >> 2 : (ht ? (st + 2) >> 2 : mid));
                else if (bx > 0) v = ht ? (st + 2) >> 2 : (hl ? (sl + 2) >> 2 : mid); /* top row, right: the row above first */
                else v = hl ? (sl + 2) >> 2 : (ht ? (st + 2) >> 2 : mid);             /* left column, below: the column first */
                for (int y = 0; y < 4; y++)
                    for (int x = 0; x < 4; x++) out[(by * 4 + y) * 8 + bx * 4 + x] = v;
            }
    } else if (mode == 1 || mode == 2) {
        for (int i = 0; i < 64; i++) out[i] = mode == 1 ? left[i / 8] : top[i % 8];
    } else {
        int hh = 0, vv = 0;
        for (int k = 0; k < 4; k++) {
            hh += (k + 1) * (top[4 + k] - (2 - k < 0 ? tl : top[2 - k]));
            vv += (k + 1) * (left[4 + k] - (2 - k < 0 ? tl : left[2 - k]));
        }
        int a = 16 * (left[7] + top[7]), b = (34 * hh + 32) >> 6, c = (34 * vv + 32) >> 6, maxv = (1 << bd) - 1;
        for (int y = 0; y < 8; y++)
            for (int x = 0; x < 8; x++) out[y * 8 + x] = clampi((a + b * (x - 3) + c * (y - 3) + 16) >> 5, 0, maxv);
    }
}

/* hadamard4, h264/idct.rs:76-95 */
static void i_hadamard4(const int c[16], int o[16]) {
    int t[16];
    for (int i = 0; i < 4; i++) {
        const int* d = c + i * 4;
        int s0 = d[0] + d[1], s1 = d[0] - d[1], s2 = d[2] + d[3], s3 = d[2] - d[3];
        t[i * 4] = s0 + s2;
        t[i * 4 + 1] = s0 - s2;
        t[i * 4 + 2] = s1 - s3;
        t[i * 4 + 3] = s1 + s3;
    }
    for (int j = 0; j < 4; j++) {
        int s0 = t[j] + t[4 + j], s1 = t[j] - t[4 + j], s2 = t[8 + j] + t[12 + j], s3 = t[8 + j] - t[12 + j];
        o[j] = s0 + s2;
        o[4 + j] = s0 - s2;
        o[8 + j] = s1 - s3;
        o[12 + j] = s1 + s3;
    }
}

/* The decision's working set: the picture being reconstructed (unfiltered), the codes so far, QP. */
typedef struct dctx {
    const fc* f;
    uint16_t* rec[3]; /* luma pw x ph, chroma cw x ch */
    ironav_mbcode* codes;
    int qp_y, qp;     /* QP_Y and QP'Y */
    int fast_t, fast_tc;
} dctx;

static void code_new(ironav_mbcode* code, int kind) { /* MbCode::new, enc/frame.rs:302-306 */
    memset(code, 0, sizeof(*code));
    memset(code->modes, 2, sizeof(code->modes));
    code->kind = (uint8_t)kind;
}

static int d_up(const struct ironav_ctx* c, int mby) { return mby > c->band_start[mby]; } /* up, enc/frame.rs:495-497 */

/* SATD of the 4x4 source block at (x, y) of plane 0 (luma) or 1/2 (chroma) against pred (4x4) */
static int d_satd4(const dctx* D, int plane, int x, int y, const int pred[16]) {
    const struct ironav_ctx* c = D->f->c;
    const uint16_t* s = plane == 0 ? c->src : c->src_c[plane - 1];
    int st = plane == 0 ? c->pw : c->mb_w * 8, d[16];
    for (int r = 0; r < 4; r++)
        for (int k = 0; k < 4; k++) d[r * 4 + k] = (int)s[(size_t)(y + r) * st + x + k] - pred[r * 4 + k];
    return satd4(d);
}

/* i16_neighbours + best_i16, enc/frame.rs:792-835 */
static void i16_nb(const dctx* D, int mbx, int mby, int top[16], int left[16], int* tl) {
    const struct ironav_ctx* c = D->f->c;
    const uint16_t* p = D->rec[0];
    int ls = c->pw, x0 = mbx * 16, y0 = mby * 16, ta = d_up(c, mby);
    for (int i = 0; i < 16; i++) {
        top[i] = ta ? p[(size_t)(y0 - 1) * ls + x0 + i] : 0;
        left[i] = mbx > 0 ? p[(size_t)(y0 + i) * ls + x0 - 1] : 0;
    }
    *tl = (mbx > 0 && ta) ? p[(size_t)(y0 - 1) * ls + x0 - 1] : 0;
}

static void best_i16(const dctx* D, int mbx, int mby, int* mode_out, int* cost_out) {
    const struct ironav_ctx* c = D->f->c;
    int ta = d_up(c, mby), la = mbx > 0, top[16], left[16], tl, pred[256];
    i16_nb(D, mbx, mby, top, left, &tl);
    int bm = 2, bc = INT32_MAX;
    for (int mode = 0; mode < 4; mode++) {
        if ((mode == 0 && !ta) || (mode == 1 && !la) || (mode == 3 && !(ta && la))) continue;
        i_pred16(mode, top, left, tl, ta, la, c->bd, pred);
        int cost = c->lambda * (mode == 2 ? 0 : 1);
        for (int b = 0; b < 16; b++) {
            int pb[16];
            for (int r = 0; r < 4; r++)
                for (int k = 0; k < 4; k++) pb[r * 4 + k] = pred[((b / 4) * 4 + r) * 16 + (b % 4) * 4 + k];
            cost += d_satd4(D, 0, mbx * 16 + (b % 4) * 4, mby * 16 + (b / 4) * 4, pb);
        }
        if (cost < bc) {
            bm = mode;
            bc = cost;
        }
    }
    *mode_out = bm;
    *cost_out = bc;
}

/* pred_i4_mode, enc/frame.rs:619-629 (a neighbour that is not Intra4x4 counts as DC) */
static int pred_i4_mode(const dctx* D, const uint8_t cur[16], int mbx, int mby, int bx, int by) {
    int a = -1, b = -1;
    if (bx > 0) a = cur[by * 4 + bx - 1];
    else {
        long i = nb_index(D->f, mbx - 1, mby, mby);
        if (i >= 0) a = kind_nxn(D->codes[i].kind) ? D->codes[i].modes[by * 4 + 3] : 2;
    }
    if (by > 0) b = cur[(by - 1) * 4 + bx];
    else {
        long i = nb_index(D->f, mbx, mby - 1, mby);
        if (i >= 0) b = kind_nxn(D->codes[i].kind) ? D->codes[i].modes[12 + bx] : 2;
    }
    return (a >= 0 && b >= 0) ? mini(a, b) : 2;
}

static int zorder4(int bx, int by) { return ((by >> 1) << 3) | ((bx >> 1) << 2) | ((by & 1) << 1) | (bx & 1); } /* enc/frame.rs:2363-2365 */

/* code_i4, enc/frame.rs:1050-1138: block by block in decoding order, each predicted from the
 * reconstruction so far, its mode the cheapest by SATD + lambda * (1 predicted, 4 otherwise), coded and
 * reconstructed in place. Returns the summed cost. */
static int code_i4(const dctx* D, int mbx, int mby, ironav_mbcode* code) {
    const struct ironav_ctx* c = D->f->c;
    code_new(code, KIND_I4);
    int ta = d_up(c, mby), la = mbx > 0, tla = la && ta, tra = ta && mbx + 1 < c->mb_w;
    uint16_t* p = D->rec[0];
    int ls = c->pw, maxv = (1 << c->bd) - 1, cost = 0;
    for (int n = 0; n < 16; n++) {
        int bx = ((n >> 2) & 1) * 2 + (n & 1), by = ((n >> 3) & 1) * 2 + ((n >> 1) & 1); /* block_pos, 108-110 */
        int x = mbx * 16 + bx * 4, y = mby * 16 + by * 4;
        i_edges e;
        memset(&e, 0, sizeof(e));
        e.have_left = bx > 0 || la;
        e.have_top = by > 0 || ta;
        e.have_topleft = bx > 0 ? (by > 0 ? 1 : ta) : (by > 0 ? la : tla);
        int have_tr = by == 0 ? (bx < 3 ? ta : tra) : (bx == 3 ? 0 : zorder4(bx + 1, by - 1) < zorder4(bx, by));
        if (e.have_top) {
            for (int i = 0; i < 4; i++) e.top[i] = p[(size_t)(y - 1) * ls + x + i];
            for (int i = 4; i < 8; i++) e.top[i] = have_tr ? p[(size_t)(y - 1) * ls + x + i] : e.top[3];
        }
        if (e.have_left)
            for (int j = 0; j < 4; j++) e.left[j] = p[(size_t)(y + j) * ls + x - 1];
        if (e.have_topleft) e.topleft = p[(size_t)(y - 1) * ls + x - 1];
        int predicted = pred_i4_mode(D, code->modes, mbx, mby, bx, by);
        int bm = 2, bc = INT32_MAX, bp[16];
        for (int mode = 0; mode < 9; mode++) {
            int ok = (mode == 0 || mode == 3 || mode == 7) ? e.have_top
                   : (mode == 1 || mode == 8) ? e.have_left
                   : mode == 2 ? 1 : (e.have_top && e.have_left && e.have_topleft);
            if (!ok) continue;
            int pr[16];
            i_pred4(mode, &e, c->bd, pr);
            int cc = d_satd4(D, 0, x, y, pr) + c->lambda * (mode == predicted ? 1 : 4);
            if (cc < bc) {
                bm = mode;
                bc = cc;
                memcpy(bp, pr, sizeof(bp));
            }
        }
        cost += bc;
        code->modes[by * 4 + bx] = (uint8_t)bm;
        int s[16], lv[16], co[16], dc;
        for (int r = 0; r < 4; r++)
            for (int k = 0; k < 4; k++) s[r * 4 + k] = c->src[(size_t)(y + r) * c->pw + x + k];
        q_block(s, bp, D->qp, 1, 0, lv, co, &dc);
        for (int r = 0; r < 4; r++)
            for (int k = 0; k < 4; k++) p[(size_t)(y + r) * ls + x + k] = (uint16_t)bp[r * 4 + k];
        int nz = 0;
        for (int k = 0; k < 16; k++) {
            code->res.luma[by * 4 + bx][k] = (int16_t)lv[k];
            nz += lv[k] != 0;
        }
        if (nz) q_idct4_add(co, p + (size_t)y * ls + x, ls, maxv);
        code->res.nnz[by * 4 + bx] = (uint8_t)nz;
    }
    for (int i8 = 0; i8 < 4; i8++) {
        int bx = (i8 & 1) * 2, by = (i8 >> 1) * 2;
        if (code->res.nnz[by * 4 + bx] || code->res.nnz[by * 4 + bx + 1] || code->res.nnz[(by + 1) * 4 + bx] || code->res.nnz[(by + 1) * 4 + bx + 1])
            code->res.cbp |= (uint8_t)(1 << i8);
    }
    return cost;
}

/* code_i16, enc/frame.rs:1140-1200: the AC of every 4x4 block, the DC through the Hadamard transform
 * (halved, quantised with doubled precision), reconstructed as a decoder does */
static void code_i16(const dctx* D, int mbx, int mby, int mode, ironav_mbcode* code) {
    const struct ironav_ctx* c = D->f->c;
    code_new(code, KIND_I16);
    code->i16_mode = (uint8_t)mode;
    int top[16], left[16], tl, pred[256];
    i16_nb(D, mbx, mby, top, left, &tl);
    i_pred16(mode, top, left, tl, d_up(c, mby), mbx > 0, c->bd, pred);
    int x0 = mbx * 16, y0 = mby * 16, ls = c->pw, qp = D->qp, maxv = (1 << c->bd) - 1;
    int dcs[16], cos[16][16], lvs[16][16], ac = 0;
    for (int b = 0; b < 16; b++) {
        int bx = b % 4, by = b / 4, s[16], pr[16];
        for (int r = 0; r < 4; r++)
            for (int k = 0; k < 4; k++) {
                s[r * 4 + k] = c->src[(size_t)(y0 + by * 4 + r) * c->pw + x0 + bx * 4 + k];
                pr[r * 4 + k] = pred[(by * 4 + r) * 16 + bx * 4 + k];
            }
        q_block(s, pr, qp, 1, 1, lvs[b], cos[b], &dcs[b]);
        for (int k = 0; k < 16; k++) ac |= lvs[b][k] != 0;
    }
    int h[16], dl[16];
    i_hadamard4(dcs, h);
    int qbits = 16 + qp / 6, f = (1 << qbits) / 3, m = qp % 6;
    for (int k = 0; k < 16; k++) {
        int l = q_quant(h[ZZ4[k]] >> 1, Q_MF[m][0], f, qbits);
        code->dc[k] = (int16_t)l;
        dl[ZZ4[k]] = l;
    }
    if (!ac) {
        memset(lvs, 0, sizeof(lvs));
        memset(cos, 0, sizeof(cos));
    }
    code->res.cbp = ac ? 15 : 0;
    int fdc[16], lsd = 16 * Q_V[m][0];
    i_hadamard4(dl, fdc);
    uint16_t* p = D->rec[0];
    for (int y = 0; y < 16; y++)
        for (int x = 0; x < 16; x++) p[(size_t)(y0 + y) * ls + x0 + x] = (uint16_t)pred[y * 16 + x];
    for (int b = 0; b < 16; b++) {
        int co[16], any = 0, nz = 0;
        memcpy(co, cos[b], sizeof(co));
        co[0] = qp >= 36 ? (fdc[b] * lsd) << (qp / 6 - 6) : (fdc[b] * lsd + (1 << (5 - qp / 6))) >> (6 - qp / 6);
        for (int k = 0; k < 16; k++) {
            any |= co[k] != 0;
            code->res.luma[b][k] = (int16_t)lvs[b][k];
            nz += lvs[b][k] != 0;
        }
        if (any) q_idct4_add(co, p + (size_t)(y0 + (b / 4) * 4) * ls + x0 + (b % 4) * 4, ls, maxv);
        code->res.nnz[b] = (uint8_t)nz;
    }
}

/* code_intra_chroma, enc/frame.rs:1807-1854: the cheapest mode by lambda * (1 DC, 3 otherwise) + both
 * components' SATD, then code_chroma with the intra rounding */
static void code_intra_chroma(const dctx* D, int mbx, int mby, ironav_mbcode* code) {
    const struct ironav_ctx* c = D->f->c;
    int la = mbx > 0, ta = d_up(c, mby), x0 = mbx * 8, y0 = mby * 8, cs = c->mb_w * 8;
    int top[2][8], left[2][8], tl[2];
    for (int cc = 0; cc < 2; cc++) {
        const uint16_t* p = D->rec[1 + cc];
        for (int i = 0; i < 8; i++) {
            top[cc][i] = ta ? p[(size_t)(y0 - 1) * cs + x0 + i] : 0;
            left[cc][i] = la ? p[(size_t)(y0 + i) * cs + x0 - 1] : 0;
        }
        tl[cc] = (la && ta) ? p[(size_t)(y0 - 1) * cs + x0 - 1] : 0;
    }
    int bm = 0, bc = INT32_MAX, bp[2][64];
    for (int mode = 0; mode < 4; mode++) {
        if ((mode == 1 && !la) || (mode == 2 && !ta) || (mode == 3 && !(la && ta))) continue;
        int pr[2][64], cost = c->lambda * (mode == 0 ? 1 : 3);
        for (int cc = 0; cc < 2; cc++) {
            i_pred_chroma(mode, top[cc], left[cc], tl[cc], ta, la, c->bd, pr[cc]);
            for (int b = 0; b < 4; b++) {
                int pb[16];
                for (int r = 0; r < 4; r++)
                    for (int k = 0; k < 4; k++) pb[r * 4 + k] = pr[cc][((b / 2) * 4 + r) * 8 + (b % 2) * 4 + k];
                cost += d_satd4(D, 1 + cc, x0 + (b % 2) * 4, y0 + (b / 2) * 4, pb);
            }
        }
        if (cost < bc) {
            bm = mode;
            bc = cost;
            memcpy(bp, pr, sizeof(bp));
        }
    }
    code->chroma_mode = (uint8_t)bm;
    uint16_t cpred[2][64];
    for (int cc = 0; cc < 2; cc++)
        for (int i = 0; i < 64; i++) cpred[cc][i] = (uint16_t)bp[cc][i];
    q_code_chroma(c, mbx, mby, D->qp_y, cpred, &code->res, D->rec + 1, cs, 1);
}

/* part_mvps, enc/frame.rs:579-594, with sub-partitions */
static void part_mvps(const fc* f, int mbx, int mby, int part, const uint8_t sub[4], const int16_t mvs[16][2], const uint8_t refs[4],
                      int16_t out[16][2]) {
    int16_t cur[16][2];
    int8_t cref[16];
    uint32_t done = 0;
    memset(cur, 0, sizeof(cur));
    memset(cref, 0, sizeof(cref));
    memset(out, 0, sizeof(int16_t) * 32);
    rect4 rs[16];
    int n = rects(part, sub, rs), dir = part == 1 ? 1 : (part == 2 ? 2 : 0);
    for (int k = 0; k < n; k++) {
        rect4 r = rs[k];
        int rf = refs[part == 3 ? (r.y / 2) * 2 + r.x / 2 : (part == 0 ? 0 : k)], p[2];
        pred_mv(f, mbx, mby, cur, cref, done, r.x, r.y, r.w, dir, rf, p);
        out[k][0] = (int16_t)p[0];
        out[k][1] = (int16_t)p[1];
        for (int by = r.y; by < r.y + r.h; by++)
            for (int bx = r.x; bx < r.x + r.w; bx++) {
                cur[by * 4 + bx][0] = mvs[k][0];
                cur[by * 4 + bx][1] = mvs[k][1];
                cref[by * 4 + bx] = (int8_t)rf;
                done |= 1u << (by * 4 + bx);
            }
    }
}

/* code_inter, enc/frame.rs:1202-1215, with the 4x4 transform, or the 8x8 transform when t8 */
static void d_code_inter(const dctx* D, int mbx, int mby, int part, const uint8_t sub[4], const uint8_t refs[4], const int16_t mvs[16][2],
                         int t8, ironav_mbcode* code) {
    const struct ironav_ctx* c = D->f->c;
    code_new(code, KIND_INTER);
    code->part = (uint8_t)part;
    memcpy(code->sub, sub, 4);
    memcpy(code->refs, refs, 4);
    memcpy(code->mvs, mvs, sizeof(code->mvs));
    int16_t mvp[16][2];
    part_mvps(D->f, mbx, mby, part, sub, mvs, refs, mvp);
    for (int n = 0; n < 16; n++)
        for (int k = 0; k < 2; k++) code->mvds[n][k] = (int16_t)(mvs[n][k] - mvp[n][k]);
    ironav_interdec d;
    memset(&d, 0, sizeof(d));
    d.mode = 2;
    d.t8 = (uint8_t)(t8 != 0);
    d.part = (uint8_t)part;
    memcpy(d.sub, sub, 4);
    memcpy(d.refs, refs, 4);
    memcpy(d.mvs, mvs, sizeof(d.mvs));
    q_code_inter(c, mbx, mby, D->qp_y, &d, &code->res, D->rec, c->pw, c->mb_w * 8);
}

/* The MbState of a decided macroblock (finish_mb, enc/frame.rs:2281-2321) */
static void d_state(const ironav_mbcode* code, ironav_mbstate* s) {
    memset(s, 0, sizeof(*s));
    if (code->kind != KIND_INTER) {
        for (int k = 0; k < 4; k++) s->refs[k] = -1;
        return;
    }
    ironav_mbresult r;
    memset(&r, 0, sizeof(r));
    r.part = code->part;
    memcpy(r.sub, code->sub, 4);
    memcpy(r.refs, code->refs, 4);
    memcpy(r.mvs, code->mvs, sizeof(r.mvs));
    state_from_result(&r, 0, s);
}

/* code_mb's P_Skip tests, enc/frame.rs:722-751: the fast one on luma and chroma SADs (live coding), then
 * code_inter with the skip vector when its SAD is under the threshold. Returns 1 when the macroblock is
 * P_Skip (code and reconstruction done), else 0 with the skip vector in sv. */
static int skip_tests(const dctx* D, int mbx, int mby, int sv[2], ironav_mbcode* code) {
    const fc* f = D->f;
    const struct ironav_ctx* c = f->c;
    int x0 = mbx * 16, y0 = mby * 16, cw = c->mb_w * 8;
    static const uint8_t zero4[4] = {0, 0, 0, 0};
    skip_mv(f, mbx, mby, sv);
    uint16_t pred[256];
    halfpel_predict(&c->refs[0].hp, x0, y0, sv[0], sv[1], 16, 16, pred);
    int sad = 0;
    for (int i = 0; i < 256; i++) sad += abs((int)c->src[(size_t)(y0 + i / 16) * c->pw + x0 + i % 16] - (int)pred[i]);
    int16_t smv[16][2];
    for (int i = 0; i < 16; i++) smv[i][0] = (int16_t)sv[0], smv[i][1] = (int16_t)sv[1];
    if (c->fast && sad < D->fast_t) {
        ironav_interdec d;
        memset(&d, 0, sizeof(d));
        memcpy(d.mvs, smv, sizeof(d.mvs));
        uint16_t lp[256], cp[2][64];
        q_inter_pred(c, mbx, mby, &d, lp, cp);
        int csad = 0;
        for (int cc = 0; cc < 2; cc++)
            for (int i = 0; i < 64; i++) csad += abs((int)c->src_c[cc][(size_t)(mby * 8 + i / 8) * cw + mbx * 8 + i % 8] - (int)cp[cc][i]);
        if (csad < D->fast_tc) {
            code_new(code, KIND_INTER);
            code->skip = 1;
            memcpy(code->mvs, smv, sizeof(code->mvs));
            for (int i = 0; i < 256; i++) D->rec[0][(size_t)(y0 + i / 16) * c->pw + x0 + i % 16] = pred[i]; /* put_pred, 1397-1403 */
            for (int cc = 0; cc < 2; cc++)
                for (int i = 0; i < 64; i++) D->rec[1 + cc][(size_t)(mby * 8 + i / 8) * cw + mbx * 8 + i % 8] = cp[cc][i];
            return 1;
        }
    }
    if (sad < c->skip_thresh) {
        d_code_inter(D, mbx, mby, 0, zero4, zero4, smv, 0, code);
        if (code->res.cbp == 0) {
            code->skip = 1;
            return 1;
        }
    }
    return 0;
}

/* code_mb for a P macroblock without CABAC, enc/frame.rs:715-790 */
static void decide_mb(const dctx* D, int mbx, int mby, ironav_mbcode* code, ironav_mbstate* st) {
    const fc* f = D->f;
    const struct ironav_ctx* c = f->c;
    int lam = c->lambda;
    int sv[2];
    if (skip_tests(D, mbx, mby, sv, code)) {
        d_state(code, st);
        return;
    }
    int i16m, i16c;
    best_i16(D, mbx, mby, &i16m, &i16c);
    int best_intra = i16c + lam * 4;
    counters cnt = {0, 0};
    ironav_mbresult r;
    memset(&r, 0, sizeof(r));
    best_inter(f, &cnt, mbx, mby, &r);
    /* Intra4x4 is tried by coding it when intra is competitive (766-779) */
    ironav_mbcode* i4 = NULL;
    ironav_mbcode i4code;
    if (best_intra < r.cost) {
        int cost = code_i4(D, mbx, mby, &i4code) + lam * 6;
        if (cost < best_intra) {
            best_intra = cost;
            i4 = &i4code;
        }
    }
    if (r.cost <= best_intra) {
        d_code_inter(D, mbx, mby, r.part, r.sub, r.refs, (const int16_t(*)[2])r.mvs, 0, code);
        if (code->res.cbp == 0 && r.part == 0 && r.mvs[0][0] == sv[0] && r.mvs[0][1] == sv[1] && r.refs[0] == 0) code->skip = 1;
        d_state(code, st);
        return;
    }
    if (i4) *code = *i4;
    else code_i16(D, mbx, mby, i16m, code);
    code_intra_chroma(D, mbx, mby, code);
    d_state(code, st);
}

/* The fast mode's P_Skip tests `sad < 256 * 0.05 * step` and `csad < 128 * 0.05 * step` (enc/frame.rs:735,
 * 740) as integer bounds, like ironav_skip_threshold */
static void fast_thresholds(int qpp, int* luma, int* chroma) {
    double step = pow(2.0, (double)qpp / 6.0);
    *luma = (int)ceil(256.0 * 0.05 * step);
    *chroma = (int)ceil(128.0 * 0.05 * step);
}

static void decide_band_cabac(const dctx* D, int row0, int row1);

int ironav_decide_p_picture(ironav_ctx* c, ironav_mbstate* states, ironav_mbcode* codes, void* rec_y, int ys, void* rec_cb, void* rec_cr,
                            int cs) {
    if (!c || !states || !codes || !rec_y || !rec_cb || !rec_cr || ys < c->pw || cs < c->pw / 2 || c->nact < 1 || !c->src_c[0])
        return IRONAV_INVALID_ARGUMENT;
    for (int r = 0; r < c->nact; r++)
        if (!c->refs[r].chroma[0]) return IRONAV_INVALID_ARGUMENT;
    long n = (long)c->mb_w * c->mb_h;
    int B = sample_bytes(c), cw = c->mb_w * 8, ch = c->mb_h * 8;
    dctx D;
    memset(&D, 0, sizeof(D));
    fc f = {c, states, NULL, 0, NULL};
    D.f = &f;
    D.rec[0] = (uint16_t*)calloc((size_t)c->pw * c->ph, sizeof(uint16_t));
    D.rec[1] = (uint16_t*)calloc((size_t)cw * ch, sizeof(uint16_t));
    D.rec[2] = (uint16_t*)calloc((size_t)cw * ch, sizeof(uint16_t));
    D.codes = codes;
    D.qp = c->qpp;
    D.qp_y = c->qpp - 6 * (c->bd - 8);
    fast_thresholds(c->qpp, &D.fast_t, &D.fast_tc);
    memset(states, 0, sizeof(ironav_mbstate) * (size_t)n);
    memset(codes, 0, sizeof(ironav_mbcode) * (size_t)n);
    int nb = 0;
    int starts[1025];
    for (int r = 0; r < c->mb_h; r++)
        if (c->band_start[r] == r) starts[nb++] = r;
    starts[nb] = c->mb_h;
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 1) num_threads(c->threads)
#endif
    for (int b = 0; b < nb; b++) {
        if (c->cabac) {
            decide_band_cabac(&D, starts[b], starts[b + 1]);
            continue;
        }
        for (int mby = starts[b]; mby < starts[b + 1]; mby++)
            for (int mbx = 0; mbx < c->mb_w; mbx++) {
                size_t i = (size_t)mby * c->mb_w + mbx;
                decide_mb(&D, mbx, mby, &codes[i], &states[i]);
            }
    }
    dbk_copy_out(rec_y, D.rec[0], B, ys, c->pw, c->ph);
    dbk_copy_out(rec_cb, D.rec[1], B, cs, cw, ch);
    dbk_copy_out(rec_cr, D.rec[2], B, cs, cw, ch);
    for (int k = 0; k < 3; k++) free(D.rec[k]);
    return IRONAV_OK;
}

int ironav_decide_p_picture_device(ironav_ctx* c, ironav_mbstate* s, ironav_mbcode* o, void* y, int ys, void* cb, void* cr, int cs) {
    (void)c; (void)s; (void)o; (void)y; (void)ys; (void)cb; (void)cr; (void)cs;
    return IRONAV_HARDWARE_UNAVAILABLE;
}

/* finish_mb's MbInfo for the deblocking filter, enc/frame.rs:2323-2339 (slice ids: enc/mod.rs:608) */
int ironav_decide_dbk_records(ironav_ctx* c, const ironav_mbcode* codes, const ironav_mbstate* states, ironav_dbk_mb* mbs) {
    if (!c || !codes || !states || !mbs || (c->nact < 1 && !c->intra_pic)) return IRONAV_INVALID_ARGUMENT;
    int band = 0, qp_y = c->qpp - 6 * (c->bd - 8);
    for (int r = 0; r < c->mb_h; r++) {
        if (r > 0 && c->band_start[r] == r) band++;
        for (int x = 0; x < c->mb_w; x++) {
            size_t i = (size_t)r * c->mb_w + x;
            const ironav_mbcode* k = &codes[i];
            ironav_dbk_mb* m = &mbs[i];
            memset(m, 0, sizeof(*m));
            m->slice = (uint16_t)(band + 1);
            m->inter = k->kind == KIND_INTER;
            m->qp = (int8_t)qp_y;
            m->t8x8 = k->res.t8x8;
            memcpy(m->nnz, k->res.nnz, 16);
            for (int l = 0; l < 2; l++)
                for (int b = 0; b < 4; b++) {
                    m->ref_idx[l][b] = -1;
                    m->ref_id[l][b] = -1;
                }
            if (m->inter)
                for (int b = 0; b < 4; b++) {
                    m->ref_idx[0][b] = states[i].refs[b];
                    m->ref_id[0][b] = 1 + states[i].refs[b];
                }
            if (m->inter) memcpy(m->mv[0], states[i].mvs, sizeof(m->mv[0]));
        }
    }
    return IRONAV_OK;
}

int ironav_decide_dbk_records_device(ironav_ctx* c, const ironav_mbcode* d_codes, const ironav_mbstate* d_states, ironav_dbk_mb* d_mbs) {
    (void)c; (void)d_codes; (void)d_states; (void)d_mbs;
    return IRONAV_HARDWARE_UNAVAILABLE;
}

int ironav_batch_deblock(ironav_batch* b, void* const* y, const int* ys, void* const* cb, void* const* cr, const int* cs,
                         const ironav_dbk_mb* const* m, const ironav_dbk_slice* const* sl, const int* ns) {
    (void)b; (void)y; (void)ys; (void)cb; (void)cr; (void)cs; (void)m; (void)sl; (void)ns;
    return IRONAV_INVALID_ARGUMENT;
}

/* ---- intra (IDR) pictures: code_mb without a reference, enc/frame.rs:752-790 ------------------------------------ */

/* The fast mode's flat-macroblock test `i16 < 256 * 0.8 * 2^(QP'/6)` (enc/frame.rs:763) as an integer bound */
static int flat_threshold(int qpp) { return (int)ceil(256.0 * 0.8 * pow(2.0, (double)qpp / 6.0)); }

/* code_mb for a macroblock of an I slice without CABAC: best_i16, the Intra4x4 trial (always, but for flat
 * macroblocks in live coding), the cheaper of the two coded, then code_intra_chroma (enc/frame.rs:752-790). */
static void decide_i_mb(const dctx* D, int mbx, int mby, int flat_t, ironav_mbcode* code, ironav_mbstate* st) {
    const struct ironav_ctx* c = D->f->c;
    int lam = c->lambda, i16m, i16c;
    best_i16(D, mbx, mby, &i16m, &i16c);
    int best_intra = i16c + lam * 4;
    int try_i4 = !(c->fast && i16c < flat_t);
    ironav_mbcode i4code;
    int i4 = 0;
    if (try_i4) {
        int cost = code_i4(D, mbx, mby, &i4code) + lam * 6;
        if (cost < best_intra) {
            best_intra = cost;
            i4 = 1;
        }
    }
    if (i4) *code = i4code;
    else code_i16(D, mbx, mby, i16m, code);
    code_intra_chroma(D, mbx, mby, code);
    d_state(code, st);
}

int ironav_begin_i_picture(ironav_ctx* c, int qpp, int lambda, int fast) {
    if (!c || lambda < 1 || qpp < 0 || qpp > 63) return IRONAV_INVALID_ARGUMENT;
    c->qpp = qpp;
    c->lambda = lambda;
    c->skip_thresh = 0;
    c->nact = 0;
    c->fast = fast ? 1 : 0;
    c->sub8 = 0;
    c->intra_pic = 1;
    return IRONAV_OK;
}

int ironav_decide_i_picture(ironav_ctx* c, ironav_mbstate* states, ironav_mbcode* codes, void* rec_y, int ys, void* rec_cb, void* rec_cr,
                            int cs) {
    if (!c || !states || !codes || !rec_y || !rec_cb || !rec_cr || ys < c->pw || cs < c->pw / 2 || !c->intra_pic || !c->src_c[0])
        return IRONAV_INVALID_ARGUMENT;
    long n = (long)c->mb_w * c->mb_h;
    int B = sample_bytes(c), cw = c->mb_w * 8, ch = c->mb_h * 8;
    dctx D;
    memset(&D, 0, sizeof(D));
    fc f = {c, states, NULL, 0, NULL};
    D.f = &f;
    D.rec[0] = (uint16_t*)calloc((size_t)c->pw * c->ph, sizeof(uint16_t));
    D.rec[1] = (uint16_t*)calloc((size_t)cw * ch, sizeof(uint16_t));
    D.rec[2] = (uint16_t*)calloc((size_t)cw * ch, sizeof(uint16_t));
    D.codes = codes;
    D.qp = c->qpp;
    D.qp_y = c->qpp - 6 * (c->bd - 8);
    int flat_t = flat_threshold(c->qpp);
    memset(states, 0, sizeof(ironav_mbstate) * (size_t)n);
    memset(codes, 0, sizeof(ironav_mbcode) * (size_t)n);
    int nb = 0;
    int starts[1025];
    for (int r = 0; r < c->mb_h; r++)
        if (c->band_start[r] == r) starts[nb++] = r;
    starts[nb] = c->mb_h;
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 1) num_threads(c->threads)
#endif
    for (int b = 0; b < nb; b++) {
        if (c->cabac) {
            decide_band_cabac(&D, starts[b], starts[b + 1]);
            continue;
        }
        for (int mby = starts[b]; mby < starts[b + 1]; mby++)
            for (int mbx = 0; mbx < c->mb_w; mbx++) {
                size_t i = (size_t)mby * c->mb_w + mbx;
                decide_i_mb(&D, mbx, mby, flat_t, &codes[i], &states[i]);
            }
    }
    dbk_copy_out(rec_y, D.rec[0], B, ys, c->pw, c->ph);
    dbk_copy_out(rec_cb, D.rec[1], B, cs, cw, ch);
    dbk_copy_out(rec_cr, D.rec[2], B, cs, cw, ch);
    for (int k = 0; k < 3; k++) free(D.rec[k]);
    return IRONAV_OK;
}

int ironav_decide_i_picture_device(ironav_ctx* c, ironav_mbstate* s, ironav_mbcode* o, void* y, int ys, void* cb, void* cr, int cs) {
    (void)c; (void)s; (void)o; (void)y; (void)ys; (void)cb; (void)cr; (void)cs;
    return IRONAV_HARDWARE_UNAVAILABLE;
}

int ironav_set_source_chroma_device(ironav_ctx* c, const void* cb, const void* cr, int stride) {
    (void)c; (void)cb; (void)cr; (void)stride;
    return IRONAV_HARDWARE_UNAVAILABLE;
}

int ironav_push_reference_chroma_device(ironav_ctx* c, const void* cb, const void* cr, int stride, int w, int h) {
    (void)c; (void)cb; (void)cr; (void)stride; (void)w; (void)h;
    return IRONAV_HARDWARE_UNAVAILABLE;
}

/* ---- the bitstream: CAVLC slices and parameter sets (Annex B) ----------------------------------------------- */

#include "cavlc_tables.h"

/* BitWriter, enc/bitw.rs:4-78: bits MSB first into bytes */
typedef struct bitw {
    uint8_t* buf;
    size_t len, cap;
    uint64_t cur;
    unsigned n;
} bitw;

static void bw_init(bitw* w) {
    memset(w, 0, sizeof(*w));
    w->cap = 4096;
    w->buf = (uint8_t*)malloc(w->cap);
}

static void bw_byte(bitw* w, uint8_t b) {
    if (w->len == w->cap) {
        w->cap *= 2;
        w->buf = (uint8_t*)realloc(w->buf, w->cap);
    }
    w->buf[w->len++] = b;
}

/* put, bitw.rs:16-25: the low n bits of v (n <= 32) */
static void bw_put(bitw* w, unsigned n, uint32_t v) {
    w->cur = (w->cur << n) | (uint64_t)v;
    w->n += n;
    while (w->n >= 8) {
        w->n -= 8;
        bw_byte(w, (uint8_t)(w->cur >> w->n));
    }
    w->cur &= (w->n ? ((1ull << w->n) - 1) : 0);
}

static void bw_flag(bitw* w, int b) { bw_put(w, 1, b ? 1u : 0u); }

/* ue, bitw.rs:31-40 */
static void bw_ue(bitw* w, uint32_t v) {
    uint64_t x = (uint64_t)v + 1;
    unsigned len = 64 - (unsigned)__builtin_clzll(x);
    if (len > 16) {
        bw_put(w, len - 1, 0);
        bw_put(w, len, (uint32_t)x);
    } else {
        bw_put(w, 2 * len - 1, (uint32_t)x);
    }
}

/* se, bitw.rs:42-44 */
static void bw_se(bitw* w, int v) { bw_ue(w, v > 0 ? 2u * (uint32_t)v - 1u : (uint32_t)(-2 * (int64_t)v)); }

/* finish, bitw.rs:69-78: rbsp_trailing_bits */
static void bw_finish(bitw* w) {
    bw_put(w, 1, 1);
    if (w->n > 0) bw_put(w, 8 - w->n, 0);
}

/* put_nal, bitw.rs:91-103: start code, NAL header, emulation prevention */
static void put_nal(bitw* out, int ref_idc, int kind, const uint8_t* rbsp, size_t n) {
    bw_byte(out, 0);
    bw_byte(out, 0);
    bw_byte(out, 0);
    bw_byte(out, 1);
    bw_byte(out, (uint8_t)((ref_idc << 5) | kind));
    int zeros = 0;
    for (size_t i = 0; i < n; i++) {
        uint8_t b = rbsp[i];
        if (zeros >= 2 && b <= 3) {
            bw_byte(out, 3);
            zeros = 0;
        }
        bw_byte(out, b);
        zeros = b == 0 ? zeros + 1 : 0;
    }
}

/* put_level, enc/cavlc.rs:12-45 */
static void put_level(bitw* w, uint32_t code, uint32_t suffix_len) {
    uint32_t rem = 0;
    int esc = 0;
    if (suffix_len == 0) {
        if (code < 14) bw_put(w, code + 1, 1);
        else if (code < 30) {
            bw_put(w, 15, 1);
            bw_put(w, 4, code - 14);
        } else {
            esc = 1;
            rem = code - 30;
        }
    } else if ((code >> suffix_len) < 15) {
        bw_put(w, (code >> suffix_len) + 1, 1);
        bw_put(w, suffix_len, code & ((1u << suffix_len) - 1));
    } else {
        esc = 1;
        rem = code - (15u << suffix_len);
    }
    if (esc) {
        if (rem < 4096) {
            bw_put(w, 16, 1);
            bw_put(w, 12, rem);
        } else {
            unsigned p = 16;
            while ((uint64_t)rem + 4096 >= (1ull << (p - 2))) p++;
            bw_put(w, p, 0);
            bw_put(w, 1, 1);
            bw_put(w, p - 3, rem + 4096 - (1u << (p - 3)));
        }
    }
}

/* write_block, enc/cavlc.rs:47-122: one residual block, levels in scan order (max = 16, 15 or 4), nc the
 * neighbour context (-1: chroma DC). Returns the non-zero count. */
static int write_block(bitw* w, int nc, const int* levels, int max) {
    int nz[16], runs[16], total = 0, last = -1;
    memset(runs, 0, sizeof(runs));
    for (int i = max - 1; i >= 0; i--)
        if (levels[i] != 0) {
            if (last >= 0) runs[total - 1] = last - i - 1;
            nz[total++] = levels[i];
            last = i;
        }
    int ones = 0;
    while (ones < (total < 3 ? total : 3) && abs(nz[ones]) == 1) ones++;
    int token = total * 4 + ones;
    if (nc == -1) bw_put(w, CAVLC_CHROMA_DC_COEFF_TOKEN_LEN[token], CAVLC_CHROMA_DC_COEFF_TOKEN_BITS[token]);
    else {
        int cls = nc <= 1 ? 0 : nc <= 3 ? 1 : nc <= 7 ? 2 : 3;
        bw_put(w, CAVLC_COEFF_TOKEN_LEN[cls][token], CAVLC_COEFF_TOKEN_BITS[cls][token]);
    }
    if (total == 0) return 0;
    for (int i = 0; i < ones; i++) bw_flag(w, nz[i] < 0);
    uint32_t suffix_len = (total > 10 && ones < 3) ? 1 : 0;
    for (int i = ones; i < total; i++) {
        int l = nz[i];
        uint32_t code = l > 0 ? 2u * (uint32_t)l - 2u : (uint32_t)(-2 * l) - 1u;
        if (i == ones && ones < 3) code -= 2;
        put_level(w, code, suffix_len);
        if (suffix_len == 0) suffix_len = 1;
        if ((uint32_t)abs(l) > (3u << (suffix_len - 1)) && suffix_len < 6) suffix_len++;
    }
    int highest = max - 1;
    while (levels[highest] == 0) highest--;
    int zeros_left = highest + 1 - total;
    if (total < max) {
        if (nc == -1) bw_put(w, CAVLC_CHROMA_DC_TOTAL_ZEROS_LEN[total - 1][zeros_left], CAVLC_CHROMA_DC_TOTAL_ZEROS_BITS[total - 1][zeros_left]);
        else bw_put(w, CAVLC_TOTAL_ZEROS_LEN[total - 1][zeros_left], CAVLC_TOTAL_ZEROS_BITS[total - 1][zeros_left]);
    }
    for (int i = 0; i < total - 1; i++) {
        if (zeros_left == 0) break;
        int zl = zeros_left < 7 ? zeros_left : 7;
        bw_put(w, CAVLC_RUN_LEN[zl - 1][runs[i]], CAVLC_RUN_BITS[zl - 1][runs[i]]);
        zeros_left -= runs[i];
    }
    return total;
}

/* One slice's writer: its bits, the skip run, and what the neighbour lookups need */
typedef struct swr {
    const struct ironav_ctx* c;
    const ironav_mbcode* codes;
    int p_slice, nref, first_row;
    uint32_t skip_run;
    bitw w;
} swr;

/* The neighbour's code when it is in this slice (nb_state, enc/frame.rs:509-515) */
static const ironav_mbcode* w_nb(const swr* s, int mbx, int mby) {
    if (mbx < 0 || mby < s->first_row || mbx >= s->c->mb_w || mby >= s->c->mb_h) return NULL;
    return &s->codes[(size_t)mby * s->c->mb_w + mbx];
}

/* nc, enc/frame.rs:2354-2361 */
static int nc_of(int ha, int a, int hb, int b) {
    if (ha && hb) return (a + b + 1) >> 1;
    if (ha) return a;
    if (hb) return b;
    return 0;
}

/* nc_luma, enc/frame.rs:606-610 */
static int w_nc_luma(const swr* s, const uint8_t cur[16], int mbx, int mby, int bx, int by) {
    int ha = 1, a = 0, hb = 1, b = 0;
    if (bx > 0) a = cur[by * 4 + bx - 1];
    else {
        const ironav_mbcode* n = w_nb(s, mbx - 1, mby);
        ha = n != NULL;
        if (n) a = n->res.nnz[by * 4 + 3];
    }
    if (by > 0) b = cur[(by - 1) * 4 + bx];
    else {
        const ironav_mbcode* n = w_nb(s, mbx, mby - 1);
        hb = n != NULL;
        if (n) b = n->res.nnz[12 + bx];
    }
    return nc_of(ha, a, hb, b);
}

/* nc_chroma, enc/frame.rs:612-616 */
static int w_nc_chroma(const swr* s, const uint8_t cur[4], int comp, int mbx, int mby, int bx, int by) {
    int ha = 1, a = 0, hb = 1, b = 0;
    if (bx > 0) a = cur[by * 2];
    else {
        const ironav_mbcode* n = w_nb(s, mbx - 1, mby);
        ha = n != NULL;
        if (n) a = n->res.cnnz[comp][by * 2 + 1];
    }
    if (by > 0) b = cur[bx];
    else {
        const ironav_mbcode* n = w_nb(s, mbx, mby - 1);
        hb = n != NULL;
        if (n) b = n->res.cnnz[comp][2 + bx];
    }
    return nc_of(ha, a, hb, b);
}

/* pred_i4_mode, enc/frame.rs:619-629 (a neighbour that is not Intra4x4 counts as DC) */
static int w_pred_i4(const swr* s, const uint8_t cur[16], int mbx, int mby, int bx, int by) {
    int a = -1, b = -1;
    if (bx > 0) a = cur[by * 4 + bx - 1];
    else {
        const ironav_mbcode* n = w_nb(s, mbx - 1, mby);
        if (n) a = kind_nxn(n->kind) ? n->modes[by * 4 + 3] : 2;
    }
    if (by > 0) b = cur[(by - 1) * 4 + bx];
    else {
        const ironav_mbcode* n = w_nb(s, mbx, mby - 1);
        if (n) b = kind_nxn(n->kind) ? n->modes[12 + bx] : 2;
    }
    return (a >= 0 && b >= 0) ? mini(a, b) : 2;
}

static int cbp_code(const uint8_t* table, int cbp) {
    for (int i = 0; i < 48; i++)
        if (table[i] == cbp) return i;
    return -1;
}

static int n_rects(int part, const uint8_t sub[4]) {
    rect4 r[16];
    return rects(part, sub, r);
}

/* write_mb, enc/frame.rs:1922-2016 */
static void write_mb(swr* s, const ironav_mbcode* code, int mbx, int mby) {
    bitw* w = &s->w;
    if (s->p_slice) {
        if (code->skip) {
            s->skip_run++;
            return;
        }
        bw_ue(w, s->skip_run);
        s->skip_run = 0;
    }
    unsigned base = s->p_slice ? 5 : 0;
    int cbpl = code->res.cbp & 15, cbpc = code->res.cbp >> 4;
    if (code->kind == KIND_I4) {
        bw_ue(w, base);
        uint8_t so_far[16];
        memset(so_far, 2, sizeof(so_far));
        for (int n = 0; n < 16; n++) {
            int bx = ((n >> 2) & 1) * 2 + (n & 1), by = ((n >> 3) & 1) * 2 + ((n >> 1) & 1);
            int mode = code->modes[by * 4 + bx];
            int pred = w_pred_i4(s, so_far, mbx, mby, bx, by);
            so_far[by * 4 + bx] = (uint8_t)mode;
            if (mode == pred) bw_flag(w, 1);
            else {
                bw_flag(w, 0);
                bw_put(w, 3, (uint32_t)(mode < pred ? mode : mode - 1));
            }
        }
        bw_ue(w, code->chroma_mode);
        bw_ue(w, (uint32_t)cbp_code(CAVLC_GOLOMB_TO_INTRA4X4_CBP, code->res.cbp));
    } else if (code->kind == KIND_I16) {
        bw_ue(w, base + 1 + code->i16_mode + 4 * (unsigned)cbpc + (cbpl ? 12 : 0));
        bw_ue(w, code->chroma_mode);
    } else {
        bw_ue(w, code->part);
        if (code->part == 3)
            for (int k = 0; k < 4; k++) bw_ue(w, code->sub[k]);
        if (s->nref > 1)
            for (int k = 0; k < NPARTS[code->part]; k++) {
                if (s->nref == 2) bw_flag(w, code->refs[k] == 0);
                else bw_ue(w, code->refs[k]);
            }
        int nr = n_rects(code->part, code->sub);
        for (int k = 0; k < nr; k++) {
            bw_se(w, code->mvds[k][0]);
            bw_se(w, code->mvds[k][1]);
        }
        bw_ue(w, (uint32_t)cbp_code(CAVLC_GOLOMB_TO_INTER_CBP, code->res.cbp));
    }
    if (code->res.cbp == 0 && code->kind != KIND_I16) return;
    bw_se(w, 0); /* mb_qp_delta */
    int lv[16];
    if (code->kind == KIND_I16) {
        for (int k = 0; k < 16; k++) lv[k] = code->dc[k];
        write_block(w, w_nc_luma(s, code->res.nnz, mbx, mby, 0, 0), lv, 16);
    }
    for (int n = 0; n < 16; n++) {
        int bx = ((n >> 2) & 1) * 2 + (n & 1), by = ((n >> 3) & 1) * 2 + ((n >> 1) & 1);
        if (!(cbpl & (1 << (n / 4)))) continue;
        int nc = w_nc_luma(s, code->res.nnz, mbx, mby, bx, by);
        const int16_t* b = code->res.luma[by * 4 + bx];
        if (code->kind == KIND_I16) {
            for (int k = 0; k < 15; k++) lv[k] = b[1 + k];
            write_block(w, nc, lv, 15);
        } else {
            for (int k = 0; k < 16; k++) lv[k] = b[k];
            write_block(w, nc, lv, 16);
        }
    }
    if (cbpc > 0)
        for (int cc = 0; cc < 2; cc++) {
            for (int k = 0; k < 4; k++) lv[k] = code->res.cdc[cc][k];
            write_block(w, -1, lv, 4);
        }
    if (cbpc == 2)
        for (int cc = 0; cc < 2; cc++)
            for (int blk = 0; blk < 4; blk++) {
                int nc = w_nc_chroma(s, code->res.cnnz[cc], cc, mbx, mby, blk & 1, blk >> 1);
                for (int k = 0; k < 15; k++) lv[k] = code->res.cac[cc][blk][1 + k];
                write_block(w, nc, lv, 15);
            }
}

static int bands_of(const struct ironav_ctx* c, int starts[1025]) {
    int nb = 0;
    for (int r = 0; r < c->mb_h; r++)
        if (c->band_start[r] == r) starts[nb++] = r;
    starts[nb] = c->mb_h;
    return nb;
}

static void write_band_cabac(const struct ironav_ctx* c, const ironav_mbcode* codes, int row0, int row1, bitw* w);

/* The picture's slices: header (enc/mod.rs:566-600), macroblocks in raster order (FrameCoder::encode,
 * enc/frame.rs:452-487), trailing skip run and rbsp bits; each a NAL unit of nal_ref_idc 3, type 5 (IDR) or
 * 1 (enc/mod.rs:641-643). */
int ironav_write_slices(ironav_ctx* c, int idr, int frame_num, int idr_pic_id, const ironav_mbcode* codes, uint8_t* out, size_t cap,
                        size_t* len) {
    if (!c || !codes || !len || (idr != 0) != (c->intra_pic != 0) || (!idr && c->nact < 1) || frame_num < 0 || frame_num > 255 ||
        idr_pic_id < 0 || idr_pic_id > 65535)
        return IRONAV_INVALID_ARGUMENT;
    int starts[1025];
    int nb = bands_of(c, starts);
    int qp = c->qpp - 6 * (c->bd - 8);
    bitw stream;
    bw_init(&stream);
    for (int b = 0; b < nb; b++) {
        swr s;
        memset(&s, 0, sizeof(s));
        s.c = c;
        s.codes = codes;
        s.p_slice = !idr;
        s.nref = idr ? 0 : c->nact;
        s.first_row = starts[b];
        bw_init(&s.w);
        bitw* w = &s.w;
        bw_ue(w, (uint32_t)(starts[b] * c->mb_w)); /* first_mb_in_slice */
        bw_ue(w, idr ? 7 : 5);                     /* slice_type: I or P, all slices alike */
        bw_ue(w, 0);                               /* pic_parameter_set_id */
        bw_put(w, 8, (uint32_t)frame_num);
        if (idr) bw_ue(w, (uint32_t)idr_pic_id);
        if (!idr) {
            if (c->nact > 1) {
                bw_flag(w, 1); /* num_ref_idx_active_override_flag */
                bw_ue(w, (uint32_t)(c->nact - 1));
            } else bw_flag(w, 0);
            bw_flag(w, 0); /* ref_pic_list_modification_flag_l0 */
        }
        if (idr) {
            bw_flag(w, 0); /* no_output_of_prior_pics_flag */
            bw_flag(w, 0); /* long_term_reference_flag */
        } else bw_flag(w, 0); /* adaptive_ref_pic_marking_mode_flag */
        if (c->cabac && !idr) bw_ue(w, 0); /* cabac_init_idc */
        bw_se(w, qp - 26);    /* slice_qp_delta */
        if (c->cabac) write_band_cabac(c, codes, starts[b], starts[b + 1], w);
        else {
            for (int mby = starts[b]; mby < starts[b + 1]; mby++)
                for (int mbx = 0; mbx < c->mb_w; mbx++) write_mb(&s, &codes[(size_t)mby * c->mb_w + mbx], mbx, mby);
            if (s.skip_run > 0) bw_ue(w, s.skip_run);
            bw_finish(w);
        }
        put_nal(&stream, 3, idr ? 5 : 1, w->buf, w->len);
        free(w->buf);
    }
    *len = stream.len;
    int st = IRONAV_OK;
    if (!out || cap < stream.len) st = IRONAV_INVALID_ARGUMENT;
    else memcpy(out, stream.buf, stream.len);
    free(stream.buf);
    return st;
}

int ironav_write_slices_device(ironav_ctx* c, int idr, int frame_num, int idr_pic_id, const ironav_mbcode* d_codes, uint8_t* out, size_t cap,
                               size_t* len) {
    (void)c; (void)idr; (void)frame_num; (void)idr_pic_id; (void)d_codes; (void)out; (void)cap; (void)len;
    return IRONAV_HARDWARE_UNAVAILABLE;
}

/* (level_idc, MaxFS, MaxMBPS) of Table A-1 (enc/mod.rs:43-63) */
static const int64_t LEVELS_A1[19][3] = {{10, 99, 1485},      {11, 396, 3000},      {12, 396, 6000},       {13, 396, 11880},
                                         {20, 396, 11880},    {21, 792, 19800},     {22, 1620, 20250},     {30, 1620, 40500},
                                         {31, 3600, 108000},  {32, 5120, 216000},   {40, 8192, 245760},    {41, 8192, 245760},
                                         {42, 8704, 522240},  {50, 22080, 589824},  {51, 36864, 983040},   {52, 36864, 2073600},
                                         {60, 139264, 4177920}, {61, 139264, 8355840}, {62, 139264, 16711680}};

/* H264Encoder::sps / pps without B pictures (enc/mod.rs:296-400) and the level choice (154-157) */
int ironav_write_parameter_sets(const ironav_stream_params* p, uint8_t* out, size_t cap, size_t* len) {
    if (!p || !len || p->width <= 0 || p->height <= 0 || (p->width & 1) || (p->height & 1) || (p->bd != 8 && p->bd != 10) || p->refs < 1 ||
        p->refs > 16)
        return IRONAV_INVALID_ARGUMENT;
    int mb_w = (p->width + 15) / 16, mb_h = (p->height + 15) / 16;
    if (mb_w > 1024 || mb_h > 1024) return IRONAV_INVALID_ARGUMENT;
    int64_t fs = (int64_t)mb_w * mb_h;
    int rate_ok = p->fps_num > 0 && p->fps_den > 0;
    double fps = rate_ok ? (double)p->fps_num / (double)p->fps_den : 25.0;
    int64_t mbps = (int64_t)ceil((double)fs * fps);
    int level = -1;
    for (int i = 0; i < 19 && level < 0; i++)
        if (LEVELS_A1[i][1] >= fs && LEVELS_A1[i][2] >= mbps) level = (int)LEVELS_A1[i][0];
    for (int i = 0; i < 19 && level < 0; i++)
        if (LEVELS_A1[i][1] >= fs) level = (int)LEVELS_A1[i][0];
    if (level < 0) level = 62;
    if (p->cabac < 0 || p->cabac > 1 || p->transform8 < 0 || p->transform8 > 1) return IRONAV_INVALID_ARGUMENT;
    int t8 = p->cabac && p->transform8, high = t8 || p->bd > 8;
    bitw w;
    bw_init(&w);
    if (p->bd > 8) {
        bw_put(&w, 8, 110); /* High 10 */
        bw_put(&w, 8, 0);
    } else if (high) {
        bw_put(&w, 8, 100); /* High */
        bw_put(&w, 8, 0);
    } else if (p->cabac) {
        bw_put(&w, 8, 77);   /* Main */
        bw_put(&w, 8, 0x40); /* constraint_set1: Main */
    } else {
        bw_put(&w, 8, 66);          /* Baseline */
        bw_put(&w, 8, 0xC0);        /* constraint_set0 and constraint_set1: Constrained Baseline */
    }
    bw_put(&w, 8, (uint32_t)level);
    bw_ue(&w, 0); /* seq_parameter_set_id */
    if (high) {
        bw_ue(&w, 1);                          /* chroma_format_idc: 4:2:0 */
        bw_ue(&w, (uint32_t)(p->bd - 8));      /* bit_depth_luma_minus8 */
        bw_ue(&w, (uint32_t)(p->bd - 8));      /* bit_depth_chroma_minus8 */
        bw_flag(&w, 0);                        /* qpprime_y_zero_transform_bypass_flag */
        bw_flag(&w, 0);                        /* seq_scaling_matrix_present_flag */
    }
    bw_ue(&w, 4); /* log2_max_frame_num_minus4 */
    bw_ue(&w, 2); /* pic_order_cnt_type: output order is decoding order */
    bw_ue(&w, (uint32_t)p->refs); /* max_num_ref_frames */
    bw_flag(&w, 0);               /* gaps_in_frame_num_value_allowed_flag */
    bw_ue(&w, (uint32_t)(mb_w - 1));
    bw_ue(&w, (uint32_t)(mb_h - 1));
    bw_flag(&w, 1); /* frame_mbs_only_flag */
    bw_flag(&w, 1); /* direct_8x8_inference_flag */
    int cr = (mb_w * 16 - p->width) / 2, cb = (mb_h * 16 - p->height) / 2;
    bw_flag(&w, cr > 0 || cb > 0);
    if (cr > 0 || cb > 0) {
        bw_ue(&w, 0);
        bw_ue(&w, (uint32_t)cr);
        bw_ue(&w, 0);
        bw_ue(&w, (uint32_t)cb);
    }
    bw_flag(&w, 1); /* vui_parameters_present_flag */
    bw_flag(&w, 0); /* aspect_ratio_info_present_flag */
    bw_flag(&w, 0); /* overscan_info_present_flag */
    bw_flag(&w, 0); /* video_signal_type_present_flag */
    bw_flag(&w, 0); /* chroma_loc_info_present_flag */
    int timing = rate_ok && 2ll * p->fps_num <= 0xFFFFFFFFll;
    bw_flag(&w, timing);
    if (timing) {
        bw_put(&w, 32, (uint32_t)p->fps_den);      /* num_units_in_tick */
        bw_put(&w, 32, 2u * (uint32_t)p->fps_num); /* time_scale: two ticks per frame */
        bw_flag(&w, 1);                            /* fixed_frame_rate_flag */
    }
    bw_flag(&w, 0); /* nal_hrd_parameters_present_flag */
    bw_flag(&w, 0); /* vcl_hrd_parameters_present_flag */
    bw_flag(&w, 0); /* pic_struct_present_flag */
    bw_flag(&w, 1); /* bitstream_restriction_flag */
    bw_flag(&w, 1); /* motion_vectors_over_pic_boundaries_flag */
    bw_ue(&w, 0);   /* max_bytes_per_pic_denom */
    bw_ue(&w, 0);   /* max_bits_per_mb_denom */
    bw_ue(&w, 15);  /* log2_max_mv_length_horizontal */
    bw_ue(&w, 15);  /* log2_max_mv_length_vertical */
    bw_ue(&w, 0);   /* max_num_reorder_frames */
    bw_ue(&w, (uint32_t)(p->refs > 1 ? p->refs : 1)); /* max_dec_frame_buffering */
    bw_finish(&w);
    bitw pps;
    bw_init(&pps);
    bw_ue(&pps, 0);      /* pic_parameter_set_id */
    bw_ue(&pps, 0);      /* seq_parameter_set_id */
    bw_flag(&pps, p->cabac); /* entropy_coding_mode_flag */
    bw_flag(&pps, 0);    /* bottom_field_pic_order_in_frame_present_flag */
    bw_ue(&pps, 0);      /* num_slice_groups_minus1 */
    bw_ue(&pps, 0);      /* num_ref_idx_l0_default_active_minus1 */
    bw_ue(&pps, 0);      /* num_ref_idx_l1_default_active_minus1 */
    bw_flag(&pps, 0);    /* weighted_pred_flag */
    bw_put(&pps, 2, 0);  /* weighted_bipred_idc */
    bw_se(&pps, 0);      /* pic_init_qp_minus26 */
    bw_se(&pps, 0);      /* pic_init_qs_minus26 */
    bw_se(&pps, 0);      /* chroma_qp_index_offset */
    bw_flag(&pps, 0);    /* deblocking_filter_control_present_flag */
    bw_flag(&pps, 0);    /* constrained_intra_pred_flag */
    bw_flag(&pps, 0);    /* redundant_pic_cnt_present_flag */
    if (t8) {
        bw_flag(&pps, 1); /* transform_8x8_mode_flag */
        bw_flag(&pps, 0); /* pic_scaling_matrix_present_flag */
        bw_se(&pps, 0);   /* second_chroma_qp_index_offset */
    }
    bw_finish(&pps);
    bitw stream;
    bw_init(&stream);
    put_nal(&stream, 3, 7, w.buf, w.len);
    put_nal(&stream, 3, 8, pps.buf, pps.len);
    free(w.buf);
    free(pps.buf);
    *len = stream.len;
    int st = IRONAV_OK;
    if (!out || cap < stream.len) st = IRONAV_INVALID_ARGUMENT;
    else memcpy(out, stream.buf, stream.len);
    free(stream.buf);
    return st;
}

/* Test hooks (oracle only): write_block of one block, and ue/se bits, for the reference's own writer tests */
int oracle_write_block(int nc, const int* levels, int max, uint8_t* out, int cap, int* nbits) {
    bitw w;
    bw_init(&w);
    int n = write_block(&w, nc, levels, max);
    *nbits = (int)(w.len * 8 + w.n);
    bw_finish(&w);
    if ((int)w.len <= cap) memcpy(out, w.buf, w.len);
    free(w.buf);
    return n;
}

int oracle_put_nal(int ref_idc, int kind, const uint8_t* rbsp, int n, uint8_t* out, int cap) {
    bitw w;
    bw_init(&w);
    put_nal(&w, ref_idc, kind, rbsp, (size_t)n);
    int len = (int)w.len;
    if (len <= cap) memcpy(out, w.buf, w.len);
    free(w.buf);
    return len;
}

int ironav_set_replay_form(ironav_ctx* c, int form) { return (!c || form < 0 || form > 3) ? IRONAV_INVALID_ARGUMENT : IRONAV_OK; }

int ironav_set_learned(ironav_ctx* c, const int16_t* cands, const uint8_t* cls, int margin, unsigned* stats) {
    if (!c || (cands && (!cls || !stats)) || margin < 0) return IRONAV_INVALID_ARGUMENT;
    c->learned = cands;
    c->learned_cls = cands ? cls : NULL;
    c->learned_stats = cands ? stats : NULL;
    c->learned_margin = margin;
    return IRONAV_OK;
}

/* The learned proposer's kernels exist only on the device */
int ironav_prop_conv3x3(const void* x, int cin, long long n, const void* w, const float* b, int relu, const void* m, void* y, unsigned* err, void* s) {
    (void)x; (void)cin; (void)n; (void)w; (void)b; (void)relu; (void)m; (void)y; (void)err; (void)s;
    return IRONAV_HARDWARE_UNAVAILABLE;
}
int ironav_prop_wgrad3x3(const void* x, int cin, const void* dz, long long n, float* dw, float* db, unsigned* err, void* s) {
    (void)x; (void)cin; (void)dz; (void)n; (void)dw; (void)db; (void)err; (void)s;
    return IRONAV_HARDWARE_UNAVAILABLE;
}
int ironav_prop_prep(const ironav_prop_sample* sm, int n, void* x, void* s) { (void)sm; (void)n; (void)x; (void)s; return IRONAV_HARDWARE_UNAVAILABLE; }
int ironav_prop_head_fwd(const void* f, int n, const float* hw, const float* hb, float* o, void* s) {
    (void)f; (void)n; (void)hw; (void)hb; (void)o; (void)s;
    return IRONAV_HARDWARE_UNAVAILABLE;
}
int ironav_prop_loss(const float* o, const int16_t* tm, const uint8_t* tp, int n, float* d, float* sums, void* s) {
    (void)o; (void)tm; (void)tp; (void)n; (void)d; (void)sums; (void)s;
    return IRONAV_HARDWARE_UNAVAILABLE;
}
int ironav_prop_head_bwd(const void* f, int n, const float* d, const float* hw, float* ghw, float* ghb, void* dz, void* s) {
    (void)f; (void)n; (void)d; (void)hw; (void)ghw; (void)ghb; (void)dz; (void)s;
    return IRONAV_HARDWARE_UNAVAILABLE;
}
int ironav_prop_adam(float* p, float* g, float* m, float* v, long long n, float lr, float b1, float b2, int step, float eps, void* s) {
    (void)p; (void)g; (void)m; (void)v; (void)n; (void)lr; (void)b1; (void)b2; (void)step; (void)eps; (void)s;
    return IRONAV_HARDWARE_UNAVAILABLE;
}
int ironav_prop_weights(const float* w, int cin, void* wf, void* wt, void* s) { (void)w; (void)cin; (void)wf; (void)wt; (void)s; return IRONAV_HARDWARE_UNAVAILABLE; }
int ironav_prop_head_pack(const float* hw, float* hwt, void* s) {
    (void)hw; (void)hwt; (void)s;
    return IRONAV_HARDWARE_UNAVAILABLE;
}
int ironav_prop_head_fwd_packed(const void* f, int n, const float* hwt, const float* hb, float* o, void* s) {
    (void)f; (void)n; (void)hwt; (void)hb; (void)o; (void)s;
    return IRONAV_HARDWARE_UNAVAILABLE;
}
int ironav_prop_propose(const float* o, int n, float min_conf, int16_t* c, uint8_t* k, void* s) {
    (void)o; (void)n; (void)min_conf; (void)c; (void)k; (void)s;
    return IRONAV_HARDWARE_UNAVAILABLE;
}

/* ==== High profile: CABAC and rate-distortion decisions (the encoder's default entropy coding) ==== */

#include "cabac_tables.h"

int ironav_set_entropy(ironav_ctx* c, int cabac, int transform8) {
    if (!c || cabac < 0 || cabac > 1 || transform8 < 0 || transform8 > 1) return IRONAV_INVALID_ARGUMENT;
    c->cabac = cabac;
    c->t8 = cabac && transform8; /* FrameCoder::new, enc/frame.rs:405: transform8 with CABAC only */
    return IRONAV_OK;
}

/* Bins, enc/cabac.rs:10-30: the arithmetic coder (CabacWriter, 42-147: w set) or the bit counter (CabacCost,
 * 150-192: w NULL). Both adapt their own contexts the same way. */
typedef struct cab {
    uint8_t st[1024]; /* per context: pStateIdx * 2 + valMPS */
    uint32_t bits;    /* the counter's total, 1/256 bits */
    bitw* w;
    uint32_t low, range, outstanding;
    int first;
} cab;

/* entropy(), enc/cabac.rs:162-173: -log2 of the MPS and LPS probabilities per pStateIdx in 1/256 bits, with
 * pLPS = 0.5 * (0.01875 / 0.5)^(p / 63) */
static uint32_t CAB_ENTROPY[64][2];

__attribute__((constructor)) static void cab_entropy_init(void) {
    for (int p = 0; p < 64; p++) {
        double lps = 0.5 * pow(0.01875 / 0.5, (double)p / 63.0);
        CAB_ENTROPY[p][0] = (uint32_t)round(-log2(1.0 - lps) * 256.0);
        CAB_ENTROPY[p][1] = (uint32_t)round(-log2(lps) * 256.0);
    }
}

/* the contexts of a slice, CabacWriter::new, enc/cabac.rs:54-64 (9.3.1.1) */
static void cab_states(uint8_t st[1024], int intra, int idc, int slice_qp) {
    int qp = clampi(slice_qp, 0, 51);
    for (int i = 0; i < 1024; i++) {
        int m = intra ? CABAC_INIT_I[i][0] : CABAC_INIT_PB[idc][i][0];
        int n = intra ? CABAC_INIT_I[i][1] : CABAC_INIT_PB[idc][i][1];
        int pre = clampi(((m * qp) >> 4) + n, 1, 126);
        st[i] = (uint8_t)(pre <= 63 ? (63 - pre) << 1 : ((pre - 64) << 1) | 1);
    }
}

/* next_state, enc/cabac.rs:32-40 */
static uint8_t cab_next(uint8_t s, int bin) {
    int p = s >> 1, mps = s & 1;
    if (bin != mps) return (uint8_t)((TRANS_LPS[p] << 1) | (p == 0 ? !mps : mps));
    return (uint8_t)(((p < 62 ? p + 1 : p) << 1) | mps);
}

/* put_bit and renorm, enc/cabac.rs:70-97 (9.3.4.2) */
static void cab_put_bit(cab* c, uint32_t b) {
    if (c->first) c->first = 0;
    else bw_put(c->w, 1, b);
    for (; c->outstanding > 0; c->outstanding--) bw_put(c->w, 1, 1 - b);
}

static void cab_renorm(cab* c) {
    while (c->range < 256) {
        if (c->low < 256) cab_put_bit(c, 0);
        else if (c->low >= 512) {
            c->low -= 512;
            cab_put_bit(c, 1);
        } else {
            c->low -= 256;
            c->outstanding++;
        }
        c->range <<= 1;
        c->low <<= 1;
    }
}

/* decision, enc/cabac.rs:105-116 (coder) and 176-180 (counter) */
static void cab_decision(cab* c, int ctx, int bin) {
    uint8_t s = c->st[ctx];
    int p = s >> 1, mps = s & 1;
    bin = bin != 0;
    c->st[ctx] = cab_next(s, bin);
    if (!c->w) {
        c->bits += CAB_ENTROPY[p][bin != mps];
        return;
    }
    uint32_t lps = LPS_RANGE[p][(c->range >> 6) & 3];
    c->range -= lps;
    if (bin != mps) {
        c->low += c->range;
        c->range = lps;
    }
    cab_renorm(c);
}

/* bypass, enc/cabac.rs:118-132 and 182-184 */
static void cab_bypass(cab* c, int bin) {
    if (!c->w) {
        c->bits += 256;
        return;
    }
    c->low <<= 1;
    if (bin) c->low += c->range;
    if (c->low >= 1024) {
        cab_put_bit(c, 1);
        c->low -= 1024;
    } else if (c->low < 512) cab_put_bit(c, 0);
    else {
        c->low -= 512;
        c->outstanding++;
    }
}

/* terminate, enc/cabac.rs:134-146 and 186-188: end_of_slice_flag, or the I_PCM test of an intra mb_type */
static void cab_terminate(cab* c, int bin) {
    if (!c->w) {
        c->bits += bin ? 7 * 256 : 1;
        return;
    }
    c->range -= 2;
    if (bin) {
        c->low += c->range;
        c->range = 2;
        cab_renorm(c);
        cab_put_bit(c, (c->low >> 9) & 1);
        bw_put(c->w, 2, ((c->low >> 7) & 3) | 1); /* the last of the two bits is the rbsp_stop_one_bit */
    } else cab_renorm(c);
}

/* exp_golomb, enc/cabac.rs:17-29: the bypass-coded k-th order Exp-Golomb suffix (9.3.2.3) */
static void cab_egk(cab* c, uint32_t v, uint32_t k) {
    while (v >= (1u << k)) {
        cab_bypass(c, 1);
        v -= 1u << k;
        k++;
    }
    cab_bypass(c, 0);
    while (k > 0) {
        k--;
        cab_bypass(c, (v >> k) & 1);
    }
}

/* write_block, enc/cabac.rs:194-250: coded_block_flag (context cbf_ctx, none when < 0) and the max levels of
 * category cat in scan order. Returns the non-zero count. */
static int cab_block(cab* c, int cat, int cbf_ctx, const int16_t* lv, int max) {
    int total = 0, last = -1;
    for (int i = 0; i < max; i++)
        if (lv[i]) {
            total++;
            last = i;
        }
    if (cbf_ctx >= 0) cab_decision(c, cbf_ctx, total > 0);
    if (total == 0) return 0;
    for (int i = 0; i < max - 1; i++) {
        /* 4:2:0 chroma DC has three significance contexts, one per position; 8x8 blocks share theirs */
        int sig = cat == 3 ? mini(i, 2) : cat == 5 ? SIG_OFF_8X8[0][i] : i;
        int lst = cat == 3 ? mini(i, 2) : cat == 5 ? LAST_OFF_8X8[i] : i;
        cab_decision(c, SIG_OFF[0][cat] + sig, lv[i] != 0);
        if (lv[i]) {
            cab_decision(c, LAST_OFF[0][cat] + lst, i == last);
            if (i == last) break;
        }
    }
    int base = ABS_OFF[cat], eq1 = 0, gt1 = 0;
    for (int i = last; i >= 0; i--) {
        int l = lv[i];
        if (!l) continue;
        uint32_t a = (uint32_t)abs(l);
        int inc0 = gt1 ? 0 : mini(1 + eq1, 4);
        if (a == 1) {
            cab_decision(c, base + inc0, 0);
            eq1++;
        } else {
            cab_decision(c, base + inc0, 1);
            int incn = base + 5 + mini(gt1, 4 - (cat == 3));
            /* abs - 2 ones and a zero, the ones capped at 13 with the rest in an Exp-Golomb suffix */
            for (uint32_t k = 0; k < (a - 2 < 13 ? a - 2 : 13); k++) cab_decision(c, incn, 1);
            if (a < 15) cab_decision(c, incn, 0);
            else cab_egk(c, a - 15, 0);
            gt1++;
        }
        cab_bypass(c, l < 0);
    }
    return total;
}

/* mvd_bins, enc/frame.rs:2393-2414: mvd_l0 of one component, sum = the neighbours' absolute differences */
static void cab_mvd(cab* c, int comp, int d, uint32_t sum) {
    int base = comp == 0 ? 40 : 47, inc = sum < 3 ? 0 : sum > 32 ? 2 : 1;
    uint32_t a = (uint32_t)abs(d);
    cab_decision(c, base + inc, a > 0);
    if (a == 0) return;
    int ctx = base + 3;
    for (uint32_t k = 1; k < (a < 9 ? a : 9); k++) {
        cab_decision(c, ctx, 1);
        if (ctx < base + 6) ctx++;
    }
    if (a < 9) cab_decision(c, ctx, 0);
    else cab_egk(c, a - 9, 3);
    cab_bypass(c, d < 0);
}

/* What the contexts read of a neighbouring macroblock (the CABAC fields of MbState, enc/frame.rs:245-272, as
 * finish_mb sets them, 2281-2321), from its code. */
typedef struct cnb {
    int skip, kind, inter, cbp, t8x8, chroma_mode, cbf_dc;
    int8_t r8[4];        /* list 0 reference index per 8x8 block (-1 intra) */
    uint8_t mvd[16][2];  /* absolute vector differences per 4x4 block, capped at 64 (mvd_grid, 238-241) */
    const uint8_t* nnz;  /* coefficients per luma 4x4 block */
    const uint8_t (*cnnz)[4];
} cnb;

static void cnb_of(const ironav_mbcode* k, cnb* n) {
    memset(n, 0, sizeof(*n));
    n->skip = k->skip;
    n->kind = k->kind;
    n->inter = k->kind == KIND_INTER;
    n->cbp = k->res.cbp;
    n->t8x8 = k->res.t8x8;
    n->chroma_mode = n->inter ? 0 : k->chroma_mode;
    int cbpc = k->res.cbp >> 4, any[3] = {0, 0, 0};
    for (int i = 0; i < 16; i++) any[0] |= k->dc[i] != 0;
    for (int i = 0; i < 4; i++) any[1] |= k->res.cdc[0][i] != 0, any[2] |= k->res.cdc[1][i] != 0;
    n->cbf_dc = (k->kind == KIND_I16 && any[0]) | ((cbpc > 0 && any[1]) << 1) | ((cbpc > 0 && any[2]) << 2);
    n->nnz = k->res.nnz;
    n->cnnz = k->res.cnnz;
    for (int b8 = 0; b8 < 4; b8++) n->r8[b8] = -1;
    if (!n->inter) return;
    /* spread of the partitions' indices, enc/frame.rs:185-196,2301-2302 */
    for (int b8 = 0; b8 < 4; b8++)
        n->r8[b8] = (int8_t)k->refs[k->part == 0 ? 0 : k->part == 1 ? b8 >> 1 : k->part == 2 ? b8 & 1 : b8];
    if (k->skip) return;
    rect4 rs[16];
    int nr = rects(k->part, k->sub, rs);
    for (int q = 0; q < nr; q++)
        for (int by = rs[q].y; by < rs[q].y + rs[q].h; by++)
            for (int bx = rs[q].x; bx < rs[q].x + rs[q].w; bx++)
                for (int comp = 0; comp < 2; comp++) n->mvd[by * 4 + bx][comp] = (uint8_t)mini(abs(k->mvds[q][comp]), 64);
}

/* What mb_bins reads besides the macroblock's own code: the picture's codes so far (its neighbours) and
 * the slice's parameters. */
typedef struct cabx {
    const struct ironav_ctx* c;
    const ironav_mbcode* codes;
    int first_row;       /* the slice band's first macroblock row */
    int p_slice, t8, nref;
} cabx;

/* nb_state, enc/frame.rs:509-515: a neighbour in the same slice, or NULL */
static const ironav_mbcode* cx_nb(const cabx* X, int mbx, int mby) {
    if (mbx < 0 || mby < X->first_row || mbx >= X->c->mb_w || mby >= X->c->mb_h) return NULL;
    return &X->codes[(size_t)mby * X->c->mb_w + mbx];
}

/* pred_i4_mode, enc/frame.rs:619-627 */
static int cx_pred_mode(const cabx* X, const uint8_t cur[16], int mbx, int mby, int bx, int by) {
    int a = -1, b = -1;
    if (bx > 0) a = cur[by * 4 + bx - 1];
    else {
        const ironav_mbcode* n = cx_nb(X, mbx - 1, mby);
        if (n) a = kind_nxn(n->kind) ? n->modes[by * 4 + 3] : 2;
    }
    if (by > 0) b = cur[(by - 1) * 4 + bx];
    else {
        const ironav_mbcode* n = cx_nb(X, mbx, mby - 1);
        if (n) b = kind_nxn(n->kind) ? n->modes[12 + bx] : 2;
    }
    return (a >= 0 && b >= 0) ? mini(a, b) : 2;
}

/* mb_bins, enc/frame.rs:2028-2279, for I and P slices: the bins of a macroblock up to end_of_slice_flag,
 * with the contexts of 9.3.3.1.1 and 9.3.3.1.3 from its neighbours in the slice */
static void mb_bins(cab* c, const cabx* X, const ironav_mbcode* code, int mbx, int mby) {
    const ironav_mbcode* lk = cx_nb(X, mbx - 1, mby);
    const ironav_mbcode* tk = cx_nb(X, mbx, mby - 1);
    cnb L, T;
    if (lk) cnb_of(lk, &L);
    if (tk) cnb_of(tk, &T);
    const cnb* l = lk ? &L : NULL;
    const cnb* t = tk ? &T : NULL;
    if (X->p_slice) {
        cab_decision(c, 11 + (l && !l->skip) + (t && !t->skip), code->skip);
        if (code->skip) return;
    }
    int kind = code->kind, cbp = code->res.cbp, cbpl = cbp & 15, cbpc = cbp >> 4;
    /* mb_type */
    if (kind == KIND_INTER) {
        /* P_L0_16x16 000, P_L0_L0_16x8 011, P_L0_L0_8x16 010, P_8x8 001 */
        static const int B1[4] = {0, 1, 1, 0}, B2[4] = {0, 1, 0, 1};
        cab_decision(c, 14, 0);
        cab_decision(c, 15, B1[code->part]);
        cab_decision(c, B1[code->part] ? 17 : 16, B2[code->part]);
    } else {
        int pre = X->p_slice, base = pre ? 17 : 3, first;
        if (pre) {
            cab_decision(c, 14, 1);
            first = 17;
        } else first = 3 + (l && !kind_nxn(l->kind)) + (t && !kind_nxn(t->kind));
        if (kind_nxn(kind)) {
            cab_decision(c, first, 0);
            if (X->t8) cab_decision(c, 399 + (l && l->t8x8) + (t && t->t8x8), kind == KIND_I8);
        } else {
            cab_decision(c, first, 1);
            cab_terminate(c, 0); /* not I_PCM */
            int b1 = pre ? base + 1 : base + 3, b2 = pre ? base + 2 : base + 4, b3 = pre ? base + 3 : base + 6;
            cab_decision(c, b1, cbpl != 0);
            cab_decision(c, b2, cbpc != 0);
            if (cbpc) cab_decision(c, pre ? base + 2 : base + 5, cbpc == 2);
            cab_decision(c, b3, (code->i16_mode >> 1) == 1);
            cab_decision(c, pre ? base + 3 : base + 7, code->i16_mode & 1);
        }
    }
    if (kind_nxn(kind)) {
        int t8 = kind == KIND_I8;
        uint8_t so_far[16];
        memset(so_far, 2, sizeof(so_far));
        for (int n = 0; n < (t8 ? 4 : 16); n++) {
            int bx = t8 ? (n & 1) * 2 : ((n >> 2) & 1) * 2 + (n & 1), by = t8 ? (n >> 1) * 2 : ((n >> 3) & 1) * 2 + ((n >> 1) & 1);
            int mode = code->modes[by * 4 + bx];
            int pred = cx_pred_mode(X, so_far, mbx, mby, bx, by);
            so_far[by * 4 + bx] = (uint8_t)mode;
            if (t8) so_far[by * 4 + bx + 1] = so_far[(by + 1) * 4 + bx] = so_far[(by + 1) * 4 + bx + 1] = (uint8_t)mode;
            cab_decision(c, 68, mode == pred);
            if (mode != pred) {
                int rem = mode < pred ? mode : mode - 1;
                for (int k = 0; k < 3; k++) cab_decision(c, 69, (rem >> k) & 1);
            }
        }
    }
    if (kind != KIND_INTER) {
        int m = code->chroma_mode;
        cab_decision(c, 64 + (l && !l->inter && l->chroma_mode != 0) + (t && !t->inter && t->chroma_mode != 0), m > 0);
        if (m > 0) {
            cab_decision(c, 67, m > 1);
            if (m > 1) cab_decision(c, 67, m > 2);
        }
    } else {
        /* sub_mb_type of each 8x8 block of P_8x8 (Table 9-38: 1, 00, 011, 010; contexts 21 to 23) */
        if (code->part == 3)
            for (int k = 0; k < 4; k++) {
                int s = code->sub[k];
                if (s == 0) cab_decision(c, 21, 1);
                else if (s == 1) {
                    cab_decision(c, 21, 0);
                    cab_decision(c, 22, 0);
                } else {
                    cab_decision(c, 21, 0);
                    cab_decision(c, 22, 1);
                    cab_decision(c, 23, s == 2);
                }
            }
        /* ref_idx_l0 per partition (per 8x8 block for P_8x8), unary, with the contexts of 9.3.3.1.1.6 */
        if (X->nref > 1) {
            uint8_t grid[4] = {0, 0, 0, 0};
            static const int P4[4][4][4] = {{{0, 0, 4, 4}}, {{0, 0, 4, 2}, {0, 2, 4, 2}}, {{0, 0, 2, 4}, {2, 0, 2, 4}},
                                            {{0, 0, 2, 2}, {2, 0, 2, 2}, {0, 2, 2, 2}, {2, 2, 2, 2}}};
            static const int NP[4] = {1, 2, 2, 4};
            for (int k = 0; k < NP[code->part]; k++) {
                int bx = P4[code->part][k][0], by = P4[code->part][k][1], w = P4[code->part][k][2], h = P4[code->part][k][3];
                int a = bx > 0 ? grid[(by / 2) * 2 + (bx - 1) / 2] > 0 : (l && l->r8[(by / 2) * 2 + 1] > 0);
                int b = by > 0 ? grid[((by - 1) / 2) * 2 + bx / 2] > 0 : (t && t->r8[2 + bx / 2] > 0);
                int r = code->refs[k], base = 54 + a + 2 * b;
                for (int i = 0; i <= r; i++) cab_decision(c, i == 0 ? base : i == 1 ? 58 : 59, i < r);
                for (int y8 = by / 2; y8 <= (by + h - 1) / 2; y8++)
                    for (int x8 = bx / 2; x8 <= (bx + w - 1) / 2; x8++) grid[y8 * 2 + x8] = code->refs[k];
            }
        }
        /* mvd_l0 per partition; the blocks left of and above a partition in the macroblock belong to earlier ones */
        cnb self;
        cnb_of(code, &self);
        rect4 rs[16];
        int nr = rects(code->part, code->sub, rs);
        for (int k = 0; k < nr; k++) {
            int bx = rs[k].x, by = rs[k].y;
            for (int comp = 0; comp < 2; comp++) {
                uint32_t a = bx > 0 ? self.mvd[by * 4 + bx - 1][comp] : (l ? l->mvd[by * 4 + 3][comp] : 0);
                uint32_t b = by > 0 ? self.mvd[(by - 1) * 4 + bx][comp] : (t ? t->mvd[12 + bx][comp] : 0);
                cab_mvd(c, comp, code->mvds[k][comp], a + b);
            }
        }
    }
    if (kind != KIND_I16) {
        int luma = 0;
        for (int b8 = 0; b8 < 4; b8++) {
            int ca = (b8 & 1) ? ((luma >> (b8 - 1)) & 1) == 0 : (l && ((l->cbp >> (b8 + 1)) & 1) == 0);
            int cb = b8 >= 2 ? ((luma >> (b8 - 2)) & 1) == 0 : (t && ((t->cbp >> (b8 + 2)) & 1) == 0);
            int bit = (cbpl >> b8) & 1;
            cab_decision(c, 73 + ca + 2 * cb, bit);
            luma |= bit << b8;
        }
        cab_decision(c, 77 + (l && (l->cbp >> 4) != 0) + 2 * (t && (t->cbp >> 4) != 0), cbpc != 0);
        if (cbpc) cab_decision(c, 81 + (l && (l->cbp >> 4) == 2) + 2 * (t && (t->cbp >> 4) == 2), cbpc == 2);
    }
    /* transform_size_8x8_flag is absent from P_8x8 with any sub-partition smaller than 8x8 */
    if (kind == KIND_INTER && X->t8 && cbpl && (code->part != 3 || !(code->sub[0] | code->sub[1] | code->sub[2] | code->sub[3])))
        cab_decision(c, 399 + (l && l->t8x8) + (t && t->t8x8), code->res.t8x8);
    if (!cbp && kind != KIND_I16) return;
    cab_decision(c, 60, 0); /* mb_qp_delta 0, after a macroblock without a change */
    /* an unavailable neighbour counts as a coded block for an intra macroblock */
    int un = kind != KIND_INTER;
#define FLAG(has, v) ((has) ? ((v) > 0) : un)
    if (kind == KIND_I16)
        cab_block(c, 0, 85 + FLAG(l, l ? l->cbf_dc & 1 : 0) + 2 * FLAG(t, t ? t->cbf_dc & 1 : 0), code->dc, 16);
    int cat = kind == KIND_I16 ? 1 : 2, base = kind == KIND_I16 ? 89 : 93;
    if (code->res.t8x8)
        for (int i8 = 0; i8 < 4; i8++)
            if (cbpl & (1 << i8)) cab_block(c, 5, -1, code->res.luma8[i8], 64);
    for (int n = 0; n < 16 && !code->res.t8x8; n++) {
        int bx = ((n >> 2) & 1) * 2 + (n & 1), by = ((n >> 3) & 1) * 2 + ((n >> 1) & 1);
        if (!(cbpl & (1 << (n / 4)))) continue;
        int ha = bx > 0 || l, hb = by > 0 || t;
        int a = bx > 0 ? code->res.nnz[by * 4 + bx - 1] : (l ? l->nnz[by * 4 + 3] : 0);
        int b = by > 0 ? code->res.nnz[(by - 1) * 4 + bx] : (t ? t->nnz[12 + bx] : 0);
        const int16_t* blk = code->res.luma[by * 4 + bx];
        cab_block(c, cat, base + FLAG(ha, a) + 2 * FLAG(hb, b), cat == 1 ? blk + 1 : blk, cat == 1 ? 15 : 16);
    }
    if (cbpc > 0)
        for (int comp = 0; comp < 2; comp++) {
            int m = 2 << comp;
            cab_block(c, 3, 97 + FLAG(l, l ? l->cbf_dc & m : 0) + 2 * FLAG(t, t ? t->cbf_dc & m : 0), code->res.cdc[comp], 4);
        }
    if (cbpc == 2)
        for (int comp = 0; comp < 2; comp++)
            for (int blk = 0; blk < 4; blk++) {
                int bx = blk & 1, by = blk >> 1;
                const uint8_t* cur = code->res.cnnz[comp];
                int ha = bx > 0 || l, hb = by > 0 || t;
                int a = bx > 0 ? cur[by * 2] : (l ? l->cnnz[comp][by * 2 + 1] : 0);
                int b = by > 0 ? cur[bx] : (t ? t->cnnz[comp][2 + bx] : 0);
                cab_block(c, 4, 101 + FLAG(ha, a) + 2 * FLAG(hb, b), code->res.cac[comp][blk] + 1, 15);
            }
#undef FLAG
}

/* Edges of an 8x8 block (h264/intra.rs:17-26: 16 samples above, the second half above-right, 8 left) */
typedef struct i_edges8 { int top[16], left[8], topleft, have_top, have_left, have_topleft; } i_edges8;

/* predict_nxn for n = 8, h264/intra.rs:30-128 (ITU-T H.264 8.3.2.2) */
static void i_pred8(int mode, const i_edges8* e, int bd, int out[64]) {
#define T(i) ((i) < 0 ? e->topleft : e->top[(i)])
#define L(j) ((j) < 0 ? e->topleft : e->left[(j)])
    for (int y = 0; y < 8; y++)
        for (int x = 0; x < 8; x++) {
            int v;
            switch (mode) {
            case 0: v = T(x); break;
            case 1: v = L(y); break;
            case 2: {
                int st = 0, sl = 0;
                for (int i = 0; i < 8; i++) st += T(i), sl += L(i);
                if (e->have_top && e->have_left) v = (st + sl + 8) >> 4;
                else if (e->have_left) v = (sl + 4) >> 3;
                else if (e->have_top) v = (st + 4) >> 3;
                else v = 1 << (bd - 1);
                break;
            }
            case 3: v = (x == 7 && y == 7) ? (T(14) + 3 * T(15) + 2) >> 2 : (T(x + y) + 2 * T(x + y + 1) + T(x + y + 2) + 2) >> 2; break;
            case 4:
                if (x > y) v = (T(x - y - 2) + 2 * T(x - y - 1) + T(x - y) + 2) >> 2;
                else if (x < y) v = (L(y - x - 2) + 2 * L(y - x - 1) + L(y - x) + 2) >> 2;
                else v = (T(0) + 2 * e->topleft + L(0) + 2) >> 2;
                break;
            case 5: {
                int z = 2 * x - y, i = x - (y >> 1);
                if (z >= 0 && (z & 1) == 0) v = (T(i - 1) + T(i) + 1) >> 1;
                else if (z >= 0) v = (T(i - 2) + 2 * T(i - 1) + T(i) + 2) >> 2;
                else if (z == -1) v = (L(0) + 2 * e->topleft + T(0) + 2) >> 2;
                else v = (L(y - 2 * x - 1) + 2 * L(y - 2 * x - 2) + L(y - 2 * x - 3) + 2) >> 2;
                break;
            }
            case 6: {
                int z = 2 * y - x, j = y - (x >> 1);
                if (z >= 0 && (z & 1) == 0) v = (L(j - 1) + L(j) + 1) >> 1;
                else if (z >= 0) v = (L(j - 2) + 2 * L(j - 1) + L(j) + 2) >> 2;
                else if (z == -1) v = (L(0) + 2 * e->topleft + T(0) + 2) >> 2;
                else v = (T(x - 2 * y - 1) + 2 * T(x - 2 * y - 2) + T(x - 2 * y - 3) + 2) >> 2;
                break;
            }
            case 7: {
                int i = x + (y >> 1);
                v = (y & 1) == 0 ? (T(i) + T(i + 1) + 1) >> 1 : (T(i) + 2 * T(i + 1) + T(i + 2) + 2) >> 2;
                break;
            }
            default: {
                int z = x + 2 * y, j = y + (x >> 1);
                if (z > 13) v = L(7);
                else if (z == 13) v = (L(6) + 3 * L(7) + 2) >> 2;
                else if ((z & 1) == 0) v = (L(j) + L(j + 1) + 1) >> 1;
                else v = (L(j) + 2 * L(j + 1) + L(j + 2) + 2) >> 2;
                break;
            }
            }
            out[y * 8 + x] = v;
        }
#undef T
#undef L
}

/* filter_8x8_edges, h264/intra.rs:131-158 (8.3.2.2.1): the reference-sample smoothing before Intra 8x8 prediction */
static void i_filter8(i_edges8* e) {
    i_edges8 p = *e;
    if (p.have_top) {
        e->top[0] = p.have_topleft ? (p.topleft + 2 * p.top[0] + p.top[1] + 2) >> 2 : (3 * p.top[0] + p.top[1] + 2) >> 2;
        for (int x = 1; x < 15; x++) e->top[x] = (p.top[x - 1] + 2 * p.top[x] + p.top[x + 1] + 2) >> 2;
        e->top[15] = (p.top[14] + 3 * p.top[15] + 2) >> 2;
    }
    if (p.have_topleft) {
        if (p.have_top && p.have_left) e->topleft = (p.top[0] + 2 * p.topleft + p.left[0] + 2) >> 2;
        else if (p.have_top) e->topleft = (3 * p.topleft + p.top[0] + 2) >> 2;
        else if (p.have_left) e->topleft = (3 * p.topleft + p.left[0] + 2) >> 2;
    }
    if (p.have_left) {
        e->left[0] = p.have_topleft ? (p.topleft + 2 * p.left[0] + p.left[1] + 2) >> 2 : (3 * p.left[0] + p.left[1] + 2) >> 2;
        for (int y = 1; y < 7; y++) e->left[y] = (p.left[y - 1] + 2 * p.left[y] + p.left[y + 1] + 2) >> 2;
        e->left[7] = (p.left[6] + 3 * p.left[7] + 2) >> 2;
    }
}

/* code_i8, enc/frame.rs:1307-1388: the luma of an Intra8x8 macroblock block by block into the reconstruction,
 * each 8x8 block's mode the cheapest by SATD + lambda * (1 predicted, 4 otherwise) over the filtered edges */
static void code_i8(const dctx* D, int mbx, int mby, ironav_mbcode* code) {
    const struct ironav_ctx* c = D->f->c;
    code_new(code, KIND_I8);
    code->res.t8x8 = 1;
    int ta = d_up(c, mby), la = mbx > 0, tla = la && ta, tra = ta && mbx + 1 < c->mb_w;
    uint16_t* p = D->rec[0];
    int ls = c->pw, maxv = (1 << c->bd) - 1;
    for (int i8 = 0; i8 < 4; i8++) {
        int bx = i8 & 1, by = i8 >> 1, x = mbx * 16 + bx * 8, y = mby * 16 + by * 8;
        i_edges8 e;
        memset(&e, 0, sizeof(e));
        e.have_left = bx > 0 || la;
        e.have_top = by > 0 || ta;
        e.have_topleft = bx > 0 ? (by > 0 ? 1 : ta) : (by > 0 ? la : tla);
        int have_tr = i8 == 0 ? ta : i8 == 1 ? tra : i8 == 2;
        if (e.have_top) {
            for (int i = 0; i < 8; i++) e.top[i] = p[(size_t)(y - 1) * ls + x + i];
            for (int i = 8; i < 16; i++) e.top[i] = have_tr ? p[(size_t)(y - 1) * ls + x + i] : e.top[7];
        }
        if (e.have_left)
            for (int j = 0; j < 8; j++) e.left[j] = p[(size_t)(y + j) * ls + x - 1];
        if (e.have_topleft) e.topleft = p[(size_t)(y - 1) * ls + x - 1];
        i_filter8(&e);
        int predicted = pred_i4_mode(D, code->modes, mbx, mby, bx * 2, by * 2);
        int bm = 2, bc = INT32_MAX, bp[64];
        for (int mode = 0; mode < 9; mode++) {
            int ok = (mode == 0 || mode == 3 || mode == 7) ? e.have_top
                   : (mode == 1 || mode == 8) ? e.have_left
                   : mode == 2 ? 1 : (e.have_top && e.have_left && e.have_topleft);
            if (!ok) continue;
            int pr[64], cc = c->lambda * (mode == predicted ? 1 : 4);
            i_pred8(mode, &e, c->bd, pr);
            for (int q = 0; q < 4; q++) {
                int pb[16];
                for (int r = 0; r < 4; r++)
                    for (int k = 0; k < 4; k++) pb[r * 4 + k] = pr[((q >> 1) * 4 + r) * 8 + (q & 1) * 4 + k];
                cc += d_satd4(D, 0, x + (q & 1) * 4, y + (q >> 1) * 4, pb);
            }
            if (cc < bc) {
                bm = mode;
                bc = cc;
                memcpy(bp, pr, sizeof(bp));
            }
        }
        int s[64], lv[64], co[64];
        for (int k = 0; k < 64; k++) s[k] = c->src[(size_t)(y + k / 8) * c->pw + x + k % 8];
        q_block8(s, bp, D->qp, 1, lv, co);
        for (int k = 0; k < 64; k++) p[(size_t)(y + k / 8) * ls + x + k % 8] = (uint16_t)bp[k];
        int n = 0;
        for (int k = 0; k < 64; k++) {
            code->res.luma8[i8][k] = (int16_t)lv[k];
            n += lv[k] != 0;
        }
        if (n) {
            q_idct8_add(co, p + (size_t)y * ls + x, ls, maxv);
            code->res.cbp |= (uint8_t)(1 << i8);
        }
        for (int j = 0; j < 4; j++) {
            int b = (by * 2 + (j >> 1)) * 4 + bx * 2 + (j & 1);
            code->modes[b] = (uint8_t)bm;
            code->res.nnz[b] = (uint8_t)n;
        }
    }
}

/* save_mb / restore_mb, enc/frame.rs:1406-1429: a macroblock's reconstruction, luma then Cb and Cr */
static void save_mb(const dctx* D, int mbx, int mby, uint16_t rec[384]) {
    const struct ironav_ctx* c = D->f->c;
    int cs = c->mb_w * 8;
    for (int r = 0; r < 16; r++) memcpy(rec + r * 16, D->rec[0] + (size_t)(mby * 16 + r) * c->pw + mbx * 16, 32);
    for (int k = 0; k < 2; k++)
        for (int r = 0; r < 8; r++) memcpy(rec + 256 + k * 64 + r * 8, D->rec[1 + k] + (size_t)(mby * 8 + r) * cs + mbx * 8, 16);
}

static void restore_mb(const dctx* D, int mbx, int mby, const uint16_t rec[384]) {
    const struct ironav_ctx* c = D->f->c;
    int cs = c->mb_w * 8;
    for (int r = 0; r < 16; r++) memcpy(D->rec[0] + (size_t)(mby * 16 + r) * c->pw + mbx * 16, rec + r * 16, 32);
    for (int k = 0; k < 2; k++)
        for (int r = 0; r < 8; r++) memcpy(D->rec[1 + k] + (size_t)(mby * 8 + r) * cs + mbx * 8, rec + 256 + k * 64 + r * 8, 16);
}

/* ssd_mb, enc/frame.rs:1432-1449: the squared error of the macroblock's reconstruction, luma and chroma */
static int64_t ssd_mb(const dctx* D, int mbx, int mby) {
    const struct ironav_ctx* c = D->f->c;
    int cs = c->mb_w * 8;
    int64_t ssd = 0;
    for (int i = 0; i < 256; i++) {
        int64_t d = (int64_t)c->src[(size_t)(mby * 16 + i / 16) * c->pw + mbx * 16 + i % 16] -
                    D->rec[0][(size_t)(mby * 16 + i / 16) * c->pw + mbx * 16 + i % 16];
        ssd += d * d;
    }
    for (int k = 0; k < 2; k++)
        for (int j = 0; j < 64; j++) {
            int64_t d = (int64_t)c->src_c[k][(size_t)(mby * 8 + j / 8) * cs + mbx * 8 + j % 8] - D->rec[1 + k][(size_t)(mby * 8 + j / 8) * cs + mbx * 8 + j % 8];
            ssd += d * d;
        }
    return ssd;
}

/* rd_cost, enc/frame.rs:1453-1457: SSD + lam2 * the bits CABAC would spend from the slice's contexts st */
static double rd_cost(const dctx* D, const cabx* X, const uint8_t st[1024], const ironav_mbcode* code, int mbx, int mby, double lam2) {
    cab k;
    memcpy(k.st, st, sizeof(k.st));
    k.bits = 0;
    k.w = NULL;
    mb_bins(&k, X, code, mbx, mby);
    return (double)ssd_mb(D, mbx, mby) + lam2 * ((double)k.bits / 256.0);
}

/* decide_rd, enc/frame.rs:1462-1513: P_Skip, the best inter partitioning (and with the 8x8 transform when no
 * 8x8 block is split), Intra16x16, Intra4x4 and Intra8x8, each coded, the one of least rate-distortion cost
 * kept (strict '<', first wins) with its reconstruction. inter NULL: an I slice. */
static void decide_rd(const dctx* D, const cabx* X, const uint8_t st[1024], int mbx, int mby, int i16, const ironav_mbresult* inter,
                      ironav_mbcode* out) {
    const struct ironav_ctx* c = D->f->c;
    /* larger than the usual 0.85 * 2^((qp - 12) / 3): the residual decisions are not RD optimised */
    double lam2 = 1.6 * pow(2.0, ((double)c->qpp - 12.0) / 3.0);
    double bj = 0.0;
    int have = 0;
    uint16_t brec[384];
    ironav_mbcode code;
#define KEEP(j)                                  \
    do {                                         \
        double j_ = (j);                         \
        if (!have || j_ < bj) {                  \
            have = 1;                            \
            bj = j_;                             \
            *out = code;                         \
            save_mb(D, mbx, mby, brec);          \
        }                                        \
    } while (0)
    if (inter) {
        int sv[2];
        skip_mv(D->f, mbx, mby, sv);
        code_new(&code, KIND_INTER);
        code.skip = 1;
        for (int i = 0; i < 16; i++) code.mvs[i][0] = (int16_t)sv[0], code.mvs[i][1] = (int16_t)sv[1];
        ironav_interdec d;
        memset(&d, 0, sizeof(d));
        d.mode = 1; /* put_inter_pred, 1391-1394: the prediction is the reconstruction */
        memcpy(d.mvs, code.mvs, sizeof(d.mvs));
        q_code_inter(c, mbx, mby, D->qp_y, &d, &code.res, D->rec, c->pw, c->mb_w * 8);
        KEEP(rd_cost(D, X, st, &code, mbx, mby, lam2));
        const int16_t(*mvs)[2] = (const int16_t(*)[2])inter->mvs;
        d_code_inter(D, mbx, mby, inter->part, inter->sub, inter->refs, mvs, 0, &code);
        /* with nothing coded and the skip vector, this is P_Skip at a higher price */
        if (!(code.res.cbp == 0 && inter->part == 0 && mvs[0][0] == sv[0] && mvs[0][1] == sv[1] && inter->refs[0] == 0))
            KEEP(rd_cost(D, X, st, &code, mbx, mby, lam2));
        /* the 8x8 transform needs every 8x8 block of P_8x8 to be a single 8x8 partition */
        if (c->t8 && !(inter->sub[0] | inter->sub[1] | inter->sub[2] | inter->sub[3])) {
            d_code_inter(D, mbx, mby, inter->part, inter->sub, inter->refs, mvs, 1, &code);
            if (code.res.t8x8) KEEP(rd_cost(D, X, st, &code, mbx, mby, lam2)); /* else the 4x4 candidate again */
        }
    }
    code_i16(D, mbx, mby, i16, &code);
    code_intra_chroma(D, mbx, mby, &code);
    KEEP(rd_cost(D, X, st, &code, mbx, mby, lam2));
    /* Intra4x4 predicts from its own reconstruction, block by block, so it can overwrite the others' */
    code_i4(D, mbx, mby, &code);
    code_intra_chroma(D, mbx, mby, &code);
    KEEP(rd_cost(D, X, st, &code, mbx, mby, lam2));
    if (c->t8) {
        code_i8(D, mbx, mby, &code);
        code_intra_chroma(D, mbx, mby, &code);
        KEEP(rd_cost(D, X, st, &code, mbx, mby, lam2));
    }
#undef KEEP
    restore_mb(D, mbx, mby, brec);
}

/* One slice band under CABAC, in raster order (FrameCoder::encode, enc/frame.rs:461-478): code_mb (its P_Skip
 * tests, best_i16 and best_inter, then decide_rd, 715-760) against the contexts the macroblocks before it
 * left, then those contexts carried past its bins as write_mb_cabac moves them. */
static void decide_band_cabac(const dctx* D, int row0, int row1) {
    const struct ironav_ctx* c = D->f->c;
    cab live;
    memset(&live, 0, sizeof(live));
    int qp_y = c->qpp - 6 * (c->bd - 8);
    cab_states(live.st, c->intra_pic, 0, qp_y);
    cabx X = {c, D->codes, row0, !c->intra_pic, c->t8, c->intra_pic ? 0 : c->nact};
    ironav_mbstate* states = (ironav_mbstate*)D->f->states;
    for (int mby = row0; mby < row1; mby++)
        for (int mbx = 0; mbx < c->mb_w; mbx++) {
            size_t i = (size_t)mby * c->mb_w + mbx;
            ironav_mbcode* code = &D->codes[i];
            int sv[2], done = 0;
            if (!c->intra_pic) done = skip_tests(D, mbx, mby, sv, code);
            if (!done) {
                int i16m, i16c;
                best_i16(D, mbx, mby, &i16m, &i16c);
                ironav_mbresult r;
                memset(&r, 0, sizeof(r));
                if (!c->intra_pic) {
                    counters cnt = {0, 0};
                    best_inter(D->f, &cnt, mbx, mby, &r);
                }
                decide_rd(D, &X, live.st, mbx, mby, i16m, c->intra_pic ? NULL : &r, code);
            }
            d_state(code, &states[i]);
            mb_bins(&live, &X, code, mbx, mby);
        }
}

/* A slice band's data under CABAC (FrameCoder::encode, enc/frame.rs:461-486): cabac_alignment_one_bit, the
 * contexts of the slice, each macroblock's bins (write_mb_cabac, 2020-2025) and end_of_slice_flag, the last
 * byte padded with zeros (into_bytes, enc/bitw.rs:60-67). */
static void write_band_cabac(const struct ironav_ctx* c, const ironav_mbcode* codes, int row0, int row1, bitw* w) {
    if (w->n > 0) bw_put(w, 8 - w->n, (1u << (8 - w->n)) - 1); /* align_ones, enc/bitw.rs:52-58 */
    cab k;
    memset(&k, 0, sizeof(k));
    k.w = w;
    k.range = 510;
    k.first = 1;
    cab_states(k.st, c->intra_pic, 0, c->qpp - 6 * (c->bd - 8));
    cabx X = {c, codes, row0, !c->intra_pic, c->t8, c->intra_pic ? 0 : c->nact};
    for (int mby = row0; mby < row1; mby++)
        for (int mbx = 0; mbx < c->mb_w; mbx++) {
            mb_bins(&k, &X, &codes[(size_t)mby * c->mb_w + mbx], mbx, mby);
            cab_terminate(&k, mby + 1 == row1 && mbx + 1 == c->mb_w);
        }
    if (w->n > 0) bw_put(w, 8 - w->n, 0);
}

/* Test hook (oracle only): the arithmetic coder on a list of bins, as the reference's coder test drives it
 * (bins_read_back_through_the_decoder, enc/cabac.rs:252-291): 5 header bits 10110 and cabac_alignment_one_bit,
 * the contexts of a slice (intra, idc, qp), then per op a decision (kind 0, context ctx[i]), a bypass (1) or a
 * terminating 0 (2), then a terminating 1 and the padded last byte. Returns the byte count, or -1 when cap is
 * too small. */
int oracle_cabac_ops(const int* kind, const int* ctx, const int* val, int n, int intra, int idc, int qp, uint8_t* out, int cap) {
    bitw w;
    bw_init(&w);
    bw_put(&w, 5, 0x16);
    if (w.n > 0) bw_put(&w, 8 - w.n, (1u << (8 - w.n)) - 1);
    cab k;
    memset(&k, 0, sizeof(k));
    k.w = &w;
    k.range = 510;
    k.first = 1;
    cab_states(k.st, intra, idc, qp);
    for (int i = 0; i < n; i++) {
        if (kind[i] == 0) cab_decision(&k, ctx[i], val[i]);
        else if (kind[i] == 1) cab_bypass(&k, val[i]);
        else cab_terminate(&k, 0);
    }
    cab_terminate(&k, 1);
    if (w.n > 0) bw_put(&w, 8 - w.n, 0);
    int len = (int)w.len;
    if (len <= cap) memcpy(out, w.buf, w.len);
    free(w.buf);
    return len <= cap ? len : -1;
}

/* Test hook (oracle only): the bits, in 1/256, the counter gives the same ops from the same contexts */
uint32_t oracle_cabac_cost(const int* kind, const int* ctx, const int* val, int n, int intra, int idc, int qp) {
    cab k;
    memset(&k, 0, sizeof(k));
    cab_states(k.st, intra, idc, qp);
    for (int i = 0; i < n; i++) {
        if (kind[i] == 0) cab_decision(&k, ctx[i], val[i]);
        else if (kind[i] == 1) cab_bypass(&k, val[i]);
        else cab_terminate(&k, 0);
    }
    return k.bits;
}
