// cabac.cuh — CABAC on the device: the contexts of a slice, and one macroblock's bins (mb_bins,
// enc/frame.rs:2028-2279, with write_block, enc/cabac.rs:194-250, and mvd_bins, enc/frame.rs:2393-2414) given
// to a sink that is either the bit counter (CabacCost, enc/cabac.rs:150-192) or the arithmetic coder
// (CabacWriter, enc/cabac.rs:42-147). A macroblock's bins are a serial walk, so one lane runs it; several
// lanes can each count another candidate's bins from their own copy of the contexts.
//
// The walk reads the macroblock's code and what the contexts need of its left and top neighbours in the
// slice (Nb, the CABAC fields of MbState, enc/frame.rs:245-272). Only I and P slices are coded here.
#pragma once
#include <stdint.h>

#include "../../include/ironav_inter.h"
#include "cabac_tables.cuh"

namespace ironav {

namespace cab {

constexpr int KIND_I4 = 1, KIND_I8 = 2, KIND_I16 = 3, KIND_INTER = 5;  // Kind, h264/mb.rs:21-30

// The contexts' step table: for state s = pStateIdx * 2 + valMPS and bin b, entry [s * 2 + b] = the next
// state (next_state, enc/cabac.rs:32-40) | the bin's cost in 1/256 bits << 8 (entropy(), enc/cabac.rs:162-173,
// computed on the host with the reference's f64 formula and copied to the kernel's shared memory).
constexpr int STEP_ENTRIES = 256;

// The contexts of a slice (CabacWriter::new, enc/cabac.rs:54-64; 9.3.1.1): lanes share the 1024 entries.
__device__ __forceinline__ void init_states(uint8_t* st, bool intra, int idc, int slice_qp, int lane, int nlanes) {
    const int qp = min(max(slice_qp, 0), 51);
    for (int i = lane; i < 1024; i += nlanes) {
        const int m = intra ? CABAC_INIT_I[i][0] : CABAC_INIT_PB[idc][i][0];
        const int n = intra ? CABAC_INIT_I[i][1] : CABAC_INIT_PB[idc][i][1];
        const int pre = min(max(((m * qp) >> 4) + n, 1), 126);
        st[i] = (uint8_t)(pre <= 63 ? (63 - pre) << 1 : ((pre - 64) << 1) | 1);
    }
}

// The bit counter over its own copy of the contexts.
struct Counter {
    uint8_t* st;
    const uint32_t* step;
    uint32_t bits;
    __device__ __forceinline__ void decision(int ctx, int bin) {
        const uint32_t e = step[st[ctx] * 2 + (bin != 0)];
        st[ctx] = (uint8_t)e;
        bits += e >> 8;
    }
    __device__ __forceinline__ void bypass(int) { bits += 256; }
    __device__ __forceinline__ void terminate(int bin) { bits += bin ? 7 * 256 : 1; }
};

// Bits MSB first into 32-bit words of a region in global memory, stored so that the bytes read in order
// (BitWriter, enc/bitw.rs:4-25). A write beyond the region sets `over` and is dropped.
struct BitOut {
    uint32_t* words;
    uint32_t cap;  // words
    uint32_t nw;
    uint64_t cur;
    int n;
    bool over;
    __device__ __forceinline__ void put(int k, uint32_t v) {  // k <= 32
        cur = (cur << k) | (uint64_t)v;
        n += k;
        if (n >= 32) {
            n -= 32;
            const uint32_t w = (uint32_t)(cur >> n);
            if (nw < cap) words[nw] = __byte_perm(w, 0, 0x0123);
            else over = true;
            nw++;
            cur &= n ? ((1ull << n) - 1) : 0ull;
        }
    }
    // the last word padded with zeros to its byte (into_bytes, enc/bitw.rs:60-67); returns the byte count
    __device__ __forceinline__ uint32_t finish() {
        uint32_t bytes = nw * 4;
        if (n > 0) {
            const int nb = (n + 7) >> 3;
            const uint32_t w = (uint32_t)(cur << (32 - n));
            if (nw < cap) words[nw] = __byte_perm(w, 0, 0x0123);
            else over = true;
            bytes += nb;
        }
        return bytes;
    }
};

// The arithmetic coder (9.3.4.2-9.3.4.5) over its contexts.
struct Coder {
    uint8_t* st;
    const uint32_t* step;
    BitOut* out;
    uint32_t low, range, outstanding;
    bool first;
    __device__ __forceinline__ void put_bit(uint32_t b) {
        if (first) first = false;
        else out->put(1, b);
        while (outstanding > 0) {
            const int k = outstanding < 32 ? (int)outstanding : 32;
            out->put(k, b ? 0u : (k == 32 ? 0xFFFFFFFFu : (1u << k) - 1));
            outstanding -= k;
        }
    }
    __device__ __forceinline__ void renorm() {
        while (range < 256) {
            if (low < 256) put_bit(0);
            else if (low >= 512) {
                low -= 512;
                put_bit(1);
            } else {
                low -= 256;
                outstanding++;
            }
            range <<= 1;
            low <<= 1;
        }
    }
    __device__ __forceinline__ void decision(int ctx, int bin) {
        const int s = st[ctx], p = s >> 1, mps = s & 1;
        bin = bin != 0;
        const uint32_t lps = LPS_RANGE[p][(range >> 6) & 3];
        range -= lps;
        if (bin != mps) {
            low += range;
            range = lps;
        }
        st[ctx] = (uint8_t)step[s * 2 + bin];
        renorm();
    }
    __device__ __forceinline__ void bypass(int bin) {
        low <<= 1;
        if (bin) low += range;
        if (low >= 1024) {
            put_bit(1);
            low -= 1024;
        } else if (low < 512) {
            put_bit(0);
        } else {
            low -= 512;
            outstanding++;
        }
    }
    __device__ __forceinline__ void terminate(int bin) {
        range -= 2;
        if (bin) {
            low += range;
            range = 2;
            renorm();
            put_bit((low >> 9) & 1);
            out->put(2, ((low >> 7) & 3) | 1);  // the last of the two bits is the rbsp_stop_one_bit
        } else {
            renorm();
        }
    }
};

// What the contexts read of a neighbouring macroblock (finish_mb's MbState fields, enc/frame.rs:2281-2321).
struct Nb {
    uint8_t avail, skip, kind, inter, cbp, t8x8, chroma_mode, cbf_dc;
    int8_t r8[4];        // list 0 reference index per 8x8 block (-1: intra)
    uint8_t mvd[16][2];  // absolute vector differences per 4x4 block, capped at 64 (mvd_grid, enc/frame.rs:238-241)
    uint8_t nnz[16];
    uint8_t cnnz[2][4];
};

__device__ __forceinline__ int rects_d(int part, const uint8_t* sub, int4* r) {
    if (part == 0) {
        r[0] = make_int4(0, 0, 4, 4);
        return 1;
    }
    if (part == 1) {
        r[0] = make_int4(0, 0, 4, 2);
        r[1] = make_int4(0, 2, 4, 2);
        return 2;
    }
    if (part == 2) {
        r[0] = make_int4(0, 0, 2, 4);
        r[1] = make_int4(2, 0, 2, 4);
        return 2;
    }
    int n = 0;
    for (int k = 0; k < 4; k++) {
        const int ox = (k & 1) * 2, oy = (k >> 1) * 2, s = sub[k];
        if (s == 0) r[n++] = make_int4(ox, oy, 2, 2);
        else if (s == 1) {
            r[n++] = make_int4(ox, oy, 2, 1);
            r[n++] = make_int4(ox, oy + 1, 2, 1);
        } else if (s == 2) {
            r[n++] = make_int4(ox, oy, 1, 2);
            r[n++] = make_int4(ox + 1, oy, 1, 2);
        } else {
            for (int q = 0; q < 4; q++) r[n++] = make_int4(ox + (q & 1), oy + (q >> 1), 1, 1);
        }
    }
    return n;
}

// The absolute vector differences of an inter, not skipped, macroblock per 4x4 block (mvd_grid).
__device__ __forceinline__ void mvd_grid(const ironav_mbcode* k, uint8_t (*g)[2]) {
    for (int i = 0; i < 16; i++) g[i][0] = g[i][1] = 0;
    if (k->kind != KIND_INTER || k->skip) return;
    int4 rs[16];
    const int nr = rects_d(k->part, k->sub, rs);
    for (int q = 0; q < nr; q++) {
        const uint8_t ax = (uint8_t)min(abs((int)k->mvds[q][0]), 64), ay = (uint8_t)min(abs((int)k->mvds[q][1]), 64);
        for (int by = rs[q].y; by < rs[q].y + rs[q].w; by++)
            for (int bx = rs[q].x; bx < rs[q].x + rs[q].z; bx++) {
                g[by * 4 + bx][0] = ax;
                g[by * 4 + bx][1] = ay;
            }
    }
}

// A neighbour's Nb from its code (one lane).
__device__ __forceinline__ void nb_of(const ironav_mbcode* k, Nb* n) {
    n->avail = 1;
    n->skip = k->skip;
    n->kind = k->kind;
    n->inter = k->kind == KIND_INTER;
    n->cbp = k->res.cbp;
    n->t8x8 = k->res.t8x8;
    n->chroma_mode = n->inter ? 0 : k->chroma_mode;
    const int cbpc = k->res.cbp >> 4;
    int any0 = 0, any1 = 0, any2 = 0;
    for (int i = 0; i < 16; i++) any0 |= k->dc[i] != 0;
    for (int i = 0; i < 4; i++) any1 |= k->res.cdc[0][i] != 0, any2 |= k->res.cdc[1][i] != 0;
    n->cbf_dc = (uint8_t)((k->kind == KIND_I16 && any0) | ((cbpc > 0 && any1) << 1) | ((cbpc > 0 && any2) << 2));
    for (int i = 0; i < 16; i++) n->nnz[i] = k->res.nnz[i];
    for (int c = 0; c < 2; c++)
        for (int i = 0; i < 4; i++) n->cnnz[c][i] = k->res.cnnz[c][i];
    for (int b8 = 0; b8 < 4; b8++)
        n->r8[b8] = n->inter ? (int8_t)k->refs[k->part == 0 ? 0 : k->part == 1 ? b8 >> 1 : k->part == 2 ? (b8 & 1) : b8] : (int8_t)-1;
    mvd_grid(k, n->mvd);
}

// The partition (rects order) that holds 4x4 block (bx, by) of a P macroblock.
__device__ __forceinline__ int part_index(int part, const uint8_t* sub, int bx, int by) {
    if (part == 0) return 0;
    if (part == 1) return by >> 1;
    if (part == 2) return bx >> 1;
    const int k = (by >> 1) * 2 + (bx >> 1);
    int n = 0;
    for (int q = 0; q < k; q++) n += sub[q] == 0 ? 1 : (sub[q] == 3 ? 4 : 2);
    const int s = sub[k];
    return n + (s == 0 ? 0 : s == 1 ? (by & 1) : s == 2 ? (bx & 1) : (by & 1) * 2 + (bx & 1));
}

constexpr int NB_WORDS = (int)(sizeof(Nb) / 4);
static_assert(sizeof(Nb) % 4 == 0, "Nb in whole words");

// nb_of with the warp: every lane calls; the code in shared or global memory.
__device__ __forceinline__ void nb_of_warp(const ironav_mbcode* k, Nb* n) {
    const int lane = threadIdx.x & 31;
    const int kind = k->kind, skip = k->skip, cbp = k->res.cbp;
    const bool inter = kind == KIND_INTER;
    bool nz = false;
    if (lane < 16) nz = k->dc[lane] != 0;
    else if (lane < 24) nz = k->res.cdc[(lane - 16) >> 2][(lane - 16) & 3] != 0;
    const unsigned bal = __ballot_sync(0xffffffffu, nz);
    if (lane < 16) {
        n->nnz[lane] = k->res.nnz[lane];
        uint8_t ax = 0, ay = 0;
        if (inter && !skip) {
            const int q = part_index(k->part, k->sub, lane & 3, lane >> 2);
            ax = (uint8_t)min(abs((int)k->mvds[q][0]), 64);
            ay = (uint8_t)min(abs((int)k->mvds[q][1]), 64);
        }
        n->mvd[lane][0] = ax;
        n->mvd[lane][1] = ay;
    } else if (lane < 24) {
        n->cnnz[(lane - 16) >> 2][(lane - 16) & 3] = k->res.cnnz[(lane - 16) >> 2][(lane - 16) & 3];
    } else if (lane < 28) {
        const int b8 = lane - 24;
        n->r8[b8] = inter ? (int8_t)k->refs[k->part == 0 ? 0 : k->part == 1 ? b8 >> 1 : k->part == 2 ? (b8 & 1) : b8] : (int8_t)-1;
    } else if (lane == 28) {
        const int cbpc = cbp >> 4;
        n->avail = 1;
        n->skip = (uint8_t)skip;
        n->kind = (uint8_t)kind;
        n->inter = inter;
        n->cbp = (uint8_t)cbp;
        n->t8x8 = k->res.t8x8;
        n->chroma_mode = inter ? 0 : k->chroma_mode;
        n->cbf_dc = (uint8_t)((kind == KIND_I16 && (bal & 0xFFFFu)) | ((cbpc > 0 && (bal & 0xF0000u)) << 1) | ((cbpc > 0 && (bal & 0xF00000u)) << 2));
    }
    __syncwarp();
}

__device__ __forceinline__ bool nxn(int kind) { return kind == KIND_I4 || kind == KIND_I8; }

// pred_i4_mode, enc/frame.rs:619-627, with the neighbours' modes in nbm (left column then top row: a mode, 2
// for a macroblock that is neither Intra4x4 nor Intra8x8, -1 unavailable).
__device__ __forceinline__ int pred_mode(const int* nbm, const uint8_t* cur, int bx, int by) {
    const int a = bx > 0 ? cur[by * 4 + bx - 1] : nbm[by];
    const int b = by > 0 ? cur[(by - 1) * 4 + bx] : nbm[4 + bx];
    return (a >= 0 && b >= 0) ? min(a, b) : 2;
}

// write_block, enc/cabac.rs:194-250: coded_block_flag (context cbf, none when < 0) and max levels of
// category cat in scan order; part 0 all of it, 1 its significance map (coded_block_flag,
// significant_coeff_flag, last_significant_coeff_flag), 2 its levels (coeff_abs_level_minus1 and the signs):
// the two parts' contexts are disjoint.
template <class S>
__device__ __forceinline__ void block(S& c, int cat, int cbf, const int16_t* lv, int max, int part = 0) {
    int last = -1;
    for (int i = 0; i < max; i++)
        if (lv[i]) last = i;
    if (cbf >= 0 && part != 2) c.decision(cbf, last >= 0);
    if (last < 0) return;
    if (part != 2) {
        const int so = SIG_OFF[0][cat], lo = LAST_OFF[0][cat];
        for (int i = 0; i < max - 1; i++) {
            // 4:2:0 chroma DC has three significance contexts, one per position; 8x8 blocks share theirs
            const int sig = cat == 3 ? min(i, 2) : cat == 5 ? SIG_OFF_8X8[0][i] : i;
            const int lst = cat == 3 ? min(i, 2) : cat == 5 ? LAST_OFF_8X8[i] : i;
            c.decision(so + sig, lv[i] != 0);
            if (lv[i]) {
                c.decision(lo + lst, i == last);
                if (i == last) break;
            }
        }
    }
    if (part == 1) return;
    const int base = ABS_OFF[cat];
    int eq1 = 0, gt1 = 0;
    for (int i = last; i >= 0; i--) {
        const int l = lv[i];
        if (!l) continue;
        const uint32_t a = (uint32_t)abs(l);
        const int inc0 = gt1 ? 0 : min(1 + eq1, 4);
        if (a == 1) {
            c.decision(base + inc0, 0);
            eq1++;
        } else {
            c.decision(base + inc0, 1);
            const int incn = base + 5 + min(gt1, 4 - (cat == 3));
            // abs - 2 ones and a zero, the ones capped at 13 with the rest in an Exp-Golomb suffix
            const uint32_t ones = a - 2 < 13 ? a - 2 : 13;
            for (uint32_t k = 0; k < ones; k++) c.decision(incn, 1);
            if (a < 15) c.decision(incn, 0);
            else {
                uint32_t v = a - 15, k = 0;  // exp_golomb(abs - 15, 0), enc/cabac.rs:17-29
                while (v >= (1u << k)) {
                    c.bypass(1);
                    v -= 1u << k;
                    k++;
                }
                c.bypass(0);
                while (k > 0) {
                    k--;
                    c.bypass((v >> k) & 1);
                }
            }
            gt1++;
        }
        c.bypass(l < 0);
    }
}

// mvd_bins, enc/frame.rs:2393-2414
template <class S>
__device__ __forceinline__ void mvd(S& c, int comp, int d, uint32_t sum) {
    const int base = comp == 0 ? 40 : 47, inc = sum < 3 ? 0 : sum > 32 ? 2 : 1;
    const uint32_t a = (uint32_t)abs(d);
    c.decision(base + inc, a > 0);
    if (a == 0) return;
    int ctx = base + 3;
    for (uint32_t k = 1; k < (a < 9 ? a : 9); k++) {
        c.decision(ctx, 1);
        if (ctx < base + 6) ctx++;
    }
    if (a < 9) c.decision(ctx, 0);
    else {
        uint32_t v = a - 9, k = 3;
        while (v >= (1u << k)) {
            c.bypass(1);
            v -= 1u << k;
            k++;
        }
        c.bypass(0);
        while (k > 0) {
            k--;
            c.bypass((v >> k) & 1);
        }
    }
    c.bypass(d < 0);
}

// The slice's parameters the walk reads.
struct Slice {
    int p_slice, t8, nref;
};

// The bins of a macroblock fall in groups whose contexts are disjoint: its syntax up to mb_qp_delta
// (contexts below 85, and 399-401), and the residual blocks of each category with their coded_block_flag
// (Intra16x16 DC; the luma blocks, 4x4 or 8x8; chroma DC; chroma AC: contexts 85-104 by category, 105 and
// up by category). So the bits of a macroblock are the sum of the groups' bits, each group walked on its
// own from the same contexts, and the contexts after it are the union of the groups' updates.
// Each category's significance map and levels use disjoint contexts too, so a category is two groups.
enum Group { ALL = -1, HEAD = 0, DC16_MAP, DC16_LEV, LUMA_MAP, LUMA_LEV, CDC_MAP, CDC_LEV, CAC_MAP, CAC_LEV, NGROUPS };

// The groups of a residual category: whether `group` walks it, and which part of its blocks.
__device__ __forceinline__ bool in_group(int group, int map_group, int* part) {
    if (group == ALL) {
        *part = 0;
        return true;
    }
    *part = group == map_group ? 1 : 2;
    return group == map_group || group == map_group + 1;
}

// mb_bins' HEAD group after mb_skip_flag (enc/frame.rs:2046-2244): mb_type, the prediction modes,
// sub_mb_type, ref_idx, mvd, coded_block_pattern, transform_size_8x8_flag and mb_qp_delta.
template <class S>
__device__ __forceinline__ void head_bins(S& c, const Slice& sl, const ironav_mbcode* code, const Nb& L, const Nb& T, const int* nbm) {
    const bool la = L.avail, ta = T.avail;
    const int kind = code->kind, cbp = code->res.cbp, cbpl = cbp & 15, cbpc = cbp >> 4;
    // mb_type
    if (kind == KIND_INTER) {
        // P_L0_16x16 000, P_L0_L0_16x8 011, P_L0_L0_8x16 010, P_8x8 001
        const int b1 = code->part == 1 || code->part == 2, b2 = code->part == 1 || code->part == 3;
        c.decision(14, 0);
        c.decision(15, b1);
        c.decision(b1 ? 17 : 16, b2);
    } else {
        const int pre = sl.p_slice, base = pre ? 17 : 3;
        int first;
        if (pre) {
            c.decision(14, 1);
            first = 17;
        } else {
            first = 3 + (la && !nxn(L.kind)) + (ta && !nxn(T.kind));
        }
        if (nxn(kind)) {
            c.decision(first, 0);
            if (sl.t8) c.decision(399 + (la && L.t8x8) + (ta && T.t8x8), kind == KIND_I8);
        } else {
            c.decision(first, 1);
            c.terminate(0);  // not I_PCM
            c.decision(pre ? base + 1 : base + 3, cbpl != 0);
            c.decision(pre ? base + 2 : base + 4, cbpc != 0);
            if (cbpc) c.decision(pre ? base + 2 : base + 5, cbpc == 2);
            c.decision(pre ? base + 3 : base + 6, (code->i16_mode >> 1) == 1);
            c.decision(pre ? base + 3 : base + 7, code->i16_mode & 1);
        }
    }
    if (nxn(kind)) {
        const bool t8 = kind == KIND_I8;
        uint8_t so_far[16];
        for (int i = 0; i < 16; i++) so_far[i] = 2;
        for (int n = 0; n < (t8 ? 4 : 16); n++) {
            const int bx = t8 ? (n & 1) * 2 : ((n >> 2) & 1) * 2 + (n & 1);
            const int by = t8 ? (n >> 1) * 2 : ((n >> 3) & 1) * 2 + ((n >> 1) & 1);
            const int mode = code->modes[by * 4 + bx];
            const int pred = pred_mode(nbm, so_far, bx, by);
            so_far[by * 4 + bx] = (uint8_t)mode;
            if (t8) so_far[by * 4 + bx + 1] = so_far[(by + 1) * 4 + bx] = so_far[(by + 1) * 4 + bx + 1] = (uint8_t)mode;
            c.decision(68, mode == pred);
            if (mode != pred) {
                const int rem = mode < pred ? mode : mode - 1;
                for (int k = 0; k < 3; k++) c.decision(69, (rem >> k) & 1);
            }
        }
    }
    if (kind != KIND_INTER) {
        const int m = code->chroma_mode;
        c.decision(64 + (la && !L.inter && L.chroma_mode != 0) + (ta && !T.inter && T.chroma_mode != 0), m > 0);
        if (m > 0) {
            c.decision(67, m > 1);
            if (m > 1) c.decision(67, m > 2);
        }
    } else {
        // sub_mb_type of each 8x8 block of P_8x8 (Table 9-38: 1, 00, 011, 010; contexts 21 to 23)
        if (code->part == 3)
            for (int k = 0; k < 4; k++) {
                const int s = code->sub[k];
                c.decision(21, s == 0);
                if (s != 0) {
                    c.decision(22, s != 1);
                    if (s != 1) c.decision(23, s == 2);
                }
            }
        // ref_idx_l0 per partition (per 8x8 block for P_8x8), unary, with the contexts of 9.3.3.1.1.6
        if (sl.nref > 1) {
            uint8_t grid[4] = {0, 0, 0, 0};
            const int np = code->part == 0 ? 1 : code->part == 3 ? 4 : 2;
            for (int k = 0; k < np; k++) {
                int bx, by, w, h;
                if (code->part == 0) bx = 0, by = 0, w = 4, h = 4;
                else if (code->part == 1) bx = 0, by = 2 * k, w = 4, h = 2;
                else if (code->part == 2) bx = 2 * k, by = 0, w = 2, h = 4;
                else bx = (k & 1) * 2, by = (k >> 1) * 2, w = 2, h = 2;
                const int a = bx > 0 ? grid[(by / 2) * 2 + (bx - 1) / 2] > 0 : (la && L.r8[(by / 2) * 2 + 1] > 0);
                const int b = by > 0 ? grid[((by - 1) / 2) * 2 + bx / 2] > 0 : (ta && T.r8[2 + bx / 2] > 0);
                const int r = code->refs[k], base = 54 + a + 2 * b;
                for (int i = 0; i <= r; i++) c.decision(i == 0 ? base : i == 1 ? 58 : 59, i < r);
                for (int y8 = by / 2; y8 <= (by + h - 1) / 2; y8++)
                    for (int x8 = bx / 2; x8 <= (bx + w - 1) / 2; x8++) grid[y8 * 2 + x8] = code->refs[k];
            }
        }
        // mvd_l0 per partition; the blocks left of and above a partition in the macroblock belong to earlier ones
        uint8_t g[16][2];
        mvd_grid(code, g);
        int4 rs[16];
        const int nr = rects_d(code->part, code->sub, rs);
        for (int k = 0; k < nr; k++) {
            const int bx = rs[k].x, by = rs[k].y;
            for (int comp = 0; comp < 2; comp++) {
                const uint32_t a = bx > 0 ? g[by * 4 + bx - 1][comp] : (la ? L.mvd[by * 4 + 3][comp] : 0);
                const uint32_t b = by > 0 ? g[(by - 1) * 4 + bx][comp] : (ta ? T.mvd[12 + bx][comp] : 0);
                mvd(c, comp, code->mvds[k][comp], a + b);
            }
        }
    }
    if (kind != KIND_I16) {
        int luma = 0;
        for (int b8 = 0; b8 < 4; b8++) {
            const int ca = (b8 & 1) ? ((luma >> (b8 - 1)) & 1) == 0 : (la && ((L.cbp >> (b8 + 1)) & 1) == 0);
            const int cb = b8 >= 2 ? ((luma >> (b8 - 2)) & 1) == 0 : (ta && ((T.cbp >> (b8 + 2)) & 1) == 0);
            const int bit = (cbpl >> b8) & 1;
            c.decision(73 + ca + 2 * cb, bit);
            luma |= bit << b8;
        }
        c.decision(77 + (la && (L.cbp >> 4) != 0) + 2 * (ta && (T.cbp >> 4) != 0), cbpc != 0);
        if (cbpc) c.decision(81 + (la && (L.cbp >> 4) == 2) + 2 * (ta && (T.cbp >> 4) == 2), cbpc == 2);
    }
    // transform_size_8x8_flag is absent from P_8x8 with any sub-partition smaller than 8x8
    if (kind == KIND_INTER && sl.t8 && cbpl && (code->part != 3 || !(code->sub[0] | code->sub[1] | code->sub[2] | code->sub[3])))
        c.decision(399 + (la && L.t8x8) + (ta && T.t8x8), code->res.t8x8);
    if (!cbp && kind != KIND_I16) return;
    c.decision(60, 0);  // mb_qp_delta 0, after a macroblock without a change
}

// mb_bins, enc/frame.rs:2028-2279, for I and P slices: the bins of the macroblock `code` up to
// end_of_slice_flag (all of them, or one group's); l and t its left and top neighbours (avail 0: not in
// the slice), nbm their Intra NxN modes as pred_mode reads them.
template <class S>
__device__ __forceinline__ void mb_bins(S& c, const Slice& sl, const ironav_mbcode* code, const Nb& L, const Nb& T, const int* nbm, int group = ALL) {
    const bool la = L.avail, ta = T.avail;
    if (sl.p_slice) {
        if (group == ALL || group == HEAD) c.decision(11 + (la && !L.skip) + (ta && !T.skip), code->skip);
        if (code->skip) return;
    }
    if (group == ALL || group == HEAD) head_bins(c, sl, code, L, T, nbm);
    const int kind = code->kind, cbp = code->res.cbp, cbpl = cbp & 15, cbpc = cbp >> 4;
    if (!cbp && kind != KIND_I16) return;
    // an unavailable neighbour counts as a coded block for an intra macroblock
    const int un = kind != KIND_INTER;
    int part;
    if (kind == KIND_I16 && in_group(group, DC16_MAP, &part))
        block(c, 0, 85 + (la ? (L.cbf_dc & 1) != 0 : un) + 2 * (ta ? (T.cbf_dc & 1) != 0 : un), code->dc, 16, part);
    const int cat = kind == KIND_I16 ? 1 : 2, base = kind == KIND_I16 ? 89 : 93;
    const bool luma = in_group(group, LUMA_MAP, &part);
    if (code->res.t8x8 && luma) {
        for (int i8 = 0; i8 < 4; i8++)
            if (cbpl & (1 << i8)) block(c, 5, -1, code->res.luma8[i8], 64, part);
    } else if (luma) {
        for (int n = 0; n < 16; n++) {
            if (!(cbpl & (1 << (n >> 2)))) continue;
            const int bx = ((n >> 2) & 1) * 2 + (n & 1), by = ((n >> 3) & 1) * 2 + ((n >> 1) & 1);
            const int fa = bx > 0 ? code->res.nnz[by * 4 + bx - 1] > 0 : (la ? L.nnz[by * 4 + 3] > 0 : un);
            const int fb = by > 0 ? code->res.nnz[(by - 1) * 4 + bx] > 0 : (ta ? T.nnz[12 + bx] > 0 : un);
            const int16_t* blk = code->res.luma[by * 4 + bx];
            block(c, cat, base + fa + 2 * fb, cat == 1 ? blk + 1 : blk, cat == 1 ? 15 : 16, part);
        }
    }
    if (cbpc > 0 && in_group(group, CDC_MAP, &part))
        for (int comp = 0; comp < 2; comp++) {
            const int m = 2 << comp;
            block(c, 3, 97 + (la ? (L.cbf_dc & m) != 0 : un) + 2 * (ta ? (T.cbf_dc & m) != 0 : un), code->res.cdc[comp], 4, part);
        }
    if (cbpc == 2 && in_group(group, CAC_MAP, &part))
        for (int comp = 0; comp < 2; comp++)
            for (int blk = 0; blk < 4; blk++) {
                const int bx = blk & 1, by = blk >> 1;
                const uint8_t* cur = code->res.cnnz[comp];
                const int fa = bx > 0 ? cur[by * 2] > 0 : (la ? L.cnnz[comp][by * 2 + 1] > 0 : un);
                const int fb = by > 0 ? cur[bx] > 0 : (ta ? T.cnnz[comp][2 + bx] > 0 : un);
                block(c, 4, 101 + fa + 2 * fb, code->res.cac[comp][blk] + 1, 15, part);
            }
}

}  // namespace cab

}  // namespace ironav
