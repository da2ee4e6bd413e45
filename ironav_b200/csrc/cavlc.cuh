// cavlc.cuh — the CAVLC slice writer on the device: every macroblock's syntax (write_mb, enc/frame.rs:1922-2016;
// residual blocks by write_block, enc/cavlc.rs:47-122), the slice header (enc/mod.rs:566-600) and the slice's
// trailing bits (enc/frame.rs:480-486), written into one RBSP buffer region per slice.
//
// Three launches:
//   1. cavlc_size_kernel (a warp per macroblock): the macroblock's bits without its mb_skip_run prefix
//      (0 for a skipped macroblock, which codes nothing of its own);
//   2. cavlc_scan_kernel (a CTA per slice): each coded macroblock's skip run (the skipped macroblocks since
//      the previous coded one), its bit offset in the slice (an exclusive scan after the header), the
//      slice's trailing run and size; it clears the slice's bytes and writes the header and the trailer;
//   3. cavlc_write_kernel (a warp per macroblock): the same syntax again, now written at its offset.
// Within a macroblock, lane 0 takes the header part (skip run, mb_type, prediction modes, sub_mb_type,
// ref_idx, mvd, coded_block_pattern, mb_qp_delta) and lanes 1..27 one residual block each (Intra16x16 DC,
// 16 luma 4x4 blocks in decoding order, 2 chroma DC, 8 chroma AC); a warp scan of their lengths places
// each lane's bits. A residual block's nC context reads only coefficient counts, which the codes hold, so
// the blocks are independent. Bits go into the buffer by atomicOr on 32-bit words holding the stream's
// bytes in order (each word byte-swapped from its MSB-first bit order), so lanes and macroblocks that
// share a word need no other ordering.
#pragma once
#include <cstdint>

#include "../../include/ironav_inter.h"
#include "cavlc_tables.cuh"

namespace ironav {

constexpr int CAVLC_KIND_I4 = 1, CAVLC_KIND_I16 = 3;
// The most bits one macroblock's syntax can take: a header of at most ~1.1k bits (sixteen mvd pairs of
// at most 27 bits each, the prediction modes, the types) and 27 residual blocks of at most 734 bits (a
// 16-bit coeff_token, 16 levels of at most 34 bits, total_zeros, 15 run_before codes of at most 11 bits).
constexpr unsigned CAVLC_MB_MAX_BITS = 24576;
constexpr unsigned CAVLC_SLICE_EXTRA_BITS = 2048;  // the slice header and the trailing skip run and bits

// Where a slice's bits go: region words at out + slice * region_words; bit positions count from its start.
struct CavlcParams {
    const ironav_mbcode* codes;
    const int* band_start;     // per macroblock row: the first row of its slice band
    const int* slice_first;    // per slice: its first macroblock (raster), slice_first[nslices] = nmb
    const int* row_slice;      // per macroblock row: its slice
    uint32_t* out;             // RBSP words (bytes in stream order), region_words per slice
    unsigned long long region_words;
    uint32_t* mb_len;          // per macroblock: its bits without the skip-run prefix (pass 1)
    uint32_t* mb_off;          // per macroblock: its bit offset in the slice, the skip-run prefix included
    uint32_t* mb_run;          // per macroblock: the skip run before it (coded macroblocks of a P slice)
    uint32_t* slice_bytes;     // per slice: RBSP bytes (rbsp_trailing_bits included)
    unsigned* err;             // bit 0: a macroblock or slice beyond its bound (nothing written past it)
    int mb_w, mb_h, nmb, nslices;
    int p_slice, nref;         // P slice and its num_ref_idx_active (ref_idx coded when > 1)
    int idr, frame_num, idr_pic_id, slice_qp_delta;
};

// A bit sink: counts (out == nullptr) or ORs bits into the region at absolute bit positions.
struct BitSink {
    uint32_t* out;
    unsigned long long pos;
    unsigned long long limit;  // the region's size in bits
    bool overflow;

    __device__ __forceinline__ void put(unsigned n, uint32_t v) {
        if (n == 0) return;
        if (out) {
            if (pos + n > limit) {
                overflow = true;
            } else {
                const unsigned long long w = pos >> 5;
                const unsigned o = (unsigned)(pos & 31);
                // v's n bits at offset o (from the word's most significant bit)
                const unsigned long long x = (unsigned long long)(v & (n == 32 ? 0xffffffffu : ((1u << n) - 1))) << (64 - o - n);
                const uint32_t hi = (uint32_t)(x >> 32), lo = (uint32_t)x;
                if (hi) atomicOr(&out[w], __byte_perm(hi, 0, 0x0123));
                if (lo) atomicOr(&out[w + 1], __byte_perm(lo, 0, 0x0123));
            }
        }
        pos += n;
    }
    __device__ __forceinline__ void flag(bool b) { put(1, b ? 1u : 0u); }
    // ue(v), enc/bitw.rs:31-40
    __device__ __forceinline__ void ue(uint32_t v) {
        const unsigned long long x = (unsigned long long)v + 1;
        const unsigned len = 64 - __clzll((long long)x);
        if (len > 16) {
            put(len - 1, 0);
            put(len, (uint32_t)x);
        } else {
            put(2 * len - 1, (uint32_t)x);
        }
    }
    // se(v), enc/bitw.rs:42-44
    __device__ __forceinline__ void se(int v) { ue(v > 0 ? 2u * (uint32_t)v - 1u : (uint32_t)(-2ll * v)); }
};

__device__ __forceinline__ unsigned ue_len(uint32_t v) { return 2 * (64 - __clzll((long long)((unsigned long long)v + 1))) - 1; }

// put_level, enc/cavlc.rs:12-45
__device__ __forceinline__ void put_level_d(BitSink& w, uint32_t code, uint32_t suffix_len) {
    bool esc = false;
    uint32_t rem = 0;
    if (suffix_len == 0) {
        if (code < 14) {
            w.put(code + 1, 1);
        } else if (code < 30) {
            w.put(15, 1);
            w.put(4, code - 14);
        } else {
            esc = true;
            rem = code - 30;
        }
    } else if ((code >> suffix_len) < 15) {
        w.put((code >> suffix_len) + 1, 1);
        w.put(suffix_len, code & ((1u << suffix_len) - 1));
    } else {
        esc = true;
        rem = code - (15u << suffix_len);
    }
    if (esc) {
        if (rem < 4096) {
            w.put(16, 1);
            w.put(12, rem);
        } else {
            unsigned p = 16;
            while ((unsigned long long)rem + 4096 >= (1ull << (p - 2))) p++;
            w.put(p, 0);
            w.put(1, 1);
            w.put(p - 3, rem + 4096 - (1u << (p - 3)));
        }
    }
}

// write_block, enc/cavlc.rs:47-122: levels[0..max) in scan order; nc = -1 for chroma DC.
__device__ void write_block_d(BitSink& w, int nc, const int (&lv)[16], int max) {
    int nz[16], runs[16], total = 0, last = -1;
#pragma unroll
    for (int i = 0; i < 16; i++) runs[i] = 0;
    for (int i = max - 1; i >= 0; i--)
        if (lv[i] != 0) {
            if (last >= 0) runs[total - 1] = last - i - 1;
            nz[total++] = lv[i];
            last = i;
        }
    int ones = 0;
    while (ones < (total < 3 ? total : 3) && abs(nz[ones]) == 1) ones++;
    const int token = total * 4 + ones;
    if (nc == -1) {
        w.put(CAVLC_CHROMA_DC_COEFF_TOKEN_LEN[token], CAVLC_CHROMA_DC_COEFF_TOKEN_BITS[token]);
    } else {
        const int cls = nc <= 1 ? 0 : nc <= 3 ? 1 : nc <= 7 ? 2 : 3;
        w.put(CAVLC_COEFF_TOKEN_LEN[cls][token], CAVLC_COEFF_TOKEN_BITS[cls][token]);
    }
    if (total == 0) return;
    for (int i = 0; i < ones; i++) w.flag(nz[i] < 0);
    uint32_t suffix_len = (total > 10 && ones < 3) ? 1 : 0;
    for (int i = ones; i < total; i++) {
        const int l = nz[i];
        uint32_t code = l > 0 ? 2u * (uint32_t)l - 2u : (uint32_t)(-2 * l) - 1u;
        if (i == ones && ones < 3) code -= 2;
        put_level_d(w, code, suffix_len);
        if (suffix_len == 0) suffix_len = 1;
        if ((uint32_t)abs(l) > (3u << (suffix_len - 1)) && suffix_len < 6) suffix_len++;
    }
    int highest = max - 1;
    while (lv[highest] == 0) highest--;
    int zeros_left = highest + 1 - total;
    if (total < max) {
        if (nc == -1)
            w.put(CAVLC_CHROMA_DC_TOTAL_ZEROS_LEN[total - 1][zeros_left], CAVLC_CHROMA_DC_TOTAL_ZEROS_BITS[total - 1][zeros_left]);
        else
            w.put(CAVLC_TOTAL_ZEROS_LEN[total - 1][zeros_left], CAVLC_TOTAL_ZEROS_BITS[total - 1][zeros_left]);
    }
    for (int i = 0; i < total - 1 && zeros_left > 0; i++) {
        const int zl = zeros_left < 7 ? zeros_left : 7;
        w.put(CAVLC_RUN_LEN[zl - 1][runs[i]], CAVLC_RUN_BITS[zl - 1][runs[i]]);
        zeros_left -= runs[i];
    }
}

// nc, enc/frame.rs:2354-2361
__device__ __forceinline__ int nc_of(bool ha, int a, bool hb, int b) {
    if (ha && hb) return (a + b + 1) >> 1;
    return ha ? a : (hb ? b : 0);
}

// The residual block of slot s (0: Intra16x16 DC; 1..16: luma in decoding order; 17, 18: chroma DC; 19..26:
// chroma AC, Cb then Cr) of macroblock `code`, if the macroblock codes it; its levels and nC context.
__device__ bool block_of(const CavlcParams& P, const ironav_mbcode& code, int mb, int s, int (&lv)[16], int* max, int* nc) {
    const int mbx = mb % P.mb_w, mby = mb / P.mb_w;
    const bool la = mbx > 0, ta = mby > P.band_start[mby];
    const ironav_mbcode* L = la ? &P.codes[mb - 1] : nullptr;
    const ironav_mbcode* U = ta ? &P.codes[mb - P.mb_w] : nullptr;
    const int cbp = code.res.cbp, cbpl = cbp & 15, cbpc = cbp >> 4;
    const bool i16 = code.kind == CAVLC_KIND_I16;
    if (cbp == 0 && !i16) return false;
    // nc_luma (enc/frame.rs:606-610) of raster block (bx, by)
    auto nc_luma = [&](int bx, int by) {
        const bool ha = bx > 0 || la, hb = by > 0 || ta;
        const int a = bx > 0 ? code.res.nnz[by * 4 + bx - 1] : (la ? L->res.nnz[by * 4 + 3] : 0);
        const int b = by > 0 ? code.res.nnz[(by - 1) * 4 + bx] : (ta ? U->res.nnz[12 + bx] : 0);
        return nc_of(ha, a, hb, b);
    };
    if (s == 0) {
        if (!i16) return false;
        for (int k = 0; k < 16; k++) lv[k] = code.dc[k];
        *max = 16;
        *nc = nc_luma(0, 0);
        return true;
    }
    if (s <= 16) {
        const int n = s - 1;
        if (!(cbpl & (1 << (n >> 2)))) return false;
        const int bx = ((n >> 2) & 1) * 2 + (n & 1), by = ((n >> 3) & 1) * 2 + ((n >> 1) & 1);  // block_pos, enc/frame.rs:108-110
        const int16_t* b = code.res.luma[by * 4 + bx];
        if (i16) {
            for (int k = 0; k < 15; k++) lv[k] = b[1 + k];
            lv[15] = 0;
            *max = 15;
        } else {
            for (int k = 0; k < 16; k++) lv[k] = b[k];
            *max = 16;
        }
        *nc = nc_luma(bx, by);
        return true;
    }
    if (s <= 18) {
        if (cbpc == 0) return false;
        const int cc = s - 17;
        for (int k = 0; k < 16; k++) lv[k] = k < 4 ? code.res.cdc[cc][k] : 0;
        *max = 4;
        *nc = -1;
        return true;
    }
    if (cbpc != 2) return false;
    const int cc = (s - 19) >> 2, blk = (s - 19) & 3, bx = blk & 1, by = blk >> 1;
    for (int k = 0; k < 15; k++) lv[k] = code.res.cac[cc][blk][1 + k];
    lv[15] = 0;
    *max = 15;
    // nc_chroma, enc/frame.rs:612-616
    const bool ha = bx > 0 || la, hb = by > 0 || ta;
    const int a = bx > 0 ? code.res.cnnz[cc][by * 2] : (la ? L->res.cnnz[cc][by * 2 + 1] : 0);
    const int b = by > 0 ? code.res.cnnz[cc][bx] : (ta ? U->res.cnnz[cc][2 + bx] : 0);
    *nc = nc_of(ha, a, hb, b);
    return true;
}

// The header part of write_mb (enc/frame.rs:1922-1977, 1978-1979): mb_type and what follows it up to
// mb_qp_delta, without the skip run.
__device__ void mb_header(const CavlcParams& P, const ironav_mbcode& code, int mb, BitSink& w) {
    const int mbx = mb % P.mb_w, mby = mb / P.mb_w;
    const bool la = mbx > 0, ta = mby > P.band_start[mby];
    const unsigned base = P.p_slice ? 5 : 0;
    const int cbp = code.res.cbp, cbpl = cbp & 15, cbpc = cbp >> 4;
    auto cbp_code = [](const uint8_t* tab, int v) {
        for (int i = 0; i < 48; i++)
            if (tab[i] == v) return i;
        return 0;
    };
    if (code.kind == CAVLC_KIND_I4) {
        w.ue(base);
        uint8_t so_far[16];
        for (int k = 0; k < 16; k++) so_far[k] = 2;
        for (int n = 0; n < 16; n++) {
            const int bx = ((n >> 2) & 1) * 2 + (n & 1), by = ((n >> 3) & 1) * 2 + ((n >> 1) & 1);
            const int mode = code.modes[by * 4 + bx];
            // pred_i4_mode, enc/frame.rs:619-629 (a neighbour that is not Intra4x4 counts as DC)
            int a = -1, b = -1;
            if (bx > 0) a = so_far[by * 4 + bx - 1];
            else if (la) {
                const ironav_mbcode& L = P.codes[mb - 1];
                a = L.kind == CAVLC_KIND_I4 ? L.modes[by * 4 + 3] : 2;
            }
            if (by > 0) b = so_far[(by - 1) * 4 + bx];
            else if (ta) {
                const ironav_mbcode& U = P.codes[mb - P.mb_w];
                b = U.kind == CAVLC_KIND_I4 ? U.modes[12 + bx] : 2;
            }
            const int pred = (a >= 0 && b >= 0) ? min(a, b) : 2;
            so_far[by * 4 + bx] = (uint8_t)mode;
            if (mode == pred) {
                w.flag(true);
            } else {
                w.flag(false);
                w.put(3, (uint32_t)(mode < pred ? mode : mode - 1));
            }
        }
        w.ue(code.chroma_mode);
        w.ue((uint32_t)cbp_code(CAVLC_GOLOMB_TO_INTRA4X4_CBP, cbp));
    } else if (code.kind == CAVLC_KIND_I16) {
        w.ue(base + 1 + code.i16_mode + 4 * (unsigned)cbpc + (cbpl ? 12 : 0));
        w.ue(code.chroma_mode);
    } else {
        w.ue(code.part);
        if (code.part == 3)
            for (int k = 0; k < 4; k++) w.ue(code.sub[k]);
        const int nparts = code.part == 0 ? 1 : (code.part == 3 ? 4 : 2);
        if (P.nref > 1)
            for (int k = 0; k < nparts; k++) {
                if (P.nref == 2) w.flag(code.refs[k] == 0);
                else w.ue(code.refs[k]);
            }
        // rects(part, sub) count: one per partition, the sub-partitions of P_8x8 (SUB, enc/frame.rs:204)
        int nr = nparts;
        if (code.part == 3) {
            nr = 0;
            for (int k = 0; k < 4; k++) nr += code.sub[k] == 0 ? 1 : (code.sub[k] == 3 ? 4 : 2);
        }
        for (int k = 0; k < nr; k++) {
            w.se(code.mvds[k][0]);
            w.se(code.mvds[k][1]);
        }
        w.ue((uint32_t)cbp_code(CAVLC_GOLOMB_TO_INTER_CBP, cbp));
    }
    if (cbp != 0 || code.kind == CAVLC_KIND_I16) w.se(0);  // mb_qp_delta
}

// One macroblock's syntax on a warp: lane 0 the skip-run prefix (when `run_prefix`) and the header, lanes
// 1..27 the residual blocks; returns the macroblock's bits (every lane). With out set, the bits go to the
// region from bit `base` on.
__device__ unsigned mb_syntax(const CavlcParams& P, int mb, uint32_t* out, unsigned long long base, unsigned long long limit,
                              bool run_prefix, uint32_t run, bool* overflow) {
    const int lane = threadIdx.x & 31;
    const ironav_mbcode& code = P.codes[mb];
    BitSink w{nullptr, 0, limit, false};
    int lv[16], max = 0, nc = 0;
    bool have = false;
    if (lane >= 1 && lane <= 27) have = block_of(P, code, mb, lane - 1, lv, &max, &nc);
    // lengths first (a counting pass), then the lanes' offsets
    if (lane == 0) {
        if (run_prefix) w.ue(run);
        mb_header(P, code, mb, w);
    } else if (have) {
        write_block_d(w, nc, lv, max);
    }
    const unsigned len = (unsigned)w.pos;
    unsigned incl = len;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const unsigned v = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d) incl += v;
    }
    const unsigned total = __shfl_sync(0xffffffffu, incl, 31);
    if (out) {
        BitSink o{out, base + (incl - len), limit, false};
        if (lane == 0) {
            if (run_prefix) o.ue(run);
            mb_header(P, code, mb, o);
        } else if (have) {
            write_block_d(o, nc, lv, max);
        }
        if (__any_sync(0xffffffffu, o.overflow)) *overflow = true;
    }
    return total;
}

// Pass 1: each macroblock's bits without the skip-run prefix (0 for a skipped macroblock of a P slice).
static __global__ void cavlc_size_kernel(const __grid_constant__ CavlcParams P) {
    const int warps = (blockDim.x >> 5) * gridDim.x;
    for (int mb = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); mb < P.nmb; mb += warps) {
        unsigned len = 0;
        if (!(P.p_slice && P.codes[mb].skip)) {
            bool ovf = false;
            len = mb_syntax(P, mb, nullptr, 0, ~0ull, false, 0, &ovf);
        }
        if ((threadIdx.x & 31) == 0) {
            if (len > CAVLC_MB_MAX_BITS) atomicOr(P.err, 1u);
            P.mb_len[mb] = len;
        }
    }
}

// Inclusive block-wide scan helpers (blockDim.x = 1024: 32 warps)
__device__ __forceinline__ unsigned block_scan_add(unsigned v, unsigned* tmp) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const unsigned t = __shfl_up_sync(0xffffffffu, v, d);
        if (lane >= d) v += t;
    }
    if (lane == 31) tmp[wid] = v;
    __syncthreads();
    if (wid == 0) {
        unsigned s = lane < (int)(blockDim.x >> 5) ? tmp[lane] : 0;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const unsigned t = __shfl_up_sync(0xffffffffu, s, d);
            if (lane >= d) s += t;
        }
        tmp[lane] = s;
    }
    __syncthreads();
    const unsigned r = v + (wid > 0 ? tmp[wid - 1] : 0);
    __syncthreads();
    return r;
}
__device__ __forceinline__ int block_scan_max(int v, int* tmp) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, v, d);
        if (lane >= d) v = max(v, t);
    }
    if (lane == 31) tmp[wid] = v;
    __syncthreads();
    if (wid == 0) {
        int s = lane < (int)(blockDim.x >> 5) ? tmp[lane] : -1;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, s, d);
            if (lane >= d) s = max(s, t);
        }
        tmp[lane] = s;
    }
    __syncthreads();
    const int r = wid > 0 ? max(v, tmp[wid - 1]) : v;
    __syncthreads();
    return r;
}

// The slice header, enc/mod.rs:566-600 (CAVLC: no cabac_init_idc; picture order type 2: no POC lsb)
__device__ void slice_header(const CavlcParams& P, int first_mb, BitSink& w) {
    w.ue((uint32_t)first_mb);    // first_mb_in_slice
    w.ue(P.idr ? 7 : 5);         // slice_type: I or P, all slices of the picture alike
    w.ue(0);                     // pic_parameter_set_id
    w.put(8, (uint32_t)P.frame_num);
    if (P.idr) w.ue((uint32_t)P.idr_pic_id);
    if (!P.idr) {
        if (P.nref > 1) {
            w.flag(true);        // num_ref_idx_active_override_flag
            w.ue((uint32_t)(P.nref - 1));
        } else {
            w.flag(false);
        }
        w.flag(false);           // ref_pic_list_modification_flag_l0
    }
    if (P.idr) {
        w.flag(false);           // no_output_of_prior_pics_flag
        w.flag(false);           // long_term_reference_flag
    } else {
        w.flag(false);           // adaptive_ref_pic_marking_mode_flag
    }
    w.se(P.slice_qp_delta);
}

// Pass 2, a CTA of 1024 threads per slice: skip runs, offsets, the slice's size; clears the slice's bytes and
// writes its header and trailer.
static __global__ void __launch_bounds__(1024) cavlc_scan_kernel(const __grid_constant__ CavlcParams P) {
    __shared__ unsigned tmpu[32];
    __shared__ int tmpi[32];
    __shared__ int s_incl[1024];
    __shared__ unsigned long long s_base, s_carry;
    __shared__ int s_last;
    const int sl = blockIdx.x;
    const int first = P.slice_first[sl], end = P.slice_first[sl + 1];
    if (threadIdx.x == 0) {
        BitSink h{nullptr, 0, ~0ull, false};
        slice_header(P, first, h);
        s_base = h.pos;
        s_carry = 0;
        s_last = first - 1;
    }
    __syncthreads();
    for (int c0 = first; c0 < end; c0 += blockDim.x) {
        const int mb = c0 + (int)threadIdx.x;
        const bool in = mb < end;
        const unsigned len = in ? P.mb_len[mb] : 0;
        const bool coded = in && (!P.p_slice || len > 0);
        // the last coded macroblock at or before mb (s_last carries the previous chunks'), and before it
        const int last_incl = max(block_scan_max(coded ? mb : -1, tmpi), s_last);
        s_incl[threadIdx.x] = last_incl;
        __syncthreads();
        const int prev = threadIdx.x == 0 ? s_last : s_incl[threadIdx.x - 1];
        const uint32_t run = coded ? (uint32_t)(mb - prev - 1) : 0;
        const unsigned bits = coded ? len + (P.p_slice ? ue_len(run) : 0) : 0;
        const unsigned incl = block_scan_add(bits, tmpu);
        if (in) {
            P.mb_off[mb] = (uint32_t)(s_base + s_carry + incl - bits);
            P.mb_run[mb] = run;
        }
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) {
            s_carry += incl;
            s_last = last_incl;
        }
        __syncthreads();
    }
    // the trailer: the skip run after the last coded macroblock, then rbsp_trailing_bits
    __shared__ unsigned long long s_end;
    __shared__ uint32_t s_trail;
    __shared__ int s_fits;
    if (threadIdx.x == 0) {
        s_trail = P.p_slice ? (uint32_t)(end - 1 - s_last) : 0;
        const unsigned long long bits = s_base + s_carry + (s_trail > 0 ? ue_len(s_trail) : 0) + 1;
        s_end = bits;
        s_fits = ((bits + 7) & ~7ull) <= P.region_words * 32ull;
        if (!s_fits) atomicOr(P.err, 1u);
        P.slice_bytes[sl] = (uint32_t)((bits + 7) >> 3);
    }
    __syncthreads();
    if (!s_fits) return;  // the same value on every thread of the CTA
    uint32_t* region = P.out + (unsigned long long)sl * P.region_words;
    const unsigned long long words = (s_end + 31) >> 5;
    for (unsigned long long k = threadIdx.x; k < words; k += blockDim.x) region[k] = 0;
    __syncthreads();
    if (threadIdx.x == 0) {
        BitSink h{region, 0, P.region_words * 32ull, false};
        slice_header(P, first, h);
        h.pos = s_base + s_carry;
        if (s_trail > 0) h.ue(s_trail);
        h.put(1, 1);  // rbsp_stop_one_bit; the alignment zeros are already there
        if (h.overflow) atomicOr(P.err, 1u);
    }
}

// Pass 3: every coded macroblock's syntax at its offset.
static __global__ void cavlc_write_kernel(const __grid_constant__ CavlcParams P) {
    if (*P.err) return;
    const int warps = (blockDim.x >> 5) * gridDim.x;
    for (int mb = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); mb < P.nmb; mb += warps) {
        if (P.p_slice && P.mb_len[mb] == 0) continue;  // skipped: counted in the next coded macroblock's run
        const int sl = P.row_slice[mb / P.mb_w];
        uint32_t* region = P.out + (unsigned long long)sl * P.region_words;
        bool ovf = false;
        mb_syntax(P, mb, region, P.mb_off[mb], P.region_words * 32ull, P.p_slice != 0, P.mb_run[mb], &ovf);
        if (ovf && (threadIdx.x & 31) == 0) atomicOr(P.err, 1u);
    }
}

}  // namespace ironav
