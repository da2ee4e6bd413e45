// decide_rd.cuh — K9: code_mb with CABAC on the device (the reference encoder's default decision: decide_rd,
// enc/frame.rs:1462-1513, after code_mb's P_Skip tests, best_i16 and best_inter, 715-760), and the CABAC
// slice writer.
//
// Under CABAC a macroblock's rate-distortion cost counts its bins against the slice's contexts as the
// macroblocks before it left them, so a slice band is one chain in raster order: a warp walks a band (one
// CTA a band, the bands side by side). For each macroblock the warp codes every candidate the reference
// tries, in its order (P_Skip, best_inter's partitioning with the 4x4 and, with transform8, the 8x8
// transform, Intra16x16, Intra4x4, Intra8x8, each intra one with its chroma), each into the picture and
// then into shared memory (code and reconstruction), with its squared error; then the candidates' bins are
// counted, each on its own copy of the contexts (the counter of cabac.cuh), a lane per group of disjoint
// contexts (nine a candidate); lane 0 keeps the least SSD + lambda2 * bits in the reference's order (strict
// '<'), and the warp copies the kept candidate's code, reconstruction and advanced contexts into place.
//
// The candidates reuse decide mode's warp-level coders (decide.cuh, residual.cuh); Intra8x8 (code_i8,
// enc/frame.rs:1307-1388) is coded here: block by block, its edges filtered (8.3.2.2.1), nine modes'
// SATD over 36 lane-units of (mode, 4x4 quadrant) from a table of the predictors (i8_entry), the chosen
// block's 8x8 transform on eight lanes.
#pragma once
#include "cabac.cuh"
#include "decide.cuh"

namespace ironav {

constexpr int RD_CANDS = 6;  // P_Skip, inter with the 4x4 transform, inter with the 8x8, Intra16x16, Intra4x4, Intra8x8

struct RdParams {
    DecideParams D;         // decide mode's parameters: the analysis, the coder, the outputs (codes, states)
    uint32_t* nbs;          // per macroblock, what the contexts read of it as a neighbour (cab::Nb, NB_WORDS words)
    const int* band_rows;   // chain i walks the rows [band_rows[i], band_rows[i + 1])
    const uint32_t* step;   // the contexts' step table (cab::STEP_ENTRIES)
    double lam2;            // 1.6 * 2^((QP'Y - 12) / 3), computed on the host in f64 as the reference does
    int nbands;
    int t8;                 // transform_8x8_mode_flag
    // the three-warp form: warps 1 and 2's scratch planes (luma, Cb, Cr of warp 1, then of warp 2), pw x ph and
    // cw x ch samples, rows scr_ys and scr_cs samples apart
    uint8_t* scr[6];
    int scr_ys, scr_cs;
};

template <class T, int W>
struct RdSmem {
    DecideSmem<T> s[W];              // each warp's working set
    ironav_mbcode cand[RD_CANDS];    // the candidates' codes
    T crec[RD_CANDS][384];           // and reconstructions (luma, Cb, Cr)
    uint8_t live[1024];              // the chain's contexts after the macroblocks before this one
    uint8_t cst[RD_CANDS][1024];     // each candidate's copy, advanced by its bins
    uint32_t step[cab::STEP_ENTRIES];
    cab::Nb nb[2];                   // the left and top neighbours as the contexts see them
    cab::Nb done;                    // the macroblock just decided, the next one's left
    ironav_mbstate state[RD_CANDS];  // each candidate's MbState
    long long ssd[RD_CANDS];
    long long cssd[RD_CANDS];        // the chroma part of ssd
    unsigned bits[RD_CANDS];
    int valid[RD_CANDS];
    int best;
    int skip;                        // the three-warp form: the P_Skip tests' verdict and the skip vector; the
    int2 sv;                         // intra chroma's coded block pattern bits; best_inter's decision for the
    uint32_t ccbp;                   // 8x8-transform candidate (warp 2), and whether that candidate is tried
    uint16_t idec[40];
    int try_t8;
    // the Intra8x8 trial
    int i8rec[256];       // its reconstruction
    int raw[25], e8[26];  // a block's edges, raw and filtered: [0] top-left, [1 + i] the 16 above, [17 + j] the 8 left,
                          // e8[25] the DC mode's value
    unsigned i8tab[9 * 64];  // i8_entry per mode and sample
    int sat[36];          // SATD per (mode, 4x4 quadrant)
    int pred8[64];
    int t8b[8][9];
    int co8b[64];
    int16_t lv8b[64];
    uint8_t i8modes[16];
    int i8meta[4];        // chosen mode, predicted mode, DC value, non-zero levels
};

// The 8x8 intra predictors as a table, as decide mode's 4x4 ones (i4_entry): every sample of every mode is
// (E[a] + 2 E[b] + E[c] + 2) >> 2 over the block's filtered edge array E (E[0] the top-left sample, E[1 + i]
// the 16 above, E[17 + j] the 8 to the left, E[25] the DC mode's value): a copy has a = b = c, a two-sample
// average (p + q + 1) >> 1 has a = c = p, b = q, and (p + 3q + 2) >> 2 has b = c = q. Entry: a | b << 5 | c << 10.
// The cases are predict_nxn's for n = 8 (h264/intra.rs:30-128; ITU-T H.264 8.3.2.2.2-8.3.2.2.10).
__device__ __forceinline__ unsigned i8_entry(int mode, int x, int y) {
    auto T = [](int i) { return i < 0 ? 0 : 1 + i; };
    auto L = [](int j) { return j < 0 ? 0 : 17 + j; };
    auto E3 = [](int a, int b, int c) { return (unsigned)(a | b << 5 | c << 10); };
    switch (mode) {
    case 0: return E3(T(x), T(x), T(x));
    case 1: return E3(L(y), L(y), L(y));
    case 2: return E3(25, 25, 25);
    case 3: return (x == 7 && y == 7) ? E3(T(14), T(15), T(15)) : E3(T(x + y), T(x + y + 1), T(x + y + 2));
    case 4:
        if (x > y) return E3(T(x - y - 2), T(x - y - 1), T(x - y));
        if (x < y) return E3(L(y - x - 2), L(y - x - 1), L(y - x));
        return E3(T(0), 0, L(0));
    case 5: {
        const int z = 2 * x - y, i = x - (y >> 1);
        if (z >= 0 && (z & 1) == 0) return E3(T(i - 1), T(i), T(i - 1));
        if (z >= 0) return E3(T(i - 2), T(i - 1), T(i));
        if (z == -1) return E3(L(0), 0, T(0));
        return E3(L(y - 2 * x - 1), L(y - 2 * x - 2), L(y - 2 * x - 3));
    }
    case 6: {
        const int z = 2 * y - x, j = y - (x >> 1);
        if (z >= 0 && (z & 1) == 0) return E3(L(j - 1), L(j), L(j - 1));
        if (z >= 0) return E3(L(j - 2), L(j - 1), L(j));
        if (z == -1) return E3(L(0), 0, T(0));
        return E3(T(x - 2 * y - 1), T(x - 2 * y - 2), T(x - 2 * y - 3));
    }
    case 7: {
        const int i = x + (y >> 1);
        return (y & 1) == 0 ? E3(T(i), T(i + 1), T(i)) : E3(T(i), T(i + 1), T(i + 2));
    }
    default: {
        const int z = x + 2 * y, j = y + (x >> 1);
        if (z > 13) return E3(L(7), L(7), L(7));
        if (z == 13) return E3(L(6), L(7), L(7));
        if ((z & 1) == 0) return E3(L(j), L(j + 1), L(j));
        return E3(L(j), L(j + 1), L(j + 2));
    }
    }
}

__device__ __forceinline__ int i8_pred(const int* E, unsigned e) { return (E[e & 31] + 2 * E[(e >> 5) & 31] + E[e >> 10] + 2) >> 2; }

// code_i8, enc/frame.rs:1307-1388: the luma of an Intra8x8 macroblock, block by block in S.i8rec (each
// block predicted from the filtered edges of the reconstruction so far, its mode the cheapest by SATD +
// lambda * (1 predicted, 4 otherwise), quantised with the intra rounding), its levels, modes and counts
// into out (zeroed by the caller with the Intra4x4 modes 2), and the reconstruction into wy.
// Returns the luma coded block pattern (every lane).
template <class T, int W>
__device__ uint32_t code_i8_d(const DecideParams& P, DecideSmem<T>& S, RdSmem<T, W>& R, int mbx, int mby, bool ta, bool la, bool tra,
                              ironav_mbcode* out, T* wy, int wys) {
    // P.C.rec: the picture the edges are read from; wy (rows wys samples apart): where the luma goes. The
    // predictor table of R.i8tab is filled once a chain (rd_chain)
    const int lane = threadIdx.x & 31;
    const CodeParams& C = P.C;
    const int bd = C.bd, maxv = (1 << bd) - 1, lam = C.A.lambda;
    const int qp = C.qp + 6 * (bd - 8), m6 = qp % 6, qbits = 16 + qp / 6, f = (1 << qbits) / 3;
    const T* Y = reinterpret_cast<const T*>(C.rec[0]);
    const int x0 = mbx * 16, y0 = mby * 16;
    if (lane < 16) R.i8modes[lane] = 2;
    __syncwarp();
    uint32_t cbp = 0;
    for (int i8 = 0; i8 < 4; i8++) {
        const int bx = i8 & 1, by = i8 >> 1;
        const bool hl = bx > 0 || la, ht = by > 0 || ta;
        const bool htl = bx > 0 ? (by > 0 ? true : ta) : (by > 0 ? la : (la && ta));
        const bool htr = i8 == 0 ? ta : (i8 == 1 ? tra : i8 == 2);
        // the raw edges: the row above (the top-right half after the rest), the column to the left, the corner
        if (lane < 8) {
            const int x = bx * 8 + lane;
            R.raw[1 + lane] = !ht ? 0 : (by == 0 ? S.top[1 + x] : R.i8rec[7 * 16 + x]);
            R.raw[17 + lane] = !hl ? 0 : (bx == 0 ? S.left[by * 8 + lane] : R.i8rec[(by * 8 + lane) * 16 + 7]);
        } else if (lane == 8) {
            int v = 0;
            if (htl) v = by == 0 ? S.top[bx * 8] : (bx == 0 ? S.left[7] : R.i8rec[7 * 16 + 7]);
            R.raw[0] = v;
        }
        __syncwarp();
        if (lane < 8) {
            int v = 0;
            if (ht) {
                if (!htr) v = R.raw[8];  // the last sample above, repeated
                else if (by == 1) v = R.i8rec[7 * 16 + 8 + lane];
                else if (bx == 0) v = S.top[1 + 8 + lane];
                else v = (int)Y[(size_t)(y0 - 1) * C.ys + x0 + 16 + lane];  // the top-right macroblock's bottom row
            }
            R.raw[9 + lane] = v;
        }
        __syncwarp();
        // filter_8x8_edges, h264/intra.rs:131-158
        if (lane < 25) {
            const int* p = R.raw;
            int v = p[lane];
            if (lane == 0) {
                if (htl) {
                    if (ht && hl) v = (p[1] + 2 * p[0] + p[17] + 2) >> 2;
                    else if (ht) v = (3 * p[0] + p[1] + 2) >> 2;
                    else if (hl) v = (3 * p[0] + p[17] + 2) >> 2;
                }
            } else if (lane <= 16) {
                const int x = lane - 1;
                if (ht) {
                    if (x == 0) v = htl ? (p[0] + 2 * p[1] + p[2] + 2) >> 2 : (3 * p[1] + p[2] + 2) >> 2;
                    else if (x == 15) v = (p[15] + 3 * p[16] + 2) >> 2;
                    else v = (p[x] + 2 * p[x + 1] + p[x + 2] + 2) >> 2;
                }
            } else {
                const int y = lane - 17;
                if (hl) {
                    if (y == 0) v = htl ? (p[0] + 2 * p[17] + p[18] + 2) >> 2 : (3 * p[17] + p[18] + 2) >> 2;
                    else if (y == 7) v = (p[23] + 3 * p[24] + 2) >> 2;
                    else v = (p[16 + y] + 2 * p[17 + y] + p[18 + y] + 2) >> 2;
                }
            }
            R.e8[lane] = v;
        }
        __syncwarp();
        if (lane == 0) {
            const int* E = R.e8;
            int st = 0, sl = 0;
            for (int i = 0; i < 8; i++) st += E[1 + i], sl += E[17 + i];
            R.i8meta[2] = (ht && hl) ? (st + sl + 8) >> 4 : (hl ? (sl + 4) >> 3 : (ht ? (st + 4) >> 3 : 1 << (bd - 1)));
            R.e8[25] = R.i8meta[2];
            R.i8meta[1] = cab::pred_mode(S.nbm, R.i8modes, bx * 2, by * 2);
        }
        __syncwarp();
        // the nine modes' SATD, a lane per (mode, 4x4 quadrant)
        for (int u = lane; u < 36; u += 32) {
            const int mode = u >> 2, q = u & 3;
            const bool ok = (mode == 0 || mode == 3 || mode == 7) ? ht : (mode == 1 || mode == 8) ? hl : mode == 2 ? true : (ht && hl && htl);
            int s = 0;
            if (ok) {
                int d[16];
#pragma unroll
                for (int r = 0; r < 4; r++)
#pragma unroll
                    for (int k = 0; k < 4; k++) {
                        const int px = (q & 1) * 4 + k, py = (q >> 1) * 4 + r;
                        d[r * 4 + k] = src_at(S.a, bx * 8 + px, by * 8 + py) - i8_pred(R.e8, R.i8tab[mode * 64 + py * 8 + px]);
                    }
                s = satd4_d(d);
            }
            R.sat[u] = ok ? s : -1;
        }
        __syncwarp();
        if (lane == 0) {
            int bm = 2, bc = 0x7fffffff;
            for (int mode = 0; mode < 9; mode++) {
                if (R.sat[mode * 4] < 0) continue;
                const int c = R.sat[mode * 4] + R.sat[mode * 4 + 1] + R.sat[mode * 4 + 2] + R.sat[mode * 4 + 3] +
                              lam * (mode == R.i8meta[1] ? 1 : 4);
                if (c < bc) bm = mode, bc = c;
            }
            R.i8meta[0] = bm;
        }
        __syncwarp();
        const int bm = R.i8meta[0];
        for (int i = lane; i < 64; i += 32) R.pred8[i] = i8_pred(R.e8, R.i8tab[bm * 64 + i]);
        __syncwarp();
        // quant8 (intra rounding) and idct8_add, enc/frame.rs:56-72 and h264/idct.rs:33-74, eight lanes
        const int j = lane & 7;
        if (lane < 8) {
            int d[8], o[8];
#pragma unroll
            for (int k = 0; k < 8; k++) d[k] = src_at(S.a, bx * 8 + k, by * 8 + j) - R.pred8[j * 8 + k];
            q_fdct8_1d_d(d, o);
#pragma unroll
            for (int k = 0; k < 8; k++) R.t8b[j][k] = o[k];
        }
        __syncwarp();
        if (lane < 8) {
            int d[8], o[8];
#pragma unroll
            for (int k = 0; k < 8; k++) d[k] = R.t8b[k][j];
            q_fdct8_1d_d(d, o);
#pragma unroll
            for (int k = 0; k < 8; k++) R.co8b[k * 8 + j] = o[k];
        }
        __syncwarp();
        int dq[8];
        int nz = 0;
        if (lane < 8) {
#pragma unroll
            for (int k = 0; k < 8; k++) {
                const int sk = j * 8 + k, pz = c_zz8[sk];
                const int l = q_quant_d(R.co8b[pz], c_q_mf8[m6][q_class8_d(pz)], f, qbits);
                R.lv8b[sk] = (int16_t)l;
                nz += l != 0;
                int v = 0;
                if (l != 0) {
                    const int vv = l * 16 * c_q_dq8[m6][q_class8_d(pz)];
                    v = qp >= 36 ? vv << (qp / 6 - 6) : (vv + (1 << (5 - qp / 6))) >> (6 - qp / 6);
                }
                dq[k] = v;
            }
        }
        __syncwarp();
        if (lane < 8) {
#pragma unroll
            for (int k = 0; k < 8; k++) R.co8b[c_zz8[j * 8 + k]] = dq[k];
        }
#pragma unroll
        for (int off = 16; off >= 1; off >>= 1) nz += __shfl_xor_sync(FULL, nz, off);
        __syncwarp();
        if (lane < 8 && nz > 0) {
            int d[8], o[8];
#pragma unroll
            for (int k = 0; k < 8; k++) d[k] = R.co8b[j * 8 + k];
            q_row8_d(d, o);
#pragma unroll
            for (int k = 0; k < 8; k++) R.t8b[j][k] = o[k];
        }
        __syncwarp();
        if (lane < 8) {
            int o[8];
            if (nz > 0) {
                int d[8];
#pragma unroll
                for (int k = 0; k < 8; k++) d[k] = R.t8b[k][j];
                q_row8_d(d, o);
            }
#pragma unroll
            for (int i = 0; i < 8; i++) {
                const int pv = R.pred8[i * 8 + j];
                R.i8rec[(by * 8 + i) * 16 + bx * 8 + j] = nz > 0 ? min(max(pv + ((o[i] + 32) >> 6), 0), maxv) : pv;
            }
        }
        for (int k = lane; k < 64; k += 32) out->res.luma8[i8][k] = R.lv8b[k];
        if (lane < 4) {
            const int b = (by * 2 + (lane >> 1)) * 4 + bx * 2 + (lane & 1);
            R.i8modes[b] = (uint8_t)bm;
            out->res.nnz[b] = (uint8_t)nz;
        }
        if (nz > 0) cbp |= 1u << i8;
        __syncwarp();
    }
    for (int i = lane; i < 256; i += 32) wy[(size_t)(y0 + (i >> 4)) * wys + x0 + (i & 15)] = (T)R.i8rec[i];
    if (lane < 16) out->modes[lane] = R.i8modes[lane];
    if (lane == 0) {
        out->kind = KIND_I8;
        out->res.t8x8 = 1;
    }
    __syncwarp();
    return cbp;
}

// MbCode::new (enc/frame.rs:302-306): zero, the Intra4x4 modes 2 (words 371-374 of the code).
__device__ __forceinline__ void code_init(ironav_mbcode* o) {
    const int lane = threadIdx.x & 31;
    uint32_t* w = reinterpret_cast<uint32_t*>(o);
    for (int k = lane; k < (int)(sizeof(ironav_mbcode) / 4); k += 32) w[k] = (k >= 371 && k < 375) ? 0x02020202u : 0u;
    __syncwarp();
}

// A candidate coded into the planes C (the picture, or a warp's scratch planes): its squared error (ssd_mb,
// enc/frame.rs:1432-1449) and a copy of its reconstruction (save_mb, 1406-1417); chroma false: the luma
// only, the chroma added later from another candidate's. The candidate counts from here on.
template <class T, int W>
__device__ void rd_take(const CodeParams& C, RdSmem<T, W>& R, const DecideSmem<T>& S, int k, int mbx, int mby, bool chroma = true) {
    const int lane = threadIdx.x & 31;
    const T* SC = reinterpret_cast<const T*>(C.src_c);
    T* dst = R.crec[k];
    __syncwarp();
    long long ssd = 0, cssd = 0;
    for (int i = lane; i < (chroma ? 384 : 256); i += 32) {
        int r, s;
        if (i < 256) {
            r = reinterpret_cast<const T*>(C.rec[0])[(size_t)(mby * 16 + (i >> 4)) * C.ys + mbx * 16 + (i & 15)];
            s = src_at(S.a, i & 15, i >> 4);
        } else {
            const int cc = (i - 256) >> 6, j = (i - 256) & 63, cy = mby * 8 + (j >> 3), cx = mbx * 8 + (j & 7);
            r = reinterpret_cast<const T*>(C.rec[1 + cc])[(size_t)cy * C.cs + cx];
            s = SC[(size_t)cc * C.cw * C.ch + (size_t)cy * C.cw + cx];
        }
        dst[i] = (T)r;
        const long long d = s - r;
        if (i < 256) ssd += d * d;
        else cssd += d * d;
    }
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) {
        ssd += __shfl_xor_sync(FULL, ssd, off);
        cssd += __shfl_xor_sync(FULL, cssd, off);
    }
    if (lane == 0) {
        R.ssd[k] = ssd + cssd;
        R.cssd[k] = cssd;
        R.valid[k] = 1;
    }
    __syncwarp();
}

// An intra candidate's chroma taken from another's (code_intra_chroma's outputs: mode, DC and AC levels, counts).
__device__ __forceinline__ void rd_chroma_copy(const ironav_mbcode& from, ironav_mbcode* o) {
    const int lane = threadIdx.x & 31;
    __syncwarp();
    const uint32_t* ac = reinterpret_cast<const uint32_t*>(from.res.cac);
    uint32_t* oc = reinterpret_cast<uint32_t*>(o->res.cac);
    for (int i = lane; i < (int)(sizeof(from.res.cac) / 4); i += 32) oc[i] = ac[i];
    if (lane < (int)(sizeof(from.res.cdc) / 4)) reinterpret_cast<uint32_t*>(o->res.cdc)[lane] = reinterpret_cast<const uint32_t*>(from.res.cdc)[lane];
    if (lane < (int)(sizeof(from.res.cnnz) / 4))
        reinterpret_cast<uint32_t*>(o->res.cnnz)[lane] = reinterpret_cast<const uint32_t*>(from.res.cnnz)[lane];
    if (lane == 0) o->chroma_mode = from.chroma_mode;
    __syncwarp();
}

// Candidates k0 .. k0 + nk - 1 priced on this warp (rd_cost, enc/frame.rs:1453-1457): each from its own copy
// of the contexts, a lane per (candidate, group of disjoint contexts), the groups' bits summed into R.bits.
// coarse: five lanes a candidate, each residual category's map and levels on one lane (six candidates fit
// the warp at once).
template <class T, int W>
__device__ void rd_count(RdSmem<T, W>& R, const cab::Slice& sl, const int* nbm, int k0, int nk, bool coarse = false) {
    const int lane = threadIdx.x & 31;
    for (int k = k0; k < k0 + nk; k++) {
        if (!R.valid[k]) continue;
        const uint32_t* s32 = reinterpret_cast<const uint32_t*>(R.live);
        uint32_t* d32 = reinterpret_cast<uint32_t*>(R.cst[k]);
        for (int i = lane; i < 256; i += 32) d32[i] = s32[i];
    }
    if (lane < nk) R.bits[k0 + lane] = 0;
    __syncwarp();
    const int ng = coarse ? (cab::NGROUPS + 1) / 2 : cab::NGROUPS;
    const int k = k0 + lane / ng, g = lane % ng;
    if (lane < nk * ng && R.valid[k]) {
        cab::Counter c = {R.cst[k], R.step, 0};
        if (!coarse || g == 0) {
            cab::mb_bins(c, sl, &R.cand[k], R.nb[0], R.nb[1], nbm, g);
        } else {
            cab::mb_bins(c, sl, &R.cand[k], R.nb[0], R.nb[1], nbm, 2 * g - 1);
            cab::mb_bins(c, sl, &R.cand[k], R.nb[0], R.nb[1], nbm, 2 * g);
        }
        if (c.bits) atomicAdd(&R.bits[k], c.bits);
    }
    __syncwarp();
}

// The MbState of a coded candidate: the inter ones' from inter_tail (S.a.out), the intra ones' without motion.
template <class T, int W>
__device__ __forceinline__ void rd_state(RdSmem<T, W>& R, const DecideSmem<T>& S, int k, bool inter) {
    const int lane = threadIdx.x & 31;
    __syncwarp();
    uint32_t* d = reinterpret_cast<uint32_t*>(&R.state[k]);
    if (inter) {
        if (lane < 18) d[lane] = reinterpret_cast<const uint32_t*>(&S.a.out)[lane];
    } else {
        // inter 0, refs -1, pad 0, no motion (bytes 0-7, then the vectors)
        if (lane < 18) d[lane] = lane == 0 ? 0xFFFFFF00u : (lane == 1 ? 0x000000FFu : 0u);
    }
    __syncwarp();
}

// decide_rd for one macroblock (after code_mb's P_Skip tests, best_i16 and best_inter; enc/frame.rs:715-760,
// 1462-1513), its bins then carried into the chain's contexts (write_mb_cabac's effect on them, 2020-2025).
template <class T>
__device__ void rd_mb(const RdParams& P, RdSmem<T, 1>& R, const unsigned* i4tab, int mb, int mbx, int mby) {
    const int lane = threadIdx.x & 31;
    const DecideParams& D = P.D;
    const AnalyseParams& A = D.C.A;
    const CodeParams& C = D.C;
    DecideSmem<T>& S = R.s[0];
    const bool ta = mby > A.band_start[mby], la = mbx > 0, tra = ta && mbx + 1 < A.mb_w;
    const cab::Slice sl = {D.intra ? 0 : 1, P.t8, D.intra ? 0 : A.nact};
    ironav_mbcode* out = &D.codes[mb];
    ironav_mbcode* cand = R.cand;
    code_init(out);
    stage_source(A, S.a);
    // the neighbours for the contexts: the left one is the macroblock just decided, the top one's was kept
    if (lane < cab::NB_WORDS) {
        uint32_t* l = reinterpret_cast<uint32_t*>(&R.nb[0]);
        uint32_t* t = reinterpret_cast<uint32_t*>(&R.nb[1]);
        l[lane] = la ? reinterpret_cast<const uint32_t*>(&R.done)[lane] : 0u;
        t[lane] = ta ? P.nbs[(size_t)(mb - A.mb_w) * cab::NB_WORDS + lane] : 0u;
    }
    if (lane < RD_CANDS) R.valid[lane] = 0;
    __syncwarp();
    int2 sv = make_int2(0, 0);
    if (!D.intra && skip_tests_d<T>(D, S, mb, mbx, mby, out, &sv)) {
        // P_Skip without a rate-distortion choice; its one bin still moves the contexts
        if (lane == 0) {
            cab::Counter c = {R.live, R.step, 0};
            cab::mb_bins(c, sl, out, R.nb[0], R.nb[1], S.nbm);
        }
        if (lane < 18) reinterpret_cast<uint32_t*>(&A.states_out[mb])[lane] = reinterpret_cast<const uint32_t*>(&S.a.out)[lane];
        __syncwarp();
        cab::nb_of_warp(out, &R.done);
        if (lane < cab::NB_WORDS) P.nbs[(size_t)mb * cab::NB_WORDS + lane] = reinterpret_cast<const uint32_t*>(&R.done)[lane];
        __syncwarp();
        return;
    }
    load_intra_neighbours(D, S, mb, mbx, mby, ta, la, tra);
    const int2 i16 = best_i16_d(D, S, ta, la);
    // best_inter, enc/frame.rs:839-849 (none in an IDR picture)
    int part = 0, cost = BIG, bestr = 0;
    uint32_t sub = 0;
    for (int r = 0; r < A.nact && !D.intra; r++) {
        const int4 bi = best_inter_or_learned(A, S.a, r);
        if (r == 0 || bi.x < cost) {
            part = bi.y;
            cost = bi.x;
            bestr = r;
            sub = (uint32_t)bi.z;
            if (lane < 16) {
                S.a.win_mvs[lane][0] = S.a.best_mvs[lane][0];
                S.a.win_mvs[lane][1] = S.a.best_mvs[lane][1];
            }
            __syncwarp();
        }
    }
    ironav_interdec& Dd = *reinterpret_cast<ironav_interdec*>(S.c.dec);
    if (!D.intra) {
        // P_Skip: the skip vector's prediction is the reconstruction (put_inter_pred, 1391-1394)
        ironav_mbcode* o = &cand[0];
        code_init(o);
        if (lane == 0) {
            Dd.mode = 1;
            Dd.part = 0;
            Dd.t8 = 0;
            for (int k = 0; k < 4; k++) Dd.sub[k] = Dd.refs[k] = 0;
        }
        if (lane < 16) {
            Dd.mvs[lane][0] = (int16_t)sv.x;
            Dd.mvs[lane][1] = (int16_t)sv.y;
        }
        __syncwarp();
        code_inter_mb<T>(C, S.c, mb, &o->res);
        inter_tail(D, S, Dd, o);
        if (lane < 16) o->mvds[lane][0] = o->mvds[lane][1] = 0;
        if (lane == 0) o->skip = 1;
        rd_state(R, S, 0, true);
        rd_take(C, R, S, 0, mbx, mby);
        // best_inter's partitioning with the 4x4 transform; with nothing coded and the skip vector, it would be
        // P_Skip at a higher price
        o = &cand[1];
        code_init(o);
        if (lane == 0) {
            Dd.mode = 2;
            Dd.part = (uint8_t)part;
            Dd.t8 = 0;
            for (int k = 0; k < 4; k++) {
                Dd.sub[k] = (uint8_t)((sub >> (8 * k)) & 0xff);
                Dd.refs[k] = (uint8_t)bestr;
            }
        }
        if (lane < 16) {
            Dd.mvs[lane][0] = S.a.win_mvs[lane][0];
            Dd.mvs[lane][1] = S.a.win_mvs[lane][1];
        }
        __syncwarp();
        const uint32_t cbp = code_inter_mb<T>(C, S.c, mb, &o->res);
        inter_tail(D, S, Dd, o);
        rd_state(R, S, 1, true);
        rd_take(C, R, S, 1, mbx, mby);
        if (lane == 0 && cbp == 0 && part == 0 && Dd.mvs[0][0] == sv.x && Dd.mvs[0][1] == sv.y && bestr == 0) R.valid[1] = 0;
        __syncwarp();
        // the 8x8 transform needs every 8x8 block of P_8x8 to be a single 8x8 partition; without luma levels it
        // would be the 4x4 candidate again
        if (P.t8 && sub == 0) {
            o = &cand[2];
            code_init(o);
            if (lane == 0) Dd.t8 = 1;
            __syncwarp();
            code_inter_mb<T>(C, S.c, mb, &o->res);
            inter_tail(D, S, Dd, o);
            rd_state(R, S, 2, true);
            rd_take(C, R, S, 2, mbx, mby);
            if (lane == 0 && !o->res.t8x8) R.valid[2] = 0;
            __syncwarp();
        }
    }
    // Intra16x16 in best_i16's mode, with its chroma. code_intra_chroma reads only the chroma around the
    // macroblock and writes only its chroma, so the Intra4x4 and Intra8x8 candidates take this one's
    // (its mode, levels, counts and pattern; the reconstruction stays in the picture)
    uint32_t ccbp = 0;
    {
        ironav_mbcode* o = &cand[3];
        code_init(o);
        uint32_t cbp = code_i16_d(D, S, mbx, mby, i16.x, ta, la, o);
        ccbp = code_intra_chroma_d(D, S, mbx, mby, ta, la, o);
        cbp |= ccbp;
        if (lane == 0) {
            o->kind = KIND_I16;
            o->i16_mode = (uint8_t)i16.x;
            o->res.cbp = (uint8_t)cbp;
        }
        rd_state(R, S, 3, false);
        rd_take(C, R, S, 3, mbx, mby);
    }
    // Intra4x4, block by block from its own reconstruction, with its chroma
    {
        ironav_mbcode* o = &cand[4];
        code_init(o);
        code_i4_trial(D, S, i4tab, ta, la, tra);
        T* RY = reinterpret_cast<T*>(C.rec[0]);
        for (int i = lane; i < 256; i += 32) RY[(size_t)(mby * 16 + (i >> 4)) * C.ys + mbx * 16 + (i & 15)] = (T)S.i4rec[i];
        if (lane < 16) {
            uint32_t* lw = reinterpret_cast<uint32_t*>(o->res.luma[lane]);
            const uint32_t* src = reinterpret_cast<const uint32_t*>(S.i4lv[lane]);
#pragma unroll
            for (int k = 0; k < 8; k++) lw[k] = src[k];
            o->res.nnz[lane] = S.i4nnz[lane];
            o->modes[lane] = S.i4modes[lane];
        }
        const unsigned bal = __ballot_sync(FULL, lane < 16 && S.i4nnz[lane] > 0);
        uint32_t cbp = 0;
#pragma unroll
        for (int i8 = 0; i8 < 4; i8++)
            if (bal & (0x33u << ((i8 >> 1) * 8 + (i8 & 1) * 2))) cbp |= 1u << i8;
        __syncwarp();
        rd_chroma_copy(cand[3], o);
        cbp |= ccbp;
        if (lane == 0) {
            o->kind = KIND_I4;
            o->res.cbp = (uint8_t)cbp;
        }
        rd_state(R, S, 4, false);
        rd_take(C, R, S, 4, mbx, mby);
    }
    // Intra8x8 with its chroma
    if (P.t8) {
        ironav_mbcode* o = &cand[5];
        code_init(o);
        uint32_t cbp = code_i8_d(D, S, R, mbx, mby, ta, la, tra, o, reinterpret_cast<T*>(C.rec[0]), C.ys);
        rd_chroma_copy(cand[3], o);
        cbp |= ccbp;
        if (lane == 0) o->res.cbp = (uint8_t)cbp;
        rd_state(R, S, 5, false);
        rd_take(C, R, S, 5, mbx, mby);
    }
    // rd_cost (1453-1457): the candidates priced at once (five lanes each); then lane 0 keeps the least SSD +
    // lam2 * bits in the reference's order (strict '<'), in f64 rounded as the reference's expression is (no
    // fused multiply-add).
    rd_count(R, sl, S.nbm, 0, RD_CANDS, true);
    if (lane == 0) {
        int best = -1;
        double bj = 0.0;
        for (int k = 0; k < RD_CANDS; k++) {
            if (!R.valid[k]) continue;
            const double j = __dadd_rn(__ll2double_rn(R.ssd[k]), __dmul_rn(P.lam2, __dmul_rn((double)R.bits[k], 0.00390625)));
            if (best < 0 || j < bj) best = k, bj = j;
        }
        R.best = best;
    }
    __syncwarp();
    const int b = R.best;
    {
        const uint32_t* s32 = reinterpret_cast<const uint32_t*>(&cand[b]);
        uint32_t* d32 = reinterpret_cast<uint32_t*>(out);
        for (int i = lane; i < (int)(sizeof(ironav_mbcode) / 4); i += 32) d32[i] = s32[i];
        const uint32_t* c32 = reinterpret_cast<const uint32_t*>(R.cst[b]);
        uint32_t* l32 = reinterpret_cast<uint32_t*>(R.live);
        for (int i = lane; i < 256; i += 32) l32[i] = c32[i];
        const T* rec = R.crec[b];
        for (int i = lane; i < 384; i += 32) {
            if (i < 256) {
                reinterpret_cast<T*>(C.rec[0])[(size_t)(mby * 16 + (i >> 4)) * C.ys + mbx * 16 + (i & 15)] = rec[i];
            } else {
                const int cc = (i - 256) >> 6, j = (i - 256) & 63;
                reinterpret_cast<T*>(C.rec[1 + cc])[(size_t)(mby * 8 + (j >> 3)) * C.cs + mbx * 8 + (j & 7)] = rec[i];
            }
        }
        if (lane < 18) reinterpret_cast<uint32_t*>(&A.states_out[mb])[lane] = reinterpret_cast<const uint32_t*>(&R.state[b])[lane];
    }
    __syncwarp();
    cab::nb_of_warp(&cand[b], &R.done);
    if (lane < cab::NB_WORDS) P.nbs[(size_t)mb * cab::NB_WORDS + lane] = reinterpret_cast<const uint32_t*>(&R.done)[lane];
    __syncwarp();
}

// One chain: slice band `band` in raster order (FrameCoder::encode, enc/frame.rs:461-478) from the slice's
// initial contexts (cabac_init_idc 0, QP_Y).
template <class T>
__device__ void rd_chain(const RdParams& P, RdSmem<T, 1>& R, const unsigned* i4tab, int band) {
    const int lane = threadIdx.x & 31;
    const AnalyseParams& A = P.D.C.A;
    for (int i = lane; i < cab::STEP_ENTRIES; i += 32) R.step[i] = P.step[i];
    for (int i = lane; i < 9 * 64; i += 32) R.i8tab[i] = i8_entry(i >> 6, i & 7, (i >> 3) & 7);
    cab::init_states(R.live, P.D.intra != 0, 0, P.D.C.qp, lane, 32);
    __syncwarp();
    for (int mby = P.band_rows[band]; mby < P.band_rows[band + 1]; mby++)
        for (int mbx = 0; mbx < A.mb_w; mbx++) {
            const int mb = mby * A.mb_w + mbx;
            if (lane == 0) {
                R.s[0].a.mb = mb;
                R.s[0].a.mbx = mbx;
                R.s[0].a.mby = mby;
            }
            __syncwarp();
            load_neighbours(A, R.s[0].a, A.states_out);
            rd_mb<T>(P, R, i4tab, mb, mbx, mby);
        }
}

// Decide mode under CABAC for one stream: CTA i, one warp, walks slice band i.
template <class T>
__global__ void __launch_bounds__(32) decide_rd_kernel(const __grid_constant__ RdParams P) {
    __shared__ RdSmem<T, 1> R;
    __shared__ unsigned i4tab[9 * 17];
    fill_i4tab(i4tab);
    if ((int)blockIdx.x >= P.nbands) return;
    rd_chain<T>(P, R, i4tab, blockIdx.x);
}

// Decide mode under CABAC for many streams in one launch: CTA i walks chains[i] = stream << 16 | band, with
// the stream's parameters from table[stream] (copied into shared memory).
template <class T>
__global__ void __launch_bounds__(32) decide_rd_batch_kernel(const RdParams* __restrict__ table, const uint32_t* __restrict__ chains,
                                                             int nchains) {
    __shared__ RdSmem<T, 1> R;
    __shared__ RdParams prm;
    __shared__ unsigned i4tab[9 * 17];
    fill_i4tab(i4tab);
    if ((int)blockIdx.x >= nchains) return;
    const int lane = threadIdx.x & 31;
    const uint32_t e = chains[blockIdx.x];
    const uint32_t* src = reinterpret_cast<const uint32_t*>(&table[e >> 16]);
    for (int k = lane; k < (int)(sizeof(RdParams) / 4); k += 32) reinterpret_cast<uint32_t*>(&prm)[k] = src[k];
    __syncwarp();
    rd_chain<T>(prm, R, i4tab, (int)(e & 0xFFFFu));
}

// ---- the three-warp form: one chain's macroblock on three warps ----------------------------------------
// Warp 0 runs code_mb's P_Skip tests; when the macroblock passes them, warp 0 runs best_inter and codes its
// partitioning with the 4x4 transform into the picture, warp 1 codes P_Skip, Intra4x4 and Intra8x8, and warp 2
// Intra16x16 (with the intra chroma) and then the partitioning with the 8x8 transform (best_inter's
// decision handed over through named barrier 1, which warp 0 arrives at and warp 2 waits on), warps 1 and
// 2 each into their own scratch planes (their edges read from the picture, which warp 0 writes only inside
// the macroblock). The three warps then price two candidates each, and warp 0 commits the kept one. The
// warps meet at CTA barriers (after the P_Skip tests; when there are candidates, after them and after the
// pricing; after the commit), every warp at every one.
constexpr int RD3_WARPS = 3;

template <class T>
__device__ void rd_mb3(const RdParams& P, const DecideParams* dw, RdSmem<T, RD3_WARPS>& R, const unsigned* i4tab, int mb, int mbx,
                       int mby) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const DecideParams& D = P.D;
    const AnalyseParams& A = D.C.A;
    const CodeParams& C = D.C;
    DecideSmem<T>& S = R.s[w];
    const bool ta = mby > A.band_start[mby], la = mbx > 0, tra = ta && mbx + 1 < A.mb_w;
    const cab::Slice sl = {D.intra ? 0 : 1, P.t8, D.intra ? 0 : A.nact};
    ironav_mbcode* out = &D.codes[mb];
    ironav_mbcode* cand = R.cand;
    if (lane == 0) {
        S.a.mb = mb;
        S.a.mbx = mbx;
        S.a.mby = mby;
    }
    __syncwarp();
    stage_source(A, S.a);
    int2 sv = make_int2(0, 0);
    if (w == 0) {
        load_neighbours(A, S.a, A.states_out);
        code_init(out);
        if (lane < cab::NB_WORDS) {
            reinterpret_cast<uint32_t*>(&R.nb[0])[lane] = la ? reinterpret_cast<const uint32_t*>(&R.done)[lane] : 0u;
            reinterpret_cast<uint32_t*>(&R.nb[1])[lane] = ta ? P.nbs[(size_t)(mb - A.mb_w) * cab::NB_WORDS + lane] : 0u;
        }
        if (lane < RD_CANDS) R.valid[lane] = 0;
        __syncwarp();
        const bool skip = !D.intra && skip_tests_d<T>(D, S, mb, mbx, mby, out, &sv);
        if (lane == 0) {
            R.skip = skip;
            R.sv = sv;
        }
    }
    __syncthreads();
    if (R.skip) {
        if (w == 0) {
            // P_Skip without a rate-distortion choice; its one bin still moves the contexts
            if (lane == 0) {
                cab::Counter c = {R.live, R.step, 0};
                cab::mb_bins(c, sl, out, R.nb[0], R.nb[1], S.nbm);
            }
            if (lane < 18) reinterpret_cast<uint32_t*>(&A.states_out[mb])[lane] = reinterpret_cast<const uint32_t*>(&S.a.out)[lane];
            __syncwarp();
            cab::nb_of_warp(out, &R.done);
            if (lane < cab::NB_WORDS) P.nbs[(size_t)mb * cab::NB_WORDS + lane] = reinterpret_cast<const uint32_t*>(&R.done)[lane];
            __syncwarp();
        }
        __syncthreads();
        return;
    }
    load_intra_neighbours(D, S, mb, mbx, mby, ta, la, tra);
    if (w == 0 && !D.intra) {
        // best_inter, enc/frame.rs:839-849; its decision goes to warp 2 (the 8x8-transform candidate) through
        // named barrier 1, and warp 0 codes it with the 4x4 transform
        int part = 0, cost = BIG, bestr = 0;
        uint32_t sub = 0;
        for (int r = 0; r < A.nact; r++) {
            const int4 bi = best_inter_or_learned(A, S.a, r);
            if (r == 0 || bi.x < cost) {
                part = bi.y;
                cost = bi.x;
                bestr = r;
                sub = (uint32_t)bi.z;
                if (lane < 16) {
                    S.a.win_mvs[lane][0] = S.a.best_mvs[lane][0];
                    S.a.win_mvs[lane][1] = S.a.best_mvs[lane][1];
                }
                __syncwarp();
            }
        }
        ironav_interdec& Dd = *reinterpret_cast<ironav_interdec*>(S.c.dec);
        if (lane == 0) {
            Dd.mode = 2;
            Dd.part = (uint8_t)part;
            Dd.t8 = 0;
            for (int k = 0; k < 4; k++) {
                Dd.sub[k] = (uint8_t)((sub >> (8 * k)) & 0xff);
                Dd.refs[k] = (uint8_t)bestr;
            }
            R.try_t8 = P.t8 && sub == 0;
        }
        if (lane < 16) {
            Dd.mvs[lane][0] = S.a.win_mvs[lane][0];
            Dd.mvs[lane][1] = S.a.win_mvs[lane][1];
        }
        __syncwarp();
        if (P.t8) {
            for (int i = lane; i < 40; i += 32) R.idec[i] = S.c.dec[i];
            __threadfence_block();
            __syncwarp();
            asm volatile("bar.arrive 1, 64;" ::: "memory");
        }
        ironav_mbcode* o = &cand[1];
        code_init(o);
        const uint32_t cbp = code_inter_mb<T>(C, S.c, mb, &o->res);
        inter_tail(D, S, Dd, o);
        rd_state(R, S, 1, true);
        rd_take(C, R, S, 1, mbx, mby);
        const int2 sv = R.sv;
        if (lane == 0 && cbp == 0 && part == 0 && Dd.mvs[0][0] == sv.x && Dd.mvs[0][1] == sv.y && bestr == 0) R.valid[1] = 0;
        __syncwarp();
    } else if (w == 1) {
        const DecideParams& Dw = dw[0];
        if (!D.intra) {
            // P_Skip: the skip vector's prediction is the reconstruction (put_inter_pred, 1391-1394), into warp
            // 1's planes; a P_Skip code carries no differences, its state the vector over the macroblock
            const int2 sv = R.sv;
            ironav_mbcode* o = &cand[0];
            code_init(o);
            ironav_interdec& Dd = *reinterpret_cast<ironav_interdec*>(S.c.dec);
            if (lane == 0) {
                Dd.mode = 1;
                Dd.part = 0;
                Dd.t8 = 0;
                for (int k = 0; k < 4; k++) Dd.sub[k] = Dd.refs[k] = 0;
                o->kind = KIND_INTER;
                o->skip = 1;
            }
            if (lane < 16) {
                Dd.mvs[lane][0] = (int16_t)sv.x;
                Dd.mvs[lane][1] = (int16_t)sv.y;
                o->mvs[lane][0] = (int16_t)sv.x;
                o->mvs[lane][1] = (int16_t)sv.y;
            }
            __syncwarp();
            code_inter_mb<T>(Dw.C, S.c, mb, &o->res);
            uint32_t* d = reinterpret_cast<uint32_t*>(&R.state[0]);
            if (lane < 18) d[lane] = lane == 0 ? 1u : (lane == 1 ? 0u : ((uint32_t)(uint16_t)sv.x | (uint32_t)(uint16_t)sv.y << 16));
            __syncwarp();
            rd_take(Dw.C, R, S, 0, mbx, mby);
        }
        // Intra4x4 into warp 1's luma plane; its chroma is Intra16x16's (taken after the barrier)
        ironav_mbcode* o = &cand[4];
        code_init(o);
        code_i4_trial(Dw, S, i4tab, ta, la, tra);
        T* RY = reinterpret_cast<T*>(Dw.C.rec[0]);
        for (int i = lane; i < 256; i += 32) RY[(size_t)(mby * 16 + (i >> 4)) * Dw.C.ys + mbx * 16 + (i & 15)] = (T)S.i4rec[i];
        if (lane < 16) {
            uint32_t* lw = reinterpret_cast<uint32_t*>(o->res.luma[lane]);
            const uint32_t* src = reinterpret_cast<const uint32_t*>(S.i4lv[lane]);
#pragma unroll
            for (int k = 0; k < 8; k++) lw[k] = src[k];
            o->res.nnz[lane] = S.i4nnz[lane];
            o->modes[lane] = S.i4modes[lane];
        }
        const unsigned bal = __ballot_sync(FULL, lane < 16 && S.i4nnz[lane] > 0);
        uint32_t cbp = 0;
#pragma unroll
        for (int i8 = 0; i8 < 4; i8++)
            if (bal & (0x33u << ((i8 >> 1) * 8 + (i8 & 1) * 2))) cbp |= 1u << i8;
        if (lane == 0) {
            o->kind = KIND_I4;
            o->res.cbp = (uint8_t)cbp;
        }
        rd_state(R, S, 4, false);
        rd_take(Dw.C, R, S, 4, mbx, mby, false);
        if (P.t8) {
            // Intra8x8 into warp 1's luma plane (its edges from the picture); its chroma too is Intra16x16's
            o = &cand[5];
            code_init(o);
            const uint32_t cbp8 = code_i8_d(D, S, R, mbx, mby, ta, la, tra, o, reinterpret_cast<T*>(Dw.C.rec[0]), Dw.C.ys);
            if (lane == 0) o->res.cbp = (uint8_t)cbp8;
            rd_state(R, S, 5, false);
            rd_take(Dw.C, R, S, 5, mbx, mby, false);
        }
    } else if (w == 2) {
        // Intra16x16 in best_i16's mode with the intra chroma, then Intra8x8, into warp 2's planes
        const DecideParams& Dw = dw[1];
        const int2 i16 = best_i16_d(Dw, S, ta, la);
        ironav_mbcode* o = &cand[3];
        code_init(o);
        uint32_t cbp = code_i16_d(Dw, S, mbx, mby, i16.x, ta, la, o);
        const uint32_t ccbp = code_intra_chroma_d(Dw, S, mbx, mby, ta, la, o);
        cbp |= ccbp;
        if (lane == 0) {
            o->kind = KIND_I16;
            o->i16_mode = (uint8_t)i16.x;
            o->res.cbp = (uint8_t)cbp;
            R.ccbp = ccbp;
        }
        rd_state(R, S, 3, false);
        rd_take(Dw.C, R, S, 3, mbx, mby);
        if (P.t8 && !D.intra) {
            // best_inter's partitioning with the 8x8 transform (when no 8x8 block is split; without luma levels it
            // would be the 4x4 candidate again), once warp 0 has handed its decision over
            asm volatile("bar.sync 1, 64;" ::: "memory");
            if (R.try_t8) {
                load_neighbours(A, S.a, A.states_out);
                for (int i = lane; i < 40; i += 32) S.c.dec[i] = R.idec[i];
                __syncwarp();
                ironav_interdec& Dd = *reinterpret_cast<ironav_interdec*>(S.c.dec);
                if (lane == 0) Dd.t8 = 1;
                __syncwarp();
                o = &cand[2];
                code_init(o);
                code_inter_mb<T>(Dw.C, S.c, mb, &o->res);
                inter_tail(D, S, Dd, o);
                rd_state(R, S, 2, true);
                rd_take(Dw.C, R, S, 2, mbx, mby);
                if (lane == 0 && !o->res.t8x8) R.valid[2] = 0;
                __syncwarp();
            }
        }
    }
    __syncthreads();
    // the candidates priced two a warp (warp 2 first gives Intra4x4 and Intra8x8 Intra16x16's chroma: code,
    // reconstruction and squared error), then warp 0 keeps the least cost in order and commits it
    if (w == 2) {
        for (int k = 4; k <= (P.t8 ? 5 : 4); k++) {
            rd_chroma_copy(cand[3], &cand[k]);
            if (lane == 0) {
                cand[k].res.cbp |= (uint8_t)R.ccbp;
                R.ssd[k] += R.cssd[3];
                R.cssd[k] = R.cssd[3];
            }
            for (int i = 256 + lane; i < 384; i += 32) R.crec[k][i] = R.crec[3][i];
            __syncwarp();
        }
    }
    rd_count(R, sl, S.nbm, 2 * w, 2);
    __syncthreads();
    if (w == 0) {
        if (lane == 0) {
            int best = -1;
            double bj = 0.0;
            for (int k = 0; k < RD_CANDS; k++) {
                if (!R.valid[k]) continue;
                const double j = __dadd_rn(__ll2double_rn(R.ssd[k]), __dmul_rn(P.lam2, __dmul_rn((double)R.bits[k], 0.00390625)));
                if (best < 0 || j < bj) best = k, bj = j;
            }
            R.best = best;
        }
        __syncwarp();
        const int b = R.best;
        const uint32_t* s32 = reinterpret_cast<const uint32_t*>(&cand[b]);
        uint32_t* d32 = reinterpret_cast<uint32_t*>(out);
        for (int i = lane; i < (int)(sizeof(ironav_mbcode) / 4); i += 32) d32[i] = s32[i];
        const uint32_t* c32 = reinterpret_cast<const uint32_t*>(R.cst[b]);
        uint32_t* l32 = reinterpret_cast<uint32_t*>(R.live);
        for (int i = lane; i < 256; i += 32) l32[i] = c32[i];
        const T* rec = R.crec[b];
        for (int i = lane; i < 384; i += 32) {
            if (i < 256) {
                reinterpret_cast<T*>(C.rec[0])[(size_t)(mby * 16 + (i >> 4)) * C.ys + mbx * 16 + (i & 15)] = rec[i];
            } else {
                const int cc = (i - 256) >> 6, j = (i - 256) & 63;
                reinterpret_cast<T*>(C.rec[1 + cc])[(size_t)(mby * 8 + (j >> 3)) * C.cs + mbx * 8 + (j & 7)] = rec[i];
            }
        }
        if (lane < 18) reinterpret_cast<uint32_t*>(&A.states_out[mb])[lane] = reinterpret_cast<const uint32_t*>(&R.state[b])[lane];
        __syncwarp();
        cab::nb_of_warp(&cand[b], &R.done);
        if (lane < cab::NB_WORDS) P.nbs[(size_t)mb * cab::NB_WORDS + lane] = reinterpret_cast<const uint32_t*>(&R.done)[lane];
        __syncwarp();
    }
    __syncthreads();
}

// The three-warp form's set-up and chain walk for the parameters P (in parameter space or shared memory):
// warps 1 and 2's parameter copies writing into their scratch planes, the CTA's tables and contexts, then
// slice band `band` in raster order.
template <class T>
__device__ void rd3_chain(const RdParams& P, DecideParams* dw, RdSmem<T, RD3_WARPS>& R, unsigned* i4tab, int band) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (w > 0) {
        const uint32_t* src = reinterpret_cast<const uint32_t*>(&P.D);
        uint32_t* dst = reinterpret_cast<uint32_t*>(&dw[w - 1]);
        for (int k = lane; k < (int)(sizeof(DecideParams) / 4); k += 32) dst[k] = src[k];
        __syncwarp();
        if (lane == 0) {
            for (int k = 0; k < 3; k++) dw[w - 1].C.rec[k] = P.scr[3 * (w - 1) + k];
            dw[w - 1].C.ys = P.scr_ys;
            dw[w - 1].C.cs = P.scr_cs;
        }
    }
    fill_i4tab(i4tab);  // its __syncthreads also publishes dw
    const AnalyseParams& A = P.D.C.A;
    for (int i = threadIdx.x; i < cab::STEP_ENTRIES; i += blockDim.x) R.step[i] = P.step[i];
    for (int i = threadIdx.x; i < 9 * 64; i += blockDim.x) R.i8tab[i] = i8_entry(i >> 6, i & 7, (i >> 3) & 7);
    cab::init_states(R.live, P.D.intra != 0, 0, P.D.C.qp, threadIdx.x, blockDim.x);
    __syncthreads();
    for (int mby = P.band_rows[band]; mby < P.band_rows[band + 1]; mby++)
        for (int mbx = 0; mbx < A.mb_w; mbx++) rd_mb3<T>(P, dw, R, i4tab, mby * A.mb_w + mbx, mbx, mby);
}

// Decide mode under CABAC for one stream, three warps a chain: CTA i walks slice band i.
template <class T>
__global__ void __launch_bounds__(RD3_WARPS * 32) decide_rd3_kernel(const __grid_constant__ RdParams P) {
    extern __shared__ __align__(16) unsigned char rd3_smem[];
    __shared__ DecideParams dw[2];
    __shared__ unsigned i4tab[9 * 17];
    if ((int)blockIdx.x >= P.nbands) return;
    rd3_chain<T>(P, dw, *reinterpret_cast<RdSmem<T, RD3_WARPS>*>(rd3_smem), i4tab, blockIdx.x);
}

// The same for many streams' chains: CTA i walks chains[i] = stream << 16 | band with the stream's
// parameters from table[stream] (copied into shared memory).
template <class T>
__global__ void __launch_bounds__(RD3_WARPS * 32) decide_rd3_batch_kernel(const RdParams* __restrict__ table,
                                                                          const uint32_t* __restrict__ chains, int nchains) {
    extern __shared__ __align__(16) unsigned char rd3_smem[];
    __shared__ RdParams prm;
    __shared__ DecideParams dw[2];
    __shared__ unsigned i4tab[9 * 17];
    if ((int)blockIdx.x >= nchains) return;
    const uint32_t e = chains[blockIdx.x];
    const uint32_t* src = reinterpret_cast<const uint32_t*>(&table[e >> 16]);
    for (int k = threadIdx.x; k < (int)(sizeof(RdParams) / 4); k += blockDim.x) reinterpret_cast<uint32_t*>(&prm)[k] = src[k];
    __syncthreads();
    rd3_chain<T>(prm, dw, *reinterpret_cast<RdSmem<T, RD3_WARPS>*>(rd3_smem), i4tab, (int)(e & 0xFFFFu));
}

template <class T>
constexpr size_t rd3_smem_bytes() { return sizeof(RdSmem<T, RD3_WARPS>); }

// ---- the CABAC slice writer ---------------------------------------------------------------------------

// What the writer reads of a macroblock as a neighbour: its Nb, and the Intra NxN modes of its right column
// and bottom row (2 for a macroblock that is neither Intra4x4 nor Intra8x8), as pred_mode reads them.
struct WrNb {
    cab::Nb nb;
    int8_t rmodes[4], bmodes[4];
};
constexpr int WRNB_WORDS = (int)(sizeof(WrNb) / 4);
static_assert(sizeof(WrNb) % 4 == 0, "WrNb in whole words");

struct CabacWriteParams {
    const ironav_mbcode* codes;
    WrNb* nbs;              // per macroblock, filled by cabac_nb_kernel
    const int* band_rows;
    const uint32_t* step;
    uint32_t* out;          // slice i's data at out + i * region_words
    uint32_t region_words;
    uint32_t* slice_bytes;  // per slice: its data's bytes; [nbands]: set when a slice outgrew its region
    int mb_w, nmb, nbands, intra, t8, nref, qp;
};

// Every macroblock's WrNb, a warp a macroblock (grid-stride): the neighbours' side of the writer's walk,
// worked out for the whole picture at once.
static __global__ void __launch_bounds__(128) cabac_nb_kernel(const __grid_constant__ CabacWriteParams P) {
    const int lane = threadIdx.x & 31;
    const int warps = (int)(gridDim.x * blockDim.x) >> 5;
    for (int mb = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); mb < P.nmb; mb += warps) {
        const ironav_mbcode* k = &P.codes[mb];
        cab::nb_of_warp(k, &P.nbs[mb].nb);
        if (lane < 8) {
            const bool n = cab::nxn(k->kind);
            if (lane < 4) P.nbs[mb].rmodes[lane] = (int8_t)(n ? k->modes[lane * 4 + 3] : 2);
            else P.nbs[mb].bmodes[lane - 4] = (int8_t)(n ? k->modes[12 + lane - 4] : 2);
        }
        __syncwarp();
    }
}

// A slice band's data (FrameCoder::encode with write_mb_cabac, enc/frame.rs:461-486): each macroblock's bins
// (mb_bins) then end_of_slice_flag, arithmetic coded from the slice's contexts; the data starts on the byte
// that follows the header's cabac_alignment_one_bit (written on the host). CTA i walks slice band i: lane 0
// codes a macroblock's bins while lanes 1-31 bring the next one's code and its neighbours' WrNb into the
// other half of a double buffer in shared memory.
static __global__ void __launch_bounds__(32) cabac_write_kernel(const __grid_constant__ CabacWriteParams P) {
    __shared__ uint8_t st[1024];
    __shared__ uint32_t step[cab::STEP_ENTRIES];
    __shared__ ironav_mbcode code[2];
    __shared__ WrNb nb[2][2];  // [buffer][left, top]
    __shared__ int over;
    const int chain = blockIdx.x, lane = threadIdx.x & 31;
    if (chain >= P.nbands) return;
    for (int i = lane; i < cab::STEP_ENTRIES; i += 32) step[i] = P.step[i];
    cab::init_states(st, P.intra != 0, 0, P.qp, lane, 32);
    if (lane == 0) over = 0;
    cab::BitOut bo = {P.out + (size_t)chain * P.region_words, P.region_words, 0, 0ull, 0, false};
    cab::Coder k = {st, step, &bo, 0u, 510u, 0u, true};
    const cab::Slice sl = {P.intra ? 0 : 1, P.t8, P.intra ? 0 : P.nref};
    const int r0 = P.band_rows[chain], r1 = P.band_rows[chain + 1];
    const int first = r0 * P.mb_w, end = r1 * P.mb_w;
    constexpr int W = (int)(sizeof(ironav_mbcode) / 4);
    // macroblock `mb`'s code and its neighbours' WrNb into buffer b, by lanes lo..31 (zeros: not in the slice)
    auto fetch = [&](int mb, int b, int lo) {
        const int mbx = mb % P.mb_w;
        const bool la = mbx > 0, ta = mb - P.mb_w >= first;
        const uint32_t* g = reinterpret_cast<const uint32_t*>(&P.codes[mb]);
        uint32_t* c = reinterpret_cast<uint32_t*>(&code[b]);
        for (int i = lane - lo; i < W; i += 32 - lo) c[i] = g[i];
        uint32_t* l = reinterpret_cast<uint32_t*>(&nb[b][0]);
        uint32_t* t = reinterpret_cast<uint32_t*>(&nb[b][1]);
        const uint32_t* gl = reinterpret_cast<const uint32_t*>(&P.nbs[la ? mb - 1 : mb]);
        const uint32_t* gt = reinterpret_cast<const uint32_t*>(&P.nbs[ta ? mb - P.mb_w : mb]);
        for (int i = lane - lo; i < 2 * WRNB_WORDS; i += 32 - lo) {
            if (i < WRNB_WORDS) l[i] = la ? gl[i] : 0u;
            else t[i - WRNB_WORDS] = ta ? gt[i - WRNB_WORDS] : 0u;
        }
    };
    fetch(first, 0, 0);
    __syncwarp();
    for (int mb = first; mb < end; mb++) {
        const int b = (mb - first) & 1;
        if (lane == 0) {
            int nbm[8];
            const bool la = nb[b][0].nb.avail, ta = nb[b][1].nb.avail;
            for (int q = 0; q < 4; q++) {
                nbm[q] = la ? nb[b][0].rmodes[q] : -1;
                nbm[4 + q] = ta ? nb[b][1].bmodes[q] : -1;
            }
            cab::mb_bins(k, sl, &code[b], nb[b][0].nb, nb[b][1].nb, nbm);
            k.terminate(mb + 1 == end);
            over = bo.over;
        } else if (mb + 1 < end) {
            fetch(mb + 1, b ^ 1, 1);
        }
        __syncwarp();
        if (over) break;
    }
    if (lane == 0) {
        const uint32_t bytes = bo.finish();
        P.slice_bytes[chain] = bytes;
        if (bo.over) atomicOr(&P.slice_bytes[P.nbands], 1u);
    }
}

}  // namespace ironav
