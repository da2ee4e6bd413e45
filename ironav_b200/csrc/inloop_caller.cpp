// inloop_caller.cpp — a native caller of in-loop mode: the encoder's slice threads (FrameCoder::encode on one
// thread per slice band, crates/ironav-codec/src/h264/enc/mod.rs:620-628 and enc/frame.rs:467-478) driving
// include/ironav_inter.h's in-loop entry points as a host encoder would. Each thread walks its band in raster
// order: it waits for a macroblock's analysis (ironav_inloop_result), makes the final decision itself and
// commits it (ironav_inloop_commit, finish_mb's MbState, enc/frame.rs:2281-2321). The decision here is the
// stage's auto policy (P_Skip when the skip SAD is under the threshold, else best_inter's partitioning), a
// stand-in for the host's own rate-distortion choice; a host encoder puts its code_mb there.
//
// It is the in-loop workload's caller in bench.py, in native threads so that what is measured is the
// device's waits and the round trips through mapped host memory, not an interpreter's.
#include <cstring>
#include <thread>
#include <vector>

#include "../../include/ironav_inter.h"

namespace {

// Sub-partitions of P_8x8 and the partitionings (SUB / PARTS, enc/frame.rs:182-204) in 4x4 blocks: x, y, w, h.
const int SUB[4][4][4] = {{{0, 0, 2, 2}}, {{0, 0, 2, 1}, {0, 1, 2, 1}}, {{0, 0, 1, 2}, {1, 0, 1, 2}},
                          {{0, 0, 1, 1}, {1, 0, 1, 1}, {0, 1, 1, 1}, {1, 1, 1, 1}}};
const int NSUB[4] = {1, 2, 2, 4};
const int PARTS[4][4][4] = {{{0, 0, 4, 4}}, {{0, 0, 4, 2}, {0, 2, 4, 2}}, {{0, 0, 2, 4}, {2, 0, 2, 4}},
                            {{0, 0, 2, 2}, {2, 0, 2, 2}, {0, 2, 2, 2}, {2, 2, 2, 2}}};
const int NPARTS[4] = {1, 2, 2, 4};

// The MbState of a decided P macroblock: P_Skip with its vector, or the best_inter partitioning's vectors
// painted over its 4x4 blocks with each 8x8 block's reference index.
void decided_state(const ironav_mbresult& r, bool skip, ironav_mbstate& s) {
    memset(&s, 0, sizeof(s));
    s.inter = 1;
    if (skip) {
        for (int i = 0; i < 16; i++) {
            s.mvs[i][0] = r.skip_mv[0];
            s.mvs[i][1] = r.skip_mv[1];
        }
        return;
    }
    int q = 0;
    for (int p = 0; p < NPARTS[r.part]; p++) {
        const int* pr = PARTS[r.part][p];
        const int nsub = r.part == 3 ? NSUB[r.sub[p]] : 1;
        for (int k = 0; k < nsub; k++, q++) {
            const int x = r.part == 3 ? pr[0] + SUB[r.sub[p]][k][0] : pr[0], y = r.part == 3 ? pr[1] + SUB[r.sub[p]][k][1] : pr[1];
            const int w = r.part == 3 ? SUB[r.sub[p]][k][2] : pr[2], h = r.part == 3 ? SUB[r.sub[p]][k][3] : pr[3];
            for (int by = y; by < y + h; by++)
                for (int bx = x; bx < x + w; bx++) {
                    s.mvs[by * 4 + bx][0] = r.mvs[q][0];
                    s.mvs[by * 4 + bx][1] = r.mvs[q][1];
                }
        }
    }
    for (int b8 = 0; b8 < 4; b8++) {
        const int bx = (b8 % 2) * 2, by = (b8 / 2) * 2;
        int k = 0;
        if (r.part == 1) k = by >= 2;
        else if (r.part == 2) k = bx >= 2;
        else if (r.part == 3) k = b8;
        s.refs[b8] = (int8_t)r.refs[k];
    }
}

}  // namespace

// Runs one P picture in in-loop mode with one caller thread per band: band_rows holds nbands + 1 macroblock
// rows (the context's bands), skip_thresh the P_Skip threshold. The decisions go to states and the results
// to results (mb_w * mb_h each). Returns the first non-zero status of any call.
extern "C" int ironav_inloop_drive_bands(ironav_ctx* ctx, int mb_w, int nbands, const int* band_rows, int skip_thresh,
                                         ironav_mbstate* states, ironav_mbresult* results) {
    int s = ironav_inloop_begin(ctx, IRONAV_INLOOP_BANDS);
    if (s != IRONAV_OK) return s;
    std::vector<int> status(nbands, IRONAV_OK);
    std::vector<std::thread> threads;
    threads.reserve(nbands);
    for (int b = 0; b < nbands; b++)
        threads.emplace_back([&, b] {
            for (int mb = band_rows[b] * mb_w; mb < band_rows[b + 1] * mb_w; mb++) {
                int st = ironav_inloop_result(ctx, mb, &results[mb], 10000);
                if (st == IRONAV_OK) {
                    decided_state(results[mb], results[mb].skip_sad < skip_thresh, states[mb]);
                    st = ironav_inloop_commit(ctx, mb, &states[mb]);
                }
                if (st != IRONAV_OK) {
                    status[b] = st;
                    return;
                }
            }
        });
    for (auto& t : threads) t.join();
    s = ironav_inloop_end(ctx);
    for (int b = 0; b < nbands; b++)
        if (status[b] != IRONAV_OK) return status[b];
    return s;
}
