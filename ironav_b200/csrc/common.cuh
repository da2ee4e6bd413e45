// common.cuh — shared definitions of the sm_100a inter-analysis kernels.
#pragma once
#include <cstdint>

#include "../../include/ironav_inter.h"

namespace ironav {

constexpr int PAD = 48;        // border kept around each half-sample plane (enc/subpel.rs:7)
constexpr int MAX_REFS = 16;   // list-0 length limit (with_refs, enc/mod.rs:265-268)

// The co-located candidate of one macroblock of the newest reference picture (col_mv,
// enc/frame.rs:944-947): mvs[5] of an inter macroblock.
struct ColMv {
    int16_t mv[2];
    int32_t valid;
};

// Everything one analysis launch reads and writes. Passed by value (kernel parameter space).
struct AnalyseParams {
    const uint8_t* src;               // padded source luma, pw x ph, rows ls bytes apart
    int ls;
    const uint8_t* planes[MAX_REFS];  // reference r (0 = newest): G, b, h, j planes, plane k at k * psize
    long long psize;
    int sw;                           // plane stride (pw + 2 * PAD)
    const ColMv* col;                 // newest reference's co-located vectors (mb_w * mb_h)
    int mb_w, mb_h, pw, ph;
    int nact, lambda, skip_thresh, fast, sub8;
    const int* band_start;            // per macroblock row: first row of its slice band
    const ironav_mbstate* states_in;  // replay mode: final decisions of every macroblock
    ironav_mbstate* states_out;       // auto mode: decisions written here
    ironav_mbresult* results;
    // work distribution and the wavefront's progress flags (auto mode)
    const int* order;                 // ticket -> macroblock index
    unsigned* ticket;                 // next ticket
    unsigned* flags;                  // per macroblock: epoch when its decision is published
    unsigned epoch;
    unsigned* err;                    // nonzero: a wait gave up (1) or an index left its plane (2)
    int nmb;
    int withhold;                     // test hook: this macroblock's flag is never published (-1: none)
    unsigned wait_limit;              // polls before a wavefront wait gives up
    // in-loop mode: the caller's final decisions and their flags, and the per-macroblock done flags, all in
    // host memory mapped into the device's address space; results go to host memory too (`results`)
    const ironav_mbstate* committed;
    const unsigned* commit_flags;
    unsigned* done_flags;
    unsigned long long wait_ns;       // how long an in-loop wait for the caller may take
    // B pictures (planes[0]: list 0's reference, planes[1]: list 1's)
    const ironav_mbstate_b* bstates_in;  // final decisions of every macroblock (both lists)
    ironav_bresult* bresults;
    const ironav_mbstate* bcol;       // the list-1 picture's decisions, or nullptr (intra)
    int tb, td;                       // picture distances (FrameCoder::dist)
    // the learned form (nullptr: the plain search): per macroblock 4 proposed vectors (x, y, quarter samples)
    // and the proposed partitioning class (0 P_Skip, 1 16x16, 2 16x8, 3 8x16, 4 8x8); the margin by which the
    // best proposal may cost more than the predictor start before the plain search takes over; counters
    // [0] macroblocks judged from the proposals, [1] fallbacks on the partitioning, [2] fallbacks on the cost
    const int16_t* learned;
    const uint8_t* learned_cls;
    int learned_margin;
    unsigned* learned_stats;
};

// Device-scope acquire load and release store of a progress word shared by warps of different CTAs.
__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(unsigned* p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

}  // namespace ironav
