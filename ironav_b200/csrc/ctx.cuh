// ctx.cuh — the state of one stream's context (ironav_ctx), shared by the translation units of the library.
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "common.cuh"

using ironav::ColMv;
using ironav::MAX_REFS;

// One stream: device buffers, the reference ring, picture parameters and the wavefront scratch.
struct ironav_ctx {
    int width = 0, height = 0, bd = 8, mb_w = 0, mb_h = 0, pw = 0, ph = 0, sw = 0, sh = 0;
    int max_refs = 0, nslices = 0, nmb = 0;
    int device = 0, nsm = 0, k2_blocks = 0;
    int g8_blocks = 0;     // the replay analysis' grid in its group forms (one macroblock per 8 / 16 lanes)
    int g16_blocks = 0, g4_blocks = 0;
    int replay_form = 0;   // replay mode's kernel: 0 8-lane groups, 1 one macroblock per warp, 2 16-lane groups, 3 4-lane groups
    cudaStream_t stream = nullptr;
    long long psize = 0;
    uint8_t* d_src = nullptr;
    uint8_t* d_stage = nullptr;  // reference luma as given, rows pw apart
    uint8_t* d_planes[MAX_REFS] = {};
    ColMv* d_col[MAX_REFS] = {};
    int slot_of[MAX_REFS] = {};  // reference index (0 = newest) -> slot
    int nrefs = 0;
    int* d_band_start = nullptr;
    int* d_order = nullptr;
    unsigned* d_flags = nullptr;
    unsigned* d_counters = nullptr;  // [0] ticket, [1] error
    unsigned epoch = 0;
    ironav_mbstate* d_states = nullptr;
    ironav_mbstate* d_col_stage = nullptr;
    ironav_mbresult* d_results = nullptr;
    // picture parameters
    int qpp = 0, lambda = 0, skip_thresh = 0, nact = 0, fast = 0, sub8 = 0;
    bool have_params = false;
    bool intra_pic = false;  // the parameters are an IDR picture's (ironav_begin_i_picture): decide mode only
    int withhold = -1;
    unsigned wait_limit = 1u << 22;
    // in-loop mode: host memory mapped into the device (allocated on first use)
    int* d_order_bands = nullptr;         // tickets: rows interleaved across bands, raster within each
    ironav_mbresult* h_results = nullptr;
    unsigned* h_done = nullptr;
    ironav_mbstate* h_committed = nullptr;
    unsigned* h_commit = nullptr;
    unsigned inloop_epoch = 0;
    bool inloop_active = false;
    unsigned long long inloop_wait_ns = 10ull * 1000 * 1000 * 1000;
    // scene-cut measure (allocated on first use): two pictures' luma, their low-resolution luma, totals
    uint8_t* d_scene_luma = nullptr;
    uint8_t* d_lowres = nullptr;
    unsigned long long* d_scene_sums = nullptr;
    // deblocking (allocated on first use): per-row progress, the slice table, and for the host-buffer form
    // the macroblock records and the three planes
    unsigned* d_dbk_progress = nullptr;
    ironav_dbk_slice* d_dbk_slices = nullptr;
    int dbk_slice_cap = 0;
    ironav_dbk_mb* d_dbk_mbs = nullptr;
    uint8_t* d_dbk_planes = nullptr;
    void* d_dbk_edges = nullptr;  // per macroblock: strengths and edge thresholds (pass 1 -> pass 2)
    // B pictures: the references used as list 0 and list 1, the list-1 picture's decisions (a copy, or the
    // caller's device pointer), picture distances; host-form buffers allocated on first use
    int b_ref[2] = {0, 0};
    int b_tb = 0, b_td = 0;
    bool b_set = false;
    ironav_mbstate* d_bcol_copy = nullptr;
    const ironav_mbstate* b_col = nullptr;
    ironav_mbstate_b* d_bstates = nullptr;
    ironav_bresult* d_bresults = nullptr;
    // inter residual coding: the source's chroma, each reference slot's chroma (Cb then Cr, 8*mb_w x
    // 8*mb_h each; c_ok: attached since the slot took its picture), host-form staging
    uint8_t* d_src_c = nullptr;
    uint8_t* d_ref_c[MAX_REFS] = {};
    bool ref_c_ok[MAX_REFS] = {};
    ironav_interdec* d_decs = nullptr;
    ironav_intercode* d_codes = nullptr;
    uint8_t* d_rec = nullptr;
    // decide mode: its persistent grid (from the kernel's occupancy, on first use) and host-form codes
    int k7_blocks = 0;
    ironav_mbcode* d_mbcodes = nullptr;
    // the CAVLC writer (allocated on first use): slice band boundaries (nslices + 1 rows), per macroblock
    // its bits, offset and skip run, per slice its bytes, the error word; each slice's first macroblock and
    // each row's slice; the slices' RBSP regions; pinned host staging for the bytes that come back
    // the learned form's proposals (device pointers, nullptr: the plain search) and counters
    const int16_t* learned = nullptr;
    const uint8_t* learned_cls = nullptr;
    int learned_margin = 0;
    unsigned* learned_stats = nullptr;
    int band_rows[1025] = {};
    uint32_t* d_cavlc = nullptr;
    int* d_slice_tab = nullptr;
    uint32_t* d_rbsp = nullptr;
    unsigned long long rbsp_region_words = 0;
    uint32_t* h_cavlc = nullptr;
    uint8_t* h_rbsp = nullptr;
    size_t h_rbsp_cap = 0;
    // CABAC (ironav_set_entropy): the setting; the contexts' step table; the slice bands' rows on the device;
    // the rate-distortion decision's per-macroblock neighbour summaries (cab::Nb); the writer's
    // per-band data regions, byte counts (and overflow word) and their pinned host copy
    int cabac = 0, t8 = 0;
    uint32_t* d_cab_step = nullptr;
    int* d_band_rows = nullptr;
    uint32_t* d_rd_nb = nullptr;
    uint8_t* d_rd_scr = nullptr;  // the three-warp decision's scratch planes
    uint32_t* d_cab_out = nullptr;
    unsigned long long cab_region_words = 0;
    uint32_t* d_cab_bytes = nullptr;
    uint8_t* d_cab_wnb = nullptr;  // the writer's per-macroblock neighbour records
    uint32_t* h_cab_bytes = nullptr;
};


// Helpers the translation units share (ironav_inter.cu).
int take_ref_slot(ironav_ctx* c);
void fill_params(const ironav_ctx* c, ironav::AnalyseParams& p);
// CABAC (ironav_cabac.cu): the step table and band rows on first use; decide mode under CABAC (the
// rate-distortion decision, one chain per slice band) on the device buffers given; the CABAC data of the
// current picture's slices from codes in device memory, one host vector of bytes per slice (each begins on
// the byte after its header's cabac_alignment_one_bit).
int cabac_setup(ironav_ctx* c);
int launch_decide_rd(ironav_ctx* c, ironav_mbstate* d_states, ironav_mbcode* d_codes, void* y, int ys, void* cb, void* cr, int cs);
int cabac_slice_data(ironav_ctx* c, int idr, const ironav_mbcode* d_codes, std::vector<std::vector<uint8_t>>* slices);
