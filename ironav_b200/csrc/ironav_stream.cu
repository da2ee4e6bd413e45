// ironav_stream.cu — the bitstream entry points of include/ironav_inter.h: the CAVLC slices of a picture
// written on the device from its codes (cavlc.cuh), or its CABAC slices (the data arithmetic coded on the
// device, ironav_cabac.cu, behind headers written here), and the sequence and picture parameter sets.
//
// A picture's slices: three launches on the context's stream (sizes, per-slice scan with header and
// trailer, the macroblocks' bits), then each slice's RBSP bytes come back to pinned host memory and go
// into NAL units with emulation prevention on the host (put_nal, enc/bitw.rs:91-103): that pass is a byte
// copy of the output, which has to reach the host anyway.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "cavlc.cuh"
#include "ctx.cuh"

using namespace ironav;

namespace {

int cuda_status(cudaError_t e) {
    if (e == cudaSuccess) return IRONAV_OK;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver || e == cudaErrorNoKernelImageForDevice)
        return IRONAV_HARDWARE_UNAVAILABLE;
    return IRONAV_INTERNAL;
}

#define CK(x)                                          \
    do {                                               \
        cudaError_t e_ = (x);                          \
        if (e_ != cudaSuccess) return cuda_status(e_); \
    } while (0)

// put_nal, enc/bitw.rs:91-103: a four-byte start code, the NAL header, the RBSP with a 3 inserted after
// every two zero bytes that a byte of at most 3 follows.
void put_nal(std::vector<uint8_t>& out, int ref_idc, int kind, const uint8_t* rbsp, size_t n) {
    out.insert(out.end(), {0, 0, 0, 1, (uint8_t)((ref_idc << 5) | kind)});
    int zeros = 0;
    for (size_t i = 0; i < n; i++) {
        const uint8_t b = rbsp[i];
        if (zeros >= 2 && b <= 3) {
            out.push_back(3);
            zeros = 0;
        }
        out.push_back(b);
        zeros = b == 0 ? zeros + 1 : 0;
    }
}

// A host bit writer for the parameter sets (BitWriter, enc/bitw.rs:4-78).
struct HostBits {
    std::vector<uint8_t> buf;
    uint64_t cur = 0;
    unsigned n = 0;
    void put(unsigned k, uint32_t v) {
        cur = (cur << k) | v;
        n += k;
        while (n >= 8) {
            n -= 8;
            buf.push_back((uint8_t)(cur >> n));
        }
        cur &= n ? ((1ull << n) - 1) : 0;
    }
    void flag(bool b) { put(1, b ? 1u : 0u); }
    void ue(uint32_t v) {
        const uint64_t x = (uint64_t)v + 1;
        const unsigned len = 64 - (unsigned)__builtin_clzll(x);
        if (len > 16) {
            put(len - 1, 0);
            put(len, (uint32_t)x);
        } else {
            put(2 * len - 1, (uint32_t)x);
        }
    }
    void se(int v) { ue(v > 0 ? 2u * (uint32_t)v - 1u : (uint32_t)(-2ll * v)); }
    void finish() {
        put(1, 1);
        if (n > 0) put(8 - n, 0);
    }
    void align_ones() {  // cabac_alignment_one_bit, enc/bitw.rs:52-58
        if (n > 0) put(8 - n, (1u << (8 - n)) - 1);
    }
};

// The writer's device buffers, on first use: per macroblock 3 words, per slice 1, the error word; the
// slice table (each slice's first macroblock, then each row's slice); one RBSP region per slice, sized for
// the largest slice at CAVLC_MB_MAX_BITS a macroblock.
int writer_setup(ironav_ctx* c) {
    if (c->d_cavlc) return IRONAV_OK;
    const int ns = c->nslices;
    int most = 0;
    std::vector<int> tab(ns + 1 + c->mb_h);
    for (int i = 0; i < ns; i++) {
        tab[i] = c->band_rows[i] * c->mb_w;
        most = std::max(most, (c->band_rows[i + 1] - c->band_rows[i]) * c->mb_w);
        for (int r = c->band_rows[i]; r < c->band_rows[i + 1]; r++) tab[ns + 1 + r] = i;
    }
    tab[ns] = c->nmb;
    c->rbsp_region_words = ((unsigned long long)most * CAVLC_MB_MAX_BITS + CAVLC_SLICE_EXTRA_BITS) / 32 + 2;
    CK(cudaMalloc(&c->d_cavlc, sizeof(uint32_t) * (3 * (size_t)c->nmb + ns + 1)));
    CK(cudaMalloc(&c->d_slice_tab, sizeof(int) * tab.size()));
    CK(cudaMalloc(&c->d_rbsp, sizeof(uint32_t) * c->rbsp_region_words * ns));
    CK(cudaMallocHost(&c->h_cavlc, sizeof(uint32_t) * (ns + 1)));
    CK(cudaMemcpy(c->d_slice_tab, tab.data(), sizeof(int) * tab.size(), cudaMemcpyHostToDevice));
    return IRONAV_OK;
}

// The CABAC slices (enc/mod.rs:566-600 and 641-643; FrameCoder::encode, enc/frame.rs:461-486): each slice's
// header with cabac_init_idc (P slices) and cabac_alignment_one_bit, then its arithmetic-coded data.
int write_slices_cabac(ironav_ctx* c, int idr, int frame_num, int idr_pic_id, const ironav_mbcode* d_codes, uint8_t* out, size_t cap,
                       size_t* len) {
    std::vector<std::vector<uint8_t>> data;
    const int s = cabac_slice_data(c, idr, d_codes, &data);
    if (s != IRONAV_OK) return s;
    std::vector<uint8_t> stream;
    for (int i = 0; i < c->nslices; i++) {
        HostBits h;
        h.ue((uint32_t)(c->band_rows[i] * c->mb_w));  // first_mb_in_slice
        h.ue(idr ? 7 : 5);                            // slice_type: I or P, all slices alike
        h.ue(0);                                      // pic_parameter_set_id
        h.put(8, (uint32_t)frame_num);
        if (idr) h.ue((uint32_t)idr_pic_id);
        if (!idr) {
            if (c->nact > 1) {
                h.flag(true);  // num_ref_idx_active_override_flag
                h.ue((uint32_t)(c->nact - 1));
            } else {
                h.flag(false);
            }
            h.flag(false);  // ref_pic_list_modification_flag_l0
        }
        if (idr) {
            h.flag(false);  // no_output_of_prior_pics_flag
            h.flag(false);  // long_term_reference_flag
        } else {
            h.flag(false);  // adaptive_ref_pic_marking_mode_flag
        }
        if (!idr) h.ue(0);                             // cabac_init_idc
        h.se((c->qpp - 6 * (c->bd - 8)) - 26);         // slice_qp_delta
        h.align_ones();
        h.buf.insert(h.buf.end(), data[i].begin(), data[i].end());
        put_nal(stream, 3, idr ? 5 : 1, h.buf.data(), h.buf.size());
    }
    *len = stream.size();
    if (!out || cap < stream.size()) return IRONAV_INVALID_ARGUMENT;
    memcpy(out, stream.data(), stream.size());
    return IRONAV_OK;
}

int write_slices(ironav_ctx* c, int idr, int frame_num, int idr_pic_id, const ironav_mbcode* d_codes, uint8_t* out, size_t cap,
                 size_t* len) {
    if (!c || !d_codes || !len || !c->have_params || (idr != 0) != c->intra_pic || (!idr && (c->nact < 1 || c->nact > c->nrefs)) ||
        frame_num < 0 || frame_num > 255 || idr_pic_id < 0 || idr_pic_id > 65535)
        return IRONAV_INVALID_ARGUMENT;
    if (reinterpret_cast<uintptr_t>(d_codes) & 3) return IRONAV_INVALID_ARGUMENT;
    if (c->cabac) return write_slices_cabac(c, idr, frame_num, idr_pic_id, d_codes, out, cap, len);
    int s = writer_setup(c);
    if (s != IRONAV_OK) return s;
    const int ns = c->nslices, nmb = c->nmb;
    CavlcParams p;
    memset(&p, 0, sizeof(p));
    p.codes = d_codes;
    p.band_start = c->d_band_start;
    p.slice_first = c->d_slice_tab;
    p.row_slice = c->d_slice_tab + ns + 1;
    p.out = c->d_rbsp;
    p.region_words = c->rbsp_region_words;
    p.mb_len = c->d_cavlc;
    p.mb_off = c->d_cavlc + nmb;
    p.mb_run = c->d_cavlc + 2 * (size_t)nmb;
    p.slice_bytes = c->d_cavlc + 3 * (size_t)nmb;
    p.err = c->d_cavlc + 3 * (size_t)nmb + ns;
    p.mb_w = c->mb_w;
    p.mb_h = c->mb_h;
    p.nmb = nmb;
    p.nslices = ns;
    p.p_slice = idr ? 0 : 1;
    p.nref = idr ? 0 : c->nact;
    p.idr = idr ? 1 : 0;
    p.frame_num = frame_num;
    p.idr_pic_id = idr_pic_id;
    p.slice_qp_delta = (c->qpp - 6 * (c->bd - 8)) - 26;
    CK(cudaMemsetAsync(p.err, 0, sizeof(uint32_t), c->stream));
    const int warps_per_block = 8;
    const int blocks = std::min((nmb + warps_per_block - 1) / warps_per_block, c->nsm * 16);
    cavlc_size_kernel<<<blocks, warps_per_block * 32, 0, c->stream>>>(p);
    cavlc_scan_kernel<<<ns, 1024, 0, c->stream>>>(p);
    cavlc_write_kernel<<<blocks, warps_per_block * 32, 0, c->stream>>>(p);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(c->h_cavlc, p.slice_bytes, sizeof(uint32_t) * (ns + 1), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (c->h_cavlc[ns]) return IRONAV_INTERNAL;  // a slice beyond its region (cannot happen within the bounds)
    size_t total = 0;
    for (int i = 0; i < ns; i++) total += c->h_cavlc[i];
    if (total > c->h_rbsp_cap) {
        cudaFreeHost(c->h_rbsp);
        c->h_rbsp = nullptr;
        c->h_rbsp_cap = 0;
        const size_t want = std::max(total, (size_t)1 << 16) * 2;
        CK(cudaMallocHost(&c->h_rbsp, want));
        c->h_rbsp_cap = want;
    }
    std::vector<size_t> at(ns + 1, 0);
    for (int i = 0; i < ns; i++) {
        at[i + 1] = at[i] + c->h_cavlc[i];
        CK(cudaMemcpyAsync(c->h_rbsp + at[i], c->d_rbsp + (size_t)i * c->rbsp_region_words, c->h_cavlc[i], cudaMemcpyDeviceToHost,
                           c->stream));
    }
    CK(cudaStreamSynchronize(c->stream));
    std::vector<uint8_t> stream;
    stream.reserve(total + total / 64 + 16 * ns);
    for (int i = 0; i < ns; i++) put_nal(stream, 3, idr ? 5 : 1, c->h_rbsp + at[i], c->h_cavlc[i]);  // enc/mod.rs:641-643
    *len = stream.size();
    if (!out || cap < stream.size()) return IRONAV_INVALID_ARGUMENT;
    memcpy(out, stream.data(), stream.size());
    return IRONAV_OK;
}

// (level_idc, MaxFS, MaxMBPS) of Table A-1 (enc/mod.rs:43-63)
const long long LEVELS[19][3] = {{10, 99, 1485},       {11, 396, 3000},       {12, 396, 6000},      {13, 396, 11880},
                                 {20, 396, 11880},     {21, 792, 19800},      {22, 1620, 20250},    {30, 1620, 40500},
                                 {31, 3600, 108000},   {32, 5120, 216000},    {40, 8192, 245760},   {41, 8192, 245760},
                                 {42, 8704, 522240},   {50, 22080, 589824},   {51, 36864, 983040},  {52, 36864, 2073600},
                                 {60, 139264, 4177920}, {61, 139264, 8355840}, {62, 139264, 16711680}};

}  // namespace

extern "C" {

int ironav_write_slices_device(ironav_ctx* c, int idr, int frame_num, int idr_pic_id, const ironav_mbcode* d_codes, uint8_t* out,
                               size_t cap, size_t* len) {
    return write_slices(c, idr, frame_num, idr_pic_id, d_codes, out, cap, len);
}

int ironav_write_slices(ironav_ctx* c, int idr, int frame_num, int idr_pic_id, const ironav_mbcode* codes, uint8_t* out, size_t cap,
                        size_t* len) {
    if (!c || !codes) return IRONAV_INVALID_ARGUMENT;
    if (!c->d_mbcodes) CK(cudaMalloc(&c->d_mbcodes, sizeof(ironav_mbcode) * c->nmb));
    CK(cudaMemcpyAsync(c->d_mbcodes, codes, sizeof(ironav_mbcode) * c->nmb, cudaMemcpyHostToDevice, c->stream));
    return write_slices(c, idr, frame_num, idr_pic_id, c->d_mbcodes, out, cap, len);
}

// H264Encoder::sps / pps without B pictures (enc/mod.rs:296-400) and its level (154-157)
int ironav_write_parameter_sets(const ironav_stream_params* p, uint8_t* out, size_t cap, size_t* len) {
    if (!p || !len || p->width <= 0 || p->height <= 0 || (p->width & 1) || (p->height & 1) || (p->bd != 8 && p->bd != 10) || p->refs < 1 ||
        p->refs > 16 || p->cabac < 0 || p->cabac > 1 || p->transform8 < 0 || p->transform8 > 1)
        return IRONAV_INVALID_ARGUMENT;
    const int mb_w = (p->width + 15) / 16, mb_h = (p->height + 15) / 16;
    if (mb_w > 1024 || mb_h > 1024) return IRONAV_INVALID_ARGUMENT;
    const long long fs = (long long)mb_w * mb_h;
    const bool rate_ok = p->fps_num > 0 && p->fps_den > 0;
    const double fps = rate_ok ? (double)p->fps_num / (double)p->fps_den : 25.0;
    const long long mbps = (long long)std::ceil((double)fs * fps);
    int level = -1;
    for (int i = 0; i < 19 && level < 0; i++)
        if (LEVELS[i][1] >= fs && LEVELS[i][2] >= mbps) level = (int)LEVELS[i][0];
    for (int i = 0; i < 19 && level < 0; i++)
        if (LEVELS[i][1] >= fs) level = (int)LEVELS[i][0];
    if (level < 0) level = 62;
    const bool t8 = p->cabac && p->transform8, high = t8 || p->bd > 8;
    HostBits w;
    if (p->bd > 8) {
        w.put(8, 110);  // High 10
        w.put(8, 0);
    } else if (high) {
        w.put(8, 100);  // High
        w.put(8, 0);
    } else if (p->cabac) {
        w.put(8, 77);    // Main
        w.put(8, 0x40);  // constraint_set1: Main
    } else {
        w.put(8, 66);    // Baseline
        w.put(8, 0xC0);  // constraint_set0 and constraint_set1: Constrained Baseline
    }
    w.put(8, (uint32_t)level);
    w.ue(0);  // seq_parameter_set_id
    if (high) {
        w.ue(1);                      // chroma_format_idc: 4:2:0
        w.ue((uint32_t)(p->bd - 8));  // bit_depth_luma_minus8
        w.ue((uint32_t)(p->bd - 8));  // bit_depth_chroma_minus8
        w.flag(false);                // qpprime_y_zero_transform_bypass_flag
        w.flag(false);                // seq_scaling_matrix_present_flag
    }
    w.ue(4);                   // log2_max_frame_num_minus4
    w.ue(2);                   // pic_order_cnt_type: output order is decoding order
    w.ue((uint32_t)p->refs);   // max_num_ref_frames
    w.flag(false);             // gaps_in_frame_num_value_allowed_flag
    w.ue((uint32_t)(mb_w - 1));
    w.ue((uint32_t)(mb_h - 1));
    w.flag(true);  // frame_mbs_only_flag
    w.flag(true);  // direct_8x8_inference_flag
    const int cr = (mb_w * 16 - p->width) / 2, cb = (mb_h * 16 - p->height) / 2;
    w.flag(cr > 0 || cb > 0);
    if (cr > 0 || cb > 0) {
        w.ue(0);
        w.ue((uint32_t)cr);
        w.ue(0);
        w.ue((uint32_t)cb);
    }
    w.flag(true);   // vui_parameters_present_flag
    w.flag(false);  // aspect_ratio_info_present_flag
    w.flag(false);  // overscan_info_present_flag
    w.flag(false);  // video_signal_type_present_flag
    w.flag(false);  // chroma_loc_info_present_flag
    const bool timing = rate_ok && 2ll * p->fps_num <= 0xFFFFFFFFll;
    w.flag(timing);
    if (timing) {
        w.put(32, (uint32_t)p->fps_den);       // num_units_in_tick
        w.put(32, 2u * (uint32_t)p->fps_num);  // time_scale: two ticks per frame
        w.flag(true);                          // fixed_frame_rate_flag
    }
    w.flag(false);  // nal_hrd_parameters_present_flag
    w.flag(false);  // vcl_hrd_parameters_present_flag
    w.flag(false);  // pic_struct_present_flag
    w.flag(true);   // bitstream_restriction_flag
    w.flag(true);   // motion_vectors_over_pic_boundaries_flag
    w.ue(0);        // max_bytes_per_pic_denom
    w.ue(0);        // max_bits_per_mb_denom
    w.ue(15);       // log2_max_mv_length_horizontal
    w.ue(15);       // log2_max_mv_length_vertical
    w.ue(0);        // max_num_reorder_frames
    w.ue((uint32_t)std::max(1, (int)p->refs));  // max_dec_frame_buffering
    w.finish();
    HostBits q;
    q.ue(0);        // pic_parameter_set_id
    q.ue(0);        // seq_parameter_set_id
    q.flag(p->cabac != 0);  // entropy_coding_mode_flag
    q.flag(false);  // bottom_field_pic_order_in_frame_present_flag
    q.ue(0);        // num_slice_groups_minus1
    q.ue(0);        // num_ref_idx_l0_default_active_minus1
    q.ue(0);        // num_ref_idx_l1_default_active_minus1
    q.flag(false);  // weighted_pred_flag
    q.put(2, 0);    // weighted_bipred_idc
    q.se(0);        // pic_init_qp_minus26
    q.se(0);        // pic_init_qs_minus26
    q.se(0);        // chroma_qp_index_offset
    q.flag(false);  // deblocking_filter_control_present_flag
    q.flag(false);  // constrained_intra_pred_flag
    q.flag(false);  // redundant_pic_cnt_present_flag
    if (t8) {
        q.flag(true);   // transform_8x8_mode_flag
        q.flag(false);  // pic_scaling_matrix_present_flag
        q.se(0);        // second_chroma_qp_index_offset
    }
    q.finish();
    std::vector<uint8_t> stream;
    put_nal(stream, 3, 7, w.buf.data(), w.buf.size());  // enc/mod.rs:637-638
    put_nal(stream, 3, 8, q.buf.data(), q.buf.size());
    *len = stream.size();
    if (!out || cap < stream.size()) return IRONAV_INVALID_ARGUMENT;
    memcpy(out, stream.data(), stream.size());
    return IRONAV_OK;
}

}  // extern "C"
