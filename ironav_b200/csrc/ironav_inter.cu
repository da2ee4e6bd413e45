// ironav_inter.cu — the C ABI of include/ironav_inter.h on B200 (sm_100a).
//
// A context owns, in device memory: the padded source luma, one slot per reference picture (its
// four half-sample planes and co-located vectors), the analysis results and decisions, and the
// wavefront's progress flags. Host-buffer entry points copy in, run the kernels and copy out on the
// context's stream and return when done; *_device entry points only queue work.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <atomic>
#include <chrono>
#include <vector>

#include "analyse.cuh"
#include "analyse_g8.cuh"
#include "bpicture.cuh"
#include "ctx.cuh"
#include "planes.cuh"
#include "peaks.cuh"
#include "scene.cuh"
#include "deblock.cuh"
#include "residual.cuh"
#include "decide.cuh"

using namespace ironav;

static_assert(sizeof(ironav_mbstate) == 72, "ironav_mbstate layout");
static_assert(sizeof(ironav_mbresult) == 104, "ironav_mbresult layout");
static_assert(sizeof(ironav_dbk_mb) == 192, "ironav_dbk_mb layout");
static_assert(sizeof(ironav_mbstate_b) == 140, "ironav_mbstate_b layout");
static_assert(sizeof(ironav_bresult) == 200, "ironav_bresult layout");
static_assert(sizeof(ironav_interdec) == 78, "ironav_interdec layout");
static_assert(sizeof(ironav_intercode) == 1324, "ironav_intercode layout");
static_assert(sizeof(ironav_mbcode) == 1516 && offsetof(ironav_mbcode, kind) == 1500 && offsetof(ironav_mbcode, modes) == 1484, "ironav_mbcode layout");
static_assert(sizeof(ironav_dbk_slice) == 20, "ironav_dbk_slice layout");

// The reference slot for a new picture: the oldest one's once max_refs are held, else a free one; the
// new picture becomes reference 0 (enc/mod.rs:663-666).
int take_ref_slot(ironav_ctx* c) {
    int slot;
    if (c->nrefs == c->max_refs) {
        slot = c->slot_of[c->max_refs - 1];
        c->nrefs--;
    } else {
        bool used[MAX_REFS] = {};
        for (int i = 0; i < c->nrefs; i++) used[c->slot_of[i]] = true;
        slot = 0;
        while (used[slot]) slot++;
    }
    for (int i = c->nrefs; i > 0; i--) c->slot_of[i] = c->slot_of[i - 1];
    c->slot_of[0] = slot;
    c->nrefs++;
    return slot;
}

// The analysis parameters of the context's current picture (everything but the mode's own fields).
void fill_params(const ironav_ctx* c, AnalyseParams& p) {
    memset(&p, 0, sizeof(p));
    p.src = c->d_src;
    p.ls = c->pw;
    for (int i = 0; i < c->nact; i++) p.planes[i] = c->d_planes[c->slot_of[i]];
    p.psize = c->psize;
    p.sw = c->sw;
    p.col = c->d_col[c->slot_of[0]];
    p.mb_w = c->mb_w;
    p.mb_h = c->mb_h;
    p.pw = c->pw;
    p.ph = c->ph;
    p.nact = c->nact;
    p.lambda = c->lambda;
    p.skip_thresh = c->skip_thresh;
    p.fast = c->fast;
    p.sub8 = c->sub8;
    p.band_start = c->d_band_start;
    p.withhold = -1;
    p.wait_limit = c->wait_limit;
    p.learned = c->learned;
    p.learned_cls = c->learned_cls;
    p.learned_margin = c->learned_margin;
    p.learned_stats = c->learned_stats;
}

namespace {

int cuda_status(cudaError_t e) {
    if (e == cudaSuccess) return IRONAV_OK;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver || e == cudaErrorNoKernelImageForDevice)
        return IRONAV_HARDWARE_UNAVAILABLE;
    return IRONAV_INTERNAL;
}

#define CK(x)                                  \
    do {                                       \
        cudaError_t e_ = (x);                  \
        if (e_ != cudaSuccess) return cuda_status(e_); \
    } while (0)

void free_ctx(ironav_ctx* c) {
    cudaFree(c->d_src);
    cudaFree(c->d_stage);
    for (int i = 0; i < MAX_REFS; i++) {
        cudaFree(c->d_planes[i]);
        cudaFree(c->d_col[i]);
    }
    cudaFree(c->d_band_start);
    cudaFree(c->d_order);
    cudaFree(c->d_flags);
    cudaFree(c->d_counters);
    cudaFree(c->d_states);
    cudaFree(c->d_col_stage);
    cudaFree(c->d_results);
    cudaFree(c->d_order_bands);
    cudaFree(c->d_scene_luma);
    cudaFree(c->d_lowres);
    cudaFree(c->d_scene_sums);
    cudaFree(c->d_dbk_progress);
    cudaFree(c->d_dbk_slices);
    cudaFree(c->d_dbk_mbs);
    cudaFree(c->d_dbk_planes);
    cudaFree(c->d_dbk_edges);
    cudaFree(c->d_bcol_copy);
    cudaFree(c->d_bstates);
    cudaFree(c->d_bresults);
    cudaFree(c->d_src_c);
    for (int i = 0; i < MAX_REFS; i++) cudaFree(c->d_ref_c[i]);
    cudaFree(c->d_decs);
    cudaFree(c->d_codes);
    cudaFree(c->d_rec);
    cudaFree(c->d_mbcodes);
    cudaFree(c->d_cavlc);
    cudaFree(c->d_slice_tab);
    cudaFree(c->d_rbsp);
    cudaFree(c->d_cab_step);
    cudaFree(c->d_band_rows);
    cudaFree(c->d_rd_nb);
    cudaFree(c->d_rd_scr);
    cudaFree(c->d_cab_out);
    cudaFree(c->d_cab_bytes);
    cudaFree(c->d_cab_wnb);
    cudaFreeHost(c->h_cab_bytes);
    cudaFreeHost(c->h_cavlc);
    cudaFreeHost(c->h_rbsp);
    cudaFreeHost(c->h_results);
    cudaFreeHost(c->h_done);
    cudaFreeHost(c->h_committed);
    cudaFreeHost(c->h_commit);
    delete c;
}

// Bytes per sample: 1 for 8-bit pictures, 2 (uint16_t) above.
inline int sample_bytes(const ironav_ctx* c) { return c->bd > 8 ? 2 : 1; }

int launch_planes(ironav_ctx* c, const void* d_luma, int stride, int w, int h, const ironav_mbstate* d_col) {
    const int slot = take_ref_slot(c);
    c->ref_c_ok[slot] = false;  // its chroma, if any, was the previous picture's
    dim3 grid((c->sw + K1_TW - 1) / K1_TW, (c->sh + K1_TH - 1) / K1_TH);
    const int maxv = (1 << c->bd) - 1;
    if (c->bd > 8)
        halfpel_planes_kernel<uint16_t><<<grid, K1_THREADS, 0, c->stream>>>(static_cast<const uint16_t*>(d_luma), stride, w, h,
                                                                           reinterpret_cast<uint16_t*>(c->d_planes[slot]), c->psize, c->sw, c->sh, maxv,
                                                                           d_col, c->d_col[slot], c->nmb);
    else
        halfpel_planes_kernel<uint8_t><<<grid, K1_THREADS, 0, c->stream>>>(static_cast<const uint8_t*>(d_luma), stride, w, h, c->d_planes[slot],
                                                                          c->psize, c->sw, c->sh, maxv, d_col, c->d_col[slot], c->nmb);
    return cuda_status(cudaGetLastError());
}

int launch_analyse(ironav_ctx* c, bool auto_mode, const ironav_mbstate* d_in, ironav_mbstate* d_out, ironav_mbresult* d_res) {
    AnalyseParams p;
    fill_params(c, p);
    p.states_in = d_in;
    p.states_out = d_out;
    p.results = d_res;
    p.order = auto_mode ? c->d_order : nullptr;
    p.ticket = c->d_counters;
    p.flags = c->d_flags;
    p.err = c->d_counters + 1;
    p.nmb = c->nmb;
    p.withhold = c->withhold;
    p.wait_limit = c->wait_limit;
    if (auto_mode) p.epoch = ++c->epoch;
    CK(cudaMemsetAsync(c->d_counters, 0, 2 * sizeof(unsigned), c->stream));
    if (!auto_mode && c->replay_form != 1 && p.learned == nullptr) {
        // replay mode: one macroblock per group of 8 (or 16) lanes
        // a grid of at most the CTAs the picture's macroblocks fill (one macroblock a group), so that no
        // SM holds warps that find no work while others hold more than their share
        auto grid = [&](int resident, int gw) {
            const int per_cta = g8::warps_for(gw) * (32 / gw);
            return std::max(1, std::min(resident, (c->nmb + per_cta - 1) / per_cta));
        };
        if (c->replay_form == 2) {
            if (c->bd > 8) g8::analyse_replay_g8_kernel<uint16_t, 16><<<grid(c->g16_blocks, 16), g8::warps_for(16) * 32, 0, c->stream>>>(p);
            else g8::analyse_replay_g8_kernel<uint8_t, 16><<<grid(c->g16_blocks, 16), g8::warps_for(16) * 32, 0, c->stream>>>(p);
        } else if (c->replay_form == 3) {
            if (c->bd > 8) g8::analyse_replay_g8_kernel<uint16_t, 4><<<grid(c->g4_blocks, 4), g8::warps_for(4) * 32, 0, c->stream>>>(p);
            else g8::analyse_replay_g8_kernel<uint8_t, 4><<<grid(c->g4_blocks, 4), g8::warps_for(4) * 32, 0, c->stream>>>(p);
        } else {
            if (c->bd > 8) g8::analyse_replay_g8_kernel<uint16_t, 8><<<grid(c->g8_blocks, 8), g8::warps_for(8) * 32, 0, c->stream>>>(p);
            else g8::analyse_replay_g8_kernel<uint8_t, 8><<<grid(c->g8_blocks, 8), g8::warps_for(8) * 32, 0, c->stream>>>(p);
        }
        return cuda_status(cudaGetLastError());
    }
    if (c->bd > 8) {
        if (auto_mode) analyse_kernel<MODE_AUTO, uint16_t><<<c->k2_blocks, K2_WARPS * 32, 0, c->stream>>>(p);
        else analyse_kernel<MODE_REPLAY, uint16_t><<<c->k2_blocks, K2_WARPS * 32, 0, c->stream>>>(p);
    } else {
        if (auto_mode) analyse_kernel<MODE_AUTO, uint8_t><<<c->k2_blocks, K2_WARPS * 32, 0, c->stream>>>(p);
        else analyse_kernel<MODE_REPLAY, uint8_t><<<c->k2_blocks, K2_WARPS * 32, 0, c->stream>>>(p);
    }
    return cuda_status(cudaGetLastError());
}

int check_device_error(ironav_ctx* c) {
    unsigned err = 0;
    CK(cudaMemcpyAsync(&err, c->d_counters + 1, sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (err & 1u) return IRONAV_TIMEOUT;
    if (err & 4u) return IRONAV_INVALID_INPUT;
    if (err) return IRONAV_INTERNAL;
    return IRONAV_OK;
}

// ---- scene-cut measure ----------------------------------------------------------------------------

int scene_alloc(ironav_ctx* c) {
    if (c->d_lowres) return IRONAV_OK;
    const size_t B = (size_t)sample_bytes(c);
    const size_t lsz = (size_t)(c->mb_w * 4) * (c->mb_h * 4) * B + 64;  // slack: rows are read as whole words
    CK(cudaMalloc(&c->d_scene_luma, 2 * (size_t)c->width * c->height * B));
    CK(cudaMalloc(&c->d_lowres, 2 * lsz));
    CK(cudaMalloc(&c->d_scene_sums, 2 * sizeof(unsigned long long)));
    CK(cudaMemset(c->d_lowres, 0, 2 * lsz));
    return IRONAV_OK;
}

template <class T>
void scene_kernels(ironav_ctx* c, const void* d_prev, int sp, const void* d_cur, int sc) {
    const int lw = c->mb_w * 4, lh = c->mb_h * 4;
    const size_t lsz = (size_t)lw * lh * sizeof(T) + 64;
    T* lp = reinterpret_cast<T*>(c->d_lowres);
    T* lc = reinterpret_cast<T*>(c->d_lowres + lsz);
    lowres_kernel<T><<<(lw * lh + 255) / 256, 256, 0, c->stream>>>(static_cast<const T*>(d_prev), sp, c->width, c->height, lw, lh, lp);
    lowres_kernel<T><<<(lw * lh + 255) / 256, 256, 0, c->stream>>>(static_cast<const T*>(d_cur), sc, c->width, c->height, lw, lh, lc);
    cudaMemsetAsync(c->d_scene_sums, 0, 2 * sizeof(unsigned long long), c->stream);
    const int nb = (lw >= 8 && lh >= 8) ? ((lw - 8) / 8 + 1) * ((lh - 8) / 8 + 1) : 0;
    if (nb > 0) change_kernel<T><<<(nb + 3) / 4, 128, 0, c->stream>>>(lp, lc, lw, lh, c->d_scene_sums);
}

int scene_run(ironav_ctx* c, const void* d_prev, int sp, const void* d_cur, int sc, int64_t* out) {
    if (c->bd > 8) scene_kernels<uint16_t>(c, d_prev, sp, d_cur, sc);
    else scene_kernels<uint8_t>(c, d_prev, sp, d_cur, sc);
    CK(cudaGetLastError());
    unsigned long long h[2];
    CK(cudaMemcpyAsync(h, c->d_scene_sums, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    out[0] = (int64_t)h[0];
    out[1] = (int64_t)h[1];
    return IRONAV_OK;
}

// ---- deblocking ------------------------------------------------------------------------------------

// Queues the filter of the picture whose planes are at d_y / d_cb / d_cr (strides in samples), with the
// macroblock records at d_mbs and the slice table from the host.
int deblock_launch(ironav_ctx* c, void* d_y, int ys, void* d_cb, void* d_cr, int cs, const ironav_dbk_mb* d_mbs,
                   const ironav_dbk_slice* slices, int nslices) {
    if (!c->d_dbk_progress) CK(cudaMalloc(&c->d_dbk_progress, sizeof(unsigned) * 2 * c->mb_h));
    if (!c->d_dbk_edges) CK(cudaMalloc(&c->d_dbk_edges, sizeof(DbkEdges) * c->nmb));
    if (nslices > c->dbk_slice_cap) {
        CK(cudaStreamSynchronize(c->stream));  // the old table may still be read by queued work
        cudaFree(c->d_dbk_slices);
        c->d_dbk_slices = nullptr;
        c->dbk_slice_cap = 0;
        const int cap = std::max(nslices, 64);
        CK(cudaMalloc(&c->d_dbk_slices, sizeof(ironav_dbk_slice) * cap));
        c->dbk_slice_cap = cap;
    }
    CK(cudaMemcpyAsync(c->d_dbk_slices, slices, sizeof(ironav_dbk_slice) * nslices, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemsetAsync(c->d_dbk_progress, 0, sizeof(unsigned) * 2 * c->mb_h, c->stream));
    CK(cudaMemsetAsync(c->d_counters, 0, 2 * sizeof(unsigned), c->stream));
    DbkParams p;
    p.planes[0] = static_cast<uint8_t*>(d_y);
    p.planes[1] = static_cast<uint8_t*>(d_cb);
    p.planes[2] = static_cast<uint8_t*>(d_cr);
    p.ys = ys;
    p.cs = cs;
    p.mbs = d_mbs;
    p.slices = c->d_dbk_slices;
    p.nslices = nslices;
    p.mb_w = c->mb_w;
    p.mb_h = c->mb_h;
    p.bd = c->bd;
    p.progress = c->d_dbk_progress;
    p.ticket = c->d_counters;
    p.err = c->d_counters + 1;
    p.wait_limit = c->wait_limit;
    DbkEdges* edges = static_cast<DbkEdges*>(c->d_dbk_edges);
    const int eblocks = std::min((c->nmb + DBK_WARPS - 1) / DBK_WARPS, c->nsm * 16);
    deblock_edges_kernel<<<eblocks, DBK_WARPS * 32, 0, c->stream>>>(p, edges);
    const int blocks = (2 * c->mb_h + DBK_WARPS - 1) / DBK_WARPS;
    if (c->bd > 8) deblock_rows_kernel<uint16_t><<<blocks, DBK_WARPS * 32, 0, c->stream>>>(p, edges);
    else deblock_rows_kernel<uint8_t><<<blocks, DBK_WARPS * 32, 0, c->stream>>>(p, edges);
    return cuda_status(cudaGetLastError());
}

// The kernel moves whole rows of a macroblock with 16-byte (luma) and 8 / 16-byte (chroma) accesses: plane
// bases 16-byte aligned, luma rows a multiple of 16 bytes apart, chroma rows a multiple of 8 samples apart.
bool deblock_args_ok(const ironav_ctx* c, const void* y, int ys, const void* cb, const void* cr, int cs, const void* mbs,
                     const ironav_dbk_slice* slices, int nslices) {
    if (!(c && y && cb && cr && mbs && slices && nslices >= 1 && nslices <= 65535 && ys >= c->pw && cs >= c->pw / 2)) return false;
    const uintptr_t align = reinterpret_cast<uintptr_t>(y) | reinterpret_cast<uintptr_t>(cb) | reinterpret_cast<uintptr_t>(cr);
    return (align & 15) == 0 && ((size_t)ys * sample_bytes(c)) % 16 == 0 && cs % 8 == 0;
}

}  // namespace

extern "C" {

int ironav_lambda(int qp) {  // enc/frame.rs:164-166
    int l = (int)std::lround(std::pow(2.0, ((double)qp - 12.0) / 6.0));
    return l < 1 ? 1 : l;
}

int ironav_skip_threshold(int qpp) {  // enc/frame.rs:730,742
    return (int)std::ceil(256.0 * 0.625 * std::pow(2.0, (double)qpp / 6.0));
}

int ironav_ue_bits(unsigned v) { return 2 * (32 - __builtin_clz(v + 1)) - 1; }  // enc/bitw.rs:81-83

int ironav_se_bits(int v) {  // enc/bitw.rs:86-89
    return ironav_ue_bits(v > 0 ? 2u * (unsigned)v - 1u : (unsigned)(-2 * (long long)v));
}

const char* ironav_version(void) { return "cuda-sm_100a ironav-inter-b200 0.1 (K1 halfpel_planes, K2 analyse)"; }

int ironav_ctx_create(ironav_ctx** out, int width, int height, int bd, int max_refs, int nslices, const int* band_rows) {
    if (!out) return IRONAV_INVALID_ARGUMENT;
    *out = nullptr;
    // 8-bit (Yuv420p) or 10-bit (Yuv420p10) pictures, the encoder's two formats (enc/mod.rs:140-143)
    if (width <= 0 || height <= 0 || (width & 1) || (height & 1) || (bd != 8 && bd != 10)) return IRONAV_INVALID_ARGUMENT;
    const int mb_w = (width + 15) / 16, mb_h = (height + 15) / 16;
    if (mb_w > 1024 || mb_h > 1024 || max_refs < 1 || max_refs > MAX_REFS || nslices < 1 || nslices > mb_h)
        return IRONAV_INVALID_ARGUMENT;
    std::vector<int> bands(nslices + 1);
    for (int i = 0; i <= nslices; i++) bands[i] = band_rows ? band_rows[i] : i * mb_h / nslices;
    if (bands[0] != 0 || bands[nslices] != mb_h) return IRONAV_INVALID_ARGUMENT;
    for (int i = 0; i < nslices; i++)
        if (bands[i + 1] <= bands[i]) return IRONAV_INVALID_ARGUMENT;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return IRONAV_HARDWARE_UNAVAILABLE;
    }
    ironav_ctx* c = new ironav_ctx();
    c->width = width;
    c->height = height;
    c->bd = bd;
    c->replay_form = bd > 8 ? 1 : 0;  // the faster replay kernel at each depth (8-lane groups at 8 bits)
    c->mb_w = mb_w;
    c->mb_h = mb_h;
    c->pw = mb_w * 16;
    c->ph = mb_h * 16;
    c->sw = c->pw + 2 * PAD;
    c->sh = c->ph + 2 * PAD;
    c->max_refs = max_refs;
    c->nslices = nslices;
    for (int i = 0; i <= nslices; i++) c->band_rows[i] = bands[i];
    c->nmb = mb_w * mb_h;
    c->psize = (long long)c->sw * c->sh;
    auto fail = [&](cudaError_t e) {
        int s = cuda_status(e);
        free_ctx(c);
        return s;
    };
    cudaError_t e = cudaGetDevice(&c->device);
    if (e != cudaSuccess) return fail(e);
    cudaDeviceProp prop;
    if ((e = cudaGetDeviceProperties(&prop, c->device)) != cudaSuccess) return fail(e);
    c->nsm = prop.multiProcessorCount;
    int per_sm = 0;
    e = bd > 8 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, analyse_kernel<MODE_AUTO, uint16_t>, K2_WARPS * 32, 0)
               : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, analyse_kernel<MODE_AUTO, uint8_t>, K2_WARPS * 32, 0);
    if (e != cudaSuccess) return fail(e);
    c->k2_blocks = std::max(1, per_sm) * c->nsm;
    per_sm = 0;
    e = bd > 8 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, g8::analyse_replay_g8_kernel<uint16_t, 8>, g8::warps_for(8) * 32, 0)
               : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, g8::analyse_replay_g8_kernel<uint8_t, 8>, g8::warps_for(8) * 32, 0);
    if (e != cudaSuccess) return fail(e);
    c->g8_blocks = std::max(1, per_sm) * c->nsm;
    per_sm = 0;
    e = bd > 8 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, g8::analyse_replay_g8_kernel<uint16_t, 16>, g8::warps_for(16) * 32, 0)
               : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, g8::analyse_replay_g8_kernel<uint8_t, 16>, g8::warps_for(16) * 32, 0);
    if (e != cudaSuccess) return fail(e);
    c->g16_blocks = std::max(1, per_sm) * c->nsm;
    per_sm = 0;
    e = bd > 8 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, g8::analyse_replay_g8_kernel<uint16_t, 4>, g8::warps_for(4) * 32, 0)
               : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, g8::analyse_replay_g8_kernel<uint8_t, 4>, g8::warps_for(4) * 32, 0);
    if (e != cudaSuccess) return fail(e);
    c->g4_blocks = std::max(1, per_sm) * c->nsm;
    const size_t slack = 256;  // word-granular reads may touch a few bytes past a plane's last sample
    const size_t bytes = (size_t)sample_bytes(c);
    if ((e = cudaMalloc(&c->d_src, (size_t)c->pw * c->ph * bytes + slack)) != cudaSuccess) return fail(e);
    if ((e = cudaMalloc(&c->d_stage, (size_t)c->pw * c->ph * bytes + slack)) != cudaSuccess) return fail(e);
    for (int i = 0; i < max_refs; i++) {
        if ((e = cudaMalloc(&c->d_planes[i], 4 * (size_t)c->psize * bytes + slack)) != cudaSuccess) return fail(e);
        if ((e = cudaMalloc(&c->d_col[i], sizeof(ColMv) * c->nmb)) != cudaSuccess) return fail(e);
    }
    if ((e = cudaMalloc(&c->d_band_start, sizeof(int) * mb_h)) != cudaSuccess) return fail(e);
    if ((e = cudaMalloc(&c->d_order, sizeof(int) * c->nmb)) != cudaSuccess) return fail(e);
    if ((e = cudaMalloc(&c->d_flags, sizeof(unsigned) * c->nmb)) != cudaSuccess) return fail(e);
    if ((e = cudaMalloc(&c->d_counters, sizeof(unsigned) * 2)) != cudaSuccess) return fail(e);
    // the ticket and the error word: a sync before any launch must read no error
    if ((e = cudaMemset(c->d_counters, 0, sizeof(unsigned) * 2)) != cudaSuccess) return fail(e);
    if ((e = cudaMalloc(&c->d_states, sizeof(ironav_mbstate) * c->nmb)) != cudaSuccess) return fail(e);
    if ((e = cudaMalloc(&c->d_col_stage, sizeof(ironav_mbstate) * c->nmb)) != cudaSuccess) return fail(e);
    if ((e = cudaMalloc(&c->d_results, sizeof(ironav_mbresult) * c->nmb)) != cudaSuccess) return fail(e);
    if ((e = cudaMemset(c->d_flags, 0, sizeof(unsigned) * c->nmb)) != cudaSuccess) return fail(e);
    // per row: its band's first row; tickets in wavefront order: t = x + 2 * (y - band start), then band
    std::vector<int> start(mb_h);
    for (int i = 0; i < nslices; i++)
        for (int r = bands[i]; r < bands[i + 1]; r++) start[r] = bands[i];
    std::vector<int> order(c->nmb);
    for (int i = 0; i < c->nmb; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        int ax = a % mb_w, ay = a / mb_w, bx = b % mb_w, by = b / mb_w;
        return ax + 2 * (ay - start[ay]) < bx + 2 * (by - start[by]);
    });
    if ((e = cudaMemcpy(c->d_band_start, start.data(), sizeof(int) * mb_h, cudaMemcpyHostToDevice)) != cudaSuccess) return fail(e);
    if ((e = cudaMemcpy(c->d_order, order.data(), sizeof(int) * c->nmb, cudaMemcpyHostToDevice)) != cudaSuccess) return fail(e);
    // in-loop tickets for one caller thread per band: row r of every band, band after band, then row r + 1
    std::vector<int> rows_order;
    rows_order.reserve(c->nmb);
    for (int r = 0; r < mb_h; r++)
        for (int i = 0; i < nslices; i++)
            if (bands[i] + r < bands[i + 1])
                for (int x = 0; x < mb_w; x++) rows_order.push_back((bands[i] + r) * mb_w + x);
    if ((e = cudaMalloc(&c->d_order_bands, sizeof(int) * c->nmb)) != cudaSuccess) return fail(e);
    if ((e = cudaMemcpy(c->d_order_bands, rows_order.data(), sizeof(int) * c->nmb, cudaMemcpyHostToDevice)) != cudaSuccess) return fail(e);
    *out = c;
    return IRONAV_OK;
}

int ironav_ctx_destroy(ironav_ctx* c) {
    if (!c) return IRONAV_INVALID_ARGUMENT;
    cudaStreamSynchronize(c->stream);
    free_ctx(c);
    return IRONAV_OK;
}

int ironav_ctx_dims(const ironav_ctx* c, int* mb_w, int* mb_h, int* sw, int* sh) {
    if (!c) return IRONAV_INVALID_ARGUMENT;
    if (mb_w) *mb_w = c->mb_w;
    if (mb_h) *mb_h = c->mb_h;
    if (sw) *sw = c->sw;
    if (sh) *sh = c->sh;
    return IRONAV_OK;
}

int ironav_ctx_set_stream(ironav_ctx* c, void* s) {
    if (!c) return IRONAV_INVALID_ARGUMENT;
    c->stream = static_cast<cudaStream_t>(s);
    return IRONAV_OK;
}

// The padded source from a picture whose rows are `stride` samples apart (kind: the copy's direction).
static int load_source(ironav_ctx* c, const void* y, int stride, cudaMemcpyKind kind) {
    const int B = sample_bytes(c);
    if (kind == cudaMemcpyDeviceToDevice) {
        // copy and padding in one pass
        const unsigned grid = (unsigned)(((long long)c->pw * c->ph / (16 / B) + 255) / 256);
        if (B == 2)
            copy_pad_kernel<uint16_t><<<grid, 256, 0, c->stream>>>(reinterpret_cast<uint16_t*>(c->d_src), c->pw, c->ph,
                                                                   static_cast<const uint16_t*>(y), stride, c->width, c->height);
        else
            copy_pad_kernel<uint8_t><<<grid, 256, 0, c->stream>>>(c->d_src, c->pw, c->ph, static_cast<const uint8_t*>(y), stride, c->width,
                                                                  c->height);
        return cuda_status(cudaGetLastError());
    }
    CK(cudaMemcpy2DAsync(c->d_src, (size_t)c->pw * B, y, (size_t)stride * B, (size_t)c->width * B, c->height, kind, c->stream));
    if (c->width != c->pw || c->height != c->ph) {
        const unsigned grid = (unsigned)((pad_edges_count(c->width, c->height, c->pw, c->ph) + 255) / 256);
        if (B == 2) pad_edges_kernel<uint16_t><<<grid, 256, 0, c->stream>>>(reinterpret_cast<uint16_t*>(c->d_src), c->width, c->height, c->pw, c->ph);
        else pad_edges_kernel<uint8_t><<<grid, 256, 0, c->stream>>>(c->d_src, c->width, c->height, c->pw, c->ph);
    }
    return cuda_status(cudaGetLastError());
}

int ironav_set_source_device(ironav_ctx* c, const void* d_y, int stride) {
    if (!c || !d_y || stride < c->width) return IRONAV_INVALID_ARGUMENT;
    return load_source(c, d_y, stride, cudaMemcpyDeviceToDevice);
}

int ironav_set_source(ironav_ctx* c, const void* y, int stride) {
    if (!c || !y || stride < c->width) return IRONAV_INVALID_ARGUMENT;
    const int s = load_source(c, y, stride, cudaMemcpyHostToDevice);
    if (s != IRONAV_OK) return s;
    CK(cudaStreamSynchronize(c->stream));
    return IRONAV_OK;
}

static bool ref_size_ok(const ironav_ctx* c, int stride, int w, int h) {
    return ((w == c->width && h == c->height) || (w == c->pw && h == c->ph)) && stride >= w;
}

int ironav_push_reference_device(ironav_ctx* c, const void* d_y, int stride, int w, int h, const ironav_mbstate* d_col) {
    if (!c || !d_y || !ref_size_ok(c, stride, w, h)) return IRONAV_INVALID_ARGUMENT;
    return launch_planes(c, d_y, stride, w, h, d_col);
}

int ironav_push_reference(ironav_ctx* c, const void* y, int stride, int w, int h, const ironav_mbstate* col) {
    if (!c || !y || !ref_size_ok(c, stride, w, h)) return IRONAV_INVALID_ARGUMENT;
    const size_t B = (size_t)sample_bytes(c);
    CK(cudaMemcpy2DAsync(c->d_stage, w * B, y, stride * B, w * B, h, cudaMemcpyHostToDevice, c->stream));
    if (col) CK(cudaMemcpyAsync(c->d_col_stage, col, sizeof(ironav_mbstate) * c->nmb, cudaMemcpyHostToDevice, c->stream));
    int s = launch_planes(c, c->d_stage, w, w, h, col ? c->d_col_stage : nullptr);
    if (s != IRONAV_OK) return s;
    CK(cudaStreamSynchronize(c->stream));
    return IRONAV_OK;
}

int ironav_clear_references(ironav_ctx* c) {
    if (!c) return IRONAV_INVALID_ARGUMENT;
    c->nrefs = 0;
    c->have_params = false;
    return IRONAV_OK;
}

int ironav_get_planes(ironav_ctx* c, int idx, void* out) {
    if (!c || !out || idx < 0 || idx >= c->nrefs) return IRONAV_INVALID_ARGUMENT;
    CK(cudaMemcpyAsync(out, c->d_planes[c->slot_of[idx]], 4 * (size_t)c->psize * sample_bytes(c), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return IRONAV_OK;
}

int ironav_begin_p_picture(ironav_ctx* c, int qpp, int lambda, int skip_thresh, int nact, int fast, int sub8) {
    if (!c || lambda < 1 || nact < 1 || nact > c->nrefs || qpp < 0 || qpp > 63) return IRONAV_INVALID_ARGUMENT;
    c->qpp = qpp;
    c->lambda = lambda;
    c->skip_thresh = skip_thresh;
    c->nact = nact;
    c->fast = fast ? 1 : 0;
    c->sub8 = sub8 ? 1 : 0;
    c->have_params = true;
    c->intra_pic = false;
    return IRONAV_OK;
}

int ironav_begin_i_picture(ironav_ctx* c, int qpp, int lambda, int fast) {
    if (!c || lambda < 1 || qpp < 0 || qpp > 63) return IRONAV_INVALID_ARGUMENT;
    c->qpp = qpp;
    c->lambda = lambda;
    c->skip_thresh = 0;
    c->nact = 0;
    c->fast = fast ? 1 : 0;
    c->sub8 = 0;
    c->have_params = true;
    c->intra_pic = true;
    return IRONAV_OK;
}

int ironav_analyse_picture_replay_device(ironav_ctx* c, const ironav_mbstate* d_states, ironav_mbresult* d_out) {
    if (!c || !d_states || !d_out || !c->have_params || c->intra_pic || c->nact > c->nrefs) return IRONAV_INVALID_ARGUMENT;
    return launch_analyse(c, false, d_states, nullptr, d_out);
}

int ironav_analyse_picture_auto_device(ironav_ctx* c, ironav_mbstate* d_states, ironav_mbresult* d_out) {
    if (!c || !d_states || !d_out || !c->have_params || c->intra_pic || c->nact > c->nrefs) return IRONAV_INVALID_ARGUMENT;
    return launch_analyse(c, true, nullptr, d_states, d_out);
}

int ironav_analyse_picture_replay(ironav_ctx* c, const ironav_mbstate* states, ironav_mbresult* out) {
    if (!c || !states || !out || !c->have_params || c->intra_pic || c->nact > c->nrefs) return IRONAV_INVALID_ARGUMENT;
    CK(cudaMemcpyAsync(c->d_states, states, sizeof(ironav_mbstate) * c->nmb, cudaMemcpyHostToDevice, c->stream));
    int s = launch_analyse(c, false, c->d_states, nullptr, c->d_results);
    if (s != IRONAV_OK) return s;
    CK(cudaMemcpyAsync(out, c->d_results, sizeof(ironav_mbresult) * c->nmb, cudaMemcpyDeviceToHost, c->stream));
    return check_device_error(c);
}

int ironav_analyse_picture_auto(ironav_ctx* c, ironav_mbstate* states, ironav_mbresult* out) {
    if (!c || !states || !out || !c->have_params || c->intra_pic || c->nact > c->nrefs) return IRONAV_INVALID_ARGUMENT;
    int s = launch_analyse(c, true, nullptr, c->d_states, c->d_results);
    if (s != IRONAV_OK) return s;
    CK(cudaMemcpyAsync(out, c->d_results, sizeof(ironav_mbresult) * c->nmb, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(states, c->d_states, sizeof(ironav_mbstate) * c->nmb, cudaMemcpyDeviceToHost, c->stream));
    return check_device_error(c);
}

int ironav_ctx_sync(ironav_ctx* c) {
    if (!c) return IRONAV_INVALID_ARGUMENT;
    CK(cudaStreamSynchronize(c->stream));
    return check_device_error(c);
}

// ---- scene-cut measure ---------------------------------------------------------------------------

int ironav_scene_change(ironav_ctx* c, const void* prev_y, const void* cur_y, int stride, int64_t* out) {
    if (!c || !prev_y || !cur_y || !out || stride < c->width) return IRONAV_INVALID_ARGUMENT;
    int s = scene_alloc(c);
    if (s != IRONAV_OK) return s;
    const size_t B = (size_t)sample_bytes(c);
    uint8_t* a = c->d_scene_luma;
    uint8_t* b = c->d_scene_luma + (size_t)c->width * c->height * B;
    CK(cudaMemcpy2DAsync(a, c->width * B, prev_y, stride * B, c->width * B, c->height, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpy2DAsync(b, c->width * B, cur_y, stride * B, c->width * B, c->height, cudaMemcpyHostToDevice, c->stream));
    return scene_run(c, a, c->width, b, c->width, out);
}

int ironav_scene_change_device(ironav_ctx* c, const void* d_prev, const void* d_cur, int stride, int64_t* out) {
    if (!c || !d_prev || !d_cur || !out || stride < c->width) return IRONAV_INVALID_ARGUMENT;
    int s = scene_alloc(c);
    if (s != IRONAV_OK) return s;
    return scene_run(c, d_prev, stride, d_cur, stride, out);
}

int ironav_deblock_picture_device(ironav_ctx* c, void* d_y, int ys, void* d_cb, void* d_cr, int cs, const ironav_dbk_mb* d_mbs,
                                  const ironav_dbk_slice* slices, int nslices) {
    if (!deblock_args_ok(c, d_y, ys, d_cb, d_cr, cs, d_mbs, slices, nslices)) return IRONAV_INVALID_ARGUMENT;
    return deblock_launch(c, d_y, ys, d_cb, d_cr, cs, d_mbs, slices, nslices);
}

int ironav_deblock_picture(ironav_ctx* c, void* y, int ys, void* cb, void* cr, int cs, const ironav_dbk_mb* mbs,
                           const ironav_dbk_slice* slices, int nslices) {
    if (!deblock_args_ok(c, y, ys, cb, cr, cs, mbs, slices, nslices)) return IRONAV_INVALID_ARGUMENT;
    const size_t B = (size_t)sample_bytes(c), pw = (size_t)c->pw, ph = (size_t)c->ph;
    if (!c->d_dbk_planes) CK(cudaMalloc(&c->d_dbk_planes, (pw * ph + 2 * (pw / 2) * (ph / 2)) * B));
    if (!c->d_dbk_mbs) CK(cudaMalloc(&c->d_dbk_mbs, sizeof(ironav_dbk_mb) * c->nmb));
    uint8_t* dy = c->d_dbk_planes;
    uint8_t* dcb = dy + pw * ph * B;
    uint8_t* dcr = dcb + (pw / 2) * (ph / 2) * B;
    CK(cudaMemcpy2DAsync(dy, pw * B, y, (size_t)ys * B, pw * B, ph, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpy2DAsync(dcb, pw / 2 * B, cb, (size_t)cs * B, pw / 2 * B, ph / 2, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpy2DAsync(dcr, pw / 2 * B, cr, (size_t)cs * B, pw / 2 * B, ph / 2, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->d_dbk_mbs, mbs, sizeof(ironav_dbk_mb) * c->nmb, cudaMemcpyHostToDevice, c->stream));
    int s = deblock_launch(c, dy, (int)pw, dcb, dcr, (int)(pw / 2), c->d_dbk_mbs, slices, nslices);
    if (s != IRONAV_OK) return s;
    CK(cudaMemcpy2DAsync(y, (size_t)ys * B, dy, pw * B, pw * B, ph, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpy2DAsync(cb, (size_t)cs * B, dcb, pw / 2 * B, pw / 2 * B, ph / 2, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpy2DAsync(cr, (size_t)cs * B, dcr, pw / 2 * B, pw / 2 * B, ph / 2, cudaMemcpyDeviceToHost, c->stream));
    return check_device_error(c);
}

// ---- B pictures -------------------------------------------------------------------------------------

static int b_params(ironav_ctx* c, int qpp, int lambda, int l0, int l1, int tb, int td, int fast) {
    if (!c || lambda < 1 || qpp < 0 || qpp > 63 || l0 < 0 || l0 >= c->nrefs || l1 < 0 || l1 >= c->nrefs || tb == 0 || td == 0)
        return IRONAV_INVALID_ARGUMENT;
    c->qpp = qpp;
    c->lambda = lambda;
    c->fast = fast ? 1 : 0;
    c->intra_pic = false;
    c->b_ref[0] = l0;
    c->b_ref[1] = l1;
    c->b_tb = tb;
    c->b_td = td;
    return IRONAV_OK;
}

int ironav_begin_b_picture(ironav_ctx* c, int qpp, int lambda, int ref_l0, int ref_l1, const ironav_mbstate* col, int tb, int td, int fast) {
    int s = b_params(c, qpp, lambda, ref_l0, ref_l1, tb, td, fast);
    if (s != IRONAV_OK) return s;
    c->b_col = nullptr;
    if (col) {
        if (!c->d_bcol_copy) CK(cudaMalloc(&c->d_bcol_copy, sizeof(ironav_mbstate) * c->nmb));
        CK(cudaMemcpyAsync(c->d_bcol_copy, col, sizeof(ironav_mbstate) * c->nmb, cudaMemcpyHostToDevice, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        c->b_col = c->d_bcol_copy;
    }
    c->b_set = true;
    return IRONAV_OK;
}

int ironav_begin_b_picture_device(ironav_ctx* c, int qpp, int lambda, int ref_l0, int ref_l1, const ironav_mbstate* d_col, int tb, int td,
                                  int fast) {
    int s = b_params(c, qpp, lambda, ref_l0, ref_l1, tb, td, fast);
    if (s != IRONAV_OK) return s;
    c->b_col = d_col;
    c->b_set = true;
    return IRONAV_OK;
}

static int launch_b(ironav_ctx* c, const ironav_mbstate_b* d_states, ironav_bresult* d_out) {
    if (!c->b_set || c->b_ref[0] >= c->nrefs || c->b_ref[1] >= c->nrefs) return IRONAV_INVALID_ARGUMENT;
    AnalyseParams p;
    fill_params(c, p);
    p.planes[0] = c->d_planes[c->slot_of[c->b_ref[0]]];
    p.planes[1] = c->d_planes[c->slot_of[c->b_ref[1]]];
    p.nact = 2;
    p.bstates_in = d_states;
    p.bresults = d_out;
    p.bcol = c->b_col;
    p.tb = c->b_tb;
    p.td = c->b_td;
    p.ticket = c->d_counters;
    p.err = c->d_counters + 1;
    p.nmb = c->nmb;
    CK(cudaMemsetAsync(c->d_counters, 0, 2 * sizeof(unsigned), c->stream));
    if (c->bd > 8) analyse_b_kernel<uint16_t><<<c->k2_blocks, K2_WARPS * 32, 0, c->stream>>>(p);
    else analyse_b_kernel<uint8_t><<<c->k2_blocks, K2_WARPS * 32, 0, c->stream>>>(p);
    return cuda_status(cudaGetLastError());
}

int ironav_analyse_b_replay_device(ironav_ctx* c, const ironav_mbstate_b* d_states, ironav_bresult* d_out) {
    if (!c || !d_states || !d_out) return IRONAV_INVALID_ARGUMENT;
    return launch_b(c, d_states, d_out);
}

int ironav_analyse_b_replay(ironav_ctx* c, const ironav_mbstate_b* states, ironav_bresult* out) {
    if (!c || !states || !out) return IRONAV_INVALID_ARGUMENT;
    if (!c->d_bstates) CK(cudaMalloc(&c->d_bstates, sizeof(ironav_mbstate_b) * c->nmb));
    if (!c->d_bresults) CK(cudaMalloc(&c->d_bresults, sizeof(ironav_bresult) * c->nmb));
    CK(cudaMemcpyAsync(c->d_bstates, states, sizeof(ironav_mbstate_b) * c->nmb, cudaMemcpyHostToDevice, c->stream));
    int s = launch_b(c, c->d_bstates, c->d_bresults);
    if (s != IRONAV_OK) return s;
    CK(cudaMemcpyAsync(out, c->d_bresults, sizeof(ironav_bresult) * c->nmb, cudaMemcpyDeviceToHost, c->stream));
    return check_device_error(c);
}

// ---- inter residual coding ----------------------------------------------------------------------------

// Copies a w x h chroma plane (rows `stride` samples apart) into dst (cw x ch, rows cw apart), padded by
// repeating its right and bottom edges.
static int load_chroma(ironav_ctx* c, uint8_t* dst, const void* src, int stride, int w, int h, cudaMemcpyKind kind) {
    const int B = sample_bytes(c), cw = c->mb_w * 8, ch = c->mb_h * 8;
    CK(cudaMemcpy2DAsync(dst, (size_t)cw * B, src, (size_t)stride * B, (size_t)w * B, h, kind, c->stream));
    if (w != cw || h != ch) {
        const unsigned grid = (unsigned)((pad_edges_count(w, h, cw, ch) + 255) / 256);
        if (B == 2) pad_edges_kernel<uint16_t><<<grid, 256, 0, c->stream>>>(reinterpret_cast<uint16_t*>(dst), w, h, cw, ch);
        else pad_edges_kernel<uint8_t><<<grid, 256, 0, c->stream>>>(dst, w, h, cw, ch);
    }
    return cuda_status(cudaGetLastError());
}

int ironav_set_source_chroma(ironav_ctx* c, const void* cb, const void* cr, int stride) {
    if (!c || !cb || !cr || stride < c->width / 2) return IRONAV_INVALID_ARGUMENT;
    const size_t plane = (size_t)c->mb_w * 8 * c->mb_h * 8 * sample_bytes(c);
    if (!c->d_src_c) CK(cudaMalloc(&c->d_src_c, 2 * plane + 256));
    int s = load_chroma(c, c->d_src_c, cb, stride, c->width / 2, c->height / 2, cudaMemcpyHostToDevice);
    if (s == IRONAV_OK) s = load_chroma(c, c->d_src_c + plane, cr, stride, c->width / 2, c->height / 2, cudaMemcpyHostToDevice);
    if (s != IRONAV_OK) return s;
    CK(cudaStreamSynchronize(c->stream));
    return IRONAV_OK;
}

int ironav_set_source_chroma_device(ironav_ctx* c, const void* d_cb, const void* d_cr, int stride) {
    if (!c || !d_cb || !d_cr || stride < c->width / 2) return IRONAV_INVALID_ARGUMENT;
    const size_t plane = (size_t)c->mb_w * 8 * c->mb_h * 8 * sample_bytes(c);
    if (!c->d_src_c) CK(cudaMalloc(&c->d_src_c, 2 * plane + 256));
    int s = load_chroma(c, c->d_src_c, d_cb, stride, c->width / 2, c->height / 2, cudaMemcpyDeviceToDevice);
    if (s == IRONAV_OK) s = load_chroma(c, c->d_src_c + plane, d_cr, stride, c->width / 2, c->height / 2, cudaMemcpyDeviceToDevice);
    return s;
}

static int push_ref_chroma(ironav_ctx* c, const void* cb, const void* cr, int stride, int w, int h, cudaMemcpyKind kind) {
    if (!c || !cb || !cr || c->nrefs < 1) return IRONAV_INVALID_ARGUMENT;
    const int cw = c->mb_w * 8, ch = c->mb_h * 8;
    if (!((w == c->width / 2 && h == c->height / 2) || (w == cw && h == ch)) || stride < w) return IRONAV_INVALID_ARGUMENT;
    const int slot = c->slot_of[0];
    const size_t plane = (size_t)cw * ch * sample_bytes(c);
    if (!c->d_ref_c[slot]) CK(cudaMalloc(&c->d_ref_c[slot], 2 * plane + 256));
    int s = load_chroma(c, c->d_ref_c[slot], cb, stride, w, h, kind);
    if (s == IRONAV_OK) s = load_chroma(c, c->d_ref_c[slot] + plane, cr, stride, w, h, kind);
    if (s != IRONAV_OK) return s;
    c->ref_c_ok[slot] = true;
    return IRONAV_OK;
}

int ironav_push_reference_chroma(ironav_ctx* c, const void* cb, const void* cr, int stride, int w, int h) {
    const int s = push_ref_chroma(c, cb, cr, stride, w, h, cudaMemcpyHostToDevice);
    if (s != IRONAV_OK) return s;
    CK(cudaStreamSynchronize(c->stream));
    return IRONAV_OK;
}

int ironav_push_reference_chroma_device(ironav_ctx* c, const void* d_cb, const void* d_cr, int stride, int w, int h) {
    return push_ref_chroma(c, d_cb, d_cr, stride, w, h, cudaMemcpyDeviceToDevice);
}

static int launch_code_inter(ironav_ctx* c, int qp, const ironav_interdec* d_decs, ironav_intercode* d_codes, void* y, int ys, void* cb,
                             void* cr, int cs) {
    if (qp < -6 * (c->bd - 8) || qp > 51 || !c->d_src_c || c->nrefs < 1) return IRONAV_INVALID_ARGUMENT;
    for (int i = 0; i < c->nrefs; i++)
        if (!c->ref_c_ok[c->slot_of[i]]) return IRONAV_INVALID_ARGUMENT;  // a reference without chroma
    CodeParams p;
    memset(&p, 0, sizeof(p));
    fill_params(c, p.A);
    for (int i = 0; i < c->nrefs; i++) {
        p.A.planes[i] = c->d_planes[c->slot_of[i]];
        p.ref_c[i] = c->d_ref_c[c->slot_of[i]];
    }
    p.src_c = c->d_src_c;
    p.cw = c->mb_w * 8;
    p.ch = c->mb_h * 8;
    p.decs = d_decs;
    p.codes = d_codes;
    p.rec[0] = static_cast<uint8_t*>(y);
    p.rec[1] = static_cast<uint8_t*>(cb);
    p.rec[2] = static_cast<uint8_t*>(cr);
    p.ys = ys;
    p.cs = cs;
    p.qp = qp;
    p.bd = c->bd;
    p.nrefs = c->nrefs;
    p.err = c->d_counters + 1;
    CK(cudaMemsetAsync(c->d_counters, 0, 2 * sizeof(unsigned), c->stream));
    const int blocks = std::min((c->nmb + 3) / 4, c->nsm * 8);
    if (c->bd > 8) code_inter_kernel<uint16_t><<<blocks, 128, 0, c->stream>>>(p);
    else code_inter_kernel<uint8_t><<<blocks, 128, 0, c->stream>>>(p);
    return cuda_status(cudaGetLastError());
}

int ironav_code_inter_picture_device(ironav_ctx* c, int qp, const ironav_interdec* d_decs, ironav_intercode* d_codes, void* y, int ys, void* cb,
                                     void* cr, int cs) {
    if (!c || !d_decs || !d_codes || !y || !cb || !cr || ys < c->pw || cs < c->pw / 2) return IRONAV_INVALID_ARGUMENT;
    // the planes: the same alignment as the deblocking filter's device form; the records: the kernel reads a
    // decision as 16-bit words and writes a code record as 32-bit words
    const uintptr_t a = reinterpret_cast<uintptr_t>(y) | reinterpret_cast<uintptr_t>(cb) | reinterpret_cast<uintptr_t>(cr);
    if ((a & 15) || ((size_t)ys * sample_bytes(c)) % 16 || cs % 8) return IRONAV_INVALID_ARGUMENT;
    if ((reinterpret_cast<uintptr_t>(d_decs) & 1) || (reinterpret_cast<uintptr_t>(d_codes) & 3)) return IRONAV_INVALID_ARGUMENT;
    return launch_code_inter(c, qp, d_decs, d_codes, y, ys, cb, cr, cs);
}

int ironav_code_inter_picture(ironav_ctx* c, int qp, const ironav_interdec* decs, ironav_intercode* codes, void* y, int ys, void* cb, void* cr,
                              int cs) {
    if (!c || !decs || !codes || !y || !cb || !cr || ys < c->pw || cs < c->pw / 2) return IRONAV_INVALID_ARGUMENT;
    const size_t B = (size_t)sample_bytes(c), pw = (size_t)c->pw, ph = (size_t)c->ph;
    if (!c->d_decs) CK(cudaMalloc(&c->d_decs, sizeof(ironav_interdec) * c->nmb));
    if (!c->d_codes) CK(cudaMalloc(&c->d_codes, sizeof(ironav_intercode) * c->nmb));
    if (!c->d_rec) CK(cudaMalloc(&c->d_rec, (pw * ph + 2 * (pw / 2) * (ph / 2)) * B));
    uint8_t* dy = c->d_rec;
    uint8_t* dcb = dy + pw * ph * B;
    uint8_t* dcr = dcb + (pw / 2) * (ph / 2) * B;
    CK(cudaMemcpyAsync(c->d_decs, decs, sizeof(ironav_interdec) * c->nmb, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpy2DAsync(dy, pw * B, y, (size_t)ys * B, pw * B, ph, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpy2DAsync(dcb, pw / 2 * B, cb, (size_t)cs * B, pw / 2 * B, ph / 2, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpy2DAsync(dcr, pw / 2 * B, cr, (size_t)cs * B, pw / 2 * B, ph / 2, cudaMemcpyHostToDevice, c->stream));
    int s = launch_code_inter(c, qp, c->d_decs, c->d_codes, dy, (int)pw, dcb, dcr, (int)(pw / 2));
    if (s != IRONAV_OK) return s;
    CK(cudaMemcpyAsync(codes, c->d_codes, sizeof(ironav_intercode) * c->nmb, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpy2DAsync(y, (size_t)ys * B, dy, pw * B, pw * B, ph, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpy2DAsync(cb, (size_t)cs * B, dcb, pw / 2 * B, pw / 2 * B, ph / 2, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpy2DAsync(cr, (size_t)cs * B, dcr, pw / 2 * B, pw / 2 * B, ph / 2, cudaMemcpyDeviceToHost, c->stream));
    return check_device_error(c);
}

// ---- decide mode ------------------------------------------------------------------------------------

// The fast mode's P_Skip tests `sad < 256 * 0.05 * step` and `csad < 128 * 0.05 * step` with step =
// 2^(QP'/6) (enc/frame.rs:735,740), as integer bounds like ironav_skip_threshold.
static void fast_thresholds(int qpp, int* luma, int* chroma) {
    const double step = std::pow(2.0, (double)qpp / 6.0);
    *luma = (int)std::ceil(256.0 * 0.05 * step);
    *chroma = (int)std::ceil(128.0 * 0.05 * step);
}

}  // extern "C"

// shared with the batched form (ironav_batch.cu)
int ironav::fill_decide_params(ironav_ctx* c, DecideParams& p, ironav_mbstate* d_states, ironav_mbcode* d_codes, void* y, int ys, void* cb, void* cr,
                               int cs) {
    if (!c->have_params || !c->d_src_c) return IRONAV_INVALID_ARGUMENT;
    if (!c->intra_pic && (c->nact < 1 || c->nact > c->nrefs)) return IRONAV_INVALID_ARGUMENT;
    for (int i = 0; i < c->nact; i++)
        if (!c->ref_c_ok[c->slot_of[i]]) return IRONAV_INVALID_ARGUMENT;  // an active reference without chroma
    memset(&p, 0, sizeof(p));
    p.intra = c->intra_pic ? 1 : 0;
    p.flat_t = (int)std::ceil(256.0 * 0.8 * std::pow(2.0, (double)c->qpp / 6.0));  // enc/frame.rs:763
    fill_params(c, p.C.A);
    p.C.A.states_out = d_states;
    p.C.A.nmb = c->nmb;
    p.C.A.withhold = c->withhold;
    for (int i = 0; i < c->nact; i++) p.C.ref_c[i] = c->d_ref_c[c->slot_of[i]];
    p.C.src_c = c->d_src_c;
    p.C.cw = c->mb_w * 8;
    p.C.ch = c->mb_h * 8;
    p.C.rec[0] = static_cast<uint8_t*>(y);
    p.C.rec[1] = static_cast<uint8_t*>(cb);
    p.C.rec[2] = static_cast<uint8_t*>(cr);
    p.C.ys = ys;
    p.C.cs = cs;
    p.C.qp = c->qpp - 6 * (c->bd - 8);
    p.C.bd = c->bd;
    p.C.nrefs = c->nact;
    p.codes = d_codes;
    fast_thresholds(c->qpp, &p.fast_t, &p.fast_tc);
    return IRONAV_OK;
}

extern "C" {

static int launch_decide(ironav_ctx* c, ironav_mbstate* d_states, ironav_mbcode* d_codes, void* y, int ys, void* cb, void* cr, int cs) {
    if (c->cabac) return launch_decide_rd(c, d_states, d_codes, y, ys, cb, cr, cs);
    DecideParams p;
    const int s = fill_decide_params(c, p, d_states, d_codes, y, ys, cb, cr, cs);
    if (s != IRONAV_OK) return s;
    if (!c->k7_blocks) {
        int per_sm = 0;
        const cudaError_t e = c->bd > 8 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, decide_kernel<uint16_t>, K7_WARPS * 32, 0)
                                        : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, decide_kernel<uint8_t>, K7_WARPS * 32, 0);
        if (e != cudaSuccess) return cuda_status(e);
        c->k7_blocks = std::max(1, per_sm) * c->nsm;
    }
    AnalyseParams& A = p.C.A;
    A.order = c->d_order;
    A.ticket = c->d_counters;
    A.flags = c->d_flags;
    A.err = c->d_counters + 1;
    A.epoch = ++c->epoch;
    p.C.err = c->d_counters + 1;
    CK(cudaMemsetAsync(c->d_counters, 0, 2 * sizeof(unsigned), c->stream));
    if (c->bd > 8) decide_kernel<uint16_t><<<c->k7_blocks, K7_WARPS * 32, 0, c->stream>>>(p);
    else decide_kernel<uint8_t><<<c->k7_blocks, K7_WARPS * 32, 0, c->stream>>>(p);
    return cuda_status(cudaGetLastError());
}

static int decide_device_checked(ironav_ctx* c, bool intra, ironav_mbstate* d_states, ironav_mbcode* d_codes, void* y, int ys, void* cb,
                                 void* cr, int cs) {
    if (!c || !d_states || !d_codes || !y || !cb || !cr || ys < c->pw || cs < c->pw / 2 || c->intra_pic != intra)
        return IRONAV_INVALID_ARGUMENT;
    // the planes as the deblocking filter's device form; states and codes are written as 32-bit words
    const uintptr_t a = reinterpret_cast<uintptr_t>(y) | reinterpret_cast<uintptr_t>(cb) | reinterpret_cast<uintptr_t>(cr);
    if ((a & 15) || ((size_t)ys * sample_bytes(c)) % 16 || cs % 8) return IRONAV_INVALID_ARGUMENT;
    if ((reinterpret_cast<uintptr_t>(d_states) | reinterpret_cast<uintptr_t>(d_codes)) & 3) return IRONAV_INVALID_ARGUMENT;
    return launch_decide(c, d_states, d_codes, y, ys, cb, cr, cs);
}

int ironav_decide_p_picture_device(ironav_ctx* c, ironav_mbstate* d_states, ironav_mbcode* d_codes, void* y, int ys, void* cb, void* cr, int cs) {
    return decide_device_checked(c, false, d_states, d_codes, y, ys, cb, cr, cs);
}

int ironav_decide_i_picture_device(ironav_ctx* c, ironav_mbstate* d_states, ironav_mbcode* d_codes, void* y, int ys, void* cb, void* cr, int cs) {
    return decide_device_checked(c, true, d_states, d_codes, y, ys, cb, cr, cs);
}

int ironav_decide_dbk_records_device(ironav_ctx* c, const ironav_mbcode* d_codes, const ironav_mbstate* d_states, ironav_dbk_mb* d_mbs) {
    if (!c || !d_codes || !d_states || !d_mbs || !c->have_params) return IRONAV_INVALID_ARGUMENT;
    if ((reinterpret_cast<uintptr_t>(d_codes) | reinterpret_cast<uintptr_t>(d_states) | reinterpret_cast<uintptr_t>(d_mbs)) & 3)
        return IRONAV_INVALID_ARGUMENT;
    dbk_records_kernel<<<(c->nmb + 127) / 128, 128, 0, c->stream>>>(d_codes, d_states, c->d_band_start, c->mb_w, c->nmb,
                                                                     c->qpp - 6 * (c->bd - 8), d_mbs);
    return cuda_status(cudaGetLastError());
}

int ironav_decide_dbk_records(ironav_ctx* c, const ironav_mbcode* codes, const ironav_mbstate* states, ironav_dbk_mb* mbs) {
    if (!c || !codes || !states || !mbs || !c->have_params) return IRONAV_INVALID_ARGUMENT;
    if (!c->d_mbcodes) CK(cudaMalloc(&c->d_mbcodes, sizeof(ironav_mbcode) * c->nmb));
    if (!c->d_dbk_mbs) CK(cudaMalloc(&c->d_dbk_mbs, sizeof(ironav_dbk_mb) * c->nmb));
    CK(cudaMemcpyAsync(c->d_mbcodes, codes, sizeof(ironav_mbcode) * c->nmb, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->d_states, states, sizeof(ironav_mbstate) * c->nmb, cudaMemcpyHostToDevice, c->stream));
    const int s = ironav_decide_dbk_records_device(c, c->d_mbcodes, c->d_states, c->d_dbk_mbs);
    if (s != IRONAV_OK) return s;
    CK(cudaMemcpyAsync(mbs, c->d_dbk_mbs, sizeof(ironav_dbk_mb) * c->nmb, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return IRONAV_OK;
}

static int decide_host(ironav_ctx* c, bool intra, ironav_mbstate* states, ironav_mbcode* codes, void* y, int ys, void* cb, void* cr, int cs) {
    if (!c || !states || !codes || !y || !cb || !cr || ys < c->pw || cs < c->pw / 2 || c->intra_pic != intra) return IRONAV_INVALID_ARGUMENT;
    const size_t B = (size_t)sample_bytes(c), pw = (size_t)c->pw, ph = (size_t)c->ph;
    if (!c->d_mbcodes) CK(cudaMalloc(&c->d_mbcodes, sizeof(ironav_mbcode) * c->nmb));
    if (!c->d_rec) CK(cudaMalloc(&c->d_rec, (pw * ph + 2 * (pw / 2) * (ph / 2)) * B));
    uint8_t* dy = c->d_rec;
    uint8_t* dcb = dy + pw * ph * B;
    uint8_t* dcr = dcb + (pw / 2) * (ph / 2) * B;
    int s = launch_decide(c, c->d_states, c->d_mbcodes, dy, (int)pw, dcb, dcr, (int)(pw / 2));
    if (s != IRONAV_OK) return s;
    CK(cudaMemcpyAsync(states, c->d_states, sizeof(ironav_mbstate) * c->nmb, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(codes, c->d_mbcodes, sizeof(ironav_mbcode) * c->nmb, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpy2DAsync(y, (size_t)ys * B, dy, pw * B, pw * B, ph, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpy2DAsync(cb, (size_t)cs * B, dcb, pw / 2 * B, pw / 2 * B, ph / 2, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpy2DAsync(cr, (size_t)cs * B, dcr, pw / 2 * B, pw / 2 * B, ph / 2, cudaMemcpyDeviceToHost, c->stream));
    return check_device_error(c);
}

int ironav_decide_p_picture(ironav_ctx* c, ironav_mbstate* states, ironav_mbcode* codes, void* y, int ys, void* cb, void* cr, int cs) {
    return decide_host(c, false, states, codes, y, ys, cb, cr, cs);
}

int ironav_decide_i_picture(ironav_ctx* c, ironav_mbstate* states, ironav_mbcode* codes, void* y, int ys, void* cb, void* cr, int cs) {
    return decide_host(c, true, states, codes, y, ys, cb, cr, cs);
}

// Measures the 32-bit integer issue rate of the current device (operations per second, 1e12 units in
// *tops): the roofline denominator for the analysis kernel (not in the public header).
int ironav_measure_int32_peak(double* tops) {
    if (!tops) return IRONAV_INVALID_ARGUMENT;
    int dev = 0, nsm = 0, per_sm = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, int32_peak_kernel, 256, 0));
    unsigned* d = nullptr;
    CK(cudaMalloc(&d, sizeof(unsigned) * nsm * per_sm));
    const int blocks = nsm * per_sm, iters = 4096;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double best = 0.0;
    for (int rep = 0; rep < 4; rep++) {
        cudaEventRecord(e0);
        int32_peak_kernel<<<blocks, 256>>>(d, iters, 12345u + rep);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        double ops = 2.0 * 16.0 * 8.0 * iters * 256.0 * blocks;
        if (rep > 0) best = std::max(best, ops / (ms * 1e-3) / 1e12);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(d);
    CK(cudaGetLastError());
    *tops = best;
    return IRONAV_OK;
}

// ---- in-loop mode ----------------------------------------------------------------------------------

int ironav_inloop_begin(ironav_ctx* c, int order) {
    if (!c || !c->have_params || c->intra_pic || c->nact > c->nrefs || (order != IRONAV_INLOOP_RASTER && order != IRONAV_INLOOP_BANDS))
        return IRONAV_INVALID_ARGUMENT;
    if (c->inloop_active) return IRONAV_INVALID_INPUT;
    if (!c->h_results) {
        CK(cudaHostAlloc(&c->h_results, sizeof(ironav_mbresult) * c->nmb, cudaHostAllocMapped));
        CK(cudaHostAlloc(&c->h_done, sizeof(unsigned) * c->nmb, cudaHostAllocMapped));
        CK(cudaHostAlloc(&c->h_committed, sizeof(ironav_mbstate) * c->nmb, cudaHostAllocMapped));
        CK(cudaHostAlloc(&c->h_commit, sizeof(unsigned) * c->nmb, cudaHostAllocMapped));
        memset(c->h_done, 0, sizeof(unsigned) * c->nmb);
        memset(c->h_commit, 0, sizeof(unsigned) * c->nmb);
    }
    AnalyseParams p;
    fill_params(c, p);
    p.order = order == IRONAV_INLOOP_BANDS ? c->d_order_bands : nullptr;
    p.ticket = c->d_counters;
    p.err = c->d_counters + 1;
    p.nmb = c->nmb;
    p.withhold = -1;
    p.epoch = ++c->inloop_epoch;
    p.wait_ns = c->inloop_wait_ns;
    CK(cudaHostGetDevicePointer((void**)&p.results, c->h_results, 0));
    CK(cudaHostGetDevicePointer((void**)&p.done_flags, c->h_done, 0));
    CK(cudaHostGetDevicePointer((void**)&p.committed, c->h_committed, 0));
    CK(cudaHostGetDevicePointer((void**)&p.commit_flags, c->h_commit, 0));
    CK(cudaMemsetAsync(c->d_counters, 0, 2 * sizeof(unsigned), c->stream));
    // few warps: the caller's pace bounds this mode, and every waiting warp polls host memory
    const int blocks = std::min(c->k2_blocks, 64);
    if (c->bd > 8) analyse_kernel<MODE_INLOOP, uint16_t><<<blocks, K2_WARPS * 32, 0, c->stream>>>(p);
    else analyse_kernel<MODE_INLOOP, uint8_t><<<blocks, K2_WARPS * 32, 0, c->stream>>>(p);
    CK(cudaGetLastError());
    c->inloop_active = true;
    return IRONAV_OK;
}

int ironav_inloop_result(ironav_ctx* c, int mb, ironav_mbresult* out, int timeout_ms) {
    if (!c || !out || mb < 0 || mb >= c->nmb || !c->inloop_active) return IRONAV_INVALID_ARGUMENT;
    const volatile unsigned* flag = c->h_done + mb;
    const auto t0 = std::chrono::steady_clock::now();
    for (unsigned i = 0; *flag != c->inloop_epoch; i++) {
        if ((i & 255) == 255 && std::chrono::steady_clock::now() - t0 > std::chrono::milliseconds(timeout_ms)) return IRONAV_TIMEOUT;
    }
    std::atomic_thread_fence(std::memory_order_acquire);
    memcpy(out, (const void*)(c->h_results + mb), sizeof(ironav_mbresult));
    return IRONAV_OK;
}

int ironav_inloop_commit(ironav_ctx* c, int mb, const ironav_mbstate* s) {
    if (!c || !s || mb < 0 || mb >= c->nmb || !c->inloop_active) return IRONAV_INVALID_ARGUMENT;
    memcpy((void*)(c->h_committed + mb), s, sizeof(ironav_mbstate));
    std::atomic_thread_fence(std::memory_order_release);
    *(volatile unsigned*)(c->h_commit + mb) = c->inloop_epoch;
    return IRONAV_OK;
}

int ironav_inloop_end(ironav_ctx* c) {
    if (!c || !c->inloop_active) return IRONAV_INVALID_ARGUMENT;
    c->inloop_active = false;
    return check_device_error(c);
}

// Replay mode's kernel: 0 one macroblock per 8-lane group (the default), 1 one macroblock per warp, 2 one
// macroblock per 16-lane group.
int ironav_set_entropy(ironav_ctx* c, int cabac, int transform8) {
    if (!c || cabac < 0 || cabac > 1 || transform8 < 0 || transform8 > 1) return IRONAV_INVALID_ARGUMENT;
    if (cabac) {
        const int s = cabac_setup(c);
        if (s != IRONAV_OK) return s;
    }
    c->cabac = cabac;
    c->t8 = cabac && transform8;  // FrameCoder::new, enc/frame.rs:405: the 8x8 transform with CABAC only
    return IRONAV_OK;
}

int ironav_set_replay_form(ironav_ctx* c, int form) {
    if (!c || form < 0 || form > 3) return IRONAV_INVALID_ARGUMENT;
    c->replay_form = form;
    return IRONAV_OK;
}

// The learned form's proposals for the context's next analyses (auto, replay and decide modes): all four
// pointers set, or d_cands NULL for the plain search again.
int ironav_set_learned(ironav_ctx* c, const int16_t* d_cands, const uint8_t* d_cls, int margin, unsigned* d_stats) {
    if (!c || (d_cands && (!d_cls || !d_stats)) || margin < 0) return IRONAV_INVALID_ARGUMENT;
    c->learned = d_cands;
    c->learned_cls = d_cands ? d_cls : nullptr;
    c->learned_stats = d_cands ? d_stats : nullptr;
    c->learned_margin = margin;
    return IRONAV_OK;
}

// How long an in-loop wait for the caller's commit may take on the device (milliseconds).
int ironav_inloop_set_wait(ironav_ctx* c, int ms) {
    if (!c || ms <= 0) return IRONAV_INVALID_ARGUMENT;
    c->inloop_wait_ns = (unsigned long long)ms * 1000000ull;
    return IRONAV_OK;
}

// Test hooks (not in the public header): a macroblock whose decision is never published, so the
// wavefront waits behind it run out, and the number of polls a wait makes before it gives up.
int ironav_debug_withhold(ironav_ctx* c, int mb) {
    if (!c || mb < -1 || mb >= c->nmb) return IRONAV_INVALID_ARGUMENT;
    c->withhold = mb;
    return IRONAV_OK;
}

int ironav_debug_wait_limit(ironav_ctx* c, unsigned polls) {
    if (!c || polls == 0) return IRONAV_INVALID_ARGUMENT;
    c->wait_limit = polls;
    return IRONAV_OK;
}

}  // extern "C"
