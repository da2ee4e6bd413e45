// ironav_batch.cu — the batched form: many streams (contexts) analysed with one launch per stage and
// frame step. The sources of every stream are copied and padded by one kernel, the new references'
// half-sample planes and co-located vectors are built by one kernel each, and one persistent launch runs
// every stream's macroblock wavefronts (auto mode) together: tickets follow the streams' merged
// wavefront order, so a waiting warp only waits on warps holding smaller tickets of its own stream.
// With many streams in flight the wavefronts fill the GPU, which one stream's wavefront cannot.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <tuple>
#include <vector>

#include "analyse.cuh"
#include "analyse_g8.cuh"
#include "ctx.cuh"
#include "decide.cuh"
#include "decide_rd.cuh"
#include "planes.cuh"

using namespace ironav;

namespace {

// One stream's new reference picture: its luma, its planes' slot and its co-located vectors.
struct PlaneJob {
    const uint8_t* luma;
    int stride, w, h;
    uint8_t* out;
    long long psize;
    int sw, sh, tiles_x, tile0;  // tile0: the job's first tile in the launch
    const ironav_mbstate* col_states;
    ColMv* col;
    int nmb, mb0;  // mb0: the job's first macroblock in the launch
};

// One stream's new source picture, copied into its context and padded to whole macroblocks.
struct SrcJob {
    const uint8_t* src;
    int stride, w, h;
    uint8_t* dst;
    int pw, ph, row0;  // row0: the job's first row in the launch
};

template <typename Job, typename Key>
__device__ __forceinline__ int find_job(const Job* jobs, int n, int idx, Key key) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (key(jobs[mid]) <= idx) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// TH: the tiles' rows (the tuner's choice, 16 or 8), 16 * TH threads a CTA.
template <class T, int TH>
__global__ void __launch_bounds__(16 * TH) planes_batch_kernel(const PlaneJob* __restrict__ jobs, int njobs, int maxv) {
    const int j = find_job(jobs, njobs, (int)blockIdx.x, [](const PlaneJob& p) { return p.tile0; });
    const PlaneJob& J = jobs[j];
    const int t = (int)blockIdx.x - J.tile0;
    if constexpr (sizeof(T) == 1)
        planes_tile8<TH>(J.luma, J.stride, J.w, J.h, J.out, J.psize, J.sw, J.sh, (t % J.tiles_x) * K1_TW, (t / J.tiles_x) * TH);
    else
        planes_tile16<TH>(reinterpret_cast<const uint16_t*>(J.luma), J.stride, J.w, J.h, reinterpret_cast<uint16_t*>(J.out), J.psize,
                          J.sw, J.sh, (t % J.tiles_x) * K1_TW, (t / J.tiles_x) * TH, maxv);
}

// col_mv, enc/frame.rs:944-947, for every stream's new reference
__global__ void col_batch_kernel(const PlaneJob* __restrict__ jobs, int njobs, int total) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const int j = find_job(jobs, njobs, i, [](const PlaneJob& p) { return p.mb0; });
    const PlaneJob& J = jobs[j];
    const int m = i - J.mb0;
    ColMv c;
    c.mv[0] = c.mv[1] = 0;
    c.valid = 0;
    if (J.col_states && J.col_states[m].inter) {
        c.mv[0] = J.col_states[m].mvs[5][0];
        c.mv[1] = J.col_states[m].mvs[5][1];
        c.valid = 1;
    }
    J.col[m] = c;
}

// H264Encoder::source (enc/mod.rs:502-519) for every stream: one block per padded row; T the samples'
// type (strides in samples).
template <class T>
__global__ void source_batch_kernel(const SrcJob* __restrict__ jobs, int njobs) {
    const int j = find_job(jobs, njobs, (int)blockIdx.x, [](const SrcJob& p) { return p.row0; });
    const SrcJob& J = jobs[j];
    const int y = (int)blockIdx.x - J.row0;
    const T* row = reinterpret_cast<const T*>(J.src) + (size_t)min(y, J.h - 1) * J.stride;
    T* out = reinterpret_cast<T*>(J.dst) + (size_t)y * J.pw;
    for (int x = threadIdx.x; x < J.pw; x += blockDim.x) out[x] = row[min(x, J.w - 1)];
}

// Every stream's auto-mode analysis in one launch (each stream's parameters in the table). MINB: the CTAs
// an SM must hold (the tuner's choice, 4 to 6), which caps the registers a thread at 128, 96 or 80.
template <class T, int MINB>
__global__ void __launch_bounds__(K2_WARPS * 32, MINB) analyse_batch_kernel(const AnalyseParams* __restrict__ table,
                                                                                     const uint32_t* __restrict__ order,
                                                                                     unsigned ntickets, unsigned* ticket,
                                                                                     const unsigned* err) {
    __shared__ WarpSmem<T> smem[K2_WARPS];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    WarpSmem<T>& S = smem[wid];
    for (;;) {
        unsigned t = 0;
        if (lane == 0) t = atomicAdd(ticket, 1u);
        t = __shfl_sync(FULL, t, 0);
        if (t >= ntickets || ld_acquire(err) != 0) break;
        const uint32_t e = order[t];
        const AnalyseParams& P = table[e >> 20];
        const int mb = (int)(e & 0xFFFFFu), mbx = mb % P.mb_w, mby = mb / P.mb_w;
        if (lane == 0) {
            S.mb = mb;
            S.mbx = mbx;
            S.mby = mby;
        }
        __syncwarp();
        const int start = P.band_start[mby];
        bool ok = true;
        if (mbx > 0) ok = wait_published(P, mb - 1);
        if (ok && mby > start) ok = wait_published(P, (mbx + 1 < P.mb_w) ? mb - P.mb_w + 1 : mb - P.mb_w);
        ok = __all_sync(FULL, ok);
        if (!ok) break;
        load_neighbours(P, S, P.states_out);
        analyse(P, S, true);
        __threadfence();
        __syncwarp();
        if (lane == 0) st_release(&P.flags[mb], P.epoch);
    }
}

int cuda_status(cudaError_t e) {
    if (e == cudaSuccess) return IRONAV_OK;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver || e == cudaErrorNoKernelImageForDevice)
        return IRONAV_HARDWARE_UNAVAILABLE;
    return IRONAV_INTERNAL;
}

#define CK(x)                                           \
    do {                                                \
        cudaError_t e_ = (x);                           \
        if (e_ != cudaSuccess) return cuda_status(e_); \
    } while (0)

}  // namespace

// The batched step's knobs (ironav_batch_tuning): the analysis' CTAs per SM (4, 5 or 6: its register cap),
// the planes' tile rows (16 or 8) and the ticket order (0: the merged wavefront, ties by stream; 1: ties
// by stream size, largest first).
constexpr int TUNE_MINB[3] = {4, 5, 6};
constexpr int TUNE_TH[2] = {16, 8};

struct ironav_batch {
    std::vector<ironav_ctx*> ctx;
    cudaStream_t stream = nullptr;
    int bd = 8;  // every stream's sample depth
    int n = 0, total_mbs = 0, total_tiles = 0, total_rows = 0, k2_blocks = 0;
    int tiles_th[2] = {0, 0};  // the planes' tiles at each tile height
    int k2_blocks_v[4] = {0, 0, 0, 0};  // the analysis' persistent grid for each variant (TUNE_MINB's, then the group form)
    int minb_i = 0, th_i = 0, order_i = 0;  // the current tuning (indices into TUNE_MINB or 3 for the group form, TUNE_TH; the order)
    std::vector<int> mb0;  // each stream's first flag
    uint32_t* d_order = nullptr;  // the two ticket orders, total_mbs each
    unsigned* d_flags = nullptr;
    unsigned* d_counters = nullptr;  // [0] ticket, [1] error
    PlaneJob* d_pjobs = nullptr;
    SrcJob* d_sjobs = nullptr;
    AnalyseParams* d_table = nullptr;
    // pinned staging of the per-step tables, reused once the previous step's copies are done
    PlaneJob* h_pjobs = nullptr;
    SrcJob* h_sjobs = nullptr;
    AnalyseParams* h_table = nullptr;
    cudaEvent_t copied = nullptr;
    bool pending = false;
    // decide mode (allocated on first use): the streams' parameters and the launch's grid
    DecideParams* d_dtable = nullptr;
    DecideParams* h_dtable = nullptr;
    int k7_blocks = 0;
    // decide mode under CABAC (allocated on first use): the streams' parameters and the chains (stream << 16 |
    // slice band), one CTA each
    RdParams* d_rdtable = nullptr;
    RdParams* h_rdtable = nullptr;
    uint32_t* d_chains = nullptr;
    int nchains = 0, nchains3 = 0;  // the first nchains3 (the longest bands) on three warps each
    cudaStream_t aux = nullptr;     // the one-warp launch runs beside the three-warp one
    cudaEvent_t fork = nullptr, join = nullptr;
    // deblocking (allocated on first use): the streams' jobs, their rows' merged ticket order, progress
    // words, and the concatenated slice tables (pinned staging reused once the previous copies are done)
    DbkJob* d_kjobs = nullptr;
    DbkJob* h_kjobs = nullptr;
    uint32_t* d_korder = nullptr;
    unsigned* d_kprogress = nullptr;
    int total_rows2 = 0;  // sum of 2 * mb_h
    ironav_dbk_slice* d_kslices = nullptr;
    ironav_dbk_slice* h_kslices = nullptr;
    int kslice_cap = 0;
};

static void free_batch(ironav_batch* b) {
    cudaFree(b->d_order);
    cudaFree(b->d_flags);
    cudaFree(b->d_counters);
    cudaFree(b->d_pjobs);
    cudaFree(b->d_sjobs);
    cudaFree(b->d_table);
    cudaFreeHost(b->h_pjobs);
    cudaFreeHost(b->h_sjobs);
    cudaFreeHost(b->h_table);
    cudaFree(b->d_dtable);
    cudaFreeHost(b->h_dtable);
    cudaFree(b->d_rdtable);
    cudaFreeHost(b->h_rdtable);
    cudaFree(b->d_chains);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->join) cudaEventDestroy(b->join);
    if (b->aux) cudaStreamDestroy(b->aux);
    cudaFree(b->d_kjobs);
    cudaFreeHost(b->h_kjobs);
    cudaFree(b->d_korder);
    cudaFree(b->d_kprogress);
    cudaFree(b->d_kslices);
    cudaFreeHost(b->h_kslices);
    if (b->copied) cudaEventDestroy(b->copied);
    delete b;
}

extern "C" int ironav_batch_create(ironav_batch** out, ironav_ctx* const* ctxs, int n) {
    if (!out || !ctxs || n < 1 || n > 4096) return IRONAV_INVALID_ARGUMENT;
    *out = nullptr;
    for (int i = 0; i < n; i++)
        if (!ctxs[i] || ctxs[i]->bd != ctxs[0]->bd || ctxs[i]->stream != ctxs[0]->stream || ctxs[i]->nmb > (1 << 20))
            return IRONAV_INVALID_ARGUMENT;
    ironav_batch* b = new ironav_batch();
    b->ctx.assign(ctxs, ctxs + n);
    b->n = n;
    b->stream = ctxs[0]->stream;
    b->bd = ctxs[0]->bd;
    // the streams' wavefronts merged: key x + 2 * (y - band start), then (order 0) stream or (order 1) the
    // stream's size, largest first, then stream, then raster
    std::vector<std::tuple<int, int, int, int>> keys[2];
    for (int i = 0; i < n; i++) {
        const ironav_ctx* c = ctxs[i];
        std::vector<int> start(c->mb_h);
        cudaMemcpy(start.data(), c->d_band_start, sizeof(int) * c->mb_h, cudaMemcpyDeviceToHost);
        b->mb0.push_back(b->total_mbs);
        for (int m = 0; m < c->nmb; m++) {
            const int x = m % c->mb_w, y = m / c->mb_w, k = x + 2 * (y - start[y]);
            keys[0].emplace_back(k, i, i, m);
            keys[1].emplace_back(k, -c->nmb, i, m);
        }
        b->total_mbs += c->nmb;
        for (int v = 0; v < 2; v++) b->tiles_th[v] += ((c->sw + K1_TW - 1) / K1_TW) * ((c->sh + TUNE_TH[v] - 1) / TUNE_TH[v]);
        b->total_rows += c->ph;
    }
    b->total_tiles = b->tiles_th[0];
    std::vector<uint32_t> order(2 * (size_t)b->total_mbs);
    for (int v = 0; v < 2; v++) {
        std::sort(keys[v].begin(), keys[v].end());
        for (size_t k = 0; k < keys[v].size(); k++)
            order[v * (size_t)b->total_mbs + k] = ((uint32_t)std::get<2>(keys[v][k]) << 20) | (uint32_t)std::get<3>(keys[v][k]);
    }
    auto fail = [&](cudaError_t e) {
        const int s = cuda_status(e);
        free_batch(b);
        return s;
    };
    cudaError_t e;
    if ((e = cudaMalloc(&b->d_order, sizeof(uint32_t) * order.size())) != cudaSuccess) return fail(e);
    if ((e = cudaMemcpy(b->d_order, order.data(), sizeof(uint32_t) * order.size(), cudaMemcpyHostToDevice)) != cudaSuccess) return fail(e);
    if ((e = cudaMalloc(&b->d_flags, sizeof(unsigned) * b->total_mbs)) != cudaSuccess) return fail(e);
    if ((e = cudaMalloc(&b->d_counters, sizeof(unsigned) * 2)) != cudaSuccess) return fail(e);
    if ((e = cudaMemset(b->d_counters, 0, sizeof(unsigned) * 2)) != cudaSuccess) return fail(e);  // read by a sync before any step
    if ((e = cudaMalloc(&b->d_pjobs, sizeof(PlaneJob) * n)) != cudaSuccess) return fail(e);
    if ((e = cudaMalloc(&b->d_sjobs, sizeof(SrcJob) * n)) != cudaSuccess) return fail(e);
    if ((e = cudaMalloc(&b->d_table, sizeof(AnalyseParams) * n)) != cudaSuccess) return fail(e);
    if ((e = cudaHostAlloc(&b->h_pjobs, sizeof(PlaneJob) * n, cudaHostAllocDefault)) != cudaSuccess) return fail(e);
    if ((e = cudaHostAlloc(&b->h_sjobs, sizeof(SrcJob) * n, cudaHostAllocDefault)) != cudaSuccess) return fail(e);
    if ((e = cudaHostAlloc(&b->h_table, sizeof(AnalyseParams) * n, cudaHostAllocDefault)) != cudaSuccess) return fail(e);
    if ((e = cudaEventCreateWithFlags(&b->copied, cudaEventDisableTiming)) != cudaSuccess) return fail(e);
    // the persistent grid of each analysis variant: every CTA the occupancy allows
    for (int v = 0; v < 3; v++) {
        int per_sm = 0;
        const void* fn = nullptr;
        if (b->bd > 8)
            fn = v == 0 ? (const void*)analyse_batch_kernel<uint16_t, 4> : v == 1 ? (const void*)analyse_batch_kernel<uint16_t, 5>
                                                                                  : (const void*)analyse_batch_kernel<uint16_t, 6>;
        else
            fn = v == 0 ? (const void*)analyse_batch_kernel<uint8_t, 4> : v == 1 ? (const void*)analyse_batch_kernel<uint8_t, 5>
                                                                                 : (const void*)analyse_batch_kernel<uint8_t, 6>;
        if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, K2_WARPS * 32, 0)) != cudaSuccess) return fail(e);
        b->k2_blocks_v[v] = std::max(1, per_sm) * ctxs[0]->nsm;
    }
    {
        int per_sm = 0;
        const void* fn = b->bd > 8 ? (const void*)g8::analyse_batch_g8_kernel<uint16_t> : (const void*)g8::analyse_batch_g8_kernel<uint8_t>;
        if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, g8::WARPS * 32, 0)) != cudaSuccess) return fail(e);
        b->k2_blocks_v[3] = std::max(1, per_sm) * ctxs[0]->nsm;
    }
    b->k2_blocks = b->k2_blocks_v[0];
    *out = b;
    return IRONAV_OK;
}

extern "C" int ironav_batch_destroy(ironav_batch* b) {
    if (!b) return IRONAV_INVALID_ARGUMENT;
    cudaStreamSynchronize(b->stream);
    free_batch(b);
    return IRONAV_OK;
}

extern "C" int ironav_batch_step(ironav_batch* b, const void* const* d_src, const void* const* d_ref,
                                 const ironav_mbstate* const* d_col, ironav_mbstate* const* d_states,
                                 ironav_mbresult* const* d_results) {
    if (!b || !d_src || !d_ref || !d_states || !d_results) return IRONAV_INVALID_ARGUMENT;
    for (int i = 0; i < b->n; i++) {
        const ironav_ctx* c = b->ctx[i];
        // the step pushes one reference: afterwards min(nrefs + 1, max_refs) are held
        if (!d_src[i] || !d_ref[i] || !d_states[i] || !d_results[i] || !c->have_params || c->intra_pic || c->nact > std::min(c->nrefs + 1, c->max_refs))
            return IRONAV_INVALID_ARGUMENT;
    }
    // the staging tables are reused: the previous step's copies must have left them
    if (b->pending) CK(cudaEventSynchronize(b->copied));
    int tile = 0, row = 0;
    for (int i = 0; i < b->n; i++) {
        ironav_ctx* c = b->ctx[i];
        const int slot = take_ref_slot(c);
        PlaneJob& pj = b->h_pjobs[i];
        pj.luma = static_cast<const uint8_t*>(d_ref[i]);
        pj.stride = c->width;
        pj.w = c->width;
        pj.h = c->height;
        pj.out = c->d_planes[slot];
        pj.psize = c->psize;
        pj.sw = c->sw;
        pj.sh = c->sh;
        pj.tiles_x = (c->sw + K1_TW - 1) / K1_TW;
        pj.tile0 = tile;
        const int th = TUNE_TH[b->th_i];
        pj.col_states = d_col ? d_col[i] : nullptr;
        pj.col = c->d_col[slot];
        pj.nmb = c->nmb;
        pj.mb0 = b->mb0[i];
        tile += pj.tiles_x * ((c->sh + th - 1) / th);
        SrcJob& sj = b->h_sjobs[i];
        sj.src = static_cast<const uint8_t*>(d_src[i]);
        sj.stride = c->width;
        sj.w = c->width;
        sj.h = c->height;
        sj.dst = c->d_src;
        sj.pw = c->pw;
        sj.ph = c->ph;
        sj.row0 = row;
        row += c->ph;
        AnalyseParams& p = b->h_table[i];
        fill_params(c, p);
        p.states_out = d_states[i];
        p.results = d_results[i];
        p.flags = b->d_flags + b->mb0[i];
        p.epoch = 1;  // the flags are cleared every step
        p.err = b->d_counters + 1;
        p.nmb = c->nmb;
    }
    CK(cudaMemcpyAsync(b->d_pjobs, b->h_pjobs, sizeof(PlaneJob) * b->n, cudaMemcpyHostToDevice, b->stream));
    CK(cudaMemcpyAsync(b->d_sjobs, b->h_sjobs, sizeof(SrcJob) * b->n, cudaMemcpyHostToDevice, b->stream));
    CK(cudaMemcpyAsync(b->d_table, b->h_table, sizeof(AnalyseParams) * b->n, cudaMemcpyHostToDevice, b->stream));
    CK(cudaEventRecord(b->copied, b->stream));
    b->pending = true;
    const int tiles = b->tiles_th[b->th_i], maxv = (1 << b->bd) - 1;
    if (b->bd > 8) {
        source_batch_kernel<uint16_t><<<b->total_rows, 128, 0, b->stream>>>(b->d_sjobs, b->n);
        if (b->th_i == 0) planes_batch_kernel<uint16_t, 16><<<tiles, 16 * 16, 0, b->stream>>>(b->d_pjobs, b->n, maxv);
        else planes_batch_kernel<uint16_t, 8><<<tiles, 16 * 8, 0, b->stream>>>(b->d_pjobs, b->n, maxv);
    } else {
        source_batch_kernel<uint8_t><<<b->total_rows, 128, 0, b->stream>>>(b->d_sjobs, b->n);
        if (b->th_i == 0) planes_batch_kernel<uint8_t, 16><<<tiles, 16 * 16, 0, b->stream>>>(b->d_pjobs, b->n, maxv);
        else planes_batch_kernel<uint8_t, 8><<<tiles, 16 * 8, 0, b->stream>>>(b->d_pjobs, b->n, maxv);
    }
    col_batch_kernel<<<(b->total_mbs + 255) / 256, 256, 0, b->stream>>>(b->d_pjobs, b->n, b->total_mbs);
    CK(cudaMemsetAsync(b->d_flags, 0, sizeof(unsigned) * b->total_mbs, b->stream));
    CK(cudaMemsetAsync(b->d_counters, 0, sizeof(unsigned) * 2, b->stream));
    const uint32_t* order = b->d_order + (size_t)b->order_i * b->total_mbs;
    const unsigned nt = (unsigned)b->total_mbs;
    unsigned* tk = b->d_counters;
    const unsigned* er = b->d_counters + 1;
    bool group = b->minb_i == 3;
    for (int i = 0; i < b->n && group; i++)
        if (b->ctx[i]->learned) group = false;  // the group form has no learned judge: the warp form then
    if (group) {
        if (b->bd > 8) g8::analyse_batch_g8_kernel<uint16_t><<<b->k2_blocks_v[3], g8::WARPS * 32, 0, b->stream>>>(b->d_table, order, nt, tk, er);
        else g8::analyse_batch_g8_kernel<uint8_t><<<b->k2_blocks_v[3], g8::WARPS * 32, 0, b->stream>>>(b->d_table, order, nt, tk, er);
        return cuda_status(cudaGetLastError());
    }
    const int minb = b->minb_i == 3 ? 0 : b->minb_i;
    const int grid = b->k2_blocks_v[minb];
    if (b->bd > 8) {
        if (minb == 0) analyse_batch_kernel<uint16_t, 4><<<grid, K2_WARPS * 32, 0, b->stream>>>(b->d_table, order, nt, tk, er);
        else if (minb == 1) analyse_batch_kernel<uint16_t, 5><<<grid, K2_WARPS * 32, 0, b->stream>>>(b->d_table, order, nt, tk, er);
        else analyse_batch_kernel<uint16_t, 6><<<grid, K2_WARPS * 32, 0, b->stream>>>(b->d_table, order, nt, tk, er);
    } else {
        if (minb == 0) analyse_batch_kernel<uint8_t, 4><<<grid, K2_WARPS * 32, 0, b->stream>>>(b->d_table, order, nt, tk, er);
        else if (minb == 1) analyse_batch_kernel<uint8_t, 5><<<grid, K2_WARPS * 32, 0, b->stream>>>(b->d_table, order, nt, tk, er);
        else analyse_batch_kernel<uint8_t, 6><<<grid, K2_WARPS * 32, 0, b->stream>>>(b->d_table, order, nt, tk, er);
    }
    return cuda_status(cudaGetLastError());
}

// ---- the batched step's tuner ---------------------------------------------------------------------------

static int tuning_index(const ironav_batch_tuning* t, int* mi, int* ti) {
    *mi = -1;
    *ti = -1;
    if (t->k2_group == 8) {
        if (t->k2_ctas_per_sm == 4) *mi = 3;
    } else if (t->k2_group == 0) {
        for (int v = 0; v < 3; v++)
            if (t->k2_ctas_per_sm == TUNE_MINB[v]) *mi = v;
    }
    for (int v = 0; v < 2; v++)
        if (t->k1_tile_rows == TUNE_TH[v]) *ti = v;
    return (*mi < 0 || *ti < 0 || t->order < 0 || t->order > 1) ? IRONAV_INVALID_ARGUMENT : IRONAV_OK;
}

extern "C" int ironav_batch_set_tuning(ironav_batch* b, const ironav_batch_tuning* t) {
    if (!b || !t) return IRONAV_INVALID_ARGUMENT;
    int mi, ti;
    if (tuning_index(t, &mi, &ti) != IRONAV_OK) return IRONAV_INVALID_ARGUMENT;
    b->minb_i = mi;
    b->th_i = ti;
    b->order_i = t->order;
    return IRONAV_OK;
}

extern "C" int ironav_batch_get_tuning(const ironav_batch* b, ironav_batch_tuning* t) {
    if (!b || !t) return IRONAV_INVALID_ARGUMENT;
    t->k2_ctas_per_sm = b->minb_i == 3 ? 4 : TUNE_MINB[b->minb_i];
    t->k1_tile_rows = TUNE_TH[b->th_i];
    t->order = b->order_i;
    t->k2_group = b->minb_i == 3 ? 8 : 0;
    t->ms = 0.f;
    return IRONAV_OK;
}

// Every candidate setting (the analysis' CTAs per SM x the planes' tile rows x the ticket order) timed on
// `reps` batched steps of the caller's inputs with CUDA events on the batch's stream; the fastest (the
// least median) is kept. Before each step every context's reference ring is put back as it was, so the
// steps all take the same slot and the batch ends exactly as after one ironav_batch_step with these inputs.
extern "C" int ironav_batch_autotune(ironav_batch* b, const void* const* d_src, const void* const* d_ref,
                                     const ironav_mbstate* const* d_col, ironav_mbstate* const* d_states,
                                     ironav_mbresult* const* d_results, int reps, ironav_batch_tuning* best,
                                     ironav_batch_tuning* all, int cap, int* n_all) {
    if (!b || reps < 1 || reps > 64 || !best) return IRONAV_INVALID_ARGUMENT;
    struct Ring {
        int nrefs;
        int slot_of[MAX_REFS];
    };
    std::vector<Ring> rings(b->n);
    for (int i = 0; i < b->n; i++) {
        rings[i].nrefs = b->ctx[i]->nrefs;
        memcpy(rings[i].slot_of, b->ctx[i]->slot_of, sizeof(rings[i].slot_of));
    }
    auto restore = [&] {
        for (int i = 0; i < b->n; i++) {
            b->ctx[i]->nrefs = rings[i].nrefs;
            memcpy(b->ctx[i]->slot_of, rings[i].slot_of, sizeof(rings[i].slot_of));
        }
    };
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    int count = 0, bm = 0, bt = 0, bo = 0;
    float best_ms = 0.f;
    int status = IRONAV_OK;
    for (int mi = 0; mi < 4 && status == IRONAV_OK; mi++)
        for (int ti = 0; ti < 2 && status == IRONAV_OK; ti++)
            for (int oi = 0; oi < 2 && status == IRONAV_OK; oi++) {
                b->minb_i = mi;
                b->th_i = ti;
                b->order_i = oi;
                std::vector<float> ms(reps + 1);
                for (int r = 0; r <= reps && status == IRONAV_OK; r++) {  // the first step is a warm-up
                    restore();
                    cudaEventRecord(e0, b->stream);
                    status = ironav_batch_step(b, d_src, d_ref, d_col, d_states, d_results);
                    cudaEventRecord(e1, b->stream);
                    if (status == IRONAV_OK) status = ironav_batch_sync(b);
                    if (status == IRONAV_OK && cudaEventElapsedTime(&ms[r], e0, e1) != cudaSuccess) status = IRONAV_INTERNAL;
                }
                if (status != IRONAV_OK) break;
                std::sort(ms.begin() + 1, ms.end());
                const float med = ms[1 + reps / 2];
                if (all && count < cap) {
                    all[count].k2_ctas_per_sm = mi == 3 ? 4 : TUNE_MINB[mi];
                    all[count].k1_tile_rows = TUNE_TH[ti];
                    all[count].order = oi;
                    all[count].k2_group = mi == 3 ? 8 : 0;
                    all[count].ms = med;
                }
                if (count == 0 || med < best_ms) {
                    best_ms = med;
                    bm = mi;
                    bt = ti;
                    bo = oi;
                }
                count++;
            }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    b->minb_i = bm;
    b->th_i = bt;
    b->order_i = bo;
    if (n_all) *n_all = count;
    if (status != IRONAV_OK) return status;
    best->k2_ctas_per_sm = bm == 3 ? 4 : TUNE_MINB[bm];
    best->k1_tile_rows = TUNE_TH[bt];
    best->order = bo;
    best->k2_group = bm == 3 ? 8 : 0;
    best->ms = best_ms;
    return IRONAV_OK;
}

extern "C" int ironav_batch_sync(ironav_batch* b) {
    if (!b) return IRONAV_INVALID_ARGUMENT;
    unsigned err = 0;
    CK(cudaMemcpyAsync(&err, b->d_counters + 1, sizeof(unsigned), cudaMemcpyDeviceToHost, b->stream));
    CK(cudaStreamSynchronize(b->stream));
    b->pending = false;  // the staging tables are free again
    if (err & 1u) return IRONAV_TIMEOUT;
    if (err & 4u) return IRONAV_INVALID_INPUT;  // a record names a slice beyond its stream's table
    return err ? IRONAV_INTERNAL : IRONAV_OK;
}

// ironav_batch_decide under CABAC: every stream's slice bands as chains of one launch (decide_rd_batch_kernel).
static int batch_decide_rd(ironav_batch* b, ironav_mbstate* const* d_states, ironav_mbcode* const* d_codes, void* const* d_y,
                           const int* y_strides, void* const* d_cb, void* const* d_cr, const int* c_strides) {
    if (!b->d_rdtable) {
        CK(cudaMalloc(&b->d_rdtable, sizeof(RdParams) * b->n));
        CK(cudaHostAlloc(&b->h_rdtable, sizeof(RdParams) * b->n, cudaHostAllocDefault));
        // the longest bands (at least 3/4 of the longest's macroblocks) first, on three warps each; the rest on one
        std::vector<std::pair<int, uint32_t>> len;
        int most = 0;
        for (int i = 0; i < b->n; i++) {
            const ironav_ctx* c = b->ctx[i];
            for (int k = 0; k < c->nslices; k++) {
                const int mbs = (c->band_rows[k + 1] - c->band_rows[k]) * c->mb_w;
                len.emplace_back(mbs, (uint32_t)i << 16 | (uint32_t)k);
                most = std::max(most, mbs);
            }
        }
        std::vector<uint32_t> chains;
        for (const auto& e : len)
            if (4 * e.first >= 3 * most) chains.push_back(e.second);
        b->nchains3 = (int)chains.size();
        for (const auto& e : len)
            if (4 * e.first < 3 * most) chains.push_back(e.second);
        CK(cudaMalloc(&b->d_chains, sizeof(uint32_t) * chains.size()));
        CK(cudaMemcpy(b->d_chains, chains.data(), sizeof(uint32_t) * chains.size(), cudaMemcpyHostToDevice));
        b->nchains = (int)chains.size();
        CK(cudaStreamCreateWithFlags(&b->aux, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&b->join, cudaEventDisableTiming));
        CK(cudaFuncSetAttribute(decide_rd3_batch_kernel<uint8_t>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rd3_smem_bytes<uint8_t>()));
        CK(cudaFuncSetAttribute(decide_rd3_batch_kernel<uint16_t>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)rd3_smem_bytes<uint16_t>()));
    }
    if (b->pending) CK(cudaEventSynchronize(b->copied));
    for (int i = 0; i < b->n; i++) {
        ironav_ctx* c = b->ctx[i];
        RdParams& p = b->h_rdtable[i];
        memset(&p, 0, sizeof(p));
        int s = fill_decide_params(c, p.D, d_states[i], d_codes[i], d_y[i], y_strides[i], d_cb[i], d_cr[i], c_strides[i]);
        if (s == IRONAV_OK) s = cabac_setup(c);
        if (s != IRONAV_OK) return s;
        p.D.C.A.err = b->d_counters + 1;
        p.D.C.err = b->d_counters + 1;
        p.nbs = c->d_rd_nb;
        p.band_rows = c->d_band_rows;
        p.step = c->d_cab_step;
        p.lam2 = 1.6 * std::pow(2.0, ((double)c->qpp - 12.0) / 3.0);  // decide_rd's lambda2, enc/frame.rs:1464
        p.nbands = c->nslices;
        p.t8 = c->t8;
        const size_t B = c->bd > 8 ? 2 : 1, ly = (size_t)c->pw * c->ph * B, cy = (size_t)(c->pw / 2) * (c->ph / 2) * B;
        for (int k = 0; k < 2; k++) {
            uint8_t* base = c->d_rd_scr + k * (ly + 2 * cy);
            p.scr[3 * k] = base;
            p.scr[3 * k + 1] = base + ly;
            p.scr[3 * k + 2] = base + ly + cy;
        }
        p.scr_ys = c->pw;
        p.scr_cs = c->pw / 2;
    }
    CK(cudaMemcpyAsync(b->d_rdtable, b->h_rdtable, sizeof(RdParams) * b->n, cudaMemcpyHostToDevice, b->stream));
    CK(cudaEventRecord(b->copied, b->stream));
    b->pending = true;
    CK(cudaMemsetAsync(b->d_counters, 0, sizeof(unsigned) * 2, b->stream));
    // the short bands' one-warp launch on the side stream, beside the long bands' three-warp launch
    const int n1 = b->nchains - b->nchains3;
    if (n1 > 0) {
        CK(cudaEventRecord(b->fork, b->stream));
        CK(cudaStreamWaitEvent(b->aux, b->fork, 0));
        if (b->bd > 8) decide_rd_batch_kernel<uint16_t><<<n1, 32, 0, b->aux>>>(b->d_rdtable, b->d_chains + b->nchains3, n1);
        else decide_rd_batch_kernel<uint8_t><<<n1, 32, 0, b->aux>>>(b->d_rdtable, b->d_chains + b->nchains3, n1);
        CK(cudaGetLastError());
    }
    if (b->bd > 8)
        decide_rd3_batch_kernel<uint16_t><<<b->nchains3, RD3_WARPS * 32, rd3_smem_bytes<uint16_t>(), b->stream>>>(b->d_rdtable, b->d_chains,
                                                                                                              b->nchains3);
    else
        decide_rd3_batch_kernel<uint8_t><<<b->nchains3, RD3_WARPS * 32, rd3_smem_bytes<uint8_t>(), b->stream>>>(b->d_rdtable, b->d_chains,
                                                                                                            b->nchains3);
    CK(cudaGetLastError());
    if (n1 > 0) {
        CK(cudaEventRecord(b->join, b->aux));
        CK(cudaStreamWaitEvent(b->stream, b->join, 0));
    }
    return IRONAV_OK;
}

extern "C" int ironav_batch_decide(ironav_batch* b, ironav_mbstate* const* d_states, ironav_mbcode* const* d_codes, void* const* d_y,
                                   const int* y_strides, void* const* d_cb, void* const* d_cr, const int* c_strides) {
    if (!b || !d_states || !d_codes || !d_y || !y_strides || !d_cb || !d_cr || !c_strides) return IRONAV_INVALID_ARGUMENT;
    for (int i = 1; i < b->n; i++)
        if (b->ctx[i]->cabac != b->ctx[0]->cabac) return IRONAV_INVALID_ARGUMENT;  // one entropy coding for the batch
    if (!b->d_dtable) {
        CK(cudaMalloc(&b->d_dtable, sizeof(DecideParams) * b->n));
        CK(cudaHostAlloc(&b->h_dtable, sizeof(DecideParams) * b->n, cudaHostAllocDefault));
        int per_sm = 0;
        if (b->bd > 8) CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, decide_batch_kernel<uint16_t>, K7_WARPS * 32, 0));
        else CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, decide_batch_kernel<uint8_t>, K7_WARPS * 32, 0));
        b->k7_blocks = std::max(1, per_sm) * b->ctx[0]->nsm;
    }
    // the staging table is reused: the previous step's copies must have left it
    if (b->pending) CK(cudaEventSynchronize(b->copied));
    for (int i = 0; i < b->n; i++) {
        ironav_ctx* c = b->ctx[i];
        if (!d_states[i] || !d_codes[i] || !d_y[i] || !d_cb[i] || !d_cr[i] || y_strides[i] < c->pw || c_strides[i] < c->pw / 2)
            return IRONAV_INVALID_ARGUMENT;
        // the planes as the single-stream device form; states and codes are written as 32-bit words
        const uintptr_t a = reinterpret_cast<uintptr_t>(d_y[i]) | reinterpret_cast<uintptr_t>(d_cb[i]) | reinterpret_cast<uintptr_t>(d_cr[i]);
        const int B = b->bd > 8 ? 2 : 1;
        if ((a & 15) || (y_strides[i] * B) % 16 || c_strides[i] % 8) return IRONAV_INVALID_ARGUMENT;
        if ((reinterpret_cast<uintptr_t>(d_states[i]) | reinterpret_cast<uintptr_t>(d_codes[i])) & 3) return IRONAV_INVALID_ARGUMENT;
        if (c->cabac) continue;
        DecideParams& p = b->h_dtable[i];
        const int s = fill_decide_params(c, p, d_states[i], d_codes[i], d_y[i], y_strides[i], d_cb[i], d_cr[i], c_strides[i]);
        if (s != IRONAV_OK) return s;
        p.C.A.flags = b->d_flags + b->mb0[i];
        p.C.A.epoch = 1;  // the flags are cleared every step
        p.C.A.err = b->d_counters + 1;
        p.C.err = b->d_counters + 1;
    }
    if (b->ctx[0]->cabac) return batch_decide_rd(b, d_states, d_codes, d_y, y_strides, d_cb, d_cr, c_strides);
    CK(cudaMemcpyAsync(b->d_dtable, b->h_dtable, sizeof(DecideParams) * b->n, cudaMemcpyHostToDevice, b->stream));
    CK(cudaEventRecord(b->copied, b->stream));
    b->pending = true;
    CK(cudaMemsetAsync(b->d_flags, 0, sizeof(unsigned) * b->total_mbs, b->stream));
    CK(cudaMemsetAsync(b->d_counters, 0, sizeof(unsigned) * 2, b->stream));
    if (b->bd > 8)
        decide_batch_kernel<uint16_t><<<b->k7_blocks, K7_WARPS * 32, 0, b->stream>>>(b->d_dtable, b->d_order, (unsigned)b->total_mbs,
                                                                                     b->d_counters, b->d_counters + 1);
    else
        decide_batch_kernel<uint8_t><<<b->k7_blocks, K7_WARPS * 32, 0, b->stream>>>(b->d_dtable, b->d_order, (unsigned)b->total_mbs,
                                                                                    b->d_counters, b->d_counters + 1);
    return cuda_status(cudaGetLastError());
}

extern "C" int ironav_batch_deblock(ironav_batch* b, void* const* d_y, const int* y_strides, void* const* d_cb, void* const* d_cr,
                                    const int* c_strides, const ironav_dbk_mb* const* d_mbs, const ironav_dbk_slice* const* slices,
                                    const int* nslices) {
    if (!b || !d_y || !y_strides || !d_cb || !d_cr || !c_strides || !d_mbs || !slices || !nslices) return IRONAV_INVALID_ARGUMENT;
    int total_slices = 0;
    for (int i = 0; i < b->n; i++) {
        const ironav_ctx* c = b->ctx[i];
        if (!d_y[i] || !d_cb[i] || !d_cr[i] || !d_mbs[i] || !slices[i] || nslices[i] < 1 || nslices[i] > 65535 || y_strides[i] < c->pw ||
            c_strides[i] < c->pw / 2)
            return IRONAV_INVALID_ARGUMENT;
        // the planes as the single-stream device form (16-byte rows); the records are read as 32-bit words
        const uintptr_t a = reinterpret_cast<uintptr_t>(d_y[i]) | reinterpret_cast<uintptr_t>(d_cb[i]) | reinterpret_cast<uintptr_t>(d_cr[i]);
        if ((a & 15) || (y_strides[i] * (b->bd > 8 ? 2 : 1)) % 16 || c_strides[i] % 8 || (reinterpret_cast<uintptr_t>(d_mbs[i]) & 3))
            return IRONAV_INVALID_ARGUMENT;
        total_slices += nslices[i];
    }
    if (!b->d_kjobs) {
        CK(cudaMalloc(&b->d_kjobs, sizeof(DbkJob) * b->n));
        CK(cudaHostAlloc(&b->h_kjobs, sizeof(DbkJob) * b->n, cudaHostAllocDefault));
        // every stream's row tickets merged by the stream's own ticket, then stream
        std::vector<std::pair<int, int>> keys;
        for (int i = 0; i < b->n; i++)
            for (int t = 0; t < 2 * b->ctx[i]->mb_h; t++) keys.emplace_back(t, i);
        std::sort(keys.begin(), keys.end());
        std::vector<uint32_t> order(keys.size());
        for (size_t k = 0; k < keys.size(); k++) order[k] = ((uint32_t)keys[k].second << 20) | (uint32_t)keys[k].first;
        b->total_rows2 = (int)order.size();
        CK(cudaMalloc(&b->d_korder, sizeof(uint32_t) * order.size()));
        CK(cudaMemcpy(b->d_korder, order.data(), sizeof(uint32_t) * order.size(), cudaMemcpyHostToDevice));
        CK(cudaMalloc(&b->d_kprogress, sizeof(unsigned) * order.size()));
        for (int i = 0; i < b->n; i++)
            if (!b->ctx[i]->d_dbk_edges) CK(cudaMalloc(&b->ctx[i]->d_dbk_edges, sizeof(DbkEdges) * b->ctx[i]->nmb));
    }
    // the staging tables are reused: the previous step's copies must have left them
    if (b->pending) CK(cudaEventSynchronize(b->copied));
    if (total_slices > b->kslice_cap) {
        CK(cudaStreamSynchronize(b->stream));  // the old table may still be read by queued work
        cudaFree(b->d_kslices);
        cudaFreeHost(b->h_kslices);
        b->d_kslices = nullptr;
        b->h_kslices = nullptr;
        b->kslice_cap = 0;
        const int cap = std::max(total_slices, 64);
        CK(cudaMalloc(&b->d_kslices, sizeof(ironav_dbk_slice) * cap));
        CK(cudaHostAlloc(&b->h_kslices, sizeof(ironav_dbk_slice) * cap, cudaHostAllocDefault));
        b->kslice_cap = cap;
    }
    int s0 = 0, row0 = 0;
    for (int i = 0; i < b->n; i++) {
        ironav_ctx* c = b->ctx[i];
        memcpy(b->h_kslices + s0, slices[i], sizeof(ironav_dbk_slice) * nslices[i]);
        DbkJob& J = b->h_kjobs[i];
        memset(&J, 0, sizeof(J));
        DbkParams& P = J.P;
        P.planes[0] = static_cast<uint8_t*>(d_y[i]);
        P.planes[1] = static_cast<uint8_t*>(d_cb[i]);
        P.planes[2] = static_cast<uint8_t*>(d_cr[i]);
        P.ys = y_strides[i];
        P.cs = c_strides[i];
        P.mbs = d_mbs[i];
        P.slices = b->d_kslices + s0;
        P.nslices = nslices[i];
        P.mb_w = c->mb_w;
        P.mb_h = c->mb_h;
        P.bd = b->bd;
        P.progress = b->d_kprogress + row0;
        P.ticket = b->d_counters;
        P.err = b->d_counters + 1;
        P.wait_limit = c->wait_limit;
        J.edges = static_cast<DbkEdges*>(c->d_dbk_edges);
        J.mb0 = b->mb0[i];
        s0 += nslices[i];
        row0 += 2 * c->mb_h;
    }
    CK(cudaMemcpyAsync(b->d_kslices, b->h_kslices, sizeof(ironav_dbk_slice) * total_slices, cudaMemcpyHostToDevice, b->stream));
    CK(cudaMemcpyAsync(b->d_kjobs, b->h_kjobs, sizeof(DbkJob) * b->n, cudaMemcpyHostToDevice, b->stream));
    CK(cudaEventRecord(b->copied, b->stream));
    b->pending = true;
    CK(cudaMemsetAsync(b->d_kprogress, 0, sizeof(unsigned) * b->total_rows2, b->stream));
    CK(cudaMemsetAsync(b->d_counters, 0, sizeof(unsigned) * 2, b->stream));
    const int nsm = b->ctx[0]->nsm;
    deblock_edges_batch_kernel<<<std::min((b->total_mbs + DBK_WARPS - 1) / DBK_WARPS, nsm * 16), DBK_WARPS * 32, 0, b->stream>>>(
        b->d_kjobs, b->n, b->total_mbs);
    const int rblocks = std::min((b->total_rows2 + DBK_WARPS - 1) / DBK_WARPS, nsm * 16);
    if (b->bd > 8)
        deblock_rows_batch_kernel<uint16_t><<<rblocks, DBK_WARPS * 32, 0, b->stream>>>(b->d_kjobs, b->d_korder, (unsigned)b->total_rows2,
                                                                                       b->d_counters, b->d_counters + 1);
    else
        deblock_rows_batch_kernel<uint8_t><<<rblocks, DBK_WARPS * 32, 0, b->stream>>>(b->d_kjobs, b->d_korder, (unsigned)b->total_rows2,
                                                                                      b->d_counters, b->d_counters + 1);
    return cuda_status(cudaGetLastError());
}
