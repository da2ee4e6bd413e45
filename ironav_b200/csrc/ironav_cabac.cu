// ironav_cabac.cu — CABAC for the library (include/ironav_inter.h, ironav_set_entropy): the contexts' step
// table, decide mode under CABAC (decide_rd_kernel: the rate-distortion decision, one chain per slice
// band) and the CABAC data of a picture's slices (cabac_write_kernel); ironav_stream.cu puts the slice
// headers in front and the NAL units around them.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "ctx.cuh"
#include "decide_rd.cuh"

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

// A slice's data region per macroblock: above the most a macroblock's bins can take (384 levels with
// their Exp-Golomb suffixes, the syntax before them); a slice that outgrows its region is reported.
constexpr unsigned long long CAB_MB_BYTES = 3200;

}  // namespace

int cabac_setup(ironav_ctx* c) {
    if (c->d_cab_step) return IRONAV_OK;
    // entropy(), enc/cabac.rs:162-173: -log2 of the MPS and LPS probabilities, pLPS = 0.5 * (0.01875 / 0.5)^(p / 63),
    // in 1/256 bits; next_state, 32-40, from transIdxLPS
    uint8_t trans[64];
    CK(cudaMemcpyFromSymbol(trans, TRANS_LPS, sizeof(trans)));
    uint32_t cost[64][2];
    for (int p = 0; p < 64; p++) {
        const double lps = 0.5 * std::pow(0.01875 / 0.5, (double)p / 63.0);
        cost[p][0] = (uint32_t)std::round(-std::log2(1.0 - lps) * 256.0);
        cost[p][1] = (uint32_t)std::round(-std::log2(lps) * 256.0);
    }
    uint32_t step[cab::STEP_ENTRIES];
    for (int s = 0; s < 128; s++)
        for (int bin = 0; bin < 2; bin++) {
            const int p = s >> 1, mps = s & 1;
            const int next = bin != mps ? (trans[p] << 1) | (p == 0 ? 1 - mps : mps) : ((p < 62 ? p + 1 : p) << 1) | mps;
            step[s * 2 + bin] = (uint32_t)next | cost[p][bin != mps] << 8;
        }
    CK(cudaMalloc(&c->d_cab_step, sizeof(step)));
    CK(cudaMemcpy(c->d_cab_step, step, sizeof(step), cudaMemcpyHostToDevice));
    CK(cudaMalloc(&c->d_band_rows, sizeof(int) * (c->nslices + 1)));
    CK(cudaMemcpy(c->d_band_rows, c->band_rows, sizeof(int) * (c->nslices + 1), cudaMemcpyHostToDevice));
    CK(cudaMalloc(&c->d_rd_nb, sizeof(cab::Nb) * c->nmb));
    // the three-warp form's scratch planes: luma, Cb and Cr of warp 1, then of warp 2
    const size_t B = c->bd > 8 ? 2 : 1, ly = (size_t)c->pw * c->ph * B, cy = (size_t)(c->pw / 2) * (c->ph / 2) * B;
    CK(cudaMalloc(&c->d_rd_scr, 2 * (ly + 2 * cy)));
    const size_t s8 = rd3_smem_bytes<uint8_t>(), s16 = rd3_smem_bytes<uint16_t>();
    CK(cudaFuncSetAttribute(decide_rd3_kernel<uint8_t>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s8));
    CK(cudaFuncSetAttribute(decide_rd3_kernel<uint16_t>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s16));
    return IRONAV_OK;
}

int launch_decide_rd(ironav_ctx* c, ironav_mbstate* d_states, ironav_mbcode* d_codes, void* y, int ys, void* cb, void* cr, int cs) {
    RdParams p;
    memset(&p, 0, sizeof(p));
    const int s = fill_decide_params(c, p.D, d_states, d_codes, y, ys, cb, cr, cs);
    if (s != IRONAV_OK) return s;
    const int t = cabac_setup(c);
    if (t != IRONAV_OK) return t;
    p.D.C.A.err = c->d_counters + 1;
    p.D.C.err = c->d_counters + 1;
    p.nbs = c->d_rd_nb;
    p.band_rows = c->d_band_rows;
    p.step = c->d_cab_step;
    // decide_rd's lambda2, enc/frame.rs:1464, in f64 on the host as the reference computes it
    p.lam2 = 1.6 * std::pow(2.0, ((double)c->qpp - 12.0) / 3.0);
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
    CK(cudaMemsetAsync(c->d_counters, 0, 2 * sizeof(unsigned), c->stream));
    // one stream: three warps a chain (its bands are few, so each chain's latency is the picture's)
    if (c->bd > 8) decide_rd3_kernel<uint16_t><<<c->nslices, RD3_WARPS * 32, rd3_smem_bytes<uint16_t>(), c->stream>>>(p);
    else decide_rd3_kernel<uint8_t><<<c->nslices, RD3_WARPS * 32, rd3_smem_bytes<uint8_t>(), c->stream>>>(p);
    return cuda_status(cudaGetLastError());
}

int cabac_slice_data(ironav_ctx* c, int idr, const ironav_mbcode* d_codes, std::vector<std::vector<uint8_t>>* slices) {
    int s = cabac_setup(c);
    if (s != IRONAV_OK) return s;
    const int ns = c->nslices;
    if (!c->d_cab_out) {
        int most = 0;
        for (int i = 0; i < ns; i++) most = std::max(most, (c->band_rows[i + 1] - c->band_rows[i]) * c->mb_w);
        c->cab_region_words = ((unsigned long long)most * CAB_MB_BYTES) / 4 + 2;
        CK(cudaMalloc(&c->d_cab_out, sizeof(uint32_t) * c->cab_region_words * ns));
        CK(cudaMalloc(&c->d_cab_bytes, sizeof(uint32_t) * (ns + 1)));
        CK(cudaMalloc(&c->d_cab_wnb, sizeof(WrNb) * c->nmb));
        CK(cudaMallocHost(&c->h_cab_bytes, sizeof(uint32_t) * (ns + 1)));
    }
    CabacWriteParams p;
    memset(&p, 0, sizeof(p));
    p.codes = d_codes;
    p.nbs = reinterpret_cast<WrNb*>(c->d_cab_wnb);
    p.nmb = c->nmb;
    p.band_rows = c->d_band_rows;
    p.step = c->d_cab_step;
    p.out = c->d_cab_out;
    p.region_words = (uint32_t)c->cab_region_words;
    p.slice_bytes = c->d_cab_bytes;
    p.mb_w = c->mb_w;
    p.nbands = ns;
    p.intra = idr ? 1 : 0;
    p.t8 = c->t8;
    p.nref = idr ? 0 : c->nact;
    p.qp = c->qpp - 6 * (c->bd - 8);
    CK(cudaMemsetAsync(c->d_cab_bytes, 0, sizeof(uint32_t) * (ns + 1), c->stream));
    cabac_nb_kernel<<<std::min((c->nmb + 3) / 4, c->nsm * 16), 128, 0, c->stream>>>(p);
    cabac_write_kernel<<<ns, 32, 0, c->stream>>>(p);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(c->h_cab_bytes, c->d_cab_bytes, sizeof(uint32_t) * (ns + 1), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (c->h_cab_bytes[ns]) return IRONAV_INTERNAL;  // a slice beyond its region
    slices->assign(ns, std::vector<uint8_t>());
    for (int i = 0; i < ns; i++) {
        (*slices)[i].resize(c->h_cab_bytes[i]);
        CK(cudaMemcpyAsync((*slices)[i].data(), c->d_cab_out + (size_t)i * c->cab_region_words, c->h_cab_bytes[i], cudaMemcpyDeviceToHost,
                           c->stream));
    }
    CK(cudaStreamSynchronize(c->stream));
    return IRONAV_OK;
}
