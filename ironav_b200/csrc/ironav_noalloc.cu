// ironav_noalloc.cu — ironav_analyse_auto_noalloc: the auto-mode (wavefront) analysis of one P picture
// for callers that cannot allocate device memory.
//
// Who needs it: code that runs where cudaMalloc is not allowed or not safe to call — inside a host
// callback or a real-time thread with a fixed memory budget, under a custom allocator that owns all
// device memory, or from a plugin host that hands out only the buffers it created. Such a caller
// cannot create an ironav_ctx (which allocates its planes, flags and staging buffers), so this entry
// point takes every input and output as the caller's device pointers and keeps its own scratch (the
// wavefront's progress flags, the ticket and error words, the slice-band table and the co-located
// vectors) in one fixed array in this library's device memory.
//
// Limits and rules:
//   - at most IRONAV_NOALLOC_MAX_MBS macroblocks (36864: 4096x2304, which covers 4K UHD) and one
//     reference picture;
//   - the scratch array is a file-scope __device__ array of 446,720 bytes (436 KiB), held by every GPU
//     that loads the library until the process exits;
//   - every call shares it and leaves its contents behind; each call clears what must start at zero.
//     Calls whose work overlaps on the GPU (two streams, or two host threads) race on it: run them one
//     after another;
//   - the first call on a device looks up the array's device address (cudaGetSymbolAddress) with that
//     device current; make that first call before any stream capture. A lookup that fails is not kept:
//     the next call on that device tries again. A device reset (cudaDeviceReset) is not supported: the
//     address kept from before it would name memory of a context that no longer exists;
//   - qp_prime is checked (0..63) but not used: the analysis reads only lambda and skip_thresh, which
//     the caller takes from ironav_lambda and ironav_skip_threshold for that QP';
//   - the call is synchronous: it returns when the analysis is done, so it can report a wavefront wait
//     that gave up (IRONAV_TIMEOUT).
#include <cuda_runtime.h>

#include <atomic>
#include <cstring>
#include <mutex>

#include "analyse.cuh"
#include "planes.cuh"

using namespace ironav;

namespace {

constexpr int NOALLOC_MAX_MBS = IRONAV_NOALLOC_MAX_MBS;
constexpr int NOALLOC_MAX_ROWS = 1024;  // H.264's limit on macroblock rows (H264Encoder::new, enc/mod.rs:150)
constexpr int MAX_DEVICES = 64;

// Scratch layout (32-bit words): [0] ticket, [1] error, [2..63] unused, [64, 64 + MAX_ROWS) band start
// of each macroblock row, then one progress flag per macroblock, then the co-located vectors (ColMv,
// 2 words each).
constexpr int SCR_TICKET = 0, SCR_ERR = 1, SCR_BANDS = 64;
constexpr int SCR_FLAGS = SCR_BANDS + NOALLOC_MAX_ROWS;
constexpr int SCR_COL = SCR_FLAGS + NOALLOC_MAX_MBS;
constexpr int SCR_WORDS = SCR_COL + 2 * NOALLOC_MAX_MBS;

static __device__ __align__(256) uint32_t g_noalloc_scratch[SCR_WORDS];

// Per device, filled once the lookups succeed (ready); a failed lookup leaves it empty for a retry.
struct DeviceSetup {
    std::mutex mu;
    std::atomic<bool> ready{false};
    uint32_t* scratch = nullptr;  // device address of g_noalloc_scratch on this device
    int blocks = 0;
};
DeviceSetup g_setup[MAX_DEVICES];

// Test hooks (ironav_debug_noalloc_wait, not in the public header): a macroblock whose decision is never
// published, and the polls a wavefront wait makes before it gives up.
std::atomic<int> g_withhold{-1};
std::atomic<unsigned> g_wait_limit{1u << 22};

// Clears the flags and counters, writes the slice bands (band i = [i*mb_h/n, (i+1)*mb_h/n), enc/mod.rs:603)
// and the co-located vectors of the reference picture (col_mv, enc/frame.rs:944-947).
__global__ void noalloc_init_kernel(uint32_t* scr, const ironav_mbstate* col, int nmb, int mb_h, int nslices) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < 2) scr[i] = 0;
    if (i < mb_h) {
        int b = 0;
        while (b + 1 < nslices && (b + 1) * mb_h / nslices <= i) b++;
        scr[SCR_BANDS + i] = (uint32_t)(b * mb_h / nslices);
    }
    if (i < nmb) {
        scr[SCR_FLAGS + i] = 0;
        ColMv c;
        c.mv[0] = c.mv[1] = 0;
        c.valid = 0;
        if (col && col[i].inter) {
            c.mv[0] = col[i].mvs[5][0];
            c.mv[1] = col[i].mvs[5][1];
            c.valid = 1;
        }
        reinterpret_cast<ColMv*>(scr + SCR_COL)[i] = c;
    }
}

// The wavefront analysis with tickets in row-interleaved order: ticket T covers row slot R = T / mb_w
// (the R / nslices-th row of band R % nslices) and column T % mb_w. A macroblock's left and top-right
// neighbours always hold smaller tickets, so a waiting warp only waits on running warps.
__global__ void __launch_bounds__(K2_WARPS * 32, K2_MIN_BLOCKS) analyse_noalloc_kernel(const __grid_constant__ AnalyseParams P, int nslices,
                                                                       int max_rows) {
    __shared__ WarpSmem<uint8_t> smem[K2_WARPS];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    WarpSmem<uint8_t>& S = smem[wid];
    const unsigned total = (unsigned)nslices * (unsigned)max_rows * (unsigned)P.mb_w;
    for (;;) {
        unsigned t = 0;
        if (lane == 0) t = atomicAdd(P.ticket, 1u);
        t = __shfl_sync(FULL, t, 0);
        if (t >= total) break;
        const int slot = (int)(t / (unsigned)P.mb_w), x = (int)(t % (unsigned)P.mb_w);
        const int r = slot / nslices, b = slot % nslices;
        const int y0 = b * P.mb_h / nslices, y1 = (b + 1) * P.mb_h / nslices;
        if (y0 + r >= y1) continue;  // this band has fewer rows
        const int mby = y0 + r, mb = mby * P.mb_w + x;
        if (lane == 0) {
            S.mb = mb;
            S.mbx = x;
            S.mby = mby;
        }
        __syncwarp();
        bool ok = true;
        if (x > 0) ok = wait_published(P, mb - 1);
        if (ok && mby > y0) ok = wait_published(P, (x + 1 < P.mb_w) ? mb - P.mb_w + 1 : mb - P.mb_w);
        ok = __all_sync(FULL, ok);
        if (!ok) break;
        load_neighbours(P, S, P.states_out);
        analyse(P, S, true);
        __threadfence();
        __syncwarp();
        if (lane == 0 && mb != P.withhold) st_release(&P.flags[mb], P.epoch);
    }
}

// The scratch array's device address and the persistent grid's size on the current device `dev`.
cudaError_t device_setup(int dev, DeviceSetup& S) {
    std::lock_guard<std::mutex> lock(S.mu);
    if (S.ready.load(std::memory_order_acquire)) return cudaSuccess;
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    int nsm = 0, per_sm = 0;
    e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, analyse_noalloc_kernel, K2_WARPS * 32, 0);
    if (e != cudaSuccess) return e;
    S.scratch = static_cast<uint32_t*>(p);
    S.blocks = (per_sm > 0 ? per_sm : 1) * nsm;
    S.ready.store(true, std::memory_order_release);
    return cudaSuccess;
}

int map_status(cudaError_t e) {
    if (e == cudaSuccess) return IRONAV_OK;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver || e == cudaErrorNoKernelImageForDevice)
        return IRONAV_HARDWARE_UNAVAILABLE;
    return IRONAV_INTERNAL;
}

}  // namespace

extern "C" int ironav_analyse_auto_noalloc(const uint8_t* d_src, int src_stride, const uint8_t* d_ref, int ref_stride,
                                           int ref_w, int ref_h, const ironav_mbstate* d_col, int width, int height,
                                           int nslices, int qp_prime, int lambda, int skip_thresh, int fast, int sub8,
                                           uint8_t* d_planes, ironav_mbstate* d_states, ironav_mbresult* d_results,
                                           void* stream) {
    if (!d_src || !d_ref || !d_planes || !d_states || !d_results) return IRONAV_INVALID_ARGUMENT;
    if (width <= 0 || height <= 0 || (width & 1) || (height & 1)) return IRONAV_INVALID_ARGUMENT;
    const int mb_w = (width + 15) / 16, mb_h = (height + 15) / 16, nmb = mb_w * mb_h;
    const int pw = mb_w * 16, ph = mb_h * 16, sw = pw + 2 * PAD, sh = ph + 2 * PAD;
    if (nmb > NOALLOC_MAX_MBS || mb_h > NOALLOC_MAX_ROWS || mb_w > 1024)
        return IRONAV_INVALID_ARGUMENT;  // beyond the scratch array's capacity
    if (nslices < 1 || nslices > mb_h || lambda < 1 || qp_prime < 0 || qp_prime > 63) return IRONAV_INVALID_ARGUMENT;
    // the source is read as 16-byte rows of whole macroblocks
    if (src_stride < pw || (src_stride & 15) || (reinterpret_cast<uintptr_t>(d_src) & 15)) return IRONAV_INVALID_ARGUMENT;
    if (!((ref_w == width && ref_h == height) || (ref_w == pw && ref_h == ph)) || ref_stride < ref_w)
        return IRONAV_INVALID_ARGUMENT;
    if (reinterpret_cast<uintptr_t>(d_planes) & 3) return IRONAV_INVALID_ARGUMENT;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return map_status(e);
    if (dev < 0 || dev >= MAX_DEVICES) return IRONAV_INTERNAL;
    // once per device, with that device current: the scratch array's device address
    DeviceSetup& S = g_setup[dev];
    if (!S.ready.load(std::memory_order_acquire)) {
        e = device_setup(dev, S);
        if (e != cudaSuccess) return map_status(e);
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    uint32_t* scr = S.scratch;

    const int init_n = nmb > mb_h ? nmb : mb_h;
    noalloc_init_kernel<<<(init_n + 255) / 256, 256, 0, s>>>(scr, d_col, nmb, mb_h, nslices);
    dim3 grid((sw + K1_TW - 1) / K1_TW, (sh + K1_TH - 1) / K1_TH);
    halfpel_planes_kernel<uint8_t><<<grid, K1_THREADS, 0, s>>>(d_ref, ref_stride, ref_w, ref_h, d_planes, (long long)sw * sh, sw, sh, 255,
                                                                nullptr, nullptr, 0);

    AnalyseParams p;
    memset(&p, 0, sizeof(p));
    p.src = d_src;
    p.ls = src_stride;
    p.planes[0] = d_planes;
    p.psize = (long long)sw * sh;
    p.sw = sw;
    p.col = reinterpret_cast<const ColMv*>(scr + SCR_COL);
    p.mb_w = mb_w;
    p.mb_h = mb_h;
    p.pw = pw;
    p.ph = ph;
    p.nact = 1;
    p.lambda = lambda;
    p.skip_thresh = skip_thresh;
    p.fast = fast ? 1 : 0;
    p.sub8 = sub8 ? 1 : 0;
    p.band_start = reinterpret_cast<const int*>(scr + SCR_BANDS);
    p.states_out = d_states;
    p.results = d_results;
    p.ticket = scr + SCR_TICKET;
    p.flags = scr + SCR_FLAGS;
    p.epoch = 1;  // the flags were cleared to 0 above
    p.err = scr + SCR_ERR;
    p.nmb = nmb;
    p.withhold = g_withhold.load();
    p.wait_limit = g_wait_limit.load();
    const int max_rows = (mb_h + nslices - 1) / nslices;
    analyse_noalloc_kernel<<<S.blocks, K2_WARPS * 32, 0, s>>>(p, nslices, max_rows);
    e = cudaGetLastError();
    if (e != cudaSuccess) return map_status(e);
    uint32_t err = 0;
    e = cudaMemcpyAsync(&err, scr + SCR_ERR, sizeof(err), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return map_status(e);
    if (err & 1u) return IRONAV_TIMEOUT;
    return err ? IRONAV_INTERNAL : IRONAV_OK;
}

// Test hook (not in the public header): withhold = a macroblock whose decision the next calls never
// publish (-1: none), polls = how often a wavefront wait polls before it gives up (0: the default).
extern "C" int ironav_debug_noalloc_wait(int withhold, unsigned polls) {
    if (withhold < -1 || withhold >= NOALLOC_MAX_MBS) return IRONAV_INVALID_ARGUMENT;
    g_withhold.store(withhold);
    g_wait_limit.store(polls ? polls : (1u << 22));
    return IRONAV_OK;
}
