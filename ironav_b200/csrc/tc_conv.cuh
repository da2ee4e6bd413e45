// tc_conv.cuh — the learned proposer's 3x3 convolutions on the 5th-generation tensor cores (tcgen05, sm_100a):
// BF16 operands in shared memory, FP32 accumulators in tensor memory (TMEM).
//
// Activation layout ("chunk-major padded"): every sample (one macroblock's input) is a 50 x 50 raster, its
// 48 x 48 interior plus a ring of zeros; rasters follow each other, Q = samples * 2500 pixels in all. A tensor
// of C channels is C / 8 planes, plane c holding channels 8c .. 8c + 7 of every pixel as 16 bytes: element
// (c, q, e) at ((c * Q) + q) * 8 + e. A 3x3 convolution of such a raster is then a 1-D convolution along q with
// the nine shifts (dy - 1) * 50 + (dx - 1): output pixel q reads input pixel q + shift, and a shift never leaves
// the sample's own raster for an interior pixel (outputs on the ring are written as zeros).
//
// A CTA takes tiles of 128 consecutive output pixels. Per tile: one TMA 3-D box load brings the input halo
// (pixels q0 - 51 .. q0 + 180 of every plane, zeros beyond the tensor) into shared memory in the same layout;
// every tap's A operand (128 pixels x 16 channels, K-major, no swizzle) is then just another start address into
// the halo, so no im2col copy is made. The weights (B: 32 output channels x CIN input channels per tap, K-major)
// sit in shared memory for the CTA's life. One thread issues 9 taps x CIN / 16 MMAs of M = 128, N = 32, K = 16
// into a TMEM accumulator (128 lanes x 32 FP32 columns); the epilogue warps read their 32 lanes (pixels) x 32
// columns (channels) back with tcgen05.ld, add the bias, apply ReLU or a gradient mask, zero the ring, and
// store BF16. Loads, MMAs and epilogues of successive tiles overlap (conv3x3p_kernel, below).
//
// The same kernel is the backward pass's data gradient (the convolution with the weights transposed and the
// taps mirrored, and the mask of the layer's ReLU in the epilogue).
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>
#include <cstdint>

namespace ironav {
namespace tc {

constexpr int RW = 50;                  // raster width (and height): 48 + 2
constexpr int RPIX = RW * RW;           // pixels a sample
constexpr int TILE = 128;               // output pixels a tile (the MMA's M)
constexpr int HALO_LO = RW + 1;         // the most negative shift
constexpr int HALO = 232;               // halo pixels staged a tile: 51 + 128 + 51, rounded up to 8
constexpr int COUT = 32;                // output channels (the MMA's N)
constexpr unsigned WAIT_LIMIT = 1u << 26;  // polls of an mbarrier before the kernel gives up

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// Waits for the mbarrier's phase `parity` to complete, at most WAIT_LIMIT polls; false when it gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity) {
    const uint32_t a = smem_u32(bar);
    for (unsigned i = 0; i < WAIT_LIMIT; i++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// TMA: a 3-D box of the tensor map into shared memory, completion counted on the mbarrier.
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
        "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
        : "memory");
}

// A shared-memory matrix descriptor for tcgen05.mma (K-major, no swizzle): start address, the byte distance
// between core matrices adjacent in K (lbo) and in M/N (sbo), version 1 (bits 46-47), layout type 0.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) | ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) |
           (1ull << 46);
}
// The instruction descriptor of kind::f16 with BF16 A and B, FP32 D, both K-major, M = 128, N = 32.
constexpr uint32_t IDESC_BF16_M128_N32 = (1u << 4) | (1u << 7) | (1u << 10) | ((COUT >> 3) << 17) | ((TILE >> 4) << 24);

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 32 lanes x 32 consecutive FP32 columns of TMEM into 32 registers of each thread (lane = the warp's lane).
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16, %17, %18, "
        "%19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]),
          "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]),
          "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
          "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

// The weight gradient of a 3x3 layer: dw[t][o][i] += sum over pixels q of dz[q][o] * x[q + shift_t][i] (FP32,
// accumulated into dw with atomics), and db[o] += sum over q of dz[q][o]. As MMAs: M = 128 rows (a group of
// 128 / CIN taps x CIN input channels), N = 32 output channels, K = pixels; both operands MN-major (a pixel's 8
// channels contiguous, pixels 16 bytes apart), so the chunk-major tensors are their own canonical layout. Per
// tile of KT pixels, TMA stages the nine tap-shifted views of x ([tap slot][plane][pixel][16 B], taps beyond
// 8 stay zero) and the tile of dz; one thread issues groups x KT / 16 MMAs into one TMEM accumulator per group
// (32 columns each), accumulating over all the CTA's tiles; at the end each warp reads its 32 rows and adds them
// to dw. xmap: x as (8, Q, CIN / 8) with boxes of KT pixels; zmap: dz as (8, Q, 4) with the same boxes.
constexpr int WG_KT = 128;  // pixels a tile (K)

template <int CIN>
constexpr int wgrad3x3_smem_bytes() {
    return ((9 + 128 / CIN - 1) / (128 / CIN)) * 128 * WG_KT * 2 + 4 * WG_KT * 16 + 2 * 8 + 16 + 32 * 4;
}

// MN-major operands for the weight gradient: M (or N) 8 channels of a pixel contiguous, K = pixels 16 bytes apart.
constexpr uint32_t IDESC_BF16_MN_M128_N32 = (1u << 4) | (1u << 7) | (1u << 10) | (1u << 15) | (1u << 16) | ((COUT >> 3) << 17) | ((TILE >> 4) << 24);

template <int CIN>
__global__ void __launch_bounds__(128, 1) wgrad3x3_kernel(const __grid_constant__ CUtensorMap xmap, const __grid_constant__ CUtensorMap zmap,
                                                          float* __restrict__ dw, float* __restrict__ db, long long Q, int tiles,
                                                          unsigned* err) {
    constexpr int KC = CIN / 8, TPG = 128 / CIN, NG = (9 + TPG - 1) / TPG;
    constexpr int PLANE = WG_KT * 16;          // bytes of one plane's tile
    constexpr int ABYTES = NG * 16 * PLANE;    // NG groups x 16 planes (TPG taps x KC planes)
    constexpr int BBYTES = 4 * PLANE;
    constexpr unsigned TX = 9 * KC * PLANE + BBYTES;
    constexpr int NCOL = NG * 32 <= 32 ? 32 : (NG * 32 <= 64 ? 64 : 128);
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t* as = smem;
    uint8_t* bs = smem + ABYTES;
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + ABYTES + BBYTES);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2);
    float* dbs = reinterpret_cast<float*>(tmem_slot + 4);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    // the slots of taps 9.. stay zero (their rows accumulate nothing)
    for (int i = tid; i < (NG * TPG - 9) * KC * PLANE / 16; i += 128)
        reinterpret_cast<uint4*>(as + 9 * KC * PLANE)[i] = make_uint4(0, 0, 0, 0);
    if (tid < 32) dbs[tid] = 0.f;
    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)), "n"(NCOL));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    bool failed = false, load_pending = false, mma_pending = false, any = false;
    unsigned it = 0;
    float dbsum = 0.f;  // this thread's share of db: channel lane, pixels warp, warp + 4, ...
    for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x, it++) {
        const long long q0 = (long long)tile * WG_KT;
        if (tid == 0) {
            mbar_expect_tx(&bars[0], TX);
            for (int t = 0; t < 9; t++) {
                const int shift = (t / 3 - 1) * RW + (t % 3 - 1);
                tma_load_3d(as + (t / TPG) * 16 * PLANE + (t % TPG) * KC * PLANE, &xmap, 0, (int)(q0 + shift), 0, &bars[0]);
            }
            tma_load_3d(bs, &zmap, 0, (int)q0, 0, &bars[0]);
        }
        const bool loaded = mbar_wait(&bars[0], it & 1);
        if (__syncthreads_or(!loaded)) {
            failed = load_pending = true;
            break;
        }
        if (tid == 0) {
            tc_fence_after();
            const uint32_t a0 = smem_u32(as), b0 = smem_u32(bs);
#pragma unroll 1
            for (int g = 0; g < NG; g++)
#pragma unroll
                for (int k = 0; k < WG_KT / 16; k++) {
                    const uint64_t ad = smem_desc(a0 + (uint32_t)(g * 16 * PLANE + k * 256), 128, PLANE);
                    const uint64_t bd = smem_desc(b0 + (uint32_t)(k * 256), 128, PLANE);
                    mma_bf16(tmem + (uint32_t)(g * 32), ad, bd, IDESC_BF16_MN_M128_N32, (any || k != 0) ? 1u : 0u);
                }
            mma_commit(&bars[1]);
        }
        any = true;
        // the bias gradient from the staged dz tile: thread (warp, lane) sums channel lane over pixels warp, warp + 4, ...
        {
            const __nv_bfloat16* z = reinterpret_cast<const __nv_bfloat16*>(bs);
            for (int p = warp; p < WG_KT; p += 4) dbsum += __bfloat162float(z[((lane >> 3) * WG_KT + p) * 8 + (lane & 7)]);
        }
        const bool computed = mbar_wait(&bars[1], it & 1);
        if (__syncthreads_or(!computed)) {
            failed = mma_pending = true;
            break;
        }
        tc_fence_before();
        __syncthreads();
    }
    if (failed && tid == 0) atomicOr(err, 1u);
    if (load_pending) mbar_wait(&bars[0], it & 1);
    if (mma_pending) mbar_wait(&bars[1], it & 1);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (!failed && any) {
        atomicAdd(&dbs[lane], dbsum);
        for (int g = 0; g < NG; g++) {
            float v[32];
            tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(g * 32), v);
            const int m = warp * 32 + lane, t = g * TPG + m / CIN, i = m % CIN;
            if (t < 9)
#pragma unroll
                for (int o = 0; o < 32; o++) atomicAdd(&dw[(t * COUT + o) * CIN + i], v[o]);
        }
        __syncthreads();
        if (tid < 32 && db != nullptr) atomicAdd(&db[tid], dbs[tid]);
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "n"(NCOL));
}



// ---- the pipelined form of the 3x3 convolution ----------------------------------------------------------
//
// The same convolution with the tile loop overlapped: warp-specialised CTAs of 6 warps. Warp 4 (one thread)
// streams the tiles' halos by TMA into a ring of CP_STAGES stages; warp 5 (one thread) issues each tile's
// MMAs into one of two TMEM accumulators as soon as its halo has landed and that accumulator is free, and
// commits them to the stage's "empty" barrier (the halo may be overwritten) and to the accumulator's
// "full" barrier; warps 0-3 read a full accumulator back (each its 32 TMEM lanes), release it at once and run
// the epilogue while the next tile's MMAs fill the other accumulator. Every wait is bounded: a role that
// gives up sets the CTA's failure flag, every other role stops at its next wait, and the tile loop ends; the
// copies and MMAs still in flight are then waited for (bounded) before the TMEM is freed.
constexpr int CP_STAGES = 4;
constexpr int CP_THREADS = 192;

// A tile of MT x 128 output pixels: MT MMAs of M = 128 a tap and K chunk. The halo it stages (51 pixels each
// side): 232 pixels for MT = 1, loaded as one box of every plane; 368 for MT = 2, each plane as two boxes of 184
// (the box limit is 256 pixels, and every box must land on a 128-byte boundary: 8 pixels). Stages: as many as
// keep two CTAs an SM (4 of 15 KB, or 3 of 23 KB, at CIN 32).
template <int MT>
__host__ __device__ constexpr int cp_halo() { return MT == 1 ? 232 : 368; }
template <int MT>
__host__ __device__ constexpr int cp_box() { return MT == 1 ? cp_halo<MT>() : cp_halo<MT>() / 2; }
template <int MT>
__host__ __device__ constexpr int cp_stages() { return MT == 1 ? 4 : 3; }
static_assert(cp_halo<1>() >= TILE + 2 * HALO_LO && cp_halo<2>() >= 2 * TILE + 2 * HALO_LO, "the halo covers every tap's rows");

template <int CIN, int MT = 1>
constexpr int conv3x3p_smem_bytes() {
    return 9 * (CIN / 8) * COUT * 16 + cp_stages<MT>() * (CIN / 8) * cp_halo<MT>() * 16 + (2 * cp_stages<MT>() + 4) * 8 + 16;
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// One 3x3 convolution layer (CIN input channels, 32 output channels) over the chunk-major padded rasters:
// y = act(conv(x, w) + bias), act = ReLU (relu != 0) or the identity, then times (mask > 0) when `mask` is set
// (the gradient through the layer's ReLU); the ring pixels of y are zero. w is [9 taps][32 out][CIN in] BF16,
// tap = 3 * dy + dx. x is read through `map` (planes CIN / 8, Q pixels, 8 channels; boxes of cp_box<MT>() pixels of
// every plane (MT = 1) or of one plane (MT = 2)). tiles = ceil(Q / (MT x 128)).
template <int CIN, int MT = 1>
__global__ void __launch_bounds__(CP_THREADS, 1) conv3x3p_kernel(const __grid_constant__ CUtensorMap map, const __nv_bfloat16* __restrict__ w,
                                                                 const float* __restrict__ bias, int relu, const __nv_bfloat16* __restrict__ mask,
                                                                 __nv_bfloat16* __restrict__ y, long long Q, int tiles, unsigned* err) {
    constexpr int KC = CIN / 8;
    constexpr int CP_STAGES = cp_stages<MT>();  // this form's ring of stages
    constexpr int WBYTES = 9 * KC * COUT * 16;
    constexpr int HP = cp_halo<MT>();                          // halo pixels a stage
    constexpr int HBYTES = KC * HP * 16;
    constexpr int TP = MT * TILE;                              // output pixels a tile
    constexpr int ACOLS = MT * COUT;                           // TMEM columns an accumulator
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t* ws = smem;                                        // weights: [tap][chunk][out][16 B]
    uint8_t* halos = smem + WBYTES;                            // CP_STAGES x [chunk][HP pixels][16 B]
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + WBYTES + CP_STAGES * HBYTES);  // [CP_STAGES]
    uint64_t* empty = full + CP_STAGES;                        // [CP_STAGES]
    uint64_t* accf = empty + CP_STAGES;                        // [2] accumulator written
    uint64_t* acce = accf + 2;                                 // [2] accumulator read back
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(acce + 2);
    volatile int* failed = reinterpret_cast<volatile int*>(tmem_slot + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int ntiles = tiles > (int)blockIdx.x ? (tiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;  // this CTA's tiles

    for (int i = tid; i < 9 * COUT * CIN; i += CP_THREADS) {
        const int t = i / (COUT * CIN), n = (i / CIN) % COUT, k = i % CIN;
        *reinterpret_cast<__nv_bfloat16*>(ws + ((t * KC + k / 8) * COUT + n) * 16 + (k % 8) * 2) = w[i];
    }
    if (tid == 0) {
        for (int s = 0; s < CP_STAGES; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int a = 0; a < 2; a++) {
            mbar_init(&accf[a], 1);
            mbar_init(&acce[a], 4);
        }
        *failed = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (warp == 5) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)), "r"(2 * ACOLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    __shared__ int s_loaded, s_issued;
    if (warp == 4) {
        // the producer: the halo of tile it into stage it % CP_STAGES once the MMAs of its previous use are done
        int loaded = 0;
        if (lane == 0) {
            for (int it = 0; it < ntiles; it++) {
                const int s = it % CP_STAGES, k = it / CP_STAGES;
                if (k > 0 && !mbar_wait(&empty[s], (k - 1) & 1)) {
                    *failed = 1;
                    break;
                }
                if (*failed) break;
                const long long q0 = ((long long)blockIdx.x + (long long)it * gridDim.x) * TP;
                mbar_expect_tx(&full[s], HBYTES);
                if constexpr (MT == 1) {
                    tma_load_3d(halos + s * HBYTES, &map, 0, (int)(q0 - HALO_LO), 0, &full[s]);
                } else {
#pragma unroll
                    for (int c = 0; c < KC; c++)
#pragma unroll
                        for (int m = 0; m < 2; m++)
                            tma_load_3d(halos + s * HBYTES + (c * HP + m * (HP / 2)) * 16, &map, 0, (int)(q0 - HALO_LO) + m * (HP / 2), c,
                                        &full[s]);
                }
                loaded = it + 1;
            }
            s_loaded = loaded;
        }
    } else if (warp == 5) {
        // the MMA issuer: tile it into accumulator it & 1
        int issued = 0;
        if (lane == 0) {
            for (int it = 0; it < ntiles; it++) {
                const int s = it % CP_STAGES, k = it / CP_STAGES, a = it & 1, j = it >> 1;
                if (!mbar_wait(&full[s], k & 1)) {
                    *failed = 1;
                    break;
                }
                if (j > 0 && !mbar_wait(&acce[a], (j - 1) & 1)) {
                    *failed = 1;
                    break;
                }
                if (*failed) break;
                tc_fence_after();
                const uint32_t h = smem_u32(halos + s * HBYTES), wb = smem_u32(ws), d = tmem + (uint32_t)(a * ACOLS);
#pragma unroll 1
                for (int t = 0; t < 9; t++) {
                    const int shift = (t / 3 - 1) * RW + (t % 3 - 1);
#pragma unroll
                    for (int kk = 0; kk < KC / 2; kk++) {
                        const uint64_t bd = smem_desc(wb + (uint32_t)((t * KC + 2 * kk) * COUT * 16), COUT * 16, 8 * 16);
#pragma unroll
                        for (int mh = 0; mh < MT; mh++) {
                            const uint64_t ad = smem_desc(h + (uint32_t)((2 * kk * HP + HALO_LO + shift + mh * TILE) * 16), HP * 16, 8 * 16);
                            mma_bf16(d + (uint32_t)(mh * COUT), ad, bd, IDESC_BF16_M128_N32, (t | kk) != 0);
                        }
                    }
                }
                mma_commit(&empty[s]);
                mma_commit(&accf[a]);
                issued = it + 1;
            }
            s_issued = issued;
        }
    } else {
        // the epilogue: warp w reads TMEM lanes 32w .. 32w + 31 (pixels), releases the accumulator, stores.
        // The bias stays in registers; a pixel's raster position comes from its tile's (one 64-bit remainder
        // a tile, the rest in 32 bits).
        float bv[32];
#pragma unroll
        for (int c = 0; c < 32; c++) bv[c] = bias != nullptr ? bias[c] : 0.f;
        for (int it = 0; it < ntiles; it++) {
            const int a = it & 1, j = it >> 1;
            const bool ok = mbar_wait(&accf[a], j & 1);
            if (!__all_sync(0xffffffffu, ok)) {
                if (lane == 0) *failed = 1;
                break;
            }
            tc_fence_after();
            float vv[MT][32];
#pragma unroll
            for (int mh = 0; mh < MT; mh++) tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(a * ACOLS + mh * COUT), vv[mh]);
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&acce[a]);
            const long long q0 = ((long long)blockIdx.x + (long long)it * gridDim.x) * TP;
            const int r0 = (int)(q0 % RPIX);
#pragma unroll
            for (int mh = 0; mh < MT; mh++) {
                const float (&v)[32] = vv[mh];
                const long long q = q0 + mh * TILE + warp * 32 + lane;
                if (q < Q) {
                    int p = r0 + mh * TILE + warp * 32 + lane;
                    if (p >= RPIX) p -= RPIX;
                    const int ry = p / RW, rx = p - ry * RW;
                    const bool ring = ry == 0 || ry == RW - 1 || rx == 0 || rx == RW - 1;
#pragma unroll
                    for (int c = 0; c < 4; c++) {
                        uint4 m4 = make_uint4(0, 0, 0, 0);
                        if (mask != nullptr) m4 = *reinterpret_cast<const uint4*>(mask + ((size_t)c * Q + q) * 8);
                        const __nv_bfloat16* mk = reinterpret_cast<const __nv_bfloat16*>(&m4);
                        __align__(16) __nv_bfloat16 o[8];
#pragma unroll
                        for (int e = 0; e < 8; e++) {
                            float f = v[c * 8 + e] + bv[c * 8 + e];
                            if (relu) f = fmaxf(f, 0.f);
                            if (mask != nullptr && !(__bfloat162float(mk[e]) > 0.f)) f = 0.f;
                            o[e] = __float2bfloat16_rn(ring ? 0.f : f);
                        }
                        *reinterpret_cast<uint4*>(y + ((size_t)c * Q + q) * 8) = *reinterpret_cast<const uint4*>(o);
                    }
                }
            }
            if (__any_sync(0xffffffffu, *failed != 0)) break;
        }
    }
    __syncthreads();
    if (tid == 0 && *failed) atomicOr(err, 1u);
    if (warp == 4 && lane == 0) {
        // copies issued but never consumed, then the MMAs' last arrivals on the stages (bounded waits)
        for (int it = s_issued; it < s_loaded; it++) mbar_wait(&full[it % CP_STAGES], (it / CP_STAGES) & 1);
        for (int it = s_issued > CP_STAGES ? s_issued - CP_STAGES : 0; it < s_issued; it++)
            mbar_wait(&empty[it % CP_STAGES], (it / CP_STAGES) & 1);
    }
    if (warp == 5 && lane == 0 && s_issued > 0) mbar_wait(&accf[(s_issued - 1) & 1], ((s_issued - 1) >> 1) & 1);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 5) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * ACOLS));
}

}  // namespace tc
}  // namespace ironav
