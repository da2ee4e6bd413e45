// ironav_proposer.cu — the learned proposer's kernels behind the C ABI (the north star's form 4): its 3x3
// convolutions and their weight gradients on the tensor cores (tc_conv.cuh), and its input, head, loss and
// optimizer on the CUDA cores (proposer.cuh). Every entry point queues its work on the given stream and
// returns; a device wait that gave up sets bit 0 of the caller's error word `err` (device memory), which the
// caller reads once a step. The TMA tensor maps are made on the host, through the driver's
// cuTensorMapEncodeTiled reached via the runtime (no link against libcuda).
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "../../include/ironav_inter.h"
#include "proposer.cuh"
#include "tc_conv.cuh"

using namespace ironav::tc;
namespace prop = ironav::prop;

static_assert(sizeof(ironav_prop_sample) == sizeof(prop::Sample), "ironav_prop_sample layout");

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

using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                 const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
                                 CUtensorMapFloatOOBfill);

// cuTensorMapEncodeTiled from the driver, through the runtime.
EncodeTiled encode_fn() {
    static EncodeTiled fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess && q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiled>(p);
    }
    return fn;
}

// The tensor map of a chunk-major padded tensor (planes x Q pixels x 8 BF16) read in boxes of `box_pixels`
// pixels of `box_planes` planes (0: every plane): dims (8, Q, planes), byte strides (16, 16 Q). Out-of-range
// pixels read as zeros.
int plane_map(CUtensorMap* map, const void* base, long long Q, int planes, int box_pixels, int box_planes = 0) {
    EncodeTiled enc = encode_fn();
    if (!enc) return IRONAV_HARDWARE_UNAVAILABLE;
    if (reinterpret_cast<uintptr_t>(base) & 15) return IRONAV_INVALID_ARGUMENT;
    const cuuint64_t dims[3] = {8, (cuuint64_t)Q, (cuuint64_t)planes};
    const cuuint64_t strides[2] = {16, (cuuint64_t)Q * 16};
    const cuuint32_t box[3] = {8, (cuuint32_t)box_pixels, (cuuint32_t)(box_planes > 0 ? box_planes : planes)};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<void*>(base), dims, strides, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? IRONAV_OK : IRONAV_INVALID_ARGUMENT;
}

int sm_count(int* nsm) {
    int dev = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(nsm, cudaDevAttrMultiProcessorCount, dev));
    return IRONAV_OK;
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

}  // namespace

extern "C" {

// The convolution's tile: CONV_MT x 128 output pixels (conv3x3p_kernel's MT).
constexpr int CONV_MT = 2;

int ironav_prop_conv3x3(const void* d_x, int cin, long long samples, const void* d_w, const float* d_bias, int relu, const void* d_mask,
                        void* d_y, unsigned* d_err, void* stream) {
    if (!d_x || !d_w || !d_y || !d_err || (cin != 16 && cin != 32) || samples < 1 || samples > (1ll << 22)) return IRONAV_INVALID_ARGUMENT;
    if (!aligned16(d_y) || !aligned16(d_mask)) return IRONAV_INVALID_ARGUMENT;
    const long long Q = samples * RPIX;
    const int tiles = (int)((Q + CONV_MT * TILE - 1) / (CONV_MT * TILE));
    CUtensorMap map;
    int s = plane_map(&map, d_x, Q, cin / 8, cp_box<CONV_MT>(), CONV_MT == 1 ? 0 : 1);
    if (s != IRONAV_OK) return s;
    int nsm = 0;
    if ((s = sm_count(&nsm)) != IRONAV_OK) return s;
    // the pipelined form: two persistent CTAs an SM
    const int grid = std::min(tiles, nsm * 2);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const __nv_bfloat16* w = static_cast<const __nv_bfloat16*>(d_w);
    const __nv_bfloat16* mask = static_cast<const __nv_bfloat16*>(d_mask);
    __nv_bfloat16* y = static_cast<__nv_bfloat16*>(d_y);
    if (cin == 32) {
        constexpr int bytes = conv3x3p_smem_bytes<32, CONV_MT>();
        CK(cudaFuncSetAttribute(conv3x3p_kernel<32, CONV_MT>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
        conv3x3p_kernel<32, CONV_MT><<<grid, CP_THREADS, bytes, st>>>(map, w, d_bias, relu, mask, y, Q, tiles, d_err);
    } else {
        constexpr int bytes = conv3x3p_smem_bytes<16, CONV_MT>();
        CK(cudaFuncSetAttribute(conv3x3p_kernel<16, CONV_MT>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
        conv3x3p_kernel<16, CONV_MT><<<grid, CP_THREADS, bytes, st>>>(map, w, d_bias, relu, mask, y, Q, tiles, d_err);
    }
    return cuda_status(cudaGetLastError());
}

int ironav_prop_wgrad3x3(const void* d_x, int cin, const void* d_dz, long long samples, float* d_dw, float* d_db, unsigned* d_err,
                         void* stream) {
    if (!d_x || !d_dz || !d_dw || !d_err || (cin != 16 && cin != 32) || samples < 1 || samples > (1ll << 22)) return IRONAV_INVALID_ARGUMENT;
    const long long Q = samples * RPIX;
    const int tiles = (int)((Q + WG_KT - 1) / WG_KT);
    CUtensorMap xmap, zmap;
    int s = plane_map(&xmap, d_x, Q, cin / 8, WG_KT);
    if (s == IRONAV_OK) s = plane_map(&zmap, d_dz, Q, 4, WG_KT);
    if (s != IRONAV_OK) return s;
    int nsm = 0;
    if ((s = sm_count(&nsm)) != IRONAV_OK) return s;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (cin == 32) {
        constexpr int bytes = wgrad3x3_smem_bytes<32>();
        CK(cudaFuncSetAttribute(wgrad3x3_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
        wgrad3x3_kernel<32><<<std::min(tiles, nsm * 2), 128, bytes, st>>>(xmap, zmap, d_dw, d_db, Q, tiles, d_err);
    } else {
        constexpr int bytes = wgrad3x3_smem_bytes<16>();
        CK(cudaFuncSetAttribute(wgrad3x3_kernel<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
        wgrad3x3_kernel<16><<<std::min(tiles, nsm * 2), 128, bytes, st>>>(xmap, zmap, d_dw, d_db, Q, tiles, d_err);
    }
    return cuda_status(cudaGetLastError());
}

int ironav_prop_prep(const ironav_prop_sample* d_samples, int n, void* d_x, void* stream) {
    if (!d_samples || !d_x || n < 1 || n > (1 << 22) || !aligned16(d_x)) return IRONAV_INVALID_ARGUMENT;
    const long long Q = (long long)n * RPIX;
    prop::prep_kernel<<<(unsigned)((Q + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<const prop::Sample*>(d_samples), n, static_cast<__nv_bfloat16*>(d_x));
    return cuda_status(cudaGetLastError());
}

int ironav_prop_head_fwd(const void* d_feat, int n, const float* d_hw, const float* d_hb, float* d_out, void* stream) {
    if (!d_feat || !d_hw || !d_hb || !d_out || n < 1 || n > (1 << 22)) return IRONAV_INVALID_ARGUMENT;
    prop::head_fwd_kernel<<<(n + prop::HEAD_SPB - 1) / prop::HEAD_SPB, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const __nv_bfloat16*>(d_feat), (long long)n * RPIX, n, d_hw, d_hb, d_out);
    return cuda_status(cudaGetLastError());
}

int ironav_prop_head_pack(const float* d_hw, float* d_hwt, void* stream) {
    if (!d_hw || !d_hwt || !aligned16(d_hwt)) return IRONAV_INVALID_ARGUMENT;
    prop::head_pack_kernel<<<(prop::NFEAT * 16 + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(d_hw, d_hwt);
    return cuda_status(cudaGetLastError());
}

int ironav_prop_head_fwd_packed(const void* d_feat, int n, const float* d_hwt, const float* d_hb, float* d_out, void* stream) {
    if (!d_feat || !d_hwt || !d_hb || !d_out || n < 1 || n > (1 << 22) || !aligned16(d_hwt)) return IRONAV_INVALID_ARGUMENT;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    CK(cudaMemsetAsync(d_out, 0, (size_t)n * prop::NOUT * sizeof(float), st));
    const dim3 grid((n + prop::HEAD_SAMPLES - 1) / prop::HEAD_SAMPLES, (48 * 48 + prop::HEAD_PIX - 1) / prop::HEAD_PIX);
    prop::head_fwd_packed_kernel<<<grid, 256, 0, st>>>(static_cast<const __nv_bfloat16*>(d_feat), (long long)n * RPIX, n,
                                                       reinterpret_cast<const float4*>(d_hwt), d_hb, d_out);
    return cuda_status(cudaGetLastError());
}

int ironav_prop_loss(const float* d_out, const int16_t* d_target_mv, const uint8_t* d_target_part, int n, float* d_dout, float* d_sums,
                     void* stream) {
    if (!d_out || !d_target_mv || !d_target_part || !d_dout || !d_sums || n < 1) return IRONAV_INVALID_ARGUMENT;
    prop::loss_kernel<<<(n + 127) / 128, 128, 0, static_cast<cudaStream_t>(stream)>>>(d_out, d_target_mv, d_target_part, n, d_dout, d_sums);
    return cuda_status(cudaGetLastError());
}

int ironav_prop_head_bwd(const void* d_feat, int n, const float* d_dout, const float* d_hw, float* d_ghw, float* d_ghb, void* d_dz,
                         void* stream) {
    if (!d_feat || !d_dout || !d_hw || !d_ghw || !d_dz || n < 1 || n > (1 << 22) || !aligned16(d_dz)) return IRONAV_INVALID_ARGUMENT;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const long long Q = (long long)n * RPIX;
    const __nv_bfloat16* feat = static_cast<const __nv_bfloat16*>(d_feat);
    // the ring of dz is zero (its interior is written below)
    CK(cudaMemsetAsync(d_dz, 0, (size_t)4 * Q * 16, st));
    prop::head_wgrad_kernel<<<(prop::NFEAT + 255) / 256, 256, 0, st>>>(feat, Q, n, d_dout, d_ghw, d_ghb);
    const long long total = (long long)n * prop::NFEAT;
    prop::head_dgrad_kernel<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(feat, Q, n, d_dout, d_hw, static_cast<__nv_bfloat16*>(d_dz));
    return cuda_status(cudaGetLastError());
}

int ironav_prop_adam(float* d_p, float* d_g, float* d_m, float* d_v, long long n, float lr, float beta1, float beta2, int step, float eps,
                     void* stream) {
    if (!d_p || !d_g || !d_m || !d_v || n < 1 || step < 1) return IRONAV_INVALID_ARGUMENT;
    const float c1 = 1.f - std::pow(beta1, (float)step), c2 = 1.f - std::pow(beta2, (float)step);
    prop::adam_kernel<<<(unsigned)((n + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(d_p, d_g, d_m, d_v, n, lr, beta1, beta2, c1,
                                                                                                   c2, eps);
    return cuda_status(cudaGetLastError());
}

int ironav_prop_weights(const float* d_w, int cin, void* d_wf, void* d_wt, void* stream) {
    if (!d_w || !d_wf || (cin != 16 && cin != 32) || (d_wt && cin != 32)) return IRONAV_INVALID_ARGUMENT;
    prop::weights_kernel<<<(9 * 32 * cin + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        d_w, cin, static_cast<__nv_bfloat16*>(d_wf), static_cast<__nv_bfloat16*>(d_wt));
    return cuda_status(cudaGetLastError());
}

int ironav_prop_propose(const float* d_out, int n, float min_conf, int16_t* d_cands, uint8_t* d_cls, void* stream) {
    if (!d_out || !d_cands || !d_cls || n < 1 || n > (1 << 22) || !(min_conf >= 0.f && min_conf <= 1.f)) return IRONAV_INVALID_ARGUMENT;
    prop::propose_kernel<<<(n + 127) / 128, 128, 0, static_cast<cudaStream_t>(stream)>>>(d_out, n, min_conf, d_cands, d_cls);
    return cuda_status(cudaGetLastError());
}

}  // extern "C"
