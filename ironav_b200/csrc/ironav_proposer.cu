// ironav_proposer.cu — the learned proposer's tensor-core building blocks (tc_conv.cuh) behind the C ABI: one
// 3x3 convolution layer over chunk-major padded rasters, its TMA tensor map made on the host.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>

#include "../../include/ironav_inter.h"
#include "tc_conv.cuh"

using namespace ironav::tc;

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

// cuTensorMapEncodeTiled from the driver, through the runtime (no link against libcuda).
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

// The tensor map of a chunk-major padded tensor (planes x Q pixels x 8 BF16) read as boxes of HALO pixels of
// every plane: dims (8, Q, planes), byte strides (16, 16 Q).
int plane_map(CUtensorMap* map, const void* base, long long Q, int planes, int box_pixels) {
    EncodeTiled enc = encode_fn();
    if (!enc) return IRONAV_HARDWARE_UNAVAILABLE;
    if (reinterpret_cast<uintptr_t>(base) & 15) return IRONAV_INVALID_ARGUMENT;
    const cuuint64_t dims[3] = {8, (cuuint64_t)Q, (cuuint64_t)planes};
    const cuuint64_t strides[2] = {16, (cuuint64_t)Q * 16};
    const cuuint32_t box[3] = {8, (cuuint32_t)box_pixels, (cuuint32_t)planes};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<void*>(base), dims, strides, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? IRONAV_OK : IRONAV_INVALID_ARGUMENT;
}

}  // namespace

extern "C" int ironav_prop_conv3x3(const void* d_x, int cin, long long samples, const void* d_w, const float* d_bias, int relu,
                                   const void* d_mask, void* d_y, void* stream) {
    if (!d_x || !d_w || !d_y || (cin != 16 && cin != 32) || samples < 1 || samples > (1ll << 24)) return IRONAV_INVALID_ARGUMENT;
    if ((reinterpret_cast<uintptr_t>(d_y) | reinterpret_cast<uintptr_t>(d_mask)) & 15) return IRONAV_INVALID_ARGUMENT;
    const long long Q = samples * RPIX;
    const int tiles = (int)((Q + TILE - 1) / TILE);
    CUtensorMap map;
    const int s = plane_map(&map, d_x, Q, cin / 8, HALO);
    if (s != IRONAV_OK) return s;
    int dev = 0, nsm = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    unsigned* err = nullptr;
    CK(cudaMallocAsync(&err, sizeof(unsigned), static_cast<cudaStream_t>(stream)));
    CK(cudaMemsetAsync(err, 0, sizeof(unsigned), static_cast<cudaStream_t>(stream)));
    const int grid = std::min(tiles, nsm * 4);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const __nv_bfloat16* w = static_cast<const __nv_bfloat16*>(d_w);
    const __nv_bfloat16* mask = static_cast<const __nv_bfloat16*>(d_mask);
    __nv_bfloat16* y = static_cast<__nv_bfloat16*>(d_y);
    if (cin == 32) conv3x3_kernel<32><<<grid, 128, conv3x3_smem_bytes<32>(), st>>>(map, w, d_bias, relu, mask, y, Q, tiles, err);
    else conv3x3_kernel<16><<<grid, 128, conv3x3_smem_bytes<16>(), st>>>(map, w, d_bias, relu, mask, y, Q, tiles, err);
    CK(cudaGetLastError());
    unsigned h = 0;
    CK(cudaMemcpyAsync(&h, err, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    CK(cudaFreeAsync(err, st));
    CK(cudaStreamSynchronize(st));
    return h ? IRONAV_TIMEOUT : IRONAV_OK;
}
