// proposer.cuh — the learned proposer's kernels that are not contractions: its input from the pictures, the
// linear head (73,728 features -> 13 outputs) forward and backward, the loss, Adam, and the transposed weights
// of the backward convolutions. The network (the north star's form 4): 4 conv3x3 layers of 32 channels with
// ReLU on a 48 x 48 input of two channels — the current macroblock's 16 x 16 luma tiled 3 x 3 (so every
// position of the window meets the current samples) and the co-located 48 x 48 reference window (the macroblock
// at its centre, 16 samples around it, edges repeated) — both u8 / 255, then a linear head giving 4 candidate
// vectors (x, y in units of 32 luma samples: +-1 covers +-32) and 5 partition logits (P_Skip, 16x16, 16x8,
// 8x16, 8x8). Layer 1 takes 16 input channels (two planes) of which channels 0 and 1 carry the input.
#pragma once
#include <cuda_bf16.h>
#include <cstdint>

#include "tc_conv.cuh"

namespace ironav {
namespace prop {

constexpr int NOUT = 13;                  // 4 vectors x 2 + 5 logits
constexpr int NFEAT = 32 * 48 * 48;       // the head's inputs: layer 4's 32 channels x 48 x 48
constexpr float MV_SCALE = 128.f;         // quarter samples per output unit (32 luma samples)

// One training or proposal sample: the macroblock (mbx, mby) of the current picture `cur` predicted from `ref`
// (luma w x h, 8-bit; rows `stride` samples apart in cur, `ref_stride` in ref, 0 meaning `stride`).
struct Sample {
    const uint8_t* cur;
    const uint8_t* ref;
    int w, h, stride, mbx, mby, ref_stride;
};

// The input planes (two: channels 0-7 and 8-15, chunk-major padded) of n samples: a thread per pixel.
__global__ void prep_kernel(const Sample* __restrict__ samples, int n, __nv_bfloat16* __restrict__ x) {
    const long long Q = (long long)n * tc::RPIX;
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= Q) return;
    const int s = (int)(q / tc::RPIX), p = (int)(q % tc::RPIX), ry = p / tc::RW, rx = p % tc::RW;
    __align__(16) __nv_bfloat16 v[8];
#pragma unroll
    for (int e = 0; e < 8; e++) v[e] = __float2bfloat16_rn(0.f);
    if (ry > 0 && ry < tc::RW - 1 && rx > 0 && rx < tc::RW - 1) {
        const Sample S = samples[s];
        const int iy = ry - 1, ix = rx - 1;
        const int cx = min(S.mbx * 16 + (ix & 15), S.w - 1), cy = min(S.mby * 16 + (iy & 15), S.h - 1);
        const int wx = min(max(S.mbx * 16 - 16 + ix, 0), S.w - 1), wy = min(max(S.mby * 16 - 16 + iy, 0), S.h - 1);
        v[0] = __float2bfloat16_rn((float)S.cur[(size_t)cy * S.stride + cx] * (1.f / 255.f));
        v[1] = __float2bfloat16_rn((float)S.ref[(size_t)wy * (S.ref_stride > 0 ? S.ref_stride : S.stride) + wx] * (1.f / 255.f));
    }
    *reinterpret_cast<uint4*>(x + (size_t)q * 8) = *reinterpret_cast<const uint4*>(v);
    *reinterpret_cast<uint4*>(x + ((size_t)Q + q) * 8) = make_uint4(0, 0, 0, 0);
}

// Feature f of the head (channel c = f % 32, interior pixel (iy, ix) = (f / 32) / 48, (f / 32) % 48) of sample s
// in the chunk-major planes of Q pixels.
__device__ __forceinline__ size_t feat_index(int s, int f, long long Q) {
    const int c = f & 31, pix = f >> 5, iy = pix / 48, ix = pix % 48;
    const long long q = (long long)s * tc::RPIX + (iy + 1) * tc::RW + (ix + 1);
    return ((size_t)(c >> 3) * Q + q) * 8 + (c & 7);
}

// out[s][j] = hb[j] + sum_f hw[j][f] * feat(s, f): a CTA of 256 threads per HEAD_SPB samples, so that each
// weight read from L2 serves HEAD_SPB samples (the head's weights are 3.8 MB; every sample needs all of them).
constexpr int HEAD_SPB = 8;

__global__ void __launch_bounds__(256) head_fwd_kernel(const __nv_bfloat16* __restrict__ feat, long long Q, int n, const float* __restrict__ hw,
                                                       const float* __restrict__ hb, float* __restrict__ out) {
    const int s0 = blockIdx.x * HEAD_SPB, tid = threadIdx.x;
    const int ns = min(HEAD_SPB, n - s0);
    float acc[HEAD_SPB][NOUT];
#pragma unroll
    for (int i = 0; i < HEAD_SPB; i++)
#pragma unroll
        for (int j = 0; j < NOUT; j++) acc[i][j] = 0.f;
    for (int f = tid; f < NFEAT; f += 256) {
        float wj[NOUT];
#pragma unroll
        for (int j = 0; j < NOUT; j++) wj[j] = __ldg(&hw[(size_t)j * NFEAT + f]);
#pragma unroll
        for (int i = 0; i < HEAD_SPB; i++) {
            const float v = i < ns ? __bfloat162float(feat[feat_index(s0 + i, f, Q)]) : 0.f;
#pragma unroll
            for (int j = 0; j < NOUT; j++) acc[i][j] += v * wj[j];
        }
    }
    __shared__ float red[8][HEAD_SPB * NOUT];
#pragma unroll
    for (int i = 0; i < HEAD_SPB; i++)
#pragma unroll
        for (int j = 0; j < NOUT; j++) {
            float a = acc[i][j];
#pragma unroll
            for (int off = 16; off >= 1; off >>= 1) a += __shfl_xor_sync(0xffffffffu, a, off);
            if ((tid & 31) == 0) red[tid >> 5][i * NOUT + j] = a;
        }
    __syncthreads();
    if (tid < HEAD_SPB * NOUT) {
        const int i = tid / NOUT, j = tid % NOUT;
        if (i < ns) {
            float a = hb[j];
            for (int w = 0; w < 8; w++) a += red[w][tid];
            out[(size_t)(s0 + i) * NOUT + j] = a;
        }
    }
}

// The head's weights packed for head_fwd_packed_kernel: hwt[f][16] = hw[j][f] for j < 13, zero after, so that
// a feature's 13 weights are four 16-byte loads.
__global__ void head_pack_kernel(const float* __restrict__ hw, float* __restrict__ hwt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= NFEAT * 16) return;
    const int f = i >> 4, j = i & 15;
    hwt[i] = j < NOUT ? hw[(size_t)j * NFEAT + f] : 0.f;
}

constexpr int HEAD_PIX = 128;   // interior pixels (of 2304) a CTA of head_fwd_packed_kernel sums over
constexpr int HEAD_CHUNK = 16;  // pixels whose packed weights a CTA holds in shared memory at a time
constexpr int HEAD_WPIX = 32 * 4 + 1;  // float4s a pixel's weights take in shared memory: 32 channels x 4, and a
                                       // pad that puts a warp's four pixels on different banks
constexpr int HEAD_SPL = 4;       // samples a lane
constexpr int HEAD_SAMPLES = 256; // samples a CTA (8 warps of 8 x HEAD_SPL samples x 4 pixels)

// The head: CTA (x, y) takes samples 256x .. 256x + 255 and interior pixels HEAD_PIX * y .. + HEAD_PIX - 1. Lane
// l of warp w takes samples 256x + 32w + 4 (l / 4) + k (k < 4) and every fourth pixel from l % 4, so a warp's
// feature loads are 64 contiguous bytes a sample (four pixels of one plane), and each weight read from shared
// memory serves four samples. The CTA stages the packed weights of HEAD_CHUNK pixels at a time in shared memory
// (coalesced); a warp reads four pixels' weights at once (four addresses on different banks). The four lanes of
// a sample are summed by shuffles and added to out (which CTAs y = 0 start from the bias; out must be zero
// before the launch).
__global__ void __launch_bounds__(256) head_fwd_packed_kernel(const __nv_bfloat16* __restrict__ feat, long long Q, int n,
                                                              const float4* __restrict__ hwt, const float* __restrict__ hb,
                                                              float* __restrict__ out) {
    __shared__ float4 ws[HEAD_CHUNK * HEAD_WPIX];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, pl = lane & 3;
    const int s0 = blockIdx.x * HEAD_SAMPLES + warp * 32 + (lane >> 2) * HEAD_SPL;
    const int p0 = blockIdx.y * HEAD_PIX;
    float acc[HEAD_SPL][16];
#pragma unroll
    for (int k = 0; k < HEAD_SPL; k++)
#pragma unroll
        for (int j = 0; j < 16; j++) acc[k][j] = 0.f;
    for (int c0 = p0; c0 < p0 + HEAD_PIX && c0 < 48 * 48; c0 += HEAD_CHUNK) {
        const int np = min(HEAD_CHUNK, 48 * 48 - c0);  // a multiple of 4: 2304 and the chunk are
        __syncthreads();
        for (int i = threadIdx.x; i < np * 128; i += 256) ws[(i >> 7) * HEAD_WPIX + (i & 127)] = __ldg(hwt + (size_t)c0 * 128 + i);
        __syncthreads();
        for (int pp = pl; pp < np; pp += 4) {
            const int pix = c0 + pp, iy = pix / 48, ix = pix - iy * 48;
            const int rq = (iy + 1) * tc::RW + (ix + 1);
            const float4* wp = ws + pp * HEAD_WPIX;
#pragma unroll 1
            for (int c = 0; c < 4; c++) {
                uint4 raw[HEAD_SPL];
#pragma unroll
                for (int k = 0; k < HEAD_SPL; k++) {
                    const int s = s0 + k;
                    raw[k] = s < n ? *reinterpret_cast<const uint4*>(feat + ((size_t)c * Q + (long long)s * tc::RPIX + rq) * 8)
                                   : make_uint4(0, 0, 0, 0);
                }
#pragma unroll
                for (int e = 0; e < 8; e++) {
                    const float4* wf = wp + ((c * 8 + e) << 2);
#pragma unroll
                    for (int kk = 0; kk < 4; kk++) {
                        const float4 w4 = wf[kk];
#pragma unroll
                        for (int k = 0; k < HEAD_SPL; k++) {
                            const float x = __bfloat162float(reinterpret_cast<const __nv_bfloat16*>(&raw[k])[e]);
                            acc[k][4 * kk] += x * w4.x;
                            acc[k][4 * kk + 1] += x * w4.y;
                            acc[k][4 * kk + 2] += x * w4.z;
                            acc[k][4 * kk + 3] += x * w4.w;
                        }
                    }
                }
            }
        }
    }
#pragma unroll
    for (int k = 0; k < HEAD_SPL; k++)
#pragma unroll
        for (int j = 0; j < NOUT; j++) {
            acc[k][j] += __shfl_xor_sync(0xffffffffu, acc[k][j], 1);
            acc[k][j] += __shfl_xor_sync(0xffffffffu, acc[k][j], 2);
        }
    if (pl == 0) {
#pragma unroll
        for (int k = 0; k < HEAD_SPL; k++)
            if (s0 + k < n)
#pragma unroll
                for (int j = 0; j < NOUT; j++) atomicAdd(&out[(size_t)(s0 + k) * NOUT + j], acc[k][j] + (blockIdx.y == 0 ? hb[j] : 0.f));
    }
}

// The loss of n samples and its gradient d_out (already divided by n): winner-takes-all L1 on the vectors (the
// candidate nearest the target, plus 0.05 of every candidate's distance so that none is left untrained) and
// cross-entropy on the partition logits. target_mv in quarter samples; target_part in 0..4. sums[0] += the
// vector loss, sums[1] += the partition loss, sums[2] += the partition hits (top-1).
__global__ void loss_kernel(const float* __restrict__ out, const int16_t* __restrict__ target_mv, const uint8_t* __restrict__ target_part, int n,
                            float* __restrict__ dout, float* __restrict__ sums) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const float* o = out + (size_t)s * NOUT;
    float* d = dout + (size_t)s * NOUT;
    const float tx = target_mv[2 * s] / MV_SCALE, ty = target_mv[2 * s + 1] / MV_SCALE;
    int best = 0;
    float bd = 1e30f, dist[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        dist[k] = fabsf(o[2 * k] - tx) + fabsf(o[2 * k + 1] - ty);
        if (dist[k] < bd) bd = dist[k], best = k;
    }
    float lmv = bd;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        lmv += 0.05f * dist[k];
        const float wk = (k == best ? 1.f : 0.f) + 0.05f;
        d[2 * k] = wk * (o[2 * k] > tx ? 1.f : (o[2 * k] < tx ? -1.f : 0.f)) / n;
        d[2 * k + 1] = wk * (o[2 * k + 1] > ty ? 1.f : (o[2 * k + 1] < ty ? -1.f : 0.f)) / n;
    }
    float m = o[8];
    int arg = 0;
    for (int c = 1; c < 5; c++)
        if (o[8 + c] > m) m = o[8 + c], arg = c;
    float z = 0.f;
    for (int c = 0; c < 5; c++) z += __expf(o[8 + c] - m);
    const int t = target_part[s];
    const float lce = logf(z) - (o[8 + t] - m);
    for (int c = 0; c < 5; c++) d[8 + c] = (__expf(o[8 + c] - m) / z - (c == t ? 1.f : 0.f)) / n;
    atomicAdd(&sums[0], lmv);
    atomicAdd(&sums[1], lce);
    atomicAdd(&sums[2], arg == t ? 1.f : 0.f);
}

// The head's weight and bias gradients, a thread per feature: ghw[j][f] += sum_s dout[s][j] * feat(s, f).
__global__ void head_wgrad_kernel(const __nv_bfloat16* __restrict__ feat, long long Q, int n, const float* __restrict__ dout,
                                  float* __restrict__ ghw, float* __restrict__ ghb) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f < NOUT && ghb != nullptr) {
        float a = 0.f;
        for (int s = 0; s < n; s++) a += dout[(size_t)s * NOUT + f];
        ghb[f] += a;
    }
    if (f >= NFEAT) return;
    float acc[NOUT];
#pragma unroll
    for (int j = 0; j < NOUT; j++) acc[j] = 0.f;
    for (int s = 0; s < n; s++) {
        const float v = __bfloat162float(feat[feat_index(s, f, Q)]);
        if (v != 0.f)
#pragma unroll
            for (int j = 0; j < NOUT; j++) acc[j] += v * dout[(size_t)s * NOUT + j];
    }
#pragma unroll
    for (int j = 0; j < NOUT; j++) ghw[(size_t)j * NFEAT + f] += acc[j];
}

// The gradient into layer 4's output through its ReLU: dz(s, f) = (feat(s, f) > 0) * sum_j dout[s][j] hw[j][f],
// written into the chunk-major planes dz (whose ring stays zero): a thread per (sample, feature).
__global__ void head_dgrad_kernel(const __nv_bfloat16* __restrict__ feat, long long Q, int n, const float* __restrict__ dout,
                                  const float* __restrict__ hw, __nv_bfloat16* __restrict__ dz) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)n * NFEAT) return;
    const int s = (int)(i / NFEAT), f = (int)(i % NFEAT);
    const size_t at = feat_index(s, f, Q);
    float a = 0.f;
    if (__bfloat162float(feat[at]) > 0.f)
#pragma unroll
        for (int j = 0; j < NOUT; j++) a += dout[(size_t)s * NOUT + j] * hw[(size_t)j * NFEAT + f];
    dz[at] = __float2bfloat16_rn(a);
}

// Adam (bias-corrected) on a flat parameter vector; the gradient is cleared after its use.
__global__ void adam_kernel(float* __restrict__ p, float* __restrict__ g, float* __restrict__ m, float* __restrict__ v, long long n, float lr,
                            float b1, float b2, float c1, float c2, float eps) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi, vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    g[i] = 0.f;
}

// The BF16 weights of a layer for its forward convolution ([9][32][cin], as the master) and, when wt is set, the
// transposed and mirrored ones of its data gradient: wt[t][i][o] = w[8 - t][o][i] (cin = 32).
__global__ void weights_kernel(const float* __restrict__ w, int cin, __nv_bfloat16* __restrict__ wf, __nv_bfloat16* __restrict__ wt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 9 * 32 * cin) return;
    wf[i] = __float2bfloat16_rn(w[i]);
    if (wt != nullptr) {
        const int t = i / (32 * cin), o = (i / cin) % 32, k = i % cin;
        wt[((8 - t) * 32 + k) * 32 + o] = __float2bfloat16_rn(w[i]);
    }
}

// The judge's inputs: 4 vectors in quarter samples (the outputs times MV_SCALE, rounded to nearest, clamped to
// the search's range) and the class of largest logit (the first on ties) when its softmax probability is at
// least min_conf, else 5 (unsure), a thread per sample.
__global__ void propose_kernel(const float* __restrict__ out, int n, float min_conf, int16_t* __restrict__ cands, uint8_t* __restrict__ cls) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const float* o = out + (size_t)s * NOUT;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const float x = fminf(fmaxf(rintf(o[2 * k] * MV_SCALE), -2048.f), 2047.f);
        const float y = fminf(fmaxf(rintf(o[2 * k + 1] * MV_SCALE), -512.f), 511.f);
        cands[(size_t)s * 8 + 2 * k] = (int16_t)x;
        cands[(size_t)s * 8 + 2 * k + 1] = (int16_t)y;
    }
    int arg = 0;
    float m = o[8];
    for (int c = 1; c < 5; c++)
        if (o[8 + c] > m) m = o[8 + c], arg = c;
    float z = 0.f;
    for (int c = 0; c < 5; c++) z += __expf(o[8 + c] - m);
    cls[s] = (uint8_t)(1.f / z >= min_conf ? arg : 5);
}

}  // namespace prop
}  // namespace ironav
