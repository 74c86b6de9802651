// The guiding network's per-tile building blocks, shared by the inference and
// training kernels (wr_guide.cu) and the guided shade kernel (wr_kernels.cu):
// feature encoding, the bf16 canonical operand tiles, the output transform to
// von Mises-Fisher lobes and their packed form.
#pragma once

#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "wr_device.cuh"
#include "wr_guide.h"
#include "wr_guide_tc.cuh"

namespace wrg {

using wrd::f3;
using wrd::mk;

constexpr int kLayers = kGuideLayers;
constexpr int kW = kGuideWidth;              // layer width (inputs and outputs)
constexpr int kParams = kGuideParams;
constexpr int kTile = 128;                   // rows per tile = threads per CTA
constexpr uint32_t kWaitIters = 1u << 24;    // bounded mbarrier waits
constexpr int kWeightBytes = kLayers * 8192; // 5 bf16 64x64 tiles
constexpr int kLastRows = 48;                // output rows of the last layer that inference computes (40 used)
constexpr int kWeightBytesInfer = (kLayers - 1) * 8192 + kLastRows * kW * 2;
constexpr int kActBytes = kTile * kW * 2;    // one 128 x 64 bf16 activation tile

// ------------------------------------------------------------------ encoding ----
// 64 features: p in [0,1]^3, sin/cos(2^f pi p) for f = 0..5, n, wo, sin/cos(pi n),
// sin/cos(pi wo), six zeros, the constant 1. The base frequency uses the hardware
// sine/cosine (__sincosf: arguments within [-pi, pi], absolute error about 4e-7); the
// higher frequencies follow by the double-angle identities (sin 2a = 2 sin a cos a,
// cos 2a = 1 - 2 sin^2 a), whose error (a few 1e-5 after five doublings) is far below
// the bf16 rounding of the features (4e-3 relative).
__device__ __forceinline__ void encode(f3 p, f3 n, f3 wo, const GuideNet &g, float *x) {
    const float q[3] = {(p.x - g.box_lo[0]) * g.box_inv[0], (p.y - g.box_lo[1]) * g.box_inv[1],
                        (p.z - g.box_lo[2]) * g.box_inv[2]};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        x[a] = q[a];
        float sn, cs;
        __sincosf(wrd::kPi * q[a], &sn, &cs);
#pragma unroll
        for (int f = 0; f < 6; ++f) {
            x[3 + 6 * f + a] = sn;
            x[6 + 6 * f + a] = cs;
            const float s2 = 2.f * sn * cs, c2 = 1.f - 2.f * sn * sn;
            sn = s2;
            cs = c2;
        }
    }
    const float nv[3] = {n.x, n.y, n.z}, wv[3] = {wo.x, wo.y, wo.z};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        x[39 + a] = nv[a];
        x[42 + a] = wv[a];
        __sincosf(wrd::kPi * nv[a], &x[45 + a], &x[48 + a]);
        __sincosf(wrd::kPi * wv[a], &x[51 + a], &x[54 + a]);
    }
#pragma unroll
    for (int k = 57; k < 63; ++k) x[k] = 0.f;
    x[63] = 1.f;
}

// columns [c0, c0 + 8 * chunks) of a row of a canonical tile from v[0..]: 16-byte stores of
// 8 bf16 each (the whole 64-wide row by default)
__device__ __forceinline__ void store_row(unsigned char *tile, int row, const float *v, int c0 = 0,
                                          int chunks = kW / 8) {
#pragma unroll
    for (int j = 0; j < chunks; ++j) {
        const float *u = v + 8 * j;
        uint4 q;
        __nv_bfloat162 h0 = __floats2bfloat162_rn(u[0], u[1]), h1 = __floats2bfloat162_rn(u[2], u[3]),
                       h2 = __floats2bfloat162_rn(u[4], u[5]), h3 = __floats2bfloat162_rn(u[6], u[7]);
        q.x = *reinterpret_cast<uint32_t *>(&h0);
        q.y = *reinterpret_cast<uint32_t *>(&h1);
        q.z = *reinterpret_cast<uint32_t *>(&h2);
        q.w = *reinterpret_cast<uint32_t *>(&h3);
        *reinterpret_cast<uint4 *>(tile + tile_offset(row, c0 + 8 * j)) = q;
    }
}

// multiplies v[0..] by the mask (x > 0) of columns [c0, c0 + 8 * chunks) of a stored row
__device__ __forceinline__ void relu_mask_row(const unsigned char *tile, int row, float *v, int c0 = 0,
                                              int chunks = kW / 8) {
#pragma unroll
    for (int c = 0; c < 8 * chunks; c += 8) {
        const uint4 q = *reinterpret_cast<const uint4 *>(tile + tile_offset(row, c0 + c));
        const uint32_t wds[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            // a bf16 is positive when its sign bit is clear and it is not +0
            const uint32_t lo = wds[j] & 0xffffu, hi = wds[j] >> 16;
            if (!(lo != 0u && lo < 0x8000u)) v[c + 2 * j] = 0.f;
            if (!(hi != 0u && hi < 0x8000u)) v[c + 2 * j + 1] = 0.f;
        }
    }
}

// The bf16 weight copies in global memory are kept as the kernels' shared-memory operand image:
// tile l (8 KB) holds W_l (or W_l^T) in the canonical layout above, so a kernel brings them in
// with a linear copy. Offset of element (row, column) of tile l, in bf16 elements:
__device__ __forceinline__ int weight_image_index(int l, int row, int col) {
    return (l * 8192 + tile_offset(row, col)) >> 1;
}

// the first `bytes` of a weight image into shared memory, 16 bytes per thread and step
__device__ __forceinline__ void load_weight_image(unsigned char *dst, const __nv_bfloat16 *src, int bytes) {
    const uint4 *s4 = reinterpret_cast<const uint4 *>(src);
    uint4 *d4 = reinterpret_cast<uint4 *>(dst);
    for (int i = threadIdx.x; i < bytes / 16; i += blockDim.x) d4[i] = __ldg(s4 + i);
}

// columns [c0, c0 + 8 * chunks) of a row of a canonical tile from FP32 values v[0..] with
// ReLU applied (cvt.rn.relu)
__device__ __forceinline__ void store_row_relu(unsigned char *tile, int row, const float *v, int c0 = 0,
                                               int chunks = kW / 8) {
#pragma unroll
    for (int j = 0; j < chunks; ++j) {
        uint4 q;
        q.x = relu_bf16x2(v[8 * j], v[8 * j + 1]);
        q.y = relu_bf16x2(v[8 * j + 2], v[8 * j + 3]);
        q.z = relu_bf16x2(v[8 * j + 4], v[8 * j + 5]);
        q.w = relu_bf16x2(v[8 * j + 6], v[8 * j + 7]);
        *reinterpret_cast<uint4 *>(tile + tile_offset(row, c0 + 8 * j)) = q;
    }
}

// -------------------------------------------------------------- output lobes ----
// lobe parameters from raw outputs (the transform of oracle/guide_oracle.py: axis
// normalised, sharpness softplus + kLambdaMin, weights softmax)
struct Lobes {
    float mu[8][3], lam[8], w[8];
};

// softplus with the hardware exp / log (relative error ~1e-6, far below the half rounding of
// the stored sharpness)
__device__ __forceinline__ float softplus(float s) { return s > 20.f ? s : __logf(1.f + __expf(s)); }

__device__ __forceinline__ void raw_to_lobes(const float *o, Lobes &L) {
    float amax = -1e30f;
#pragma unroll
    for (int k = 0; k < 8; ++k) amax = fmaxf(amax, o[5 * k + 4]);
    float wsum = 0.f;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const float rx = o[5 * k], ry = o[5 * k + 1], rz = o[5 * k + 2];
        const float n2 = rx * rx + ry * ry + rz * rz;
        if (n2 > 1e-24f) {
            const float inv = rsqrtf(n2);
            L.mu[k][0] = rx * inv; L.mu[k][1] = ry * inv; L.mu[k][2] = rz * inv;
        } else {
            L.mu[k][0] = 0.f; L.mu[k][1] = 1.f; L.mu[k][2] = 0.f;
        }
        L.lam[k] = fminf(softplus(o[5 * k + 3]) + kLambdaMin, kLambdaMax);
        L.w[k] = __expf(o[5 * k + 4] - amax);
        wsum += L.w[k];
    }
    const float inv_sum = 1.f / wsum;
#pragma unroll
    for (int k = 0; k < 8; ++k) L.w[k] *= inv_sum;
}

// ------------------------------------------------------------ packed lobes ----
// The render keeps each path's lobes as halves in five 16-byte chunks, stored
// chunk-major in HBM (chunk c of wavefront slot i at c * capacity + i, coalesced):
//   chunk 0/1/2 = axis x/y/z of lobes 0..7, chunk 3 = sharpness, chunk 4 = weight.
// The shade kernel loads the five chunks of its path once into registers. Sampling and
// density evaluation both use these rounded values (the axis is renormalised after
// loading, the weights divided by their sum), so the density used for MIS is exactly the
// density that is sampled.
struct PackedLobes {
    uint4 c[kPackedChunks];

    __device__ __forceinline__ void load(int chunk, float *v) const {
        const uint4 q = c[chunk];
        const uint32_t wds[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const float2 f = __half22float2(*reinterpret_cast<const __half2 *>(&wds[j]));
            v[2 * j] = f.x;
            v[2 * j + 1] = f.y;
        }
    }
};

__device__ __forceinline__ void store_packed_lobes(uint4 *base, size_t stride, size_t slot, const Lobes &L,
                                                   bool valid) {
    float v[kPackedChunks][8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        v[0][k] = L.mu[k][0];
        v[1][k] = L.mu[k][1];
        v[2][k] = L.mu[k][2];
        v[3][k] = L.lam[k];
        v[4][k] = valid ? L.w[k] : 0.f;   // zero weights: no guide for this slot
    }
#pragma unroll
    for (int c = 0; c < kPackedChunks; ++c) {
        uint4 q;
        __half2 h0 = __floats2half2_rn(v[c][0], v[c][1]), h1 = __floats2half2_rn(v[c][2], v[c][3]),
                h2 = __floats2half2_rn(v[c][4], v[c][5]), h3 = __floats2half2_rn(v[c][6], v[c][7]);
        q.x = *reinterpret_cast<uint32_t *>(&h0);
        q.y = *reinterpret_cast<uint32_t *>(&h1);
        q.z = *reinterpret_cast<uint32_t *>(&h2);
        q.w = *reinterpret_cast<uint32_t *>(&h3);
        base[c * stride + slot] = q;
    }
}

}  // namespace wrg
