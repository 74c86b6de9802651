// Device functions of the learned guiding proposal used inside the shade and
// shadow kernels: the lobe-mixture density and its sampling, the one-sample MIS
// mixture with BSDF sampling, and the training-record bookkeeping.
//
// The lobes (packed halves in shared memory, wrg::PackedLobes) are 8 von Mises-Fisher
// lobes (axis mu, sharpness lambda, weight w):
//     q(d) = sum_k w_k lambda_k / (2 pi (1 - exp(-2 lambda_k))) exp(lambda_k (mu_k . d - 1)).
// Lobe selection uses the weights divided by their sum (the same normalisation as the
// density); sampling a lobe uses the inversion of
// W. Jakob, "Numerically stable sampling of the von Mises-Fisher distribution
// on S2" (2012): cos(theta) = 1 + log(u + (1 - u) exp(-2 lambda)) / lambda.
#pragma once

#include "wr_device.cuh"
#include "wr_guide.h"
#include "wr_guide_net.cuh"

namespace wrd {

// probability of sampling the guide instead of the BSDF (0.65 measured best of 0.5 / 0.65 / 0.75 /
// 0.85 in equal-time error on the door-gap room)
constexpr float kGuideAlpha = 0.65f;

__device__ __forceinline__ float guide_weight_sum(const wrg::PackedLobes &L) {
    float w[8];
    L.load(4, w);
    return ((w[0] + w[1]) + (w[2] + w[3])) + ((w[4] + w[5]) + (w[6] + w[7]));
}

// The lobes of one path vertex, prepared once for that vertex's density evaluations and its
// sample: the packed halves, and per lobe the factor a_k = lambda_k / |m_k| (the sharpness over the
// length of the stored axis m_k, so that lambda_k (mu_k . d) = a_k (m_k . d)) and the coefficient
// coef_k = (w_k / sum w) lambda_k / (2 pi (1 - exp(-2 lambda_k))). The density
//     q(d) = sum_k coef_k exp(a_k (m_k . d) - lambda_k)
// is the same mixture as the one guide_sample draws from (lobe k with probability w_k / sum w,
// then the vMF lobe with axis m_k / |m_k| and sharpness lambda_k).
struct GuideVertex {
    const wrg::PackedLobes *L;
    float a[8], coef[8];
};

__device__ __forceinline__ void guide_prepare(const wrg::PackedLobes &L, GuideVertex &g) {
    float mx[8], my[8], mz[8], lam[8], w[8];
    L.load(0, mx);
    L.load(1, my);
    L.load(2, mz);
    L.load(3, lam);
    L.load(4, w);
    const float inv_total = __fdividef(1.f, ((w[0] + w[1]) + (w[2] + w[3])) + ((w[4] + w[5]) + (w[6] + w[7])));
    g.L = &L;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        g.a[k] = lam[k] * rsqrtf(mx[k] * mx[k] + my[k] * my[k] + mz[k] * mz[k]);
        // lambda >= 0.5: 1 - exp(-2 lambda) >= 0.63, no cancellation
        g.coef[k] = w[k] * inv_total * __fdividef(lam[k], 2.f * kPi * (1.f - __expf(-2.f * lam[k])));
    }
}

__device__ __forceinline__ float guide_pdf(const GuideVertex &g, f3 d) {
    float mx[8], my[8], mz[8], lam[8];
    g.L->load(0, mx);
    g.L->load(1, my);
    g.L->load(2, mz);
    g.L->load(3, lam);
    float p = 0.f;
#pragma unroll
    for (int k = 0; k < 8; ++k)
        p = fmaf(g.coef[k], __expf(fmaf(g.a[k], mx[k] * d.x + my[k] * d.y + mz[k] * d.z, -lam[k])), p);
    return p;
}

// draws a direction from the mixture: u_sel picks the lobe (by weight), (u1, u2) the direction
__device__ __forceinline__ f3 guide_sample(const GuideVertex &g, float u_sel, float u1, float u2) {
    const wrg::PackedLobes &L = *g.L;
    float w[8], mx[8], my[8], mz[8], lam[8];
    L.load(4, w);
    const float total = ((w[0] + w[1]) + (w[2] + w[3])) + ((w[4] + w[5]) + (w[6] + w[7]));
    const float target = u_sel * total;
    float acc = 0.f;
    int pick = 7;
#pragma unroll
    for (int k = 0; k < 7; ++k) {
        acc += w[k];
        if (pick == 7 && target < acc) pick = k;
    }
    L.load(0, mx);
    L.load(1, my);
    L.load(2, mz);
    L.load(3, lam);
    float ax = mx[7], ay = my[7], az = mz[7], lm = lam[7];
#pragma unroll
    for (int k = 0; k < 7; ++k)
        if (k == pick) { ax = mx[k]; ay = my[k]; az = mz[k]; lm = lam[k]; }
    const float inv = rsqrtf(ax * ax + ay * ay + az * az);
    const float v = 1.f - u1;   // in (0, 1]
    float ct = 1.f + __fdividef(__logf(v + (1.f - v) * __expf(-2.f * lm)), lm);
    ct = fminf(fmaxf(ct, -1.f), 1.f);
    const float st = sqrtf(fmaxf(0.f, 1.f - ct * ct));
    float sp, cp;
    __sincosf(2.f * kPi * u2, &sp, &cp);
    const Frame fr(mk(ax * inv, ay * inv, az * inv));   // y axis = lobe axis
    return normalize(fr.to_world(mk(st * cp, ct, st * sp)));
}

__device__ __forceinline__ float luminance(f3 c) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; }

// adds a path contribution c (film units) to the training records of the path: record r
// receives luminance(c / throughput_r), the part of its one-sample estimate f cos L_i / pdf
__device__ __forceinline__ void record_contribution(float4 *records, uint32_t rec, f3 c) {
    for (int guard = 0; rec != wrg::kNoRecord && guard < 64; ++guard) {
        float4 *r = records + wrg::kRecordFloat4 * size_t(rec);
        const float4 t = r[4];
        const f3 q = mk(t.x > 0.f ? c.x / t.x : 0.f, t.y > 0.f ? c.y / t.y : 0.f, t.z > 0.f ? c.z / t.z : 0.f);
        const float add = luminance(q);
        if (add > 0.f && isfinite(add)) atomicAdd(&r[0].w, add);
        rec = __float_as_uint(r[1].w);
    }
}

}  // namespace wrd
