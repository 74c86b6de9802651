// Learned guiding proposal: network state, training-record layout and host entry
// points of the tcgen05 kernels in wr_guide.cu (failures throw wr::Error).
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>

#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace wrg {

constexpr int kGuideLayers = 5;
constexpr int kGuideWidth = 64;
constexpr int kGuideParams = kGuideLayers * kGuideWidth * kGuideWidth;   // 20,480
constexpr int kGuideLobes = 8;
constexpr float kLambdaMin = 0.5f;     // lobe sharpness = softplus(s) + kLambdaMin
constexpr float kLambdaMax = 5000.f;   // sharpness cap (keeps the vMF normaliser finite in FP32)
constexpr float kCMax = 100.f;         // default clamp of the per-sample loss weight
constexpr uint32_t kNoRecord = 0xFFFFFFFFu;

// Per-path lobe record written by the inference kernel: 10 float4 per wavefront slot,
//   [0..7] (axis.xyz, sharpness)   [8] weights 0..3   [9] weights 4..7 (all zero: no guide here)
constexpr int kLobeFloat4 = 10;
// The render's per-path lobes: 5 chunks of 8 halves (axis x, y, z, sharpness, weight)
constexpr int kPackedChunks = 5;

// Training record, 5 float4 per guided vertex:
//   r0 (position.xyz, c)  r1 (normal.xyz, parent record bits)  r2 (outgoing.xyz, -)
//   r3 (sampled direction.xyz, -)  r4 (throughput arriving at the vertex .rgb, -)
// c accumulates luminance(contribution / throughput) over every contribution that the
// rest of the path makes, i.e. a one-sample estimate of f cos L_i / pdf for the sampled
// direction; the loss of the record is -min(c, c_max) log q(direction).
constexpr int kRecordFloat4 = 5;

struct GuideNet {
    __nv_bfloat16 *w = nullptr;    // bf16 W of each layer as its shared-memory operand tile (8 KB per layer)
    float *master = nullptr;       // FP32 master weights [layer][out][in]
    float *grad = nullptr;         // FP32 gradient summed over samples (filled by guide_sum_gradient)
    float *partial = nullptr;      // per-CTA partial gradients, slots x kGuideParams (layout: partial_offset)
    int slots = 0;                 // training CTAs (one per SM)
    float *m = nullptr, *v = nullptr;   // Adam moments
    uint32_t *err = nullptr;       // set to 1 when a tensor-core completion wait timed out
    float box_lo[3] = {0.f, 0.f, 0.f};
    float box_inv[3] = {1.f, 1.f, 1.f};   // position feature = (p - box_lo) * box_inv
};

// normal given to the network: the geometric normal turned toward the outgoing direction
// (both the inference kernel and the training records use it)
#ifdef __CUDACC__
template <class V>
__host__ __device__ __forceinline__ V guide_normal(V ng, V wo) {
    return (ng.x * wo.x + ng.y * wo.y + ng.z * wo.z) < 0.f ? V{-ng.x, -ng.y, -ng.z} : ng;
}
#endif

void guide_alloc(GuideNet &g);
void guide_free(GuideNet &g);
void guide_init(GuideNet &g, uint32_t seed, cudaStream_t st);
void guide_set_master(GuideNet &g, const float *host_w, cudaStream_t st);
void guide_get_master(const GuideNet &g, float *host_w, cudaStream_t st);

// lobes for explicit (position, normal, outgoing) rows, 9 floats each
void guide_infer_rows(const GuideNet &g, const float *rows_dev, uint32_t n, float4 *lobes_dev, int sms, cudaStream_t st);
// packed lobes for every live path of the wavefront (hit point, geometric normal turned
// toward the outgoing direction, outgoing direction); count is the device counter of live
// paths; chunk c of slot i goes to lobes_packed[c * stride + i]
void guide_infer_wavefront(const GuideNet &g, const float4 *o, const float4 *d, const float4 *hit, const uint32_t *count,
                           const float4 *tris, const uint32_t *tri_mat, uint4 *lobes_packed, size_t stride, int sms,
                           cudaStream_t st);
// the loss gradient of minibatch rows [first, count) into the per-CTA partial slots (and the
// summed loss added to *loss_dev when given); row r reads record (r * stride) % total. Returns
// the number of partial slots written (pass it to guide_sum_gradient / guide_adam).
// overlap: launched with programmatic stream serialization, so that its set-up and first gather
// run under the previous kernel of the stream (which must be a guide_adam step or need no wait).
int guide_gradient(GuideNet &g, const float4 *records_dev, uint32_t count, uint32_t first, uint32_t total,
                   uint32_t stride, float c_max, double *loss_dev, cudaStream_t st, bool overlap = false);
// out_dev[0] = sum of c over records [0, n) with c > 0, out_dev[1] = their number (FP64)
void guide_cstats(const float4 *records_dev, uint32_t n, double *out_dev, int sms, cudaStream_t st);
// the gradient of the last guide_gradient call, summed over its nslots partial slots in a fixed
// order, into g.grad
void guide_sum_gradient(GuideNet &g, int nslots, cudaStream_t st);
// one Adam step on the gradient of the last guide_gradient call (nslots partial slots), scaled by
// `scale`
void guide_adam(GuideNet &g, float lr, float scale, int step, int nslots, cudaStream_t st, bool overlap = false);

}  // namespace wrg
