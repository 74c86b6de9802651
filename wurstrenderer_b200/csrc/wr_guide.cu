// Learned guiding proposal: a small MLP trained online on incident-radiance
// samples produced by the path tracer, predicting 8 von Mises-Fisher lobes that
// serve as a directional sampling density (combined with BSDF sampling by
// one-sample MIS in k_shade, so the estimator stays unbiased). It has no
// counterpart in the reference; the plain NEE+MIS path is unchanged when it is off.
//
// Network: 64 encoded inputs (57 features + zeros + a constant 1), 4 hidden
// layers of 64 ReLU units, 64 outputs of which 40 are used (8 x axis, sharpness,
// weight). Unit 63 of every hidden layer is held at 1 (its weight row is e_63),
// so column 63 of the following layer is that layer's bias.
// Arithmetic: BF16 weights and activations, FP32 accumulation on the 5th-gen
// tensor cores (tcgen05.mma, accumulators in TMEM), FP32 master weights and Adam.
//
//   k_guide_infer   128-row tiles: encode -> 5 x (tcgen05.mma M128 N64 K64 -> TMEM ->
//                   ReLU -> smem) -> lobe parameters per path
//   k_guide_train   forward (activations kept in smem), mixture-NLL gradient, backward:
//                   dX = dH W (M128 N64 K64), dW += dH^T X (M64 N64 K128, MN-major operands,
//                   accumulated in TMEM across all tiles of the CTA), the CTA's dW stored into
//                   its own partial-gradient slot
//   k_guide_adam    fixed-order sum of the partial slots, Adam on the FP32 master weights, and
//                   the BF16 W image in the kernels' shared-memory operand layout
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <string>
#include <vector>

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "wr_device.cuh"
#include "wr_trace.cuh"
#include "wr_guide.h"
#include "wr_host.h"
#include "wr_guide_net.cuh"
#include "wr_guide_tc.cuh"

namespace wrg {

// --------------------------------------------------------------- inference ----
// Inputs come either from the wavefront (hit point of every live path) or from an
// explicit array of (p, n, wo) rows (validation).
struct InferSource {
    // wavefront
    const float4 *o, *d, *hit;
    const uint32_t *count;      // device counter of live paths
    const float4 *tris;
    const uint32_t *tri_mat;
    // explicit rows: 9 floats (p, n, wo)
    const float *rows;
    uint32_t nrows;
};

__device__ __forceinline__ bool fetch_point(const InferSource &s, uint32_t i, f3 &p, f3 &n, f3 &wo) {
    if (s.rows) {
        const float *r = s.rows + 9 * size_t(i);
        p = mk(r[0], r[1], r[2]); n = mk(r[3], r[4], r[5]); wo = mk(r[6], r[7], r[8]);
        return true;
    }
    // the path's records first (independent loads), then the triangle they name
    const float4 h = s.hit[i], o = s.o[i], d = s.d[i];
    const uint32_t tri = __float_as_uint(h.w);
    if (tri == wrd::MISS) return false;
    const uint32_t mat = __ldg(s.tri_mat + tri);
    const float4 a = __ldg(s.tris + 3 * tri), b = __ldg(s.tris + 3 * tri + 1), c = __ldg(s.tris + 3 * tri + 2);
    if (mat & wrd::LIGHT_BIT) return false;
    const f3 dd = mk(d.x, d.y, d.z);
    p = mk(o.x, o.y, o.z) + dd * h.x;
    wo = -dd;
    n = guide_normal(wrd::surface_normal(a, b, c, h.y, h.z), wo);
    return true;
}

// Inference: kGroups warpgroups per CTA, and each warpgroup keeps kPair 128-row tiles in
// flight, each with its own activation tile, 64 TMEM columns and mbarrier. The group's
// first thread issues a tile's layer as soon as that tile's previous epilogue is stored, so
// while the group converts one tile's accumulators (tcgen05.ld, ReLU, bf16, st.shared) the
// tensor core runs the other tile's MMAs: kGroups x kPair = 4 tiles per CTA, 8 per SM, over
// weights loaded once per CTA. The next pair's path records are prefetched into L2 while the
// current pair runs.
// Output: lobes as FP32 (kLobeFloat4 float4 per row, the validation API) or packed
// halves (chunk-major with `packed_stride`, the render).
constexpr int kGroups = 2;
constexpr int kPair = 2;
constexpr int kInferCtasPerSm = 2;
constexpr size_t kInferSmem = size_t(kWeightBytesInfer) + size_t(kGroups * kPair) * kActBytes + 64;

__device__ __forceinline__ void prefetch_l2(const void *p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

// gathers and encodes row `row` of a tile into `at` (all-zero features when the row is past the
// end or its path did not hit a surface); returns whether the row has a guide point
__device__ __forceinline__ bool stage_row(const InferSource &src, const GuideNet &g, unsigned char *at, int r,
                                          uint32_t row, uint32_t n_rows) {
    float x[kW];
    f3 p, n, wo;
    const bool valid = row < n_rows && fetch_point(src, row, p, n, wo);
    if (valid) encode(p, n, wo, g, x);
    else {
#pragma unroll
        for (int k = 0; k < kW; ++k) x[k] = 0.f;
    }
    store_row(at, r, x);
    return valid;
}

__device__ __forceinline__ void issue_layer(unsigned char *at, const unsigned char *wt, int l, uint32_t tmem,
                                            uint64_t *mbar) {
    const uint32_t idesc = idesc_bf16(128, l == kLayers - 1 ? kLastRows : kW, 0, 0);
    const uint32_t a0 = smem_addr(at), b0 = smem_addr(wt + l * 8192);
#pragma unroll
    for (int ks = 0; ks < 4; ++ks)
        mma_bf16(tmem, smem_desc(a0 + ks * 256, 128, 1024), smem_desc(b0 + ks * 256, 128, 1024), idesc,
                 ks > 0 ? 1u : 0u);
    mma_commit(smem_addr(mbar));
}

__global__ void __launch_bounds__(kTile *kGroups, kInferCtasPerSm) k_guide_infer(GuideNet g, InferSource src,
                                                                                float4 *lobes_f, uint4 *lobes_packed,
                                                                                size_t packed_stride) {
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char *wt = smem;                                   // weight tiles (last layer: 48 rows)
    const int tid = threadIdx.x, grp = tid >> 7, r = tid & 127, warp = tid >> 5;
    unsigned char *act[kPair];                                  // this group's activation tiles
#pragma unroll
    for (int j = 0; j < kPair; ++j) act[j] = smem + kWeightBytesInfer + (grp * kPair + j) * kActBytes;
    uint64_t *mbar = reinterpret_cast<uint64_t *>(smem + kWeightBytesInfer + kGroups * kPair * kActBytes) + grp * kPair;
    uint32_t *slot = reinterpret_cast<uint32_t *>(smem + kWeightBytesInfer + kGroups * kPair * kActBytes +
                                                  8 * kGroups * kPair);
    if (warp == 0) tmem_alloc(smem_addr(slot), 64 * kGroups * kPair);
    if (r == 0)
        for (int j = 0; j < kPair; ++j) mbar_init(smem_addr(mbar + j), 1);
    load_weight_image(wt, g.w, kWeightBytesInfer);
    fence_async_smem();
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tmem0 = *slot + uint32_t(64 * kPair * grp);
    const uint32_t lane_base = uint32_t((warp & 3) * 32) << 16;
    const int bar = 1 + grp;
    const uint32_t n_rows = src.rows ? src.nrows : *src.count;
    const uint32_t npairs = (n_rows + kTile * kPair - 1) / (kTile * kPair);
    const uint32_t pair_step = gridDim.x * kGroups;
    uint32_t phase[kPair] = {0u, 0u};
    bool failed = false;
    for (uint32_t pr = blockIdx.x * kGroups + grp; pr < npairs && !failed; pr += pair_step) {
        if (!src.rows) {   // the next pair's path records toward L2 while this pair runs
            const uint32_t nrow = (pr + pair_step) * (kTile * kPair) + r;
#pragma unroll
            for (int j = 0; j < kPair; ++j)
                if (nrow + j * kTile < n_rows) {
                    prefetch_l2(src.hit + nrow + j * kTile);
                    prefetch_l2(src.o + nrow + j * kTile);
                    prefetch_l2(src.d + nrow + j * kTile);
                }
        }
        uint32_t row[kPair];
        bool valid[kPair];
#pragma unroll
        for (int j = 0; j < kPair; ++j) {
            row[j] = (pr * kPair + j) * kTile + r;
            valid[j] = stage_row(src, g, act[j], r, row[j], n_rows);
        }
        fence_async_smem();
        fence_before_sync();
        group_sync(bar);
        fence_after_sync();
        if (r == 0)
#pragma unroll
            for (int j = 0; j < kPair; ++j) issue_layer(act[j], wt, 0, tmem0 + 64 * j, mbar + j);
        float out[kW];
        for (int l = 0; l < kLayers; ++l) {
#pragma unroll
            for (int j = 0; j < kPair; ++j) {
                const uint32_t tm = tmem0 + 64 * j;
                // every thread waits on the tile's mbarrier (bounded); a wait that gave up is
                // voted on once per pair, so that the group's barriers stay in step
                if (!mbar_wait(smem_addr(mbar + j), phase[j], kWaitIters)) failed = true;
                phase[j] ^= 1u;
                fence_after_sync();
                if (l < kLayers - 1) {   // hidden layer: ReLU, bf16, back into the tile in place
                    tmem_ld32(tm + lane_base, out);
                    store_row_relu(act[j], r, out, 0, 4);
                    tmem_ld32(tm + lane_base + 32, out);
                    store_row_relu(act[j], r, out, 32, 4);
                    fence_async_smem();
                    fence_before_sync();
                    group_sync(bar);
                    fence_after_sync();
                    if (r == 0) issue_layer(act[j], wt, l + 1, tm, mbar + j);
                    continue;
                }
                tmem_ld32(tm + lane_base, out);   // outputs 0..47
                tmem_ld16(tm + lane_base + 32, out + 32);
                if (row[j] < n_rows) {
                    Lobes L;
                    raw_to_lobes(out, L);
                    if (lobes_packed) {
                        store_packed_lobes(lobes_packed, packed_stride, row[j], L, valid[j]);
                    } else {
                        float4 *o4 = lobes_f + kLobeFloat4 * size_t(row[j]);
                        if (valid[j]) {
#pragma unroll
                            for (int k = 0; k < 8; ++k) o4[k] = make_float4(L.mu[k][0], L.mu[k][1], L.mu[k][2], L.lam[k]);
                            o4[8] = make_float4(L.w[0], L.w[1], L.w[2], L.w[3]);
                            o4[9] = make_float4(L.w[4], L.w[5], L.w[6], L.w[7]);
                        } else {
                            o4[8] = make_float4(0.f, 0.f, 0.f, 0.f);   // zero weights: no lobe
                            o4[9] = make_float4(0.f, 0.f, 0.f, 0.f);
                        }
                    }
                }
            }
        }
        // every thread has read its TMEM lanes and the tensor core no longer reads the tiles;
        // the vote ends the group's work when any of its waits gave up
        fence_before_sync();
        failed = group_any(bar, failed);
        fence_after_sync();
        if (failed) break;
    }
    if (failed && r == 0) atomicExch(g.err, 1u);
    fence_before_sync();
    __syncthreads();
    if (warp == 0) tmem_dealloc(*slot, 64 * kGroups * kPair);
}

// ----------------------------------------------------------------- training ----
// A training tile is 128 rows (records); the CTA's 512 threads are four warpgroups over the same
// rows. Warp w reads TMEM lanes 32 (w % 4) .. 32 (w % 4) + 31, so the thread of warpgroup j and
// row r takes, in every epilogue, columns [16 j, 16 j + 16) of row r, and in the loss gradient
// lobes 2 j and 2 j + 1 (the row's mixture density is summed over the four threads through
// shared memory). One elected thread issues the MMAs. The backward pass keeps every layer's
// output gradient dH_l: the chain of dX products runs first (B = the W tile read MN-major, so no
// transposed copy is needed), and the five dW products follow together after it, so none of them
// delays a dX.
constexpr int kTrainGroups = 4;
constexpr int kTrainThreads = kTile * kTrainGroups;

// Layout of a partial-gradient slot, in the order the training CTA writes it: for layer l,
// column block col / 16 and column quad (col % 16) / 4, the 64 output rows n hold their 4
// consecutive columns, so the 16 threads of a warp that own rows n..n+15 store 256 contiguous
// bytes per instruction.
__host__ __device__ constexpr int partial_offset(int l, int n, int col) {
    return ((l * 4 + (col >> 4)) * 4 + ((col >> 2) & 3)) * 256 + n * 4 + (col & 3);
}
// the inverse: parameter index (l * 4096 + n * 64 + col) of slot offset u
__device__ __forceinline__ int partial_param(int u) {
    const int l = u >> 12, col = ((u >> 10) & 3) * 16 + ((u >> 8) & 3) * 4 + (u & 3), n = (u >> 2) & 63;
    return (l * kW + n) * kW + col;
}

// shared memory: the W image 40 KB, X_0..X_4 80 KB (the layer inputs), dH_0..dH_4 80 KB (the
// loss gradient at each layer's output) followed by 8 KB of zeros (the operand reach of the
// weight-gradient MMA stays inside the allocation for either reading of the descriptor's two
// strides), the density exchange (2 x 4 x 128 floats), two mbarriers and the TMEM address slot
constexpr int kTrainW = 0, kTrainX = kWeightBytes;
constexpr int kTrainDh = kTrainX + kLayers * kActBytes;
constexpr int kTrainExch = kTrainDh + kLayers * kActBytes + 8192;
constexpr int kTrainBarrier = kTrainExch + 2 * kTrainGroups * kTile * 4;
constexpr size_t kTrainSmem = size_t(kTrainBarrier) + 64;
static_assert(kTrainSmem <= 227 * 1024, "training tile does not fit in shared memory");

// Terms of the mixture-NLL gradient (oracle: loss_grad_output) for lobes 2 J and 2 J + 1 of a
// row, from the row's 40 used outputs o (5 per lobe: axis, sharpness, weight logit) and the
// sample direction d. The mixture weights are w_k = e_k / sum_k e_k with e_k = exp(logit_k - max);
// the thread returns its two lobes' sums of e_k f_k and of e_k (the row's four threads add them up
// through shared memory), so each lobe's exponential is evaluated by one thread only.
struct LobeTerms {
    float e[2], f[2], lam[2], cosk[2], mu[2][3], inr[2], e2[2], inv1me2[2], sig[2];
};

template <int J>
__device__ __forceinline__ float2 lobe_terms(const float *o, f3 d, LobeTerms &t) {
    float amax = -1e30f;
#pragma unroll
    for (int k = 0; k < 8; ++k) amax = fmaxf(amax, o[5 * k + 4]);
    float2 part = make_float2(0.f, 0.f);   // (sum e_k f_k, sum e_k) over this thread's lobes
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        const int k = 2 * J + j;
        const float rx = o[5 * k], ry = o[5 * k + 1], rz = o[5 * k + 2];
        t.inr[j] = rsqrtf(fmaxf(rx * rx + ry * ry + rz * rz, 1e-24f));   // 1 / max(|r|, 1e-12)
        t.mu[j][0] = rx * t.inr[j];
        t.mu[j][1] = ry * t.inr[j];
        t.mu[j][2] = rz * t.inr[j];
        // softplus(s) = log(1 + e^s) and its derivative, the sigmoid e^s / (1 + e^s), from one exp
        const float s = o[5 * k + 3];
        float sp;
        if (s > 20.f) {
            sp = s;
            t.sig[j] = 1.f;
        } else {
            const float es = __expf(s);
            sp = __logf(1.f + es);
            t.sig[j] = __fdividef(es, 1.f + es);
        }
        t.lam[j] = fminf(sp + kLambdaMin, kLambdaMax);
        t.e[j] = __expf(o[5 * k + 4] - amax);
        t.cosk[j] = t.mu[j][0] * d.x + t.mu[j][1] * d.y + t.mu[j][2] * d.z;
        t.e2[j] = __expf(-2.f * t.lam[j]);   // lam >= kLambdaMin: 1 - e2 >= 0.63
        t.inv1me2[j] = __fdividef(1.f, 1.f - t.e2[j]);
        t.f[j] = t.lam[j] * t.inv1me2[j] * (0.5f / wrd::kPi) * __expf(t.lam[j] * (t.cosk[j] - 1.f));
        part.x += t.e[j] * t.f[j];
        part.y += t.e[j];
    }
    return part;
}

// d(-c log p)/d(outputs) of the two lobes (cc = the clamped loss weight, ip = 1 / p, iw = 1 / sum e)
// into columns [10 J, 10 J + 10) of a row of the dH tile; the thread of lobes 6 and 7 also zeroes
// the unused columns 40..63
template <int J>
__device__ __forceinline__ void lobe_grads_store(const LobeTerms &t, f3 d, float cc, float ip, float iw, bool active,
                                                 unsigned char *tile, int row) {
    float go[10];
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        const float w = t.e[j] * iw;
        const float resp = w * t.f[j] * ip;
        const float dldl = __fdividef(1.f, t.lam[j]) - 2.f * t.e2[j] * t.inv1me2[j] + (t.cosk[j] - 1.f);
        const float a = -cc * resp * t.lam[j] * t.inr[j];
        go[5 * j + 0] = a * (d.x - t.mu[j][0] * t.cosk[j]);
        go[5 * j + 1] = a * (d.y - t.mu[j][1] * t.cosk[j]);
        go[5 * j + 2] = a * (d.z - t.mu[j][2] * t.cosk[j]);
        go[5 * j + 3] = -cc * resp * dldl * t.sig[j];
        go[5 * j + 4] = -cc * (resp - w);
    }
#pragma unroll
    for (int i = 0; i < 5; ++i) {
        const __nv_bfloat162 h = active ? __floats2bfloat162_rn(go[2 * i], go[2 * i + 1]) : __floats2bfloat162_rn(0.f, 0.f);
        *reinterpret_cast<__nv_bfloat162 *>(tile + tile_offset(row, 10 * J + 2 * i)) = h;
    }
    if (J == 3)
#pragma unroll
        for (int c = 40; c < kW; c += 8) *reinterpret_cast<uint4 *>(tile + tile_offset(row, c)) = make_uint4(0u, 0u, 0u, 0u);
}

__device__ __forceinline__ float2 lobe_terms_of(int j, const float *o, f3 d, LobeTerms &t) {
    switch (j) {
    case 0: return lobe_terms<0>(o, d, t);
    case 1: return lobe_terms<1>(o, d, t);
    case 2: return lobe_terms<2>(o, d, t);
    default: return lobe_terms<3>(o, d, t);
    }
}

__device__ __forceinline__ void lobe_grads_store_of(int j, const LobeTerms &t, f3 d, float cc, float ip, float iw,
                                                    bool active, unsigned char *tile, int row) {
    switch (j) {
    case 0: lobe_grads_store<0>(t, d, cc, ip, iw, active, tile, row); break;
    case 1: lobe_grads_store<1>(t, d, cc, ip, iw, active, tile, row); break;
    case 2: lobe_grads_store<2>(t, d, cc, ip, iw, active, tile, row); break;
    default: lobe_grads_store<3>(t, d, cc, ip, iw, active, tile, row); break;
    }
}

// columns [16 j, 16 j + 16) of a 64-wide row x into a tile
__device__ __forceinline__ void store_row_part(unsigned char *tile, int row, const float *x, int j) {
    switch (j) {
    case 0: store_row(tile, row, x, 0, 2); break;
    case 1: store_row(tile, row, x + 16, 16, 2); break;
    case 2: store_row(tile, row, x + 32, 32, 2); break;
    default: store_row(tile, row, x + 48, 48, 2); break;
    }
}

// training records: kRecordFloat4 float4 each (layout in wr_guide.h)
// rows [first, count) of the minibatch map to records (row * stride) % total (a fixed shuffle
// when stride and total are coprime)
__global__ void __launch_bounds__(kTrainThreads, 1) k_guide_train(GuideNet g, const float4 *records, uint32_t count,
                                                                 uint32_t first, uint32_t total, uint32_t stride,
                                                                 float c_max, double *loss_out) {
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char *wt = smem + kTrainW;      // W image   5 x 8 KB
    unsigned char *xt = smem + kTrainX;      // X_0..X_4  5 x 16 KB (the layer inputs, kept for backward)
    unsigned char *dht = smem + kTrainDh;    // dH_0..dH_4 5 x 16 KB (the gradients at the layer outputs)
    float *exch = reinterpret_cast<float *>(smem + kTrainExch);
    uint64_t *mbar = reinterpret_cast<uint64_t *>(smem + kTrainBarrier);   // [0] MMA completion, [1] weights
    uint32_t *slot = reinterpret_cast<uint32_t *>(smem + kTrainBarrier + 16);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int grp = warp >> 2;                 // column slice and lobe pair of this thread
    const int r = (warp & 3) * 32 + lane;      // row of the tile = TMEM lane
    const uint32_t n = count > first ? count - first : 0u;
    const uint32_t ntiles = (n + kTile - 1) / kTile;
    const bool has_tiles = blockIdx.x < ntiles;
    const uint32_t mb = smem_addr(mbar), mbw = smem_addr(mbar + 1);
    // The optimiser step that follows may be scheduled now: it waits for this grid before it reads
    // the partial gradients. In turn this kernel runs its set-up and the first tile's gather and
    // encoding before it waits for the previous optimiser step, whose weights it then loads.
    griddep_launch_dependents();
    if (warp == 0) tmem_alloc(smem_addr(slot), 512);
    if (tid == 0) {
        mbar_init(mb, 1);
        mbar_init(mbw, 1);
    }
    for (int i = tid; i < 512; i += kTrainThreads)   // the zeros behind the dH tiles
        reinterpret_cast<uint4 *>(dht + kLayers * kActBytes)[i] = make_uint4(0u, 0u, 0u, 0u);
    fence_async_smem();
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tmem = *slot;
    const uint32_t tD = tmem, tdW = tmem + 64;   // columns [0, 64) scratch, [64, 384) dW of layers 0..4
    const uint32_t lane_base = uint32_t((warp & 3) * 32) << 16;
    const uint32_t id_fwd = idesc_bf16(128, 64, 0, 0);
    const uint32_t id_dx = idesc_bf16(128, 64, 0, 1);   // B = the W tile read MN-major (rows = K = out)
    const uint32_t id_dw = idesc_bf16(64, 64, 1, 1);
    uint32_t phase = 0;
    // failed: a wait of this thread gave up; stop: the CTA's vote on it at the next barrier (a
    // failure is acted on only after the vote, so that every thread leaves at the same barrier)
    bool failed = false, stop = false, any_tile = false, weights_in = !has_tiles;
    double loss = 0.0;
    for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const uint32_t row = tile * kTile + r;
        const bool valid = row < n;
        float x[kW];
        f3 dir = mk(0.f, 1.f, 0.f);
        float c = 0.f;
        if (valid) {
            const uint32_t ri = uint32_t((uint64_t(first + row) * stride) % (total ? total : 1u));
            const float4 *rec = records + kRecordFloat4 * size_t(ri);
            const float4 s0 = rec[0], s1 = rec[1], s2 = rec[2], s3 = rec[3];
            encode(mk(s0.x, s0.y, s0.z), mk(s1.x, s1.y, s1.z), mk(s2.x, s2.y, s2.z), g, x);
            dir = mk(s3.x, s3.y, s3.z);
            c = s0.w;
        } else {
#pragma unroll
            for (int k = 0; k < kW; ++k) x[k] = 0.f;
        }
        store_row_part(xt, r, x, grp);
        if (tile == blockIdx.x) {
            // the previous kernels of the stream are complete from here on: the weight image may
            // be read and this CTA's partial-gradient slot written
            griddep_wait();
            if (tid == 0) {   // the weight image in one bulk copy
                mbar_expect_tx(mbw, kWeightBytes);
                bulk_load(smem_addr(wt), g.w, kWeightBytes, mbw);
            }
        }
        fence_async_smem();
        fence_before_sync();
        __syncthreads();
        fence_after_sync();
        // forward; X_l kept for the backward pass
        float out[48];
        for (int l = 0; l < kLayers; ++l) {
            if (tid == 0) {
                if (!weights_in) {
                    weights_in = mbar_wait(mbw, 0, kWaitIters);
                    failed = failed || !weights_in;
                }
                if (weights_in) {
                    const uint32_t a0 = smem_addr(xt + l * kActBytes), b0 = smem_addr(wt + l * 8192);
#pragma unroll
                    for (int ks = 0; ks < 4; ++ks)
                        mma_bf16(tD, smem_desc(a0 + ks * 256, 128, 1024), smem_desc(b0 + ks * 256, 128, 1024), id_fwd,
                                 ks > 0 ? 1u : 0u);
                }
                mma_commit(mb);
            }
            if (!mbar_wait(mb, phase, kWaitIters)) failed = true;
            phase ^= 1u;
            fence_after_sync();
            if (l == kLayers - 1) {   // outputs 0..47 for the loss
                tmem_ld32(tD + lane_base, out);
                tmem_ld16(tD + lane_base + 32, out + 32);
                break;
            }
            float v[16];
            tmem_ld16(tD + lane_base + 16 * grp, v);
            store_row_relu(xt + (l + 1) * kActBytes, r, v, 16 * grp, 2);
            fence_async_smem();
            fence_before_sync();
            stop = __syncthreads_or(failed);
            fence_after_sync();
            if (stop) break;
        }
        if (stop) break;
        // loss gradient at the outputs -> dH_4 (bf16)
        const bool active = valid && c > 0.f;
        LobeTerms lt{};
        const float2 part = active ? lobe_terms_of(grp, out, dir, lt) : make_float2(0.f, 0.f);
        exch[grp * kTile + r] = part.x;
        exch[(kTrainGroups + grp) * kTile + r] = part.y;
        fence_before_sync();
        stop = __syncthreads_or(failed);
        fence_after_sync();
        if (stop) break;
        const float sum_ef = (exch[r] + exch[kTile + r]) + (exch[2 * kTile + r] + exch[3 * kTile + r]);
        const float sum_e = (exch[4 * kTile + r] + exch[5 * kTile + r]) + (exch[6 * kTile + r] + exch[7 * kTile + r]);
        const float iw = active ? __fdividef(1.f, sum_e) : 0.f;
        const float p = fmaxf(sum_ef * iw, 1e-30f);
        const float cc = fminf(c, c_max);
        if (active && grp == 0) loss += double(-cc * __logf(p));
        lobe_grads_store_of(grp, lt, dir, cc, __fdividef(1.f, p), iw, active, dht + (kLayers - 1) * kActBytes, r);
        fence_async_smem();
        fence_before_sync();
        __syncthreads();
        fence_after_sync();
        // backward: the dX chain dH_l -> dH_{l-1}, then every layer's dW at once
        for (int l = kLayers - 1; l >= 0; --l) {
            if (tid == 0) {
                if (l > 0) {
                    // dX = dH_l W_l : M = 128, N = 64 (in), K = 64 (out); B = the W tile, MN-major
                    const uint32_t a0 = smem_addr(dht + l * kActBytes), b0 = smem_addr(wt + l * 8192);
#pragma unroll
                    for (int ks = 0; ks < 4; ++ks)
                        mma_bf16(tD, smem_desc(a0 + ks * 256, 128, 1024), smem_desc(b0 + ks * 2048, 1024, 128), id_dx,
                                 ks > 0 ? 1u : 0u);
                } else {
                    // dW_l += dH_l^T X_l for every layer: M = 64 (out), N = 64 (in), K = 128 (rows),
                    // MN-major operands, accumulated in TMEM over the CTA's tiles
#pragma unroll 1
                    for (int k = kLayers - 1; k >= 0; --k) {
                        const uint32_t a0 = smem_addr(dht + k * kActBytes), b0 = smem_addr(xt + k * kActBytes);
#pragma unroll
                        for (int ks = 0; ks < 8; ++ks)
                            mma_bf16(tdW + 64 * k, smem_desc(a0 + ks * 2048, 1024, 128),
                                     smem_desc(b0 + ks * 2048, 1024, 128), id_dw, (any_tile || ks > 0) ? 1u : 0u);
                    }
                }
                mma_commit(mb);
            }
            if (!mbar_wait(mb, phase, kWaitIters)) failed = true;
            phase ^= 1u;
            fence_after_sync();
            if (l > 0) {
                float v[16];
                tmem_ld16(tD + lane_base + 16 * grp, v);
                relu_mask_row(xt + l * kActBytes, r, v, 16 * grp, 2);   // input of layer l = ReLU output of layer l-1
                store_row(dht + (l - 1) * kActBytes, r, v, 16 * grp, 2);
            }
            fence_async_smem();
            fence_before_sync();
            stop = __syncthreads_or(failed);
            fence_after_sync();
            if (stop) break;
        }
        if (stop) break;
        any_tile = true;
    }
    if (tid == 0 && !weights_in) mbar_wait(mbw, 0, kWaitIters);   // no copy into shared memory outlives the CTA
    if (stop) {
        if (tid == 0) atomicExch(g.err, 1u);
    } else if (any_tile) {
        // this CTA's dW into its own partial slot (summed in a fixed order by the optimiser, so
        // the gradient is deterministic). M = 64 accumulator row n lives in TMEM lane
        // (n % 16) + 32 (n / 16). CTA b has tiles exactly when b < ceil(rows / 128), and only
        // those slots are summed.
        float *slot_base = g.partial + size_t(blockIdx.x) * kParams;
        const int nrow = 16 * (warp & 3) + lane;
        for (int l = 0; l < kLayers; ++l) {
            float v[16];
            tmem_ld16(tdW + 64 * l + 16 * grp + lane_base, v);
            if (lane < 16) {
                float4 *gr = reinterpret_cast<float4 *>(slot_base + partial_offset(l, nrow, 16 * grp));
#pragma unroll
                for (int k = 0; k < 4; ++k)   // column quad k: 256 floats further on
                    gr[64 * k] = make_float4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
            }
        }
    }
    if (loss_out) {   // only the first warpgroup carries loss terms
        __shared__ double red[kTrainThreads / 32];
        double v = loss;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) red[warp] = v;
        __syncthreads();
        if (tid == 0) {
            double t = 0.0;
            for (int w = 0; w < kTrainThreads / 32; ++w) t += red[w];
            atomicAdd(loss_out, t);
        }
    }
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    if (warp == 0) tmem_dealloc(tmem, 512);
}

// ------------------------------------------------------------- optimiser ----
// Deterministic sum of the per-CTA partial gradients: a block covers kRedParams consecutive
// slot offsets with kRedGroups groups of threads; group j adds slots j, j + kRedGroups, ... eight
// loads at a time in a fixed order, then group 0 adds the group sums in order. Returns the total
// on group-0 threads.
constexpr int kRedParams = 64;
constexpr int kRedGroups = 8;
constexpr int kRedThreads = kRedParams * kRedGroups;

__device__ __forceinline__ float reduce_partials(const GuideNet &g, int u, int nslots) {
    __shared__ float red[kRedGroups][kRedParams];
    const int p = threadIdx.x % kRedParams, grp = threadIdx.x / kRedParams;
    const float *part = g.partial + u;
    float s = 0.f;
    for (int k0 = grp; k0 < nslots; k0 += 8 * kRedGroups) {
        float v[8];
#pragma unroll
        for (int t = 0; t < 8; ++t) {
            const int k = k0 + t * kRedGroups;
            v[t] = k < nslots ? part[size_t(k) * kParams] : 0.f;
        }
        s += ((v[0] + v[1]) + (v[2] + v[3])) + ((v[4] + v[5]) + (v[6] + v[7]));
    }
    red[grp][p] = s;
    __syncthreads();
    float total = 0.f;
    if (grp == 0)
#pragma unroll
        for (int j = 0; j < kRedGroups; ++j) total += red[j][p];
    return total;
}

// the summed gradient into g.grad (for callers that read it)
__global__ void __launch_bounds__(kRedThreads) k_guide_sum(GuideNet g, int nslots) {
    const int u = blockIdx.x * kRedParams + threadIdx.x % kRedParams;
    const float total = reduce_partials(g, u, nslots);
    if (threadIdx.x < kRedParams) g.grad[partial_param(u)] = total;
}

// one Adam step on the summed gradient (apply = 0: only the constant-unit rows and the bf16
// copies are refreshed from the master weights)
__global__ void __launch_bounds__(kRedThreads) k_guide_adam(GuideNet g, float lr, float scale, int step, int apply,
                                                            int nslots) {
    griddep_launch_dependents();   // the next training step may set up; it waits for this grid
    griddep_wait();                // the partial gradients are complete; no kernel reads the weights
    const int u = blockIdx.x * kRedParams + threadIdx.x % kRedParams;
    const float gsum = apply ? reduce_partials(g, u, nslots) : 0.f;
    if (threadIdx.x >= kRedParams) return;
    const int i = partial_param(u);
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float c1 = 1.f - powf(b1, float(step)), c2 = 1.f - powf(b2, float(step));
    const int l = i / (kW * kW), nrow = (i / kW) % kW, k = i % kW;
    float w = g.master[i];
    if (apply) {
        const float gr = gsum * scale;
        const float m = b1 * g.m[i] + (1.f - b1) * gr;
        const float v = b2 * g.v[i] + (1.f - b2) * gr * gr;
        g.m[i] = m;
        g.v[i] = v;
        w -= lr * (m / c1) / (sqrtf(v / c2) + eps);
    }
    if (l < kLayers - 1 && nrow == kW - 1) w = (k == kW - 1) ? 1.f : 0.f;   // the constant unit
    g.master[i] = w;
    const __nv_bfloat16 h = __float2bfloat16_rn(w);
    g.w[weight_image_index(l, nrow, k)] = h;
}

// sum of c and number of records with c > 0 over records [0, n)
__global__ void k_guide_cstats(const float4 *records, uint32_t n, double *out) {
    __shared__ double red[2][256];
    double sum = 0.0, cnt = 0.0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float c = records[kRecordFloat4 * size_t(i)].w;
        if (c > 0.f && isfinite(c)) { sum += double(c); cnt += 1.0; }
    }
    red[0][threadIdx.x] = sum;
    red[1][threadIdx.x] = cnt;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (int(threadIdx.x) < s) {
            red[0][threadIdx.x] += red[0][threadIdx.x + s];
            red[1][threadIdx.x] += red[1][threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        atomicAdd(out, red[0][0]);
        atomicAdd(out + 1, red[1][0]);
    }
}

__global__ void k_guide_init(GuideNet g, uint32_t seed) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kParams; i += gridDim.x * blockDim.x) {
        const int l = i / (kW * kW);
        const uint4 h = wrd::pcg4d(make_uint4(uint32_t(i), seed, 0x6a09e667u, 77u));
        const float u = wrd::u01(h.x) * 2.f - 1.f;
        const float limit = sqrtf(6.f / float(kW + kW)) * (l == kLayers - 1 ? 0.1f : 1.f);
        g.master[i] = u * limit;
        g.m[i] = 0.f;
        g.v[i] = 0.f;
        g.grad[i] = 0.f;
    }
}

}  // namespace wrg

// ------------------------------------------------------------------ host ----
namespace wrg {

static void check(cudaError_t e, const char *what) {
    if (e != cudaSuccess)
        throw wr::Error(e == cudaErrorMemoryAllocation ? WR_ERR_OUT_OF_MEMORY : WR_ERR_CUDA,
                        std::string(what) + ": " + cudaGetErrorString(e));
}

void guide_alloc(GuideNet &g) {
    check(cudaMalloc(&g.w, kParams * 2), "guide alloc");
    check(cudaMalloc(&g.master, kParams * 4), "guide alloc");
    check(cudaMalloc(&g.grad, kParams * 4), "guide alloc");
    int dev = 0, sms = 148;
    check(cudaGetDevice(&dev), "guide alloc");
    check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "guide alloc");
    g.slots = sms;
    check(cudaMalloc(&g.partial, size_t(g.slots) * kParams * 4), "guide alloc");
    check(cudaMalloc(&g.m, kParams * 4), "guide alloc");
    check(cudaMalloc(&g.v, kParams * 4), "guide alloc");
    check(cudaMalloc(&g.err, 4), "guide alloc");
    check(cudaMemset(g.err, 0, 4), "guide memset");
    check(cudaFuncSetAttribute(k_guide_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kInferSmem)),
          "guide smem attribute");
    check(cudaFuncSetAttribute(k_guide_train, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kTrainSmem)),
          "guide smem attribute");
}

void guide_free(GuideNet &g) {
    for (void *p : {(void *)g.w, (void *)g.master, (void *)g.grad, (void *)g.partial, (void *)g.m,
                    (void *)g.v,
                    (void *)g.err})
        if (p) cudaFree(p);
    g = GuideNet{};
}

void guide_init(GuideNet &g, uint32_t seed, cudaStream_t st) {
    k_guide_init<<<40, 512, 0, st>>>(g, seed);
    k_guide_adam<<<kParams / kRedParams, kRedThreads, 0, st>>>(g, 0.f, 0.f, 1, 0, 0);   // constant unit, bf16 copies
    check(cudaGetLastError(), "guide init");
}

void guide_set_master(GuideNet &g, const float *host_w, cudaStream_t st) {
    check(cudaMemcpyAsync(g.master, host_w, kParams * 4, cudaMemcpyHostToDevice, st), "guide set");
    k_guide_adam<<<kParams / kRedParams, kRedThreads, 0, st>>>(g, 0.f, 0.f, 1, 0, 0);
    check(cudaGetLastError(), "guide set");
}

void guide_get_master(const GuideNet &g, float *host_w, cudaStream_t st) {
    check(cudaMemcpyAsync(host_w, g.master, kParams * 4, cudaMemcpyDeviceToHost, st), "guide get");
    check(cudaStreamSynchronize(st), "guide get");
}

int infer_grid(int sms) { return sms * kInferCtasPerSm; }   // CTAs per SM allowed by shared memory and TMEM

void guide_infer_rows(const GuideNet &g, const float *rows_dev, uint32_t n, float4 *lobes_dev, int sms, cudaStream_t st) {
    InferSource s{};
    s.rows = rows_dev;
    s.nrows = n;
    k_guide_infer<<<infer_grid(sms), kTile * kGroups, kInferSmem, st>>>(g, s, lobes_dev, nullptr, 0);
    check(cudaGetLastError(), "guide infer");
}

void guide_infer_wavefront(const GuideNet &g, const float4 *o, const float4 *d, const float4 *hit, const uint32_t *count,
                           const float4 *tris, const uint32_t *tri_mat, uint4 *lobes_packed, size_t stride, int sms,
                           cudaStream_t st) {
    InferSource s{};
    s.o = o; s.d = d; s.hit = hit; s.count = count; s.tris = tris; s.tri_mat = tri_mat;
    k_guide_infer<<<infer_grid(sms), kTile * kGroups, kInferSmem, st>>>(g, s, nullptr, lobes_packed, stride);
}

// launches a kernel, with programmatic stream serialization when `overlap` is set (the kernel
// may then start before the previous one ends and waits for it with griddepcontrol.wait)
template <class... Params, class... Args>
static void launch(void (*kernel)(Params...), int grid, int block, size_t smem, cudaStream_t st, bool overlap,
                   const char *what, Args... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(unsigned(grid));
    cfg.blockDim = dim3(unsigned(block));
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = overlap ? 1 : 0;
    check(cudaLaunchKernelEx(&cfg, kernel, args...), what);
}

int guide_gradient(GuideNet &g, const float4 *records_dev, uint32_t count, uint32_t first, uint32_t total,
                   uint32_t stride, float c_max, double *loss_dev, cudaStream_t st, bool overlap) {
    // one CTA per partial-gradient slot (the shared memory allows one CTA per SM)
    launch(k_guide_train, g.slots, kTrainThreads, kTrainSmem, st, overlap, "guide train", g, records_dev, count, first,
           total, stride, c_max, loss_dev);
    const uint32_t rows = count > first ? count - first : 0u;
    return int(std::min<uint32_t>(uint32_t(g.slots), (rows + kTile - 1) / kTile));
}

void guide_cstats(const float4 *records_dev, uint32_t n, double *out_dev, int sms, cudaStream_t st) {
    check(cudaMemsetAsync(out_dev, 0, 16, st), "guide cstats");
    if (n) k_guide_cstats<<<sms * 2, 256, 0, st>>>(records_dev, n, out_dev);
    check(cudaGetLastError(), "guide cstats");
}

void guide_sum_gradient(GuideNet &g, int nslots, cudaStream_t st) {
    k_guide_sum<<<kParams / kRedParams, kRedThreads, 0, st>>>(g, nslots);
    check(cudaGetLastError(), "guide sum");
}

void guide_adam(GuideNet &g, float lr, float scale, int step, int nslots, cudaStream_t st, bool overlap) {
    launch(k_guide_adam, kParams / kRedParams, kRedThreads, 0, st, overlap, "guide adam", g, lr, scale, step, 1, nslots);
}

}  // namespace wrg
