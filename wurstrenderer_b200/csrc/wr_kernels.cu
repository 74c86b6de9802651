// sm_100a kernels of the wavefront NEE+MIS path tracer.
//
// The reference integrator (src/renderer/pathnextevent.h:41-191 driving
// src/pathsampler/generalsubpathsampler.h:13-323) is recursive per pixel
// sample. Here every sample is a slot in a wavefront; one iteration of the
// bounce loop is five persistent, grid-stride kernels:
//   extend  closest hit for every live path                       (Scene::intersect)
//   shade   emitter hit (strategy B) or NEE at a surface (strategy A, emits a
//           shadow ray), then BSDF sampling; surviving paths are compacted into
//           the next wavefront by warp ballot/popc + one atomic per warp
//   raygen  fills the freed slots with new camera samples: light vertex,
//           camera vertex, light->camera connection (strategy C, emits a shadow
//           ray into the splat film), primary ray
//   shadow  any-hit test of every queued shadow ray; unoccluded contributions
//           are added to the FP64 film with FP64 atomics
//   advance one thread: queue bookkeeping for the next iteration
// Counters live on the device, so an iteration needs no host round trip and a
// pair of iterations is captured once into a CUDA graph by the host.
// Arithmetic is FP32; FP64 is used for the film and for building the light /
// environment CDF tables (the prefix sums at the end of this file).

#include <cstdint>
#include <cuda_runtime.h>

#include "wr_device.cuh"
#include "wr_guide.h"
#include "wr_guide_dev.cuh"
#include "wr_guide_net.cuh"
#include "wr_kernels.h"
#include "wr_trace.cuh"

namespace wrd {

// ------------------------------------------------------------------ BSDFs ----
// TwoSided(inner) of src/bsdf/twosided.h:25-63 with inner one of Lambert
// (lambertdiffuse.h:16-51), Oren-Nayar (orennayar.h:14-83), modified Phong
// (phong.h:22-93) or Mixed(diffuse, Phong) (mixed.h:20-60). Directions are in
// the local frame with y = normal.

__device__ __forceinline__ f3 lambert_or_on_eval(const DevMaterial &m, f3 in, f3 out) {
    if (in.y <= 0.f || out.y <= 0.f) return mk(0.f, 0.f, 0.f);
    const f3 kd = mk(m.kd[0], m.kd[1], m.kd[2]);
    if (!(m.flags & MAT_OREN_NAYAR)) return kd * kInvPi;
    const float sinI = sqrtf(fminf(fmaxf(1.f - in.y * in.y, 0.f), 1.f));
    const float sinO = sqrtf(fminf(fmaxf(1.f - out.y * out.y, 0.f), 1.f));
    float maxCos = 0.f, sinAlpha = 0.f, tanBeta = 0.f;
    if (sinI > 1e-4f && sinO > 1e-4f) {
        const float cI = in.x / sinI, sI = in.z / sinI, cO = out.x / sinO, sO = out.z / sinO;
        maxCos = fmaxf(0.f, cI * cO + sI * sO);
        if (fabsf(in.y) > fabsf(out.y)) { sinAlpha = sinO; tanBeta = sinI / in.y; }
        else { sinAlpha = sinI; tanBeta = sinO / out.y; }
    }
    return kd * (kInvPi * (m.on_a + m.on_b * maxCos * sinAlpha * tanBeta));
}

__device__ __forceinline__ float diffuse_pdf(f3 in, f3 out) {
    if (in.y <= 0.f || out.y <= 0.f) return 0.f;
    return out.y * kInvPi;
}

__device__ __forceinline__ f3 phong_eval(const DevMaterial &m, f3 in, f3 out) {
    if (in.y <= 0.f || out.y <= 0.f) return mk(0.f, 0.f, 0.f);
    const f3 refl = mk(-in.x, in.y, -in.z);   // Local3::Reflect(-in)
    const float cr = dot(refl, out);
    if (cr <= 0.f) return mk(0.f, 0.f, 0.f);
    const float n = m.exponent;
    return mk(m.ks[0], m.ks[1], m.ks[2]) * ((n + 2.f) * __powf(cr, n) * (kInvPi * 0.5f));
}

__device__ __forceinline__ float phong_pdf(const DevMaterial &m, f3 in, f3 out) {
    if (in.y <= 0.f && out.y <= 0.f) return 0.f;
    const f3 refl = mk(-in.x, in.y, -in.z);
    const float cr = dot(refl, out);
    if (cr <= 0.f) return 0.f;
    const float n = m.exponent;
    return (n + 1.f) * __powf(cr, n) * (kInvPi * 0.5f);
}

__device__ __forceinline__ f3 inner_eval(const DevMaterial &m, f3 in, f3 out) {
    f3 r = mk(0.f, 0.f, 0.f);
    if (m.flags & MAT_DIFFUSE) r = lambert_or_on_eval(m, in, out);
    if (m.flags & MAT_GLOSSY) r = r + phong_eval(m, in, out);
    return r;
}

__device__ __forceinline__ float inner_pdf(const DevMaterial &m, f3 in, f3 out) {
    const int both = (m.flags & MAT_DIFFUSE) && (m.flags & MAT_GLOSSY);
    float p = 0.f;
    if (m.flags & MAT_DIFFUSE) p = diffuse_pdf(in, out);
    if (m.flags & MAT_GLOSSY) p += phong_pdf(m, in, out);
    return both ? p * 0.5f : p;
}

__device__ __forceinline__ f3 cosine_hemisphere(float s0, float s1) {
    float sn, cs;
    __sincosf(2.f * kPi * s1, &sn, &cs);
    const float sinPhi = sqrtf(fmaxf(1.f - s0, 0.f));
    return mk(cs * sinPhi, sqrtf(s0), sn * sinPhi);
}

// lobe about the mirror direction (phong.h:58-72)
__device__ __forceinline__ f3 phong_direction(float n, f3 in, float s0, float s1) {
    const f3 refl = mk(-in.x, in.y, -in.z);
    const float cosT = __powf(s0, 1.f / (n + 1.f));
    const float sinT = sqrtf(fmaxf(1.f - cosT * cosT, 0.f));
    float sn, cs;
    __sincosf(2.f * kPi * s1, &sn, &cs);
    const Frame rf(refl);
    return rf.to_world(mk(sinT * cs, cosT, sinT * sn));
}

// Bsdf::sampleBsdfCosByPdf on the inner BSDF (front side): returns bsdf*cos/pdf
// (zero terminates the path) and writes the direction and its pdf.
__device__ __forceinline__ f3 inner_sample(const DevMaterial &m, f3 in, float s0, float s1, f3 &out, float &pdf) {
    const bool dif = m.flags & MAT_DIFFUSE, gl = m.flags & MAT_GLOSSY;
    pdf = 0.f;
    if (dif && gl) {
        // MixedBsdf: pick a component with s0, evaluate the mixture at the result
        const int k = s0 < 0.5f ? 0 : 1;
        const float r0 = fminf(s0 * 2.f - float(k), 0.99999994f);
        out = mk(0.f, 0.f, 0.f);
        if (k == 0) {
            if ((m.flags & MAT_OREN_NAYAR) ? in.y >= 0.f : in.y > 0.f) out = cosine_hemisphere(r0, s1);
        } else {
            if (in.y > 0.f) out = phong_direction(m.exponent, in, r0, s1);
        }
        const f3 f = inner_eval(m, in, out);
        pdf = inner_pdf(m, in, out);
        if (pdf == 0.f) return mk(0.f, 0.f, 0.f);
        return f * (out.y / pdf);
    }
    if (dif) {
        if (m.flags & MAT_OREN_NAYAR) {
            if (in.y < 0.f) return mk(0.f, 0.f, 0.f);
            out = cosine_hemisphere(s0, s1);
            pdf = out.y * kInvPi;
            return lambert_or_on_eval(m, out, in) * kPi;
        }
        if (in.y <= 0.f) return mk(0.f, 0.f, 0.f);
        out = cosine_hemisphere(s0, s1);
        pdf = fmaxf(out.y, 0.f) * kInvPi;
        if (out.y <= 0.f) return mk(0.f, 0.f, 0.f);
        return mk(m.kd[0], m.kd[1], m.kd[2]);
    }
    // Phong only
    if (in.y <= 0.f) return mk(0.f, 0.f, 0.f);
    const float n = m.exponent;
    const f3 refl = mk(-in.x, in.y, -in.z);
    out = phong_direction(n, in, s0, s1);
    const float cr = dot(out, refl);
    pdf = (n + 1.f) * 0.5f * kInvPi * __powf(fmaxf(cr, 0.f), n);
    if (refl.y <= 0.f || out.y <= 0.f || cr <= 0.f) return mk(0.f, 0.f, 0.f);
    return mk(m.ks[0], m.ks[1], m.ks[2]) * ((n + 2.f) / (n + 1.f) * out.y);
}

__device__ __forceinline__ f3 flip_y(f3 v) { return mk(v.x, -v.y, v.z); }

__device__ __forceinline__ f3 bsdf_eval(const DevMaterial &m, f3 in, f3 out) {
    if (in.y > 0.f && out.y > 0.f) return inner_eval(m, in, out);
    if (in.y <= 0.f && out.y <= 0.f) return inner_eval(m, flip_y(in), flip_y(out));
    return mk(0.f, 0.f, 0.f);
}

__device__ __forceinline__ float bsdf_pdf(const DevMaterial &m, f3 in, f3 out) {
    if (in.y > 0.f && out.y > 0.f) return inner_pdf(m, in, out);
    if (in.y <= 0.f && out.y <= 0.f) return inner_pdf(m, flip_y(in), flip_y(out));
    return 0.f;
}

__device__ __forceinline__ f3 bsdf_sample(const DevMaterial &m, f3 in, float s0, float s1, f3 &out, float &pdf) {
    if (in.y > 0.f) return inner_sample(m, in, s0, s1, out, pdf);
    f3 o;
    const f3 w = inner_sample(m, flip_y(in), s0, s1, o, pdf);
    out = flip_y(o);
    return w;
}

// ------------------------------------------------------------ environment ----
// EnvmapLight + EquiRectRep (src/light/envmap.h:22-101,
// src/sphericalrepresentation/equirectangular.h:66-123, mapping.h:91-96,302-323)
__device__ __forceinline__ void panorama(f3 d, float &u, float &v) {
    u = atan2f(-d.z, -d.x) * (kInvPi * 0.5f) + 0.5f;
    v = acosf(fminf(fmaxf(d.y, -1.f), 1.f)) * kInvPi;
}

__device__ __forceinline__ f3 env_texel(const DevScene &s, int x, int y) {
    x %= s.env_w;
    if (x < 0) x += s.env_w;
    y = min(max(y, 0), s.env_h - 1);
    return xyz(__ldg(s.env_texels + size_t(y) * s.env_w + x));
}

__device__ __forceinline__ f3 env_eval(const DevScene &s, f3 d) {
    float u, v;
    panorama(d, u, v);
    const float su = u * float(s.env_w) - 0.5f, sv = v * float(s.env_h) - 0.5f;
    const float fx = floorf(su), fy = floorf(sv);
    const int x = int(fx), y = int(fy);
    const float dx1 = su - fx, dy1 = sv - fy, dx2 = 1.f - dx1, dy2 = 1.f - dy1;
    return env_texel(s, x, y) * (dx2 * dy2) + env_texel(s, x, y + 1) * (dx2 * dy1) +
           env_texel(s, x + 1, y) * (dx1 * dy2) + env_texel(s, x + 1, y + 1) * (dx1 * dy1);
}

// directional pdf (solid angle) of EquiRectRep::pdfA
__device__ __forceinline__ float env_pdf(const DevScene &s, f3 d) {
    float u, v;
    panorama(d, u, v);
    if (!(u >= 0.f && v >= 0.f)) return 0.f;   // non-finite direction
    const int px = min(int(u * float(s.env_w)), s.env_w - 1), py = min(int(v * float(s.env_h)), s.env_h - 1);
    const float sine = sqrtf(fminf(fmaxf(1.f - d.y * d.y, 0.f), 1.f));
    if (sine <= 1e-12f) return 0.f;
    return __ldg(s.env_pixel_pdf + size_t(py) * s.env_w + px) * float(s.env_w * s.env_h) / sine * (kInvPi * kInvPi * 0.5f);
}

// ------------------------------------------------------------ light vertex ----
struct LightVtx {
    f3 pos;       // area: point; environment: direction toward the environment
    f3 n;
    f3 contrib;   // Le0 / pdf of the light subpath (mPathContrib)
    float pdfA;   // lPdfA
    bool env;
};

// GeneralSubpathSampler::createLightSubpath with one vertex (generalsubpathsampler.h:185-268)
__device__ __forceinline__ LightVtx sample_light(const DevScene &s, float u0, float u1) {
    LightVtx l;
    if (s.num_select == 0) {   // no emitter and no environment: nothing to connect to
        l.env = false;
        l.pos = mk(0.f, 0.f, 0.f);
        l.n = mk(0.f, 1.f, 0.f);
        l.contrib = mk(0.f, 0.f, 0.f);
        l.pdfA = 0.f;
        return l;
    }
    const int li = cdf_lower_bound(s.light_cdf, s.num_select, u0);
    const float pl = li < s.num_lights ? __ldg(&s.lights[li].select_pdf) : s.env_select_pdf;
    float r0 = cdf_remap(s.light_cdf, li, pl, u0);
    if (li >= s.num_lights) {
        // environment: pixel by the row / column tables, uniform within the pixel
        const int row = cdf_lower_bound(s.env_row_cdf, s.env_h, r0);
        const float rp = __ldg(s.env_row_pdf + row);
        const float r1 = cdf_remap(s.env_row_cdf, row, rp, r0);
        const float *ccdf = s.env_col_cdf + size_t(row) * s.env_w;
        const int col = cdf_lower_bound(ccdf, s.env_w, r1);
        const float cp = __ldg(s.env_col_pdf + size_t(row) * s.env_w + col);
        const float r2 = cdf_remap(ccdf, col, cp, r1);
        const float uu = (float(col) + r2) / float(s.env_w), vv = (float(row) + u1) / float(s.env_h);
        float st, ct, sp, cp2;
        sincosf(uu * 2.f * kPi, &st, &ct);
        sincosf(vv * kPi, &sp, &cp2);
        const f3 d = mk(ct * sp, cp2, st * sp);
        const float sine = sqrtf(fminf(fmaxf(1.f - d.y * d.y, 0.f), 1.f));
        const float pix = __ldg(s.env_pixel_pdf + size_t(row) * s.env_w + col);
        const float pdfDir = sine <= 1e-12f ? 0.f : pix * float(s.env_w * s.env_h) / sine * (kInvPi * kInvPi * 0.5f);
        l.env = true;
        l.pos = d;
        l.n = mk(0.f, 1.f, 0.f);
        l.contrib = pdfDir > 0.f ? env_eval(s, d) * (1.f / (pdfDir * pl)) : mk(0.f, 0.f, 0.f);
        l.pdfA = pl * pdfDir;
        return l;
    }
    const DevLight &L = s.lights[li];
    const float *tcdf = s.light_tri_cdf + L.tri_offset;
    const int ti = cdf_lower_bound(tcdf, int(L.tri_count), r0);
    const float tp = __ldg(tcdf + ti) - (ti == 0 ? 0.f : __ldg(tcdf + ti - 1));
    const float r1 = cdf_remap(tcdf, ti, tp, r0);
    const float4 *lt = s.light_tris + 3 * size_t(L.tri_offset + ti);
    const f3 p0 = xyz(__ldg(lt)), p1 = xyz(__ldg(lt + 1)), p2 = xyz(__ldg(lt + 2));
    const float sq = sqrtf(r1);
    const float b1 = sq * (1.f - u1), b2 = u1 * sq;   // BarycentricFromSquare (mapping.h:21-27)
    l.env = false;
    l.pos = p0 * (1.f - b1 - b2) + p1 * b1 + p2 * b2;
    l.n = normalize(cross(p1 - p0, p2 - p0));
    l.contrib = mk(L.intensity[0], L.intensity[1], L.intensity[2]) * (kPi / (L.inv_area * pl));
    l.pdfA = pl * L.inv_area;
    return l;
}

// ----------------------------------------------------------------- kernels ----
struct PathState {
    float4 *o, *d, *thr;
    uint32_t *meta;     // depth (bits 0-7) | job (bits 8-31)
    uint32_t *rec;      // newest training record of the path (only while records are collected)
};

struct ShadowQueue {
    float4 *o, *d, *c;
};

struct WaveArgs {
    PathState cur, nxt;
    float4 *hit;
    ShadowQueue sq;
    double *film;          // base film (total_pix*3) followed by the splat film (total_pix*3)
    uint32_t *ctr;         // device counters (Counter)
    unsigned long long *sample_next;
    unsigned long long total_samples;
    uint32_t capacity;
    uint32_t shadow_capacity;
    const DevJob *jobs;    // job table in device memory, or nullptr: the single job `job0`
    DevJob job0;
    int num_jobs;
    uint32_t total_pix;
    uint32_t iter_limit;   // bookkeeping stops the loop after this many iterations
    cudaGraphConditionalHandle cond;   // while-loop condition of the captured graph (0: none)
    int has_cond;
    unsigned long long *prof;   // profiling totals (nullptr when off): items[6], extend nv/nt, shadow nv/nt
    // learned guiding (nullptr when off)
    const uint4 *lobes;    // packed lobes of the current wavefront (chunk c of slot i at c * capacity + i)
    float4 *records;       // training records (kRecordFloat4 float4 each), nullptr: not collected
    uint32_t *rec_count;
    uint32_t rec_capacity;
    int fetch_min;         // traversal: refill idle lanes when fewer lanes than this still traverse
};

__device__ __forceinline__ const DevJob &job_at(const WaveArgs &w, uint32_t j) { return w.jobs ? w.jobs[j] : w.job0; }

// job owning global sample `id`: last job whose sample_begin <= id
__device__ __forceinline__ uint32_t job_of_sample(const WaveArgs &w, unsigned long long id) {
    if (!w.jobs) return 0;
    int lo = 0, hi = w.num_jobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(&w.jobs[mid].sample_begin) <= id) lo = mid; else hi = mid - 1;
    }
    return uint32_t(lo);
}

__device__ __forceinline__ uint32_t job_of_pixel(const DevJob *jobs, int n, uint32_t pix) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(&jobs[mid].pix_offset) <= pix) lo = mid; else hi = mid - 1;
    }
    return uint32_t(lo);
}

__device__ __forceinline__ uint32_t job_seed(const DevJob &J, uint32_t job) { return J.seed + job * 0x9E3779B9u; }

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

// warp-aggregated append: one atomic per warp, lane offsets from ballot/popc
__device__ __forceinline__ uint32_t warp_append(uint32_t *counter, bool pred, uint32_t &total_out) {
    const uint32_t mask = __ballot_sync(0xffffffffu, pred);
    const uint32_t n = __popc(mask);
    uint32_t base = 0;
    const uint32_t leader = mask ? (__ffs(mask) - 1) : 0;
    if (n && lane_id() == leader) base = atomicAdd(counter, n);
    base = __shfl_sync(0xffffffffu, base, leader);
    total_out = n;
    return base + __popc(mask & ((1u << lane_id()) - 1u));
}

__device__ __forceinline__ void push_shadow(const WaveArgs &w, bool pred, f3 o, f3 d, float tmax, uint32_t slot, f3 c,
                                            uint32_t rec = wrg::kNoRecord) {
    uint32_t n;
    const uint32_t idx = warp_append(w.ctr + CTR_SHADOW, pred, n);
    if (pred && idx < w.shadow_capacity) {
        // streaming stores (evict-first in L2): the queues pass through L2 once per bounce and
        // should not push the BVH out of it
        __stcs(&w.sq.o[idx], make_float4(o.x, o.y, o.z, tmax));
        __stcs(&w.sq.d[idx], make_float4(d.x, d.y, d.z, __uint_as_float(slot)));
        __stcs(&w.sq.c[idx], make_float4(c.x, c.y, c.z, __uint_as_float(rec)));
    }
}

__device__ __forceinline__ void film_add(const WaveArgs &w, uint32_t slot, f3 c) {
    double *f = w.film + ((slot & SPLAT_BIT) ? 3 * size_t(w.total_pix) : size_t(0)) + 3 * size_t(slot & ~SPLAT_BIT);
    atomicAdd(f + 0, double(c.x));
    atomicAdd(f + 1, double(c.y));
    atomicAdd(f + 2, double(c.z));
}

// Persistent traversal of a ray queue with dynamic ray fetching: every lane keeps one ray
// in flight; a warp whose traversing lanes drop below w.fetch_min leaves the traversal
// loop and its idle lanes take the next rays of the queue (one atomic per warp), so that
// SIMD lanes are not left idle while a few long rays finish (Aila & Laine, HPG 2009). Once
// the queue is exhausted the remaining rays run to completion.
//   SHADOW = false: extend -- closest hit of every live path into the hit records
//   SHADOW = true:  shadow -- any hit of every queued shadow ray; unoccluded contributions
//                   are added to the FP64 film (and to the path's training records)

//   count_ctr: the counter holding the queue length (CTR_ACTIVE; CTR_SHADOW, or
//              CTR_SHADOW_PENDING for the previous iteration's queue)

template <int BLOCK, bool SHADOW, bool PHONG, bool WIDE>
__device__ __forceinline__ void trace_queue(const DevScene &s, const WaveArgs &w, uint32_t *stack, int count_ctr) {
    const uint32_t n = SHADOW ? min(w.ctr[count_ctr], w.shadow_capacity) : w.ctr[count_ctr];
    uint32_t *fetch = w.ctr + (SHADOW ? CTR_SHADOW_FETCH : CTR_EXTEND_FETCH);
    TraceStack st;
    st.smem = stack + threadIdx.x;
    st.stride = BLOCK;
    st.sp = 0;
    RayPre r{};
    PatchRay pr{};   // read only by the PHONG instantiation
    float t = 0.f, bu = 0.f, bv = 0.f;
    uint32_t tri = MISS, ray = 0, nv = 0, nt = 0;
    int node = kTraceDone, leaf = 0;
    WideState ws{-1, 0u, 0u, 0u};   // WIDE: compressed 8-wide traversal state
    uint32_t oct = 0;
    bool busy = false, exhausted = false;
    const uint32_t lane = lane_id();
    while (true) {
        const uint32_t need = __ballot_sync(0xffffffffu, !busy && !exhausted);
        if (need) {
            const uint32_t leader = __ffs(need) - 1u;
            uint32_t base = 0;
            if (lane == leader) base = atomicAdd(fetch, uint32_t(__popc(need)));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (!busy && !exhausted) {
                ray = base + uint32_t(__popc(need & ((1u << lane) - 1u)));
                if (ray < n) {
                    float4 o, d;
                    float tmax;
                    if (SHADOW) { o = __ldcs(&w.sq.o[ray]); d = __ldcs(&w.sq.d[ray]); tmax = o.w; }
                    else { o = w.cur.o[ray]; d = w.cur.d[ray]; tmax = __int_as_float(0x7f800000); }
                    r = ray_setup(xyz(o), xyz(d));
                    if (PHONG) pr = PatchRay{o.x, o.y, o.z, d.x, d.y, d.z};
                    if (WIDE) {
                        ws = WideState{0, 0u, 0u, 0u};
                        oct = ray_octant(xyz(d));
                    }
                    t = tmax; tri = MISS; bu = 0.f; bv = 0.f;
                    node = 0; leaf = 0; st.sp = 0;
                    busy = true;
                } else {
                    exhausted = true;   // the queue counter only grows: no lane gets another ray
                }
            }
        }
        if (!__any_sync(0xffffffffu, busy)) break;
        const int min_active = __any_sync(0xffffffffu, exhausted) ? 0 : w.fetch_min;
        bool finished = false;
        if (busy) {
            if (WIDE)
                finished = traverse_steps_w8<SHADOW, PHONG>(s.wnodes, s.tris, r, oct, kRayEps, t, tri, bu, bv, ws, st,
                                                             nv, nt, min_active, s.patches, pr);
            else
                finished = traverse_steps<SHADOW, PHONG>(s.nodes, s.tris, r, kRayEps, t, tri, bu, bv, node, leaf, st,
                                                          nv, nt, min_active, s.patches, pr);
        }
        if (finished) {
            busy = false;
            if (SHADOW) {
                if (tri == MISS) {   // unoccluded
                    const float4 c = __ldcs(&w.sq.c[ray]);
                    film_add(w, __float_as_uint(__ldcs(&w.sq.d[ray]).w), mk(c.x, c.y, c.z));
                    if (w.records) record_contribution(w.records, __float_as_uint(c.w), mk(c.x, c.y, c.z));
                }
            } else {
                w.hit[ray] = make_float4(t, bu, bv, __uint_as_float(tri));
            }
        }
    }
    if (w.prof) {   // the whole warp leaves the loop together: one atomic per warp and counter
        const uint32_t wnv = __reduce_add_sync(0xffffffffu, nv), wnt = __reduce_add_sync(0xffffffffu, nt);
        if (lane == 0) {
            atomicAdd(w.prof + (SHADOW ? 8 : 6), (unsigned long long)wnv);
            atomicAdd(w.prof + (SHADOW ? 9 : 7), (unsigned long long)wnt);
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(w.prof + (SHADOW ? 3 : 0), (unsigned long long)n);
    }
}

template <int BLOCK, bool PHONG, bool WIDE>
__global__ void __launch_bounds__(BLOCK) k_extend(DevScene s, WaveArgs w) {
    __shared__ uint32_t stack[kSmemStack * BLOCK];
    trace_queue<BLOCK, false, PHONG, WIDE>(s, w, stack, CTR_ACTIVE);
}

// lens point of a sample's camera vertex (ThinlensCamera::sampleWe0ByPdf, thinlens.h:121-136; the
// pinhole origin when the aperture is zero) from the sample's dimension group 1
__device__ __forceinline__ f3 lens_point(const DevCamera &cam, uint32_t lpix, uint32_t sample, uint32_t seed) {
    const f3 cfx = ld3(cam.fx), cfy = ld3(cam.fy), corg = ld3(cam.origin);
    if (!(cam.aperture > 0.f)) return corg;
    const Rand4 r1 = rand4(lpix, sample, 1, seed);
    const float ax = 2.f * r1.a - 1.f, ay = 2.f * r1.b - 1.f;
    float rr = 0.f, phi = 0.f;
    if (ax != 0.f || ay != 0.f) {
        if (ax * ax > ay * ay) { rr = ax; phi = (kPi / 4.f) * (ay / ax); }
        else { rr = ay; phi = (kPi / 2.f) - (kPi / 4.f) * (ax / ay); }
    }
    float sn, cs;
    sincosf(phi, &sn, &cs);
    return corg + cfx * (rr * cs * cam.aperture) + cfy * (rr * sn * cam.aperture);
}

// Connection of a vertex to the lens point c0: direction and distance camera -> vertex, the
// geometry term (cosine at the vertex only when it is not an environment vertex), the camera
// importance evalWe1 with its raster position (thinlens.h:63-80) and the camera's area pdf of
// the vertex (for MIS). Returns false when the vertex is behind the camera or off the film.
struct CamLink {
    f3 w;            // unit direction camera -> vertex
    float len;       // distance (0 for an environment vertex)
    float G;         // geometry term
    float we;        // camera importance We1
    float camPdfA;   // per-pixel camera pdf of the vertex in area measure
    uint32_t slot;   // splat film slot (SPLAT_BIT set)
};

__device__ __forceinline__ bool camera_link(const DevJob &J, f3 c0, f3 p, f3 n, bool env, CamLink &k) {
    const DevCamera &cam = J.cam;
    const f3 cfx = ld3(cam.fx), cfy = ld3(cam.fy), cfz = ld3(cam.fz), corg = ld3(cam.origin);
    float conv;
    if (env) {
        k.w = p;
        k.len = 0.f;
        k.G = fabsf(dot(cfz, k.w));
        conv = 1.f;
    } else {
        const f3 uv = p - c0;
        const float d2 = len2(uv);
        k.len = sqrtf(d2);
        k.w = uv / k.len;
        conv = fabsf(dot(n, k.w)) / d2;
        k.G = fabsf(dot(cfz, k.w)) * conv;
    }
    const float cosT = dot(k.w, cfz);
    if (!(k.G > 0.f) || !(cosT > 0.f)) return false;
    const f3 cp = c0 - corg;
    const f3 pl = mk(dot(cp, cfx), dot(cp, cfy), dot(cp, cfz));
    const f3 dl = mk(dot(k.w, cfx), dot(k.w, cfy), cosT);
    const f3 fpp = dl * (cam.focal / cosT) + pl;
    const float fxp = -fpp.x / cam.focal * cam.dist, fyp = -fpp.y / cam.focal * cam.dist;
    const float rx = (fxp / float(cam.width) + 0.5f) * float(cam.width);
    const float ry = (fyp / float(cam.height) + 0.5f) * float(cam.height);
    if (!(rx >= 0.f && rx < float(cam.width) && ry >= 0.f && ry < float(cam.height))) return false;
    const float c2 = cosT * cosT;
    k.we = cam.per_film / (c2 * c2);
    k.camPdfA = cam.per_pixel / (c2 * cosT) * conv;
    const uint32_t sx = min(uint32_t(rx), uint32_t(cam.width - 1));
    const uint32_t sy = min(uint32_t(ry), uint32_t(cam.height - 1));
    k.slot = (J.pix_offset + sy * uint32_t(cam.width) + sx) | SPLAT_BIT;
    return true;
}

// a ray that leaves the scene's bounding sphere upward (a slot with no path to trace)
__device__ __forceinline__ void dead_ray(const DevScene &s, f3 &o, f3 &d) {
    o = mk(s.scene_center[0], s.scene_center[1] + 2.f * s.scene_radius + 1.f, s.scene_center[2]);
    d = mk(0.f, 1.f, 0.f);
}

// One path of the current wavefront: emitter hit (strategy B) or NEE at a surface
// (strategy A, one shadow ray), then BSDF sampling -- or, with lobes `gl` of the learned
// proposal, one-sample MIS between the guide and the BSDF -- and compaction of the
// continued path into the next wavefront. Called by all 32 lanes of a warp together
// (warp-aggregated appends); `valid` is false for lanes past the end of the wavefront.
template <bool NEE_ONLY, bool RECORD>
__device__ __forceinline__ void shade_path(const DevScene &s, const WaveArgs &w, uint32_t i, bool valid,
                                           const wrg::PackedLobes *gl) {
    float4 *const records = RECORD ? w.records : nullptr;   // training records (guided training passes)
    bool alive = false, shadow = false;
    f3 so = mk(0, 0, 0), sd = mk(0, 0, 1), sc = mk(0, 0, 0);
    float stmax = 0.f;
    f3 no = mk(0, 0, 0), nd = mk(0, 0, 1), nthr = mk(0, 0, 0);
    float npdf = 0.f;
    uint32_t pixel = 0, sample = 0, meta = 0;
    uint32_t shadow_slot = MISS;        // film slot of the shadow record when it is not the path's pixel
    uint32_t rec = wrg::kNoRecord;      // newest training record of this path
    uint32_t nrec = wrg::kNoRecord;     // record of the continued path
    bool want_rec = false;              // a record is created for this vertex
    f3 rec_pos = mk(0, 0, 0), rec_n = mk(0, 1, 0), rec_wo = mk(0, 1, 0), rec_thr = mk(0, 0, 0);
    if (valid) {
        // last reads of this bounce's path state (streaming: evict-first in L2)
        const float4 o4 = __ldcs(&w.cur.o[i]), d4 = __ldcs(&w.cur.d[i]), t4 = __ldcs(&w.cur.thr[i]);
        meta = __ldcs(&w.cur.meta[i]);
        if (records) rec = __ldcs(&w.cur.rec[i]);
        const uint32_t depth = meta & 0xffu, job = meta >> 8;
        const DevJob &J = job_at(w, job);
        const float4 h = __ldcs(&w.hit[i]);
        const f3 o = xyz(o4), d = xyz(d4), thr = xyz(t4);
        const float prevPdfW = o4.w;
        pixel = __float_as_uint(d4.w);   // global film pixel
        sample = __float_as_uint(t4.w);
        const uint32_t tri = __float_as_uint(h.w);
        const float t = h.x;
        const bool primitive = !NEE_ONLY && J.integrator == INTEGRATOR_PRIMITIVE;
        if (!NEE_ONLY && J.integrator == INTEGRATOR_LIGHT) {
            // light_splatting: a vertex of the light subpath (randomWalk callback,
            // lightsplatting.h:85-104); emitter hits and misses end the subpath
            if (tri != MISS && !(__ldg(s.tri_mat + tri) & LIGHT_BIT)) {
                const float4 a = __ldg(s.tris + 3 * tri), b = __ldg(s.tris + 3 * tri + 1), cc = __ldg(s.tris + 3 * tri + 2);
                const f3 ng = surface_normal(a, b, cc, h.y, h.z);
                const f3 pos = o + d * t;
                const DevMaterial mm = s.materials[__ldg(s.tri_mat + tri)];
                const Frame fr(ng);
                const f3 inL = fr.to_local(-d);
                const uint32_t lpix = pixel - J.pix_offset, seed = job_seed(J, job);
                // connection to the sample's lens point: We1 * G * transmittance * bsdf(previous -> here
                // -> camera) * path contribution, splatted with weight 1 / (spp * W * H) by the resolve
                const f3 c0 = lens_point(J.cam, lpix, sample, seed);
                CamLink cl;
                if (camera_link(J, c0, pos, ng, false, cl)) {
                    const f3 f = bsdf_eval(mm, inL, fr.to_local(-cl.w));
                    const f3 c = thr * f * (cl.we * cl.G);
                    if (!is_zero(c) && isfinite(c.x + c.y + c.z)) {
                        shadow = true;
                        so = pos; sd = -cl.w; sc = c;
                        stmax = cl.len - kRayEps;
                        shadow_slot = cl.slot;   // splat film (the path keeps its own pixel key)
                    }
                }
                // the subpath has num_path_vertices - 2 walk vertices; this is walk vertex depth + 1
                if (int(depth) + 3 < J.nverts) {
                    const Rand4 rb = rand4(lpix, sample, 2 + depth, seed);
                    f3 outL;
                    float pdfW;
                    const f3 wgt = bsdf_sample(mm, inL, rb.a, rb.b, outL, pdfW);
                    if (!is_zero(wgt) && isfinite(wgt.x + wgt.y + wgt.z)) {
                        alive = true;
                        no = pos;
                        nd = normalize(fr.to_world(outL));
                        nthr = thr * wgt;
                        npdf = pdfW;
                    }
                }
            }
        } else if (tri == MISS) {
            if (s.has_env) {
                // strategy B on the environment (pathnextevent.h:128-146); the primitive tracer
                // takes the emission with weight one (primitivepath.h:49-53)
                const float cPdfA = prevPdfW;   // ConvertToArea to an environment vertex: 1/|d|^2
                const float lPdfA = primitive ? 0.f : s.env_select_pdf * env_pdf(s, d);
                const float mis = primitive ? 1.f : cPdfA / (lPdfA + cPdfA);
                const f3 c = thr * env_eval(s, d) * mis;
                if (!is_zero(c) && isfinite(c.x + c.y + c.z)) {
                    film_add(w, pixel, c);
                    if (records) record_contribution(records, rec, c);
                }
            }
        } else {
            const float4 a = __ldg(s.tris + 3 * tri), b = __ldg(s.tris + 3 * tri + 1), cc = __ldg(s.tris + 3 * tri + 2);
            const f3 ng = surface_normal(a, b, cc, h.y, h.z);
            const f3 pos = o + d * t;
            const uint32_t mat = __ldg(s.tri_mat + tri);
            if (mat & LIGHT_BIT) {
                // strategy B: BSDF-sampled hit on an emitter
                const uint32_t li = mat & ~LIGHT_BIT;
                const float cosl = dot(ng, d);
                if (cosl <= 0.f) {   // front face: evalLe1 (diffusearealight.h:48-53)
                    const float cPdfA = prevPdfW * fabsf(cosl) / (t * t);
                    const float lPdfA = __ldg(&s.lights[li].select_pdf) * __ldg(&s.lights[li].inv_area);
                    const float mis = primitive ? 1.f : cPdfA / (lPdfA + cPdfA);
                    const f3 c = thr * mk(__ldg(&s.lights[li].intensity[0]), __ldg(&s.lights[li].intensity[1]),
                                          __ldg(&s.lights[li].intensity[2])) * mis;
                    if (!is_zero(c) && isfinite(c.x + c.y + c.z)) {
                        film_add(w, pixel, c);
                        if (records) record_contribution(records, rec, c);
                    }
                }
            } else if (int(depth) + 2 < J.nverts) {
                const DevMaterial mm = s.materials[mat];
                const Frame fr(ng);
                const f3 wi = -d;
                const f3 inL = fr.to_local(wi);
                const uint32_t lpix = pixel - J.pix_offset, seed = job_seed(J, job);
                // learned proposal at this vertex (one-sample MIS with BSDF sampling)
                const bool guided = gl && !primitive && guide_weight_sum(*gl) > 0.f;
                GuideVertex gv;
                if (guided) guide_prepare(*gl, gv);
                // strategy A: next-event estimation toward this sample's light vertex
                const Rand4 r0 = rand4(lpix, sample, 0, seed);
                LightVtx l{};
                if (primitive) l.pdfA = 0.f;   // no connection to the light (primitivepath.h)
                else l = sample_light(s, r0.a, r0.b);
                f3 wo;
                float G, convA, dist = 0.f;
                if (l.env) {
                    wo = l.pos;
                    G = fabsf(dot(ng, wo));
                    convA = 1.f;
                } else {
                    const f3 uv = l.pos - pos;
                    const float d2 = len2(uv);
                    dist = sqrtf(d2);
                    wo = uv / dist;
                    const float cl = fabsf(dot(l.n, wo));
                    convA = cl / d2;
                    G = fabsf(dot(ng, wo)) * convA;
                }
                const bool front = l.env || dot(l.n, wo) <= 0.f;   // light emits toward -wo
                if (G > 0.f && front && l.pdfA > 0.f) {
                    const f3 outL = fr.to_local(wo);
                    const f3 f = bsdf_eval(mm, inL, outL);
                    if (!is_zero(f)) {
                        float pdfW = bsdf_pdf(mm, inL, outL);
                        if (guided) pdfW = kGuideAlpha * guide_pdf(gv, wo) + (1.f - kGuideAlpha) * pdfW;
                        const float bsdfPdfA = pdfW * convA;
                        const float mis = l.pdfA / (l.pdfA + bsdfPdfA);
                        const float le1 = l.env ? 1.f : kInvPi;
                        const f3 c = thr * f * (le1 * G * mis) * l.contrib;
                        if (!is_zero(c) && isfinite(c.x + c.y + c.z)) {
                            shadow = true;
                            so = pos; sd = wo; sc = c;
                            stmax = l.env ? __int_as_float(0x7f800000) : dist - kRayEps;
                        }
                    }
                }
                // BSDF sampling (or, when guided, the guide/BSDF mixture) continues the path
                const Rand4 rb = rand4(lpix, sample, 2 + depth, seed);
                f3 outL;
                float pdfW;
                f3 wgt;
                if (!guided) {
                    wgt = bsdf_sample(mm, inL, rb.a, rb.b, outL, pdfW);
                } else {
                    // one-sample MIS: the direction from the guide (probability kGuideAlpha) or from the
                    // BSDF, weighted by f cos / (alpha q + (1 - alpha) p_bsdf); both techniques share
                    // the density evaluation (no divergent second evaluation)
                    f3 dw;
                    if (rb.c < kGuideAlpha) {
                        dw = guide_sample(gv, rb.c * (1.f / kGuideAlpha), rb.a, rb.b);
                        outL = fr.to_local(dw);
                    } else {
                        float pb_unused;
                        bsdf_sample(mm, inL, rb.a, rb.b, outL, pb_unused);
                        dw = normalize(fr.to_world(outL));
                    }
                    pdfW = kGuideAlpha * guide_pdf(gv, dw) + (1.f - kGuideAlpha) * bsdf_pdf(mm, inL, outL);
                    const f3 f = bsdf_eval(mm, inL, outL);
                    wgt = (pdfW > 0.f && !is_zero(f)) ? f * (fabsf(outL.y) / pdfW) : mk(0.f, 0.f, 0.f);
                }
                if (!is_zero(wgt) && isfinite(wgt.x + wgt.y + wgt.z)) {
                    alive = true;
                    no = pos;
                    nd = normalize(fr.to_world(outL));
                    nthr = thr * wgt;
                    npdf = pdfW;
                    if (records) {
                        want_rec = true;
                        rec_pos = pos;
                        rec_wo = wi;
                        rec_n = wrg::guide_normal(ng, wi);
                        rec_thr = thr;
                    }
                }
            }
        }
    }
    push_shadow(w, shadow, so, sd, stmax, shadow_slot == MISS ? pixel : shadow_slot, sc, rec);
    if (records) {   // training record of this vertex (parent: the path's previous record)
        uint32_t nr;
        const uint32_t r = warp_append(w.rec_count, want_rec, nr);
        nrec = rec;
        if (want_rec && r < w.rec_capacity) {
            float4 *R = records + wrg::kRecordFloat4 * size_t(r);
            R[0] = make_float4(rec_pos.x, rec_pos.y, rec_pos.z, 0.f);
            R[1] = make_float4(rec_n.x, rec_n.y, rec_n.z, __uint_as_float(rec));
            R[2] = make_float4(rec_wo.x, rec_wo.y, rec_wo.z, 0.f);
            R[3] = make_float4(nd.x, nd.y, nd.z, 0.f);
            R[4] = make_float4(rec_thr.x, rec_thr.y, rec_thr.z, 0.f);
            nrec = r;
        }
    }
    uint32_t cnt;
    const uint32_t j = warp_append(w.ctr + CTR_NEXT, alive, cnt);
    if (alive) {
        __stcs(&w.nxt.o[j], make_float4(no.x, no.y, no.z, npdf));
        __stcs(&w.nxt.d[j], make_float4(nd.x, nd.y, nd.z, __uint_as_float(pixel)));
        __stcs(&w.nxt.thr[j], make_float4(nthr.x, nthr.y, nthr.z, __uint_as_float(sample)));
        __stcs(&w.nxt.meta[j], meta + 1u);
        if (records) __stcs(&w.nxt.rec[j], nrec);
    }
}

// GUIDED: the learned proposal is on (w.lobes); a separate instantiation keeps the plain
// shade kernel's register count unchanged. NEE_ONLY: every job of the launch is
// nextevent_path_tracer, so the primitive-tracer and light-splatting branches are compiled out
// (fewer spills: 657.9 against 650.8 Mpaths/s on the 1M-triangle render; guided renders are
// always NEE). RECORD: the launch collects training records (guided training passes only); the
// other launches, the final guided pass among them, run without that code. Both run 3 blocks per SM: the guided kernel is
// latency-bound, and at 80 registers (with spills) it measured faster than at 128 registers and
// 2 blocks per SM (80.2 against 93.6 ms of shading in a 64-spp render of the door-gap room); 4
// blocks (64 registers) gained nothing on it and cost 0.7 % on the plain 1M-triangle render.
template <bool GUIDED, bool NEE_ONLY, bool RECORD>
__global__ void __launch_bounds__(kShadeBlock, 3) k_shade(DevScene s, WaveArgs w) {
    const uint32_t n = w.ctr[CTR_ACTIVE];
    if (w.prof && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(w.prof + 1, (unsigned long long)n);
    const uint32_t warp_global = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t base = warp_global * 32u; base < n; base += nwarps * 32u) {
        const uint32_t i = base + lane_id();
        if (GUIDED) {   // learned proposal: this path's packed lobes, loaded once
            wrg::PackedLobes pl;
            if (i < n) {
#pragma unroll
                for (int c = 0; c < wrg::kPackedChunks; ++c) pl.c[c] = w.lobes[c * size_t(w.capacity) + i];
            } else {
#pragma unroll
                for (int c = 0; c < wrg::kPackedChunks; ++c) pl.c[c] = make_uint4(0u, 0u, 0u, 0u);
            }
            shade_path<NEE_ONLY, RECORD>(s, w, i, i < n, &pl);
        } else {
            shade_path<NEE_ONLY, RECORD>(s, w, i, i < n, nullptr);
        }
    }
}


__device__ __forceinline__ uint32_t new_samples(const WaveArgs &w, uint32_t filled, unsigned long long issued) {
    const unsigned long long remaining = w.total_samples > issued ? w.total_samples - issued : 0ull;
    const uint32_t room = w.capacity > filled ? w.capacity - filled : 0u;
    return uint32_t(remaining < room ? remaining : room);
}

// new camera samples into the free tail of the next wavefront
// new camera samples into the free tail of the next wavefront; for light_splatting the sample's
// light subpath starts there instead
// The pixel of the q-th sample of a sample layer. Consecutive samples cover 8 x 4 pixel tiles (one
// warp's 32 new paths start from a compact patch of the film, so their rays stay closer in space
// and direction over the first bounces than a 32 x 1 scanline run: 651 vs 641 Mpaths/s on the 1M
// workload); pixels outside the whole tiles follow in scanline order, right strip then bottom strip.
// A bijection of [0, W*H): every pixel still gets every sample index, with its own random streams.
__device__ __forceinline__ uint32_t tile_order_pixel(uint32_t q, uint32_t W, uint32_t H) {
    const uint32_t W8 = W & ~7u, H4 = H & ~3u;
    const uint32_t inner = W8 * H4;
    if (q < inner) {
        const uint32_t tile = q >> 5, r = q & 31u, tiles_x = W8 >> 3;
        return ((tile / tiles_x) * 4u + (r >> 3)) * W + (tile % tiles_x) * 8u + (r & 7u);
    }
    q -= inner;
    const uint32_t rw = W - W8;                  // right strip, rows [0, H4)
    if (q < H4 * rw) return (q / rw) * W + W8 + q % rw;
    q -= H4 * rw;                                // bottom strip, rows [H4, H)
    return (H4 + q / W) * W + q % W;
}

__global__ void __launch_bounds__(kShadeBlock) k_raygen(DevScene s, WaveArgs w) {
    const uint32_t filled = w.ctr[CTR_NEXT];
    const unsigned long long issued = *w.sample_next;
    const uint32_t n_new = new_samples(w, filled, issued);
    if (w.prof && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(w.prof + 2, (unsigned long long)n_new);
    const uint32_t warp_global = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t base = warp_global * 32u; base < n_new; base += nwarps * 32u) {
        const uint32_t k = base + lane_id();
        const bool valid = k < n_new;
        bool shadow = false;
        f3 so = mk(0, 0, 0), sd = mk(0, 0, 1), sc = mk(0, 0, 0);
        float stmax = 0.f;
        uint32_t slot = 0;
        if (valid) {
            const unsigned long long id = issued + k;
            const uint32_t job = job_of_sample(w, id);
            const DevJob &J = job_at(w, job);
            const DevCamera &cam = J.cam;
            const f3 cfx = ld3(cam.fx), cfy = ld3(cam.fy), cfz = ld3(cam.fz), corg = ld3(cam.origin);
            const unsigned long long lid = id - J.sample_begin;
            const uint32_t lpix = tile_order_pixel(uint32_t(lid % J.npix), uint32_t(cam.width), uint32_t(cam.height));
            const uint32_t sample = J.sample_offset + uint32_t(lid / J.npix);
            const uint32_t seed = job_seed(J, job);
            const uint32_t px = lpix % uint32_t(cam.width), py = lpix / uint32_t(cam.width);
            const Rand4 r0 = rand4(lpix, sample, 0, seed);
            LightVtx l{};
            if (J.integrator == INTEGRATOR_PRIMITIVE) l.pdfA = 0.f;   // camera subpath only
            else l = sample_light(s, r0.a, r0.b);
            // camera vertex: lens point (pinhole when the aperture is zero)
            const f3 c0 = lens_point(cam, lpix, sample, seed);
            const uint32_t j = filled + k;
            if (J.integrator == INTEGRATOR_LIGHT) {
                // light_splatting (lightsplatting.h:47-108): the light vertex connected to the lens
                // point with weight one, then the light subpath's first ray
                CamLink cl;
                if (l.pdfA > 0.f && camera_link(J, c0, l.pos, l.n, l.env, cl)) {
                    const float le1 = l.env ? 1.f : (dot(l.n, -cl.w) >= 0.f ? kInvPi : 0.f);
                    const f3 c = l.contrib * (cl.we * cl.G * le1);
                    if (!is_zero(c) && isfinite(c.x + c.y + c.z)) {
                        shadow = true;
                        slot = cl.slot;
                        sc = c;
                        if (l.env) { so = c0; sd = cl.w; stmax = __int_as_float(0x7f800000); }
                        else { so = l.pos; sd = -cl.w; stmax = cl.len - kRayEps; }
                    }
                }
                f3 o, d, thr = mk(0.f, 0.f, 0.f);
                dead_ray(s, o, d);
                if (l.pdfA > 0.f && !l.env && J.nverts > 2) {
                    // sampleLe1CosByPdf (diffusearealight.h:73-81): cosine-weighted about the normal
                    const Frame lf(l.n);
                    o = l.pos;
                    d = normalize(lf.to_world(cosine_hemisphere(r0.c, r0.d)));
                    thr = l.contrib;
                } else if (l.pdfA > 0.f && l.env && J.nverts > 2) {
                    // sampleLe1CosByPdf (envmap.h:83-101): a point on the disk of the scene's bounding
                    // sphere facing the sampled direction
                    const float ax = 2.f * r0.c - 1.f, ay = 2.f * r0.d - 1.f;
                    float rr = 0.f, phi = 0.f;
                    if (ax != 0.f || ay != 0.f) {
                        if (ax * ax > ay * ay) { rr = ax; phi = (kPi / 4.f) * (ay / ax); }
                        else { rr = ay; phi = (kPi / 2.f) - (kPi / 4.f) * (ax / ay); }
                    }
                    float sn, cs;
                    sincosf(phi, &sn, &cs);
                    const float R = s.scene_radius;
                    const Frame df(-l.pos);
                    o = df.to_world(mk(rr * cs * R, -R, rr * sn * R)) +
                        mk(s.scene_center[0], s.scene_center[1], s.scene_center[2]);
                    d = -l.pos;
                    thr = l.contrib * (kPi * R * R);
                }
                __stcs(&w.nxt.o[j], make_float4(o.x, o.y, o.z, 0.f));
                __stcs(&w.nxt.d[j], make_float4(d.x, d.y, d.z, __uint_as_float(J.pix_offset + lpix)));
                __stcs(&w.nxt.thr[j], make_float4(thr.x, thr.y, thr.z, __uint_as_float(sample)));
                __stcs(&w.nxt.meta[j], job << 8);
                if (w.records) __stcs(&w.nxt.rec[j], wrg::kNoRecord);
            } else {
                // strategy C: connect the light vertex to the camera (pathnextevent.h:75-99)
                CamLink cl;
                if (l.pdfA > 0.f && camera_link(J, c0, l.pos, l.n, l.env, cl)) {
                    const bool front = l.env || dot(l.n, cl.w) <= 0.f;   // the light emits toward the camera
                    const float mis = l.pdfA / (l.pdfA + cl.camPdfA);
                    const float le1 = l.env ? 1.f : kInvPi;
                    const f3 c = l.contrib * (mis * cl.we * cl.G * le1);
                    if (front && !is_zero(c) && isfinite(c.x + c.y + c.z)) {
                        shadow = true;
                        slot = cl.slot;
                        sc = c;
                        if (l.env) { so = c0; sd = cl.w; stmax = __int_as_float(0x7f800000); }
                        else { so = l.pos; sd = -cl.w; stmax = cl.len - kRayEps; }
                    }
                }
                // primary ray through the jittered pixel position (thinlens.h:138-165)
                const float nsx = (float(px) + r0.c) / float(cam.width), nsy = (float(py) + r0.d) / float(cam.height);
                const f3 film = mk((nsx - 0.5f) * float(cam.width), (nsy - 0.5f) * float(cam.height), -cam.dist);
                const f3 fpp = film * (cam.focal / film.z);
                const f3 cpl = mk(dot(c0 - corg, cfx), dot(c0 - corg, cfy), dot(c0 - corg, cfz));
                const f3 dir = normalize(fpp - cpl);
                const float ct = dir.z;
                const float pdfW = cam.per_film / (ct * ct * ct) / float(J.npix);
                const f3 dw = normalize(cfx * dir.x + cfy * dir.y + cfz * dir.z);
                __stcs(&w.nxt.o[j], make_float4(c0.x, c0.y, c0.z, pdfW));
                __stcs(&w.nxt.d[j], make_float4(dw.x, dw.y, dw.z, __uint_as_float(J.pix_offset + lpix)));
                __stcs(&w.nxt.thr[j], make_float4(1.f, 1.f, 1.f, __uint_as_float(sample)));
                __stcs(&w.nxt.meta[j], job << 8);
                if (w.records) __stcs(&w.nxt.rec[j], wrg::kNoRecord);
            }
        }
        push_shadow(w, shadow, so, sd, stmax, slot, sc);
    }
}

template <int BLOCK, bool PHONG, bool WIDE>
__global__ void __launch_bounds__(BLOCK) k_shadow(DevScene s, WaveArgs w, int count_ctr) {
    __shared__ uint32_t stack[kSmemStack * BLOCK];
    trace_queue<BLOCK, true, PHONG, WIDE>(s, w, stack, count_ctr);
}

// Extend of this iteration and the shadow rays of the previous one in one persistent launch:
// a warp that finds the extend queue exhausted and its lanes finished moves on to the shadow
// queue, so the shadow rays fill the extend launch's tail instead of waiting for it. The two
// queues are independent: extend reads this wavefront's rays and writes hit records; the
// shadow rays were queued by the previous shade / raygen and only add to the film (the next
// shade appends to the shadow queue only after this launch).
template <int BLOCK, bool PHONG, bool WIDE>
__device__ __forceinline__ void trace_pair(const DevScene &s, const WaveArgs &w) {
    __shared__ uint32_t stack[kSmemStack * BLOCK];
    trace_queue<BLOCK, false, PHONG, WIDE>(s, w, stack, CTR_ACTIVE);
    trace_queue<BLOCK, true, PHONG, WIDE>(s, w, stack, CTR_SHADOW_PENDING);
}

template <int BLOCK, bool WIDE>
__global__ void __launch_bounds__(BLOCK) k_trace_pair(DevScene s, WaveArgs w) {
    trace_pair<BLOCK, false, WIDE>(s, w);
}

// With Phong patches both FP64 patch tests in one kernel would take 190 registers (2 blocks of
// 128 per SM); the bound keeps the 384 resident threads per SM of the separate kernels.
template <int BLOCK, bool WIDE>
__global__ void __launch_bounds__(BLOCK, (384 / BLOCK > 0 ? 384 / BLOCK : 1)) k_trace_pair_phong(DevScene s, WaveArgs w) {
    trace_pair<BLOCK, true, WIDE>(s, w);
}

// queue bookkeeping between iterations (one thread); also drives the graph's while loop
__global__ void k_advance(WaveArgs w) {
    const uint32_t filled = w.ctr[CTR_NEXT];
    const unsigned long long issued = *w.sample_next;
    const uint32_t n_new = new_samples(w, filled, issued);
    if (w.ctr[CTR_SHADOW] > w.ctr[CTR_SHADOW_MAX]) w.ctr[CTR_SHADOW_MAX] = w.ctr[CTR_SHADOW];
    if (w.ctr[CTR_SHADOW] > w.shadow_capacity) w.ctr[CTR_OVERFLOW] = 1;
    w.ctr[CTR_SHADOW_PENDING] = w.ctr[CTR_SHADOW];   // for a fused launch that traces them next
    w.ctr[CTR_ACTIVE] = filled + n_new;
    w.ctr[CTR_NEXT] = 0;
    w.ctr[CTR_SHADOW] = 0;
    w.ctr[CTR_EXTEND_FETCH] = 0;
    w.ctr[CTR_SHADOW_FETCH] = 0;
    const uint32_t iter = w.ctr[CTR_ITER] + 1;
    w.ctr[CTR_ITER] = iter;
    *w.sample_next = issued + n_new;
    bool done = filled + n_new == 0u;
    if (!done && iter >= w.iter_limit) {   // never loop unbounded: stop and report
        w.ctr[CTR_TIMEOUT] = 1;
        done = true;
    }
    w.ctr[CTR_DONE] = done ? 1u : 0u;
    if (w.has_cond) cudaGraphSetConditional(w.cond, done ? 0u : 1u);
}

// final image = base / spp + splat / (spp * W * H) per job (film.h:70-90)
__global__ void k_resolve(const double *film, double *out, uint32_t total_pix, const DevJob *jobs, int njobs,
                          DevJob job0) {
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < 3 * size_t(total_pix);
         i += size_t(gridDim.x) * blockDim.x) {
        const uint32_t pix = uint32_t(i / 3);
        const DevJob &J = jobs ? jobs[job_of_pixel(jobs, njobs, pix)] : job0;
        const double spp = double(J.spp_norm > 0 ? J.spp_norm : J.spp);
        const double bs = 1.0 / spp, as = 1.0 / spp / double(J.npix);
        double c = 0.0;
        c += film[i] * bs;
        c += film[3 * size_t(total_pix) + i] * as;
        out[i] = c;
    }
}

// ----------------------------------------------------------- ray batches ----
// rays: n x 8 floats (ox, oy, oz, tnear, dx, dy, dz, tfar)
// out: 3 float4 per ray -- (geomID, primID, t, leaf index), (u, v, 0, 0) with the triangle's
// barycentrics (zero on a patch, whose texture coordinate the reference leaves at zero), and
// (unit geometry normal, 0)
template <bool PHONG, bool WIDE>
__global__ void __launch_bounds__(kTraceBlock) k_trace_batch(DevScene s, const float4 *rays, uint32_t n, int any_hit,
                                                           float4 *out, uint32_t *visits) {
    __shared__ uint32_t stack[kSmemStack * kTraceBlock];
    uint32_t nv = 0, nt = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 a = rays[2 * i], b = rays[2 * i + 1];
        float t, bu = 0.f, bv = 0.f;
        uint32_t tri;
        bool hit;
        if (WIDE && any_hit)
            hit = traverse_w8<true, PHONG>(s.wnodes, s.tris, xyz(a), xyz(b), a.w, b.w, stack, t, tri, bu, bv, &nv,
                                           &nt, s.patches);
        else if (WIDE)
            hit = traverse_w8<false, PHONG>(s.wnodes, s.tris, xyz(a), xyz(b), a.w, b.w, stack, t, tri, bu, bv, &nv,
                                            &nt, s.patches);
        else if (any_hit)
            hit = traverse<true, PHONG>(s.nodes, s.tris, xyz(a), xyz(b), a.w, b.w, stack, t, tri, bu, bv, &nv, &nt,
                                        s.patches);
        else
            hit = traverse<false, PHONG>(s.nodes, s.tris, xyz(a), xyz(b), a.w, b.w, stack, t, tri, bu, bv, &nv, &nt,
                                         s.patches);
        uint32_t gid = MISS, pid = MISS;
        f3 ng = mk(0.f, 0.f, 0.f);
        if (hit) {
            const float4 ta = __ldg(s.tris + 3 * tri), tb = __ldg(s.tris + 3 * tri + 1), tc = __ldg(s.tris + 3 * tri + 2);
            gid = __float_as_uint(tb.w);
            pid = __float_as_uint(tc.w);
            ng = surface_normal(ta, tb, tc, bu, bv);
            if (__float_as_uint(ta.w) & wrp::kPatchFlag) { bu = 0.f; bv = 0.f; }
        }
        out[3 * i] = make_float4(__uint_as_float(gid), __uint_as_float(pid), hit ? t : __int_as_float(0x7f800000),
                                 __uint_as_float(tri));
        out[3 * i + 1] = make_float4(bu, bv, 0.f, 0.f);
        out[3 * i + 2] = make_float4(ng.x, ng.y, ng.z, 0.f);
    }
    if (visits) {
        atomicAdd(visits, nv);
        atomicAdd(visits + 1, nt);
    }
}

// ------------------------------------------------------ FP64 CDF builders ----
// CdfTable construction (src/common/cdftable.h:10-30) as FP64 prefix sums on
// the device, one block per table; the tables are stored as float for
// sampling. pdf_i = |w_i| / sum, cdf_i = sum_{j<=i} pdf_j, cdf_last = 1.
__global__ void k_cdf_build(const double *weights, const uint32_t *offsets, uint32_t ntables, float *cdf_out,
                            float *pdf_out, double *sums_out) {
    __shared__ double part[1024];
    __shared__ double carry;
    const uint32_t tb = blockIdx.x;
    if (tb >= ntables) return;
    const uint32_t b0 = offsets[tb], b1 = offsets[tb + 1], n = b1 - b0;
    // total
    double acc = 0.0;
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) acc += fabs(weights[b0 + i]);
    part[threadIdx.x] = acc;
    __syncthreads();
    for (uint32_t s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) part[threadIdx.x] += part[threadIdx.x + s];
        __syncthreads();
    }
    const double total = part[0];
    __syncthreads();
    if (threadIdx.x == 0) { carry = 0.0; if (sums_out) sums_out[tb] = total; }
    __syncthreads();
    const double inv = total > 0.0 ? 1.0 / total : 0.0;
    // chunked inclusive scan of the pdfs
    for (uint32_t c0 = 0; c0 < n; c0 += blockDim.x) {
        const uint32_t i = c0 + threadIdx.x;
        const double p = i < n ? fabs(weights[b0 + i]) * inv : 0.0;
        part[threadIdx.x] = p;
        __syncthreads();
        for (uint32_t off = 1; off < blockDim.x; off <<= 1) {
            const double v = threadIdx.x >= off ? part[threadIdx.x - off] : 0.0;
            __syncthreads();
            part[threadIdx.x] += v;
            __syncthreads();
        }
        if (i < n) {
            const double c = carry + part[threadIdx.x];
            cdf_out[b0 + i] = (i == n - 1) ? 1.0f : float(c);
            pdf_out[b0 + i] = float(p);
        }
        __syncthreads();
        if (threadIdx.x == 0) carry += part[blockDim.x - 1];
        __syncthreads();
    }
}

// environment weights sin(theta_row) * |L| (equirectangular.h:40-61)
__global__ void k_env_weights(const float4 *texels, int w, int h, double *out) {
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < size_t(w) * h; i += size_t(gridDim.x) * blockDim.x) {
        const int y = int(i / w);
        const double v = (double(y) + 0.5) / double(h);
        const double sine = sin(v * 3.14159265358979323846);
        const float4 t = texels[i];
        out[i] = sine * sqrt(double(t.x) * t.x + double(t.y) * t.y + double(t.z) * t.z);
    }
}

__global__ void k_scale_pdf(const double *weights, double total, float *pdf, size_t n) {
    const double inv = total > 0.0 ? 1.0 / total : 0.0;
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        pdf[i] = float(fabs(weights[i]) * inv);
}

}  // namespace wrd

// ------------------------------------------------------------ launch API ----
namespace wrk {

using namespace wrd;

static WaveArgs make_args(const WaveBuffers &b, int parity, const RenderLaunch &r) {
    WaveArgs w;
    const int c = parity & 1, n = c ^ 1;
    w.cur = {b.o[c], b.d[c], b.thr[c], b.meta[c], b.rec[c]};
    w.nxt = {b.o[n], b.d[n], b.thr[n], b.meta[n], b.rec[n]};
    w.hit = b.hit;
    w.sq = {b.sh_o, b.sh_d, b.sh_c};
    w.film = b.film;
    w.ctr = b.ctr;
    w.sample_next = b.sample_next;
    w.total_samples = r.total_samples;
    w.capacity = b.capacity;
    w.shadow_capacity = b.shadow_capacity;
    w.jobs = r.jobs;
    w.job0 = r.job0;
    w.num_jobs = r.num_jobs;
    w.total_pix = r.total_pix;
    w.iter_limit = r.iter_limit;
    w.cond = r.cond;
    w.has_cond = r.has_cond;
    w.prof = r.prof;
    w.lobes = r.guide ? b.lobes : nullptr;
    w.records = r.record ? b.records : nullptr;
    w.rec_count = b.rec_count;
    w.rec_capacity = b.rec_capacity;
    w.fetch_min = (r.fetch_min >= 1 && r.fetch_min <= 32) ? r.fetch_min : 20;
    return w;
}

// the traversal kernel instantiation for the scene: block size x (Phong patches) x (BVH width)
enum TraceLaunch { TRACE_EXTEND, TRACE_SHADOW, TRACE_SHADOW_PENDING, TRACE_PAIR };

template <int BLOCK, bool PHONG, bool WIDE>
void launch_trace_4(TraceLaunch what, const DevScene &s, const WaveArgs &w, const RenderLaunch &r, cudaStream_t st) {
    switch (what) {
        case TRACE_EXTEND: k_extend<BLOCK, PHONG, WIDE><<<r.grid_trace, BLOCK, 0, st>>>(s, w); break;
        case TRACE_SHADOW: k_shadow<BLOCK, PHONG, WIDE><<<r.grid_trace, BLOCK, 0, st>>>(s, w, CTR_SHADOW); break;
        case TRACE_SHADOW_PENDING:
            k_shadow<BLOCK, PHONG, WIDE><<<r.grid_trace, BLOCK, 0, st>>>(s, w, CTR_SHADOW_PENDING);
            break;
        case TRACE_PAIR:
            if (PHONG) k_trace_pair_phong<BLOCK, WIDE><<<r.grid_trace, BLOCK, 0, st>>>(s, w);
            else k_trace_pair<BLOCK, WIDE><<<r.grid_trace, BLOCK, 0, st>>>(s, w);
            break;
    }
}

template <int BLOCK>
void launch_trace_3(TraceLaunch what, const DevScene &s, const WaveArgs &w, const RenderLaunch &r, cudaStream_t st) {
    if (s.patches && s.wnodes) launch_trace_4<BLOCK, true, true>(what, s, w, r, st);
    else if (s.patches) launch_trace_4<BLOCK, true, false>(what, s, w, r, st);
    else if (s.wnodes) launch_trace_4<BLOCK, false, true>(what, s, w, r, st);
    else launch_trace_4<BLOCK, false, false>(what, s, w, r, st);
}

void launch_trace(TraceLaunch what, const DevScene &s, const WaveArgs &w, const RenderLaunch &r, cudaStream_t st) {
    if (r.trace_block == 64) launch_trace_3<64>(what, s, w, r, st);
    else if (r.trace_block == 256) launch_trace_3<256>(what, s, w, r, st);
    else launch_trace_3<128>(what, s, w, r, st);
}

void launch_kernel(int which, const DevScene &s, const WaveBuffers &b, const RenderLaunch &r, int parity,
                   cudaStream_t st) {
    const WaveArgs w = make_args(b, parity, r);
    switch (which) {
        case KERNEL_EXTEND: launch_trace(TRACE_EXTEND, s, w, r, st); break;
        case KERNEL_SHADE:
            if (w.lobes && w.records) k_shade<true, true, true><<<r.grid_shade, kShadeBlock, 0, st>>>(s, w);
            else if (w.lobes) k_shade<true, true, false><<<r.grid_shade, kShadeBlock, 0, st>>>(s, w);
            else if (w.records) k_shade<false, false, true><<<r.grid_shade, kShadeBlock, 0, st>>>(s, w);
            else if (r.nee_only) k_shade<false, true, false><<<r.grid_shade, kShadeBlock, 0, st>>>(s, w);
            else k_shade<false, false, false><<<r.grid_shade, kShadeBlock, 0, st>>>(s, w);
            break;
        case KERNEL_GUIDE:
            if (r.guide)
                wrg::guide_infer_wavefront(*r.guide, w.cur.o, w.cur.d, w.hit, w.ctr + CTR_ACTIVE, s.tris, s.tri_mat,
                                           b.lobes, b.capacity, r.guide_sms, st);
            break;
        case KERNEL_RAYGEN: k_raygen<<<r.grid_shade, kShadeBlock, 0, st>>>(s, w); break;
        case KERNEL_SHADOW: launch_trace(TRACE_SHADOW, s, w, r, st); break;
        case KERNEL_TRACE_PAIR: launch_trace(TRACE_PAIR, s, w, r, st); break;
        case KERNEL_SHADOW_FLUSH: launch_trace(TRACE_SHADOW_PENDING, s, w, r, st); break;
        case KERNEL_ADVANCE: k_advance<<<1, 1, 0, st>>>(w); break;
        default: break;
    }
}

void launch_iteration(const DevScene &s, const WaveBuffers &b, const RenderLaunch &r, int parity, cudaStream_t st) {
    for (int k : {KERNEL_EXTEND, KERNEL_GUIDE, KERNEL_SHADE, KERNEL_RAYGEN, KERNEL_SHADOW, KERNEL_ADVANCE})
        if (k != KERNEL_GUIDE || r.guide) launch_kernel(k, s, b, r, parity, st);
}

// Fused schedule: each iteration's extend shares one launch with the previous iteration's
// shadow rays (k_trace_pair); the first wavefront's shadow rays go with the first extend, and
// the last iteration's are traced by launch_shadow_flush after the loop. Same rays, same
// film contributions as the separate schedule; only the FP64 atomic order differs.
void launch_prime_fused(const DevScene &s, const WaveBuffers &b, const RenderLaunch &r, cudaStream_t st) {
    RenderLaunch r0 = r;
    r0.has_cond = 0;
    for (int k : {KERNEL_RAYGEN, KERNEL_ADVANCE}) launch_kernel(k, s, b, r0, 1, st);
}

void launch_iteration_fused(const DevScene &s, const WaveBuffers &b, const RenderLaunch &r, int parity,
                            cudaStream_t st) {
    launch_trace(TRACE_PAIR, s, make_args(b, parity, r), r, st);
    for (int k : {KERNEL_GUIDE, KERNEL_SHADE, KERNEL_RAYGEN, KERNEL_ADVANCE})
        if (k != KERNEL_GUIDE || r.guide) launch_kernel(k, s, b, r, parity, st);
}

void launch_shadow_flush(const DevScene &s, const WaveBuffers &b, const RenderLaunch &r, cudaStream_t st) {
    RenderLaunch r0 = r;
    r0.has_cond = 0;
    launch_trace(TRACE_SHADOW_PENDING, s, make_args(b, 0, r0), r0, st);
}

void launch_prime(const DevScene &s, const WaveBuffers &b, const RenderLaunch &r, cudaStream_t st) {
    // the first wavefront: raygen into buffer 0 (parity 1 makes buffer 0 the "next" one), then bookkeeping;
    // the graph condition is not touched here (it is only set inside the loop body)
    RenderLaunch r0 = r;
    r0.has_cond = 0;
    for (int k : {KERNEL_RAYGEN, KERNEL_SHADOW, KERNEL_ADVANCE}) launch_kernel(k, s, b, r0, 1, st);
}

void launch_resolve(const double *film, double *out, const RenderLaunch &r, cudaStream_t st) {
    k_resolve<<<592, 256, 0, st>>>(film, out, r.total_pix, r.jobs, r.num_jobs, r.job0);
}

void launch_trace_batch(const DevScene &s, const float4 *rays, uint32_t n, int any_hit, float4 *out, uint32_t *visits,
                        int grid, cudaStream_t st) {
    if (s.patches && s.wnodes) k_trace_batch<true, true><<<grid, kTraceBlock, 0, st>>>(s, rays, n, any_hit, out, visits);
    else if (s.patches) k_trace_batch<true, false><<<grid, kTraceBlock, 0, st>>>(s, rays, n, any_hit, out, visits);
    else if (s.wnodes) k_trace_batch<false, true><<<grid, kTraceBlock, 0, st>>>(s, rays, n, any_hit, out, visits);
    else k_trace_batch<false, false><<<grid, kTraceBlock, 0, st>>>(s, rays, n, any_hit, out, visits);
}

void launch_cdf_build(const double *weights, const uint32_t *offsets, uint32_t ntables, float *cdf, float *pdf,
                      double *sums, cudaStream_t st) {
    if (ntables) k_cdf_build<<<ntables, 1024, 0, st>>>(weights, offsets, ntables, cdf, pdf, sums);
}

void launch_env_weights(const float4 *texels, int w, int h, double *out, cudaStream_t st) {
    k_env_weights<<<592, 256, 0, st>>>(texels, w, h, out);
}

void launch_scale_pdf(const double *weights, double total, float *pdf, size_t n, cudaStream_t st) {
    k_scale_pdf<<<592, 256, 0, st>>>(weights, total, pdf, n);
}

template <int BLOCK, bool PHONG, bool WIDE> int extend_occupancy() {
    int nb = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_extend<BLOCK, PHONG, WIDE>, BLOCK, 0);
    return nb;
}

template <int BLOCK> int extend_occupancy_3(bool phong, bool wide) {
    if (phong && wide) return extend_occupancy<BLOCK, true, true>();
    if (phong) return extend_occupancy<BLOCK, true, false>();
    if (wide) return extend_occupancy<BLOCK, false, true>();
    return extend_occupancy<BLOCK, false, false>();
}

int occupancy_blocks(int which, int trace_block, bool phong, bool wide) {
    int nb = 0;
    if (which == 0) {
        if (trace_block == 64) nb = extend_occupancy_3<64>(phong, wide);
        else if (trace_block == 256) nb = extend_occupancy_3<256>(phong, wide);
        else nb = extend_occupancy_3<128>(phong, wide);
    } else {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_shade<false, false, false>, kShadeBlock, 0);
    }
    return nb;
}

}  // namespace wrk
