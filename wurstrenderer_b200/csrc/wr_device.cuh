// Device-side data layout and inline math of the B200 NEE+MIS renderer.
//
// Scene data in HBM (all 16-byte aligned, read through the non-coherent path):
//   nodes      4 x float4 per binary BVH node (layout in wr_bvh.cpp)
//   tris       3 x float4 per triangle in leaf order: v0.xyz|global id, v1.xyz|mesh id, v2.xyz|prim id
//   tri_mat    uint32 per leaf-order triangle: material index, or LIGHT_BIT | light index
//   materials  DevMaterial per surface material
//   lights     DevLight per area light, light_tris 3 x float4 per emitter triangle
//   env        float4 texels + FP64-built pdf/cdf tables stored as float
// Path state (one wavefront slot per path, structure of arrays, ping-ponged
// between bounces so that every kernel reads and writes it contiguously):
//   ray_o  float4 (origin.xyz, prev pdfW)     ray_d  float4 (dir.xyz, pixel index bits)
//   thr    float4 (throughput.rgb, sample index bits)   meta uint32 (depth)
// Hit records: float4 (t, u, v, leaf triangle | MISS)
// Shadow queue: float4 (origin.xyz, tmax), float4 (dir.xyz, film slot bits),
//               float4 (contribution.rgb, unused)
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace wrd {

constexpr uint32_t LIGHT_BIT = 0x80000000u;
constexpr uint32_t SPLAT_BIT = 0x80000000u;   // shadow target in the splat film
constexpr uint32_t MISS = 0xFFFFFFFFu;
constexpr float kPi = 3.14159265358979323846f;
constexpr float kInvPi = 0.318309886183790671538f;
constexpr float kRayEps = 1e-4f;              // Ray<Vec>::Epsilon (src/common/math/ray.h:8)

constexpr int kTraceBlock = 128;   // threads per block of the traversal kernels
constexpr int kShadeBlock = 256;   // threads per block of shade / raygen
constexpr int kSmemStack = 8;      // traversal stack entries kept in shared memory per ray (the rest in local memory)
constexpr int kMaxStack = 64;      // total traversal stack entries (the BVH builder stays below)

// device counters of the wavefront loop (uint32 each)
enum Counter {
    CTR_ACTIVE = 0,      // live paths in the current wavefront
    CTR_NEXT = 1,        // paths appended to the next wavefront by shade
    CTR_SHADOW = 2,      // shadow rays queued this iteration
    CTR_DONE = 3,        // 1 when no live path is left and every sample was issued
    CTR_ITER = 4,        // iterations executed
    CTR_SHADOW_MAX = 5,  // largest shadow queue seen
    CTR_OVERFLOW = 6,    // shadow queue overflowed (not expected: its capacity is 2x the wavefront)
    CTR_TIMEOUT = 7,     // the iteration bound was reached before the wavefront drained
    CTR_EXTEND_FETCH = 8,   // next ray of the current extend launch (dynamic fetching)
    CTR_SHADOW_FETCH = 9,   // next shadow ray of the current shadow launch
    CTR_SHADOW_PENDING = 10,   // shadow rays of the previous iteration, traced by the next fused launch
    CTR_COUNT = 11
};

struct DevMaterial {
    float kd[3];
    float ks[3];
    float exponent;
    float on_a, on_b;      // Oren-Nayar A, B (sigma >= 0)
    int flags;             // 1 diffuse, 2 glossy, 4 Oren-Nayar diffuse
    float pad[2];
};
constexpr int MAT_DIFFUSE = 1, MAT_GLOSSY = 2, MAT_OREN_NAYAR = 4;

struct DevLight {
    float intensity[3];
    float inv_area;
    uint32_t tri_offset, tri_count;
    float select_pdf;      // light-selection probability (FP64-built CDF table)
    float pad;
};

struct DevCamera {
    float origin[3];
    float fx[3], fy[3], fz[3];   // camera frame (thinlens.h:44-50)
    float dist;                  // lens-to-film distance
    float per_film, per_pixel;   // mPerFilmNormFactor, mPerPixelNormFactor
    float focal, aperture, inv_lens_area;
    int width, height;
};

// one render job of a batch: its camera, sample count and film slice
struct DevJob {
    DevCamera cam;
    int spp, nverts;
    uint32_t pix_offset;              // first pixel of this job in the batch film
    uint32_t npix;
    unsigned long long sample_begin;  // first global sample id of this job
    uint32_t seed;
    int integrator;                   // INTEGRATOR_NEE or INTEGRATOR_PRIMITIVE
    uint32_t sample_offset;           // per-pixel sample index of the first sample (renders split in passes)
    int spp_norm;                     // film normalisation spp (0: spp)
};
constexpr int INTEGRATOR_NEE = 0;        // nextevent_path_tracer (src/renderer/pathnextevent.h)
constexpr int INTEGRATOR_PRIMITIVE = 1;  // primitive_path_tracer (src/renderer/primitivepath.h)
constexpr int INTEGRATOR_LIGHT = 2;      // light_splatting (src/renderer/lightsplatting.h)

struct DevScene {
    const float4 *nodes;            // binary BVH (4 x float4 per node)
    const uint4 *wnodes;            // compressed 8-wide BVH (5 x uint4 per node), nullptr when binary
    const float4 *tris;             // leaf order: p0, p1, p2 (.w: index | patch flag, mesh, primitive)
    const double *patches;          // Phong tessellation patches (wrp::kPatchDoubles per leaf primitive),
                                    // nullptr when the scene has none
    const uint32_t *tri_mat;
    const DevMaterial *materials;
    const DevLight *lights;
    const float4 *light_tris;       // p0, p1, p2 per emitter triangle (mesh order)
    const float *light_tri_cdf;     // per emitter triangle, within its light
    const float *light_cdf;         // num_lights (+1 when env) entries
    int num_lights;
    int num_select;                 // num_lights + has_env
    float scene_center[3];          // bounding sphere of all triangles (EmbreeAccel::boundingSphere,
    float scene_radius;             //   src/accel/embreeaccel.h:326-334)
    // environment
    int has_env, env_w, env_h;
    float env_select_pdf;
    const float4 *env_texels;       // row 0 = top
    const float *env_pixel_pdf;     // w_i / sum w (FP64-built)
    const float *env_row_cdf;       // env_h entries
    const float *env_row_pdf;
    const float *env_col_cdf;       // env_h x env_w, per-row normalised
    const float *env_col_pdf;
};

// ------------------------------------------------------------- float3 ----
struct f3 { float x, y, z; };
__device__ __forceinline__ f3 mk(float x, float y, float z) { return {x, y, z}; }
__device__ __forceinline__ f3 operator+(f3 a, f3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ f3 operator-(f3 a, f3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ f3 operator-(f3 a) { return {-a.x, -a.y, -a.z}; }
__device__ __forceinline__ f3 operator*(f3 a, f3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
__device__ __forceinline__ f3 operator*(f3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ f3 operator*(float s, f3 a) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ f3 operator/(f3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
__device__ __forceinline__ float dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ f3 cross(f3 a, f3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
__device__ __forceinline__ float len2(f3 a) { return dot(a, a); }
__device__ __forceinline__ f3 normalize(f3 a) { return a * rsqrtf(dot(a, a)); }
__device__ __forceinline__ bool is_zero(f3 a) { return a.x == 0.f && a.y == 0.f && a.z == 0.f; }
__device__ __forceinline__ f3 xyz(float4 v) { return {v.x, v.y, v.z}; }
__device__ __forceinline__ f3 ld3(const float *p) { return {p[0], p[1], p[2]}; }

// CoordFrame3 with y = normal: Duff et al. 2017, "Building an orthonormal basis, revisited"
struct Frame {
    f3 x, y, z;
    __device__ __forceinline__ explicit Frame(f3 n) {
        y = n;
        const float sign = copysignf(1.0f, n.y);
        const float a = -1.0f / (sign + n.y);
        const float b = n.z * n.x * a;
        x = mk(sign + n.x * n.x * a, -n.x, b);
        z = mk(sign * b, -sign * n.z, 1.0f + sign * n.z * n.z * a);
    }
    __device__ __forceinline__ f3 to_local(f3 g) const { return {dot(g, x), dot(g, y), dot(g, z)}; }
    __device__ __forceinline__ f3 to_world(f3 l) const { return x * l.x + y * l.y + z * l.z; }
};

// ---------------------------------------------------------------- RNG ----
// Counter-based generator: pcg4d (Jarzynski & Olano, "Hash Functions for GPU
// Rendering", JCGT 2020) keyed by (pixel, sample, dimension group, seed). Each
// call yields four independent uniform numbers; no generator state is stored
// in the wavefront. Streams are statistically, not bitwise, equivalent to the
// reference's per-tile std::mt19937_64.
__device__ __forceinline__ uint4 pcg4d(uint4 v) {
    v.x = v.x * 1664525u + 1013904223u; v.y = v.y * 1664525u + 1013904223u;
    v.z = v.z * 1664525u + 1013904223u; v.w = v.w * 1664525u + 1013904223u;
    v.x += v.y * v.w; v.y += v.z * v.x; v.z += v.x * v.y; v.w += v.y * v.z;
    v.x ^= v.x >> 16; v.y ^= v.y >> 16; v.z ^= v.z >> 16; v.w ^= v.w >> 16;
    v.x += v.y * v.w; v.y += v.z * v.x; v.z += v.x * v.y; v.w += v.y * v.z;
    return v;
}
__device__ __forceinline__ float u01(uint32_t x) { return float(x >> 8) * (1.0f / 16777216.0f); }

struct Rand4 { float a, b, c, d; };
// dimension groups: 0 light selection + pixel jitter, 1 lens, 2 + k BSDF at vertex k
__device__ __forceinline__ Rand4 rand4(uint32_t pixel, uint32_t sample, uint32_t group, uint32_t seed) {
    uint4 h = pcg4d(make_uint4(pixel, sample, group, seed));
    return {u01(h.x), u01(h.y), u01(h.z), u01(h.w)};
}

// --------------------------------------------------------- CDF search ----
// CdfTable::sample (src/common/cdftable.h:36-44): first index with cdf >= u,
// sample remapped into that bin and clamped below one.
__device__ __forceinline__ int cdf_lower_bound(const float *cdf, int n, float u) {
    int lo = 0, hi = n;   // [lo, hi)
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (__ldg(cdf + mid) < u) lo = mid + 1; else hi = mid;
    }
    return min(lo, n - 1);
}
__device__ __forceinline__ float cdf_remap(const float *cdf, int i, float pdf_i, float u) {
    const float prev = i == 0 ? 0.f : __ldg(cdf + i - 1);
    const float r = pdf_i > 0.f ? (u - prev) / pdf_i : 0.f;
    return fminf(fmaxf(r, 0.f), 0.99999994f);
}

}  // namespace wrd
