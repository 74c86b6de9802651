// C ABI of the B200 renderer (include/wurst_b200.h): scene upload, the
// wavefront render loop, ray-batch queries and the simple2 CLI flow.
//
// Scene creation mirrors Simple2Parser::ParseScene + the GeneralSubpathSampler
// constructor (src/sceneio/simple2parser.h:27-68,
// src/pathsampler/generalsubpathsampler.h:162-183): meshes are flattened in
// Embree attach order, the BVH is built, and the light-selection CDF
// (|average Ke| per emitter, 1.23 for the environment, src/light/diffusearealight.h:21-24,
// src/light/envmap.h:22-26), the per-emitter triangle-area CDFs
// (src/geometry/trianglemesh.h:110-129) and the environment's sin-weighted
// luminance CDF (src/sphericalrepresentation/equirectangular.h:33-64) are
// built as FP64 prefix sums on the device.

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/wurst_b200.h"
#include "wr_guide.h"
#include "wr_host.h"
#include "wr_kernels.h"
#include "wr_phong.cuh"

using wr::Error;

namespace wr {
BvhBuildResult build_bvh_lbvh(const std::vector<float> &tri_vertices, cudaStream_t st, double *device_ms);
}

namespace {

thread_local std::string g_last_error;

#define WR_CUDA(call)                                                                                  \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess)                                                                         \
            throw Error(e_ == cudaErrorMemoryAllocation ? WR_ERR_OUT_OF_MEMORY : WR_ERR_CUDA,  \
                        std::string(#call) + ": " + cudaGetErrorString(e_));                          \
    } while (0)

struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    DevBuf() {}
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    void alloc(size_t n) {
        if (n <= bytes && p) return;
        release();
        WR_CUDA(cudaMalloc(&p, std::max<size_t>(n, 16)));
        bytes = n;
    }
    template <typename T> T *as() const { return static_cast<T *>(p); }
};

template <typename T> void upload(DevBuf &b, const std::vector<T> &v, cudaStream_t st) {
    b.alloc(v.size() * sizeof(T));
    if (!v.empty()) WR_CUDA(cudaMemcpyAsync(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st));
}

}  // namespace

struct wr_scene {
    wr::Scene host;
    cudaStream_t stream = nullptr;
    int device = 0;
    // scene data
    DevBuf nodes, wnodes, tris, patches, tri_mat, materials, lights, light_tris, light_tri_cdf, light_tri_pdf, light_cdf, light_pdf;
    uint32_t num_patches = 0;
    DevBuf env_texels, env_pixel_pdf, env_row_cdf, env_row_pdf, env_col_cdf, env_col_pdf;
    wrd::DevScene dev{};
    wr_scene_options opts{};
    int bvh_nodes = 0, bvh_depth = 0;
    double sah_cost = 0.0, build_ms = 0.0, bvh_ms = 0.0;
    // wavefront buffers
    DevBuf w_o[2], w_d[2], w_thr[2], w_meta[2], w_hit, w_sho, w_shd, w_shc, w_film, w_ctr, w_sample, w_out, w_prof,
        w_jobs;
    std::vector<cudaEvent_t> kev;
    // learned guiding: network, per-slot lobes / record links, training records
    wrg::GuideNet guide{};
    bool guide_ready = false;
    int guide_step = 0;
    float box_lo[3] = {0.f, 0.f, 0.f}, box_inv[3] = {1.f, 1.f, 1.f};
    DevBuf w_rec[2], w_lobes, w_records, w_rec_count, g_scratch, g_scratch2, g_loss;
    uint32_t w_guide_capacity = 0, w_record_capacity = 0;
    uint32_t w_capacity = 0;
    size_t w_npix = 0;
    uint32_t *pinned = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    wr_render_stats stats{};
    ~wr_scene() {
        if (guide_ready) wrg::guide_free(guide);
        if (pinned) cudaFreeHost(pinned);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        for (auto e : kev) cudaEventDestroy(e);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

int fail(const Error &e) {
    g_last_error = e.what();
    return e.code;
}

// ------------------------------------------------------------ scene upload ----
void build_device_scene(wr_scene &s) {
    const auto t0 = std::chrono::steady_clock::now();
    wr::Scene &h = s.host;
    WR_CUDA(cudaGetDevice(&s.device));
    WR_CUDA(cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking));
    WR_CUDA(cudaEventCreate(&s.ev0));
    WR_CUDA(cudaEventCreate(&s.ev1));
    WR_CUDA(cudaMallocHost(reinterpret_cast<void **>(&s.pinned), 64));
    cudaStream_t st = s.stream;

    // flatten triangles in attach order
    const uint64_t ntri64 = h.num_triangles();
    if (ntri64 >= (1ull << 27)) throw Error(WR_ERR_UNSUPPORTED, "scene has more than 2^27 triangles");
    const uint32_t ntri = uint32_t(ntri64);
    std::vector<float> verts(size_t(ntri) * 9);
    std::vector<uint32_t> tri_mesh(ntri), tri_prim(ntri), tri_code(ntri);
    // Phong tessellation patches: FP64 unit normals and boxes per patch (global order)
    std::vector<uint8_t> is_patch(ntri, 0);
    std::vector<double> patch_n;          // 9 per triangle (only patches are filled)
    std::vector<float> box_near, box_out; // 6 per triangle: the bound rounded to nearest / outward
    uint32_t npatch = 0;
    for (const wr::Mesh &m : h.meshes) if (m.phong) npatch += m.num_triangles();
    if (npatch) {
        patch_n.assign(size_t(ntri) * 9, 0.0);
        box_near.assign(size_t(ntri) * 6, 0.f);
        box_out.assign(size_t(ntri) * 6, 0.f);
    }
    {
        size_t g = 0;
        for (size_t mi = 0; mi < h.meshes.size(); ++mi) {
            const wr::Mesh &m = h.meshes[mi];
            const uint32_t code = m.light >= 0 ? (wrd::LIGHT_BIT | uint32_t(m.light)) : uint32_t(m.material);
            if (m.phong && m.normals.size() != m.positions.size())
                throw Error(WR_ERR_PARSE, "phong mesh '" + m.name + "' needs one normal per vertex");
            for (uint32_t t = 0; t < m.num_triangles(); ++t, ++g) {
                for (int c = 0; c < 3; ++c) {
                    const uint32_t vi = m.indices[3 * t + c];
                    if (size_t(vi) * 3 + 2 >= m.positions.size()) throw Error(WR_ERR_PARSE, "mesh index out of range");
                    for (int k = 0; k < 3; ++k) verts[9 * g + 3 * c + k] = m.positions[3 * size_t(vi) + k];
                }
                tri_mesh[g] = uint32_t(mi);
                tri_prim[g] = t;
                tri_code[g] = code;
                if (!m.phong) continue;
                // the PhongMeshGeometry of this triangle: normals as AssimpInOut stores them
                // (zero when of ~zero length, else normalised in FP64; assimpio.h:211-223)
                wrp::Patch<double> P;
                for (int c = 0; c < 3; ++c) {
                    const uint32_t vi = m.indices[3 * t + c];
                    const float *q = &m.positions[3 * size_t(vi)];
                    const float *nn = &m.normals[3 * size_t(vi)];
                    P.p[c] = wrp::v3<double>(q[0], q[1], q[2]);
                    const wrp::V<double> n = wrp::v3<double>(nn[0], nn[1], nn[2]);
                    P.n[c] = wrp::is_approx_zero(wrp::length(n)) ? wrp::v3<double>(0.0, 0.0, 0.0) : wrp::normalize(n);
                    patch_n[9 * g + 3 * c + 0] = P.n[c].x;
                    patch_n[9 * g + 3 * c + 1] = P.n[c].y;
                    patch_n[9 * g + 3 * c + 2] = P.n[c].z;
                }
                double lo[3], hi[3];
                wrp::patch_bound(P, lo, hi);
                for (int k = 0; k < 3; ++k) {
                    // Embree keeps float(bound) (embreeaccel.h:63-75); the BVH uses the box
                    // rounded outward so that it contains the FP64 bound
                    float fl = float(lo[k]), fh = float(hi[k]);
                    box_near[6 * g + k] = fl;
                    box_near[6 * g + 3 + k] = fh;
                    if (double(fl) > lo[k]) fl = std::nextafter(fl, -INFINITY);
                    if (double(fh) < hi[k]) fh = std::nextafter(fh, INFINITY);
                    box_out[6 * g + k] = fl;
                    box_out[6 * g + 3 + k] = fh;
                }
                is_patch[g] = 1;
            }
        }
    }
    {   // scene box of the guiding network's position feature (1% margin per side), over the
        // triangles and the patch bounds (the accel's bounds, rtcGetSceneBounds)
        float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (uint32_t g = 0; g < ntri; ++g) {
            if (is_patch[g]) {
                for (int k = 0; k < 3; ++k) {
                    lo[k] = std::min(lo[k], box_near[6 * size_t(g) + k]);
                    hi[k] = std::max(hi[k], box_near[6 * size_t(g) + 3 + k]);
                }
                continue;
            }
            for (int c = 0; c < 3; ++c)
                for (int k = 0; k < 3; ++k) {
                    lo[k] = std::min(lo[k], verts[9 * size_t(g) + 3 * c + k]);
                    hi[k] = std::max(hi[k], verts[9 * size_t(g) + 3 * c + k]);
                }
        }
        double d2 = 0.0;
        for (int k = 0; k < 3; ++k) {
            if (!(lo[k] <= hi[k])) { lo[k] = 0.f; hi[k] = 1.f; }
            const float ext = std::max(hi[k] - lo[k], 1e-6f);
            s.box_lo[k] = lo[k] - 0.01f * ext;
            s.box_inv[k] = 1.f / (1.02f * ext);
            s.dev.scene_center[k] = float((double(lo[k]) + double(hi[k])) * 0.5);
            d2 += (double(hi[k]) - double(lo[k])) * (double(hi[k]) - double(lo[k]));
        }
        // the bounding sphere of EmbreeAccel::boundingSphere (src/accel/embreeaccel.h:326-334)
        s.dev.scene_radius = float(std::sqrt(d2) * 0.5);
    }
    // the builders bound each primitive by the min/max of three points: a patch enters as the
    // pseudo-triangle (lo, hi, hi) of its outward-rounded box
    std::vector<float> bvh_verts;
    if (npatch) {
        bvh_verts = verts;
        for (uint32_t g = 0; g < ntri; ++g) {
            if (!is_patch[g]) continue;
            float *o = &bvh_verts[9 * size_t(g)];
            for (int k = 0; k < 3; ++k) {
                o[k] = box_out[6 * size_t(g) + k];
                o[3 + k] = o[6 + k] = box_out[6 * size_t(g) + 3 + k];
            }
        }
    }
    const std::vector<float> &build_in = npatch ? bvh_verts : verts;
    const bool wide = s.opts.bvh_width == 8;
    wr::BvhBuildResult bvh;
    const auto tb = std::chrono::steady_clock::now();
    if (s.opts.bvh_builder == WR_BVH_DEVICE_LBVH) {
        bvh = wr::build_bvh_lbvh(build_in, st, &s.bvh_ms);
    } else {
        // the compressed 8-wide tree encodes at most 3 triangles per leaf
        const int ml = s.opts.max_leaf > 0 ? s.opts.max_leaf : WR_MAX_LEAF_DEFAULT;
        const double ct = s.opts.sah_trav_cost_milli > 0 ? s.opts.sah_trav_cost_milli * 1e-3 : 1.0;
        // a Phong patch test (FP64 cubic and quadratics) costs many triangle tests: weighting
        // patches in the SAH keeps them in small leaves of their own
        std::vector<float> prim_cost;
        if (npatch) {
            const double cp = s.opts.sah_patch_cost_milli > 0 ? s.opts.sah_patch_cost_milli * 1e-3
                                                              : double(WR_SAH_PATCH_COST_DEFAULT);
            prim_cost.resize(ntri);
            for (uint32_t g = 0; g < ntri; ++g) prim_cost[g] = is_patch[g] ? float(cp) : 1.f;
        }
        bvh = wr::build_bvh_sah(build_in, wide ? std::min(ml, 3) : ml, 0, ct, npatch ? &prim_cost : nullptr);
        s.bvh_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tb).count();
    }
    wr::WideBvh wbvh;
    if (wide) {
        const auto tw = std::chrono::steady_clock::now();
        wbvh = wr::build_wide8(bvh);
        s.bvh_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tw).count();
        bvh.tri_order = wbvh.order;   // leaf order of the wide tree
        bvh.depth = wbvh.depth;
    }
    s.bvh_nodes = wide ? int(wbvh.nodes.size() / 20) : int(bvh.nodes.size() / 16);
    s.bvh_depth = bvh.depth;
    s.sah_cost = bvh.sah_cost;
    if (bvh.depth > wrd::kMaxStack) throw Error(WR_ERR_UNSUPPORTED, "BVH deeper than the traversal stack");
    std::vector<float> trisf(size_t(ntri) * 12);
    std::vector<uint32_t> leaf_mat(ntri);
    std::vector<double> patchd(npatch ? size_t(ntri) * wrp::kPatchDoubles : 0, 0.0);
    for (uint32_t i = 0; i < ntri; ++i) {
        const uint32_t g = bvh.tri_order[i];
        float *o = &trisf[12 * size_t(i)];
        for (int c = 0; c < 3; ++c)
            for (int k = 0; k < 3; ++k) o[4 * c + k] = verts[9 * size_t(g) + 3 * c + k];
        const uint32_t gw = g | (is_patch[g] ? wrp::kPatchFlag : 0u);
        memcpy(&o[3], &gw, 4);
        memcpy(&o[7], &tri_mesh[g], 4);
        memcpy(&o[11], &tri_prim[g], 4);
        leaf_mat[i] = tri_code[g];
        if (is_patch[g]) {   // n1 n2 n3, then the outward box as 6 floats in the last 3 doubles
            double *pd = &patchd[size_t(wrp::kPatchDoubles) * i];
            for (int k = 0; k < 9; ++k) pd[k] = patch_n[9 * size_t(g) + k];
            memcpy(pd + 9, &box_out[6 * size_t(g)], 24);
        }
    }
    if (wide) upload(s.wnodes, wbvh.nodes, st);
    else upload(s.nodes, bvh.nodes, st);
    upload(s.tris, trisf, st);
    upload(s.tri_mat, leaf_mat, st);
    s.num_patches = npatch;
    if (npatch) upload(s.patches, patchd, st);

    // materials
    std::vector<wrd::DevMaterial> mats(std::max<size_t>(h.materials.size(), 1));
    for (size_t i = 0; i < h.materials.size(); ++i) {
        const wr::Material &m = h.materials[i];
        wrd::DevMaterial d{};
        for (int k = 0; k < 3; ++k) { d.kd[k] = m.kd[k]; d.ks[k] = m.ks[k]; }
        d.exponent = m.exponent;
        d.flags = (m.has_diffuse ? wrd::MAT_DIFFUSE : 0) | (m.has_glossy ? wrd::MAT_GLOSSY : 0);
        if (m.sigma >= 0.f && m.has_diffuse) {
            const double s2 = double(m.sigma) * m.sigma;
            d.on_a = float(1.0 - s2 / (2 * (s2 + 0.33)));
            d.on_b = float(0.45 * s2 / (s2 + 0.09));
            d.flags |= wrd::MAT_OREN_NAYAR;
        } else {
            d.on_a = 1.f;
            d.on_b = 0.f;
        }
        mats[i] = d;
    }
    upload(s.materials, mats, st);

    // emitters: triangles in mesh order, FP64 area CDF per emitter, FP64 selection CDF
    const int nl = int(h.lights.size());
    std::vector<float> ltris;
    std::vector<double> areas;
    std::vector<uint32_t> offsets{0};
    std::vector<wrd::DevLight> lights(std::max(nl, 1));
    for (int li = 0; li < nl; ++li) {
        const wr::Mesh &m = h.meshes[h.lights[li].mesh];
        lights[li].tri_offset = uint32_t(areas.size());
        lights[li].tri_count = m.num_triangles();
        for (int k = 0; k < 3; ++k) lights[li].intensity[k] = h.lights[li].intensity[k];
        for (uint32_t t = 0; t < m.num_triangles(); ++t) {
            double p[3][3];
            for (int c = 0; c < 3; ++c) {
                for (int k = 0; k < 3; ++k) {
                    p[c][k] = m.positions[3 * size_t(m.indices[3 * t + c]) + k];
                    ltris.push_back(float(p[c][k]));
                }
                ltris.push_back(0.f);
            }
            const double e1[3] = {p[1][0] - p[0][0], p[1][1] - p[0][1], p[1][2] - p[0][2]};
            const double e2[3] = {p[2][0] - p[0][0], p[2][1] - p[0][1], p[2][2] - p[0][2]};
            const double cx = e1[1] * e2[2] - e1[2] * e2[1], cy = e1[2] * e2[0] - e1[0] * e2[2], cz = e1[0] * e2[1] - e1[1] * e2[0];
            areas.push_back(std::sqrt(cx * cx + cy * cy + cz * cz) / 2.0);
        }
        offsets.push_back(uint32_t(areas.size()));
    }
    // selection weights: emitters then the environment
    std::vector<double> sel;
    for (int li = 0; li < nl; ++li) {
        const float *I = h.lights[li].intensity;
        sel.push_back(std::sqrt(double(I[0]) * I[0] + double(I[1]) * I[1] + double(I[2]) * I[2]));
    }
    if (h.has_env) sel.push_back(1.23);
    const int nsel = int(sel.size());
    std::vector<double> tri_sums(std::max(nl, 1), 0.0);
    std::vector<float> sel_pdf(std::max(nsel, 1), 0.f);
    {
        DevBuf w, off, sums;
        upload(w, areas, st);
        upload(off, offsets, st);
        s.light_tri_cdf.alloc(std::max<size_t>(areas.size(), 1) * 4);
        s.light_tri_pdf.alloc(std::max<size_t>(areas.size(), 1) * 4);
        sums.alloc(std::max(nl, 1) * 8);
        wrk::launch_cdf_build(w.as<double>(), off.as<uint32_t>(), uint32_t(nl), s.light_tri_cdf.as<float>(),
                              s.light_tri_pdf.as<float>(), sums.as<double>(), st);
        WR_CUDA(cudaGetLastError());
        if (nl) WR_CUDA(cudaMemcpyAsync(tri_sums.data(), sums.p, nl * 8, cudaMemcpyDeviceToHost, st));
        DevBuf w2, off2;
        upload(w2, sel, st);
        std::vector<uint32_t> o2{0, uint32_t(nsel)};
        upload(off2, o2, st);
        s.light_cdf.alloc(std::max(nsel, 1) * 4);
        s.light_pdf.alloc(std::max(nsel, 1) * 4);
        wrk::launch_cdf_build(w2.as<double>(), off2.as<uint32_t>(), nsel ? 1u : 0u, s.light_cdf.as<float>(),
                              s.light_pdf.as<float>(), nullptr, st);
        WR_CUDA(cudaGetLastError());
        if (nsel) WR_CUDA(cudaMemcpyAsync(sel_pdf.data(), s.light_pdf.p, nsel * 4, cudaMemcpyDeviceToHost, st));
        WR_CUDA(cudaStreamSynchronize(st));
    }
    for (int li = 0; li < nl; ++li) {
        lights[li].inv_area = float(1.0 / tri_sums[li]);
        lights[li].select_pdf = sel_pdf[li];
    }
    upload(s.lights, lights, st);
    if (ltris.empty()) ltris.assign(12, 0.f);
    upload(s.light_tris, ltris, st);

    wrd::DevScene &d = s.dev;
    d.nodes = wide ? nullptr : s.nodes.as<float4>();
    d.wnodes = wide ? s.wnodes.as<uint4>() : nullptr;
    d.tris = s.tris.as<float4>();
    d.patches = npatch ? s.patches.as<double>() : nullptr;
    d.tri_mat = s.tri_mat.as<uint32_t>();
    d.materials = s.materials.as<wrd::DevMaterial>();
    d.lights = s.lights.as<wrd::DevLight>();
    d.light_tris = s.light_tris.as<float4>();
    d.light_tri_cdf = s.light_tri_cdf.as<float>();
    d.light_cdf = s.light_cdf.as<float>();
    d.num_lights = nl;
    d.num_select = nsel;
    d.has_env = h.has_env ? 1 : 0;
    d.env_select_pdf = h.has_env ? sel_pdf[nsel - 1] : 0.f;

    if (h.has_env) {
        const int W = h.env.width, H = h.env.height;
        const size_t N = size_t(W) * H;
        std::vector<float> tex(N * 4);
        for (size_t i = 0; i < N; ++i) {
            for (int k = 0; k < 3; ++k) tex[4 * i + k] = h.env.rgb[3 * i + k];
            tex[4 * i + 3] = 0.f;
        }
        upload(s.env_texels, tex, st);
        DevBuf wts, off, rowsum, off2;
        wts.alloc(N * 8);
        wrk::launch_env_weights(s.env_texels.as<float4>(), W, H, wts.as<double>(), st);
        std::vector<uint32_t> offs(H + 1);
        for (int y = 0; y <= H; ++y) offs[y] = uint32_t(size_t(y) * W);
        upload(off, offs, st);
        s.env_col_cdf.alloc(N * 4);
        s.env_col_pdf.alloc(N * 4);
        rowsum.alloc(size_t(H) * 8);
        wrk::launch_cdf_build(wts.as<double>(), off.as<uint32_t>(), uint32_t(H), s.env_col_cdf.as<float>(),
                              s.env_col_pdf.as<float>(), rowsum.as<double>(), st);
        std::vector<uint32_t> o2{0, uint32_t(H)};
        upload(off2, o2, st);
        s.env_row_cdf.alloc(size_t(H) * 4);
        s.env_row_pdf.alloc(size_t(H) * 4);
        DevBuf total;
        total.alloc(8);
        wrk::launch_cdf_build(rowsum.as<double>(), off2.as<uint32_t>(), 1u, s.env_row_cdf.as<float>(),
                              s.env_row_pdf.as<float>(), total.as<double>(), st);
        double tot = 0.0;
        WR_CUDA(cudaMemcpyAsync(&tot, total.p, 8, cudaMemcpyDeviceToHost, st));
        WR_CUDA(cudaStreamSynchronize(st));
        s.env_pixel_pdf.alloc(N * 4);
        wrk::launch_scale_pdf(wts.as<double>(), tot, s.env_pixel_pdf.as<float>(), N, st);
        WR_CUDA(cudaGetLastError());
        WR_CUDA(cudaStreamSynchronize(st));
        d.env_w = W;
        d.env_h = H;
        d.env_texels = s.env_texels.as<float4>();
        d.env_pixel_pdf = s.env_pixel_pdf.as<float>();
        d.env_row_cdf = s.env_row_cdf.as<float>();
        d.env_row_pdf = s.env_row_pdf.as<float>();
        d.env_col_cdf = s.env_col_cdf.as<float>();
        d.env_col_pdf = s.env_col_pdf.as<float>();
    }
    WR_CUDA(cudaStreamSynchronize(st));
    s.build_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

// camera constants of ThinlensCamera (src/camera/thinlens.h:40-61, src/common/camera.h:9-18), in FP64
wrd::DevCamera make_camera(const wr::Camera &c) {
    auto sub = [](const double *a, const double *b, double *o) { for (int k = 0; k < 3; ++k) o[k] = a[k] - b[k]; };
    auto crs = [](const double *a, const double *b, double *o) {
        o[0] = a[1] * b[2] - a[2] * b[1]; o[1] = a[2] * b[0] - a[0] * b[2]; o[2] = a[0] * b[1] - a[1] * b[0];
    };
    auto nrm = [](double *a) { double l = std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]); for (int k = 0; k < 3; ++k) a[k] /= l; };
    double z[3], x[3], y[3];
    sub(c.lookat, c.pos, z); nrm(z);
    crs(c.up, z, x); nrm(x);
    crs(z, x, y); nrm(y);
    const double fov = c.fovy_deg * 3.141592653589793238462643 / 180.0;
    const double dist = double(c.height) * 0.5 / std::tan(fov * 0.5);
    wrd::DevCamera d{};
    for (int k = 0; k < 3; ++k) {
        d.origin[k] = float(c.pos[k]); d.fx[k] = float(x[k]); d.fy[k] = float(y[k]); d.fz[k] = float(z[k]);
    }
    d.dist = float(dist);
    d.per_film = float(dist * dist);
    d.per_pixel = float(dist * dist / (double(c.width) * double(c.height)));
    d.focal = float(c.focal);
    d.aperture = float(c.aperture);
    d.inv_lens_area = c.aperture > 0 ? float(1.0 / (3.141592653589793 * c.aperture * c.aperture)) : 1.f;
    d.width = c.width;
    d.height = c.height;
    return d;
}

void ensure_wave(wr_scene &s, uint32_t capacity, size_t npix) {
    if (s.w_capacity != capacity) {
        for (int p = 0; p < 2; ++p) {
            s.w_o[p].alloc(size_t(capacity) * 16);
            s.w_d[p].alloc(size_t(capacity) * 16);
            s.w_thr[p].alloc(size_t(capacity) * 16);
            s.w_meta[p].alloc(size_t(capacity) * 4);
        }
        s.w_hit.alloc(size_t(capacity) * 16);
        s.w_sho.alloc(size_t(capacity) * 2 * 16);
        s.w_shd.alloc(size_t(capacity) * 2 * 16);
        s.w_shc.alloc(size_t(capacity) * 2 * 16);
        s.w_ctr.alloc(wrd::CTR_COUNT * 4);
        s.w_sample.alloc(8);
        s.w_capacity = capacity;
    }
    if (s.w_npix != npix) {
        s.w_film.alloc(npix * 6 * 8);
        s.w_out.alloc(npix * 3 * 8);
        s.w_npix = npix;
    }
}

struct HostJob {
    wr::Camera cam;
    int spp = 16, nverts = 10;
    uint32_t seed = 0;
    int integrator = wrd::INTEGRATOR_NEE;
    uint32_t sample_offset = 0;   // per-pixel index of the first sample (renders split in passes)
    int spp_norm = 0;             // film normalisation (0: spp)
};

// options of one render pass (guided renders are a sequence of passes over one film)
struct PassOpts {
    const wrg::GuideNet *guide = nullptr;   // lobes for shading (nullptr: plain NEE+MIS)
    bool record = false;                    // collect training records
    bool keep_film = false;                 // add to the film of the previous pass
    uint32_t record_capacity = 0;
};

void ensure_guide_wave(wr_scene &s, uint32_t capacity, uint32_t record_capacity) {
    if (s.w_guide_capacity != capacity) {
        s.w_rec[0].alloc(size_t(capacity) * 4);
        s.w_rec[1].alloc(size_t(capacity) * 4);
        s.w_lobes.alloc(size_t(capacity) * wrg::kPackedChunks * 16);
        s.w_guide_capacity = capacity;
    }
    if (record_capacity > s.w_record_capacity) {
        s.w_records.alloc(size_t(record_capacity) * wrg::kRecordFloat4 * 16);
        s.w_record_capacity = record_capacity;
    }
    s.w_rec_count.alloc(16);
}

int integrator_of(const std::string &name) {
    if (name.empty() || name == "nextevent_path_tracer") return wrd::INTEGRATOR_NEE;
    if (name == "primitive_path_tracer") return wrd::INTEGRATOR_PRIMITIVE;
    if (name == "light_splatting") return wrd::INTEGRATOR_LIGHT;
    throw Error(WR_ERR_UNSUPPORTED, "integrator '" + name + "' is not provided by this build");
}

// Renders a batch of jobs (one camera, spp and depth each) over the scene in one wavefront.
// The images land in `out` (host or device) concatenated in job order.
void render_jobs(wr_scene &s, const std::vector<HostJob> &jobs, const wr_render_desc &desc, double *out,
                 bool out_on_host, const PassOpts &po = PassOpts{}) {
    if (jobs.empty()) throw Error(WR_ERR_INVALID_ARGUMENT, "no jobs");
    std::vector<wrd::DevJob> table(jobs.size());
    unsigned long long total = 0;
    size_t total_pix = 0;
    int max_nverts = 0;
    for (size_t j = 0; j < jobs.size(); ++j) {
        const HostJob &hj = jobs[j];
        if (hj.spp <= 0) throw Error(WR_ERR_INVALID_ARGUMENT, "num_spp must be positive");
        if (hj.cam.width <= 0 || hj.cam.height <= 0) throw Error(WR_ERR_INVALID_ARGUMENT, "resolution must be positive");
        wrd::DevJob &d = table[j];
        d = wrd::DevJob{};
        d.cam = make_camera(hj.cam);
        d.spp = hj.spp;
        d.nverts = hj.nverts;
        d.npix = uint32_t(size_t(hj.cam.width) * hj.cam.height);
        d.pix_offset = uint32_t(total_pix);
        d.sample_begin = total;
        d.seed = hj.seed;
        d.integrator = hj.integrator;
        d.sample_offset = hj.sample_offset;
        d.spp_norm = hj.spp_norm;
        total += (unsigned long long)d.npix * unsigned(hj.spp);
        total_pix += d.npix;
        max_nverts = std::max(max_nverts, hj.nverts);
        if (hj.integrator == wrd::INTEGRATOR_PRIMITIVE && hj.nverts <= 1) table[j].nverts = 1;
        if (total_pix >= (1ull << 31)) throw Error(WR_ERR_UNSUPPORTED, "batch film larger than 2^31 pixels");
        if (jobs.size() >= (1u << 24)) throw Error(WR_ERR_UNSUPPORTED, "more than 2^24 jobs");
    }
    int sms = 148;
    WR_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s.device));
    uint32_t capacity = desc.queue_capacity > 0 ? uint32_t(desc.queue_capacity) : (1u << 21);
    capacity = uint32_t(std::min<unsigned long long>(capacity, std::max<unsigned long long>(total, 1024ull)));
    ensure_wave(s, capacity, total_pix);
    cudaStream_t st = s.stream;

    wrk::WaveBuffers b{};
    for (int p = 0; p < 2; ++p) {
        b.o[p] = s.w_o[p].as<float4>();
        b.d[p] = s.w_d[p].as<float4>();
        b.thr[p] = s.w_thr[p].as<float4>();
        b.meta[p] = s.w_meta[p].as<uint32_t>();
    }
    b.hit = s.w_hit.as<float4>();
    b.sh_o = s.w_sho.as<float4>();
    b.sh_d = s.w_shd.as<float4>();
    b.sh_c = s.w_shc.as<float4>();
    b.film = s.w_film.as<double>();
    b.ctr = s.w_ctr.as<uint32_t>();
    b.sample_next = s.w_sample.as<unsigned long long>();
    b.capacity = capacity;
    b.shadow_capacity = 2 * capacity;
    const bool guided = po.guide || po.record;
    if (guided) {
        ensure_guide_wave(s, capacity, po.record_capacity);
        b.rec[0] = s.w_rec[0].as<uint32_t>();
        b.rec[1] = s.w_rec[1].as<uint32_t>();
        b.lobes = s.w_lobes.as<uint4>();
        b.records = s.w_records.as<float4>();
        b.rec_count = s.w_rec_count.as<uint32_t>();
        b.rec_capacity = s.w_record_capacity;
    }

    wrk::RenderLaunch r{};
    r.guide = po.guide;
    r.record = po.record ? 1 : 0;
    r.guide_sms = sms;
    if (desc.fetch_threshold < 0 || desc.fetch_threshold > 32)
        throw Error(WR_ERR_INVALID_ARGUMENT, "fetch_threshold must be 0..32");
    r.fetch_min = desc.fetch_threshold > 0 ? desc.fetch_threshold : 20;
    r.num_jobs = int(table.size());
    r.job0 = table[0];
    r.nee_only = 1;
    for (const auto &j : table) r.nee_only &= j.integrator == wrd::INTEGRATOR_NEE ? 1 : 0;
    if (table.size() > 1) {
        upload(s.w_jobs, table, st);
        r.jobs = s.w_jobs.as<wrd::DevJob>();
    }
    r.total_pix = uint32_t(total_pix);
    r.total_samples = total;
    const unsigned long long waves = (total + capacity - 1) / capacity;
    r.iter_limit = uint32_t(std::min<unsigned long long>((waves + 2) * (unsigned long long)(max_nverts + 2) + 64,
                                                         0xffffffffull));
    if (desc.max_iterations < 0) throw Error(WR_ERR_INVALID_ARGUMENT, "max_iterations must be >= 0");
    if (desc.max_iterations > 0) r.iter_limit = std::min(r.iter_limit, uint32_t(desc.max_iterations));
    r.trace_block = (desc.trace_block == 64 || desc.trace_block == 256) ? desc.trace_block : 128;
    r.grid_trace = desc.grid_trace > 0 ? desc.grid_trace : sms * std::max(1, wrk::occupancy_blocks(0, r.trace_block, s.dev.patches != nullptr, s.dev.wnodes != nullptr));
    r.grid_shade = desc.grid_shade > 0 ? desc.grid_shade : sms * std::max(1, wrk::occupancy_blocks(1));

    const int profile = desc.profile;
    s.w_prof.alloc(16 * 8);
    r.prof = profile >= 2 ? s.w_prof.as<unsigned long long>() : nullptr;
    s.stats = wr_render_stats{};
    double *dst = (out_on_host || !out) ? s.w_out.as<double>() : out;
    unsigned long long launches = 0;

    auto clear = [&]() {
        if (!po.keep_film) WR_CUDA(cudaMemsetAsync(b.film, 0, total_pix * 6 * 8, st));
        if (po.record) WR_CUDA(cudaMemsetAsync(b.rec_count, 0, 4, st));
        WR_CUDA(cudaMemsetAsync(b.ctr, 0, wrd::CTR_COUNT * 4, st));
        WR_CUDA(cudaMemsetAsync(b.sample_next, 0, 8, st));
    };
    const bool trace = max_nverts > 1;
    if (profile) {
        // one kernel at a time, bracketed by events, to attribute device time per kernel
        WR_CUDA(cudaMemsetAsync(s.w_prof.p, 0, 16 * 8, st));
        clear();
        WR_CUDA(cudaEventRecord(s.ev0, st));
        if (s.kev.empty()) {
            s.kev.resize(2);
            for (auto &e : s.kev) WR_CUDA(cudaEventCreate(&e));
        }
        auto timed = [&](int which, int parity) {
            WR_CUDA(cudaEventRecord(s.kev[0], st));
            if (which == wrk::KERNEL_RESOLVE) wrk::launch_resolve(b.film, dst, r, st);
            else wrk::launch_kernel(which, s.dev, b, r, parity, st);
            WR_CUDA(cudaGetLastError());
            WR_CUDA(cudaEventRecord(s.kev[1], st));
            WR_CUDA(cudaEventSynchronize(s.kev[1]));
            float ms = 0.f;
            WR_CUDA(cudaEventElapsedTime(&ms, s.kev[0], s.kev[1]));
            // profile 3 (fused schedule): the pair kernel is booked as extend, the flush as shadow
            const int slot = which == wrk::KERNEL_TRACE_PAIR ? WR_K_EXTEND
                           : which == wrk::KERNEL_SHADOW_FLUSH ? WR_K_SHADOW : which;
            s.stats.kernel_ms[slot] += ms;
            s.stats.kernel_count[slot] += 1;
            launches += 1;
        };
        if (trace && profile >= 3) {
            timed(wrk::KERNEL_RAYGEN, 1);
            timed(wrk::KERNEL_ADVANCE, 1);
            int parity = 0;
            while (true) {
                for (int k : {wrk::KERNEL_TRACE_PAIR, wrk::KERNEL_GUIDE, wrk::KERNEL_SHADE, wrk::KERNEL_RAYGEN,
                              wrk::KERNEL_ADVANCE})
                    if (k != wrk::KERNEL_GUIDE || po.guide) timed(k, parity);
                parity ^= 1;
                WR_CUDA(cudaMemcpyAsync(s.pinned, b.ctr, wrd::CTR_COUNT * 4, cudaMemcpyDeviceToHost, st));
                WR_CUDA(cudaStreamSynchronize(st));
                if (s.pinned[wrd::CTR_DONE]) break;
            }
            timed(wrk::KERNEL_SHADOW_FLUSH, 0);
        } else if (trace) {
            timed(wrk::KERNEL_RAYGEN, 1);
            timed(wrk::KERNEL_SHADOW, 1);
            timed(wrk::KERNEL_ADVANCE, 1);
            int parity = 0;
            while (true) {
                for (int k : {wrk::KERNEL_EXTEND, wrk::KERNEL_GUIDE, wrk::KERNEL_SHADE, wrk::KERNEL_RAYGEN,
                              wrk::KERNEL_SHADOW, wrk::KERNEL_ADVANCE})
                    if (k != wrk::KERNEL_GUIDE || po.guide) timed(k, parity);
                parity ^= 1;
                WR_CUDA(cudaMemcpyAsync(s.pinned, b.ctr, wrd::CTR_COUNT * 4, cudaMemcpyDeviceToHost, st));
                WR_CUDA(cudaStreamSynchronize(st));
                if (s.pinned[wrd::CTR_DONE]) break;
            }
        }
        timed(wrk::KERNEL_RESOLVE, 0);
        s.stats.kernel_items[wrk::KERNEL_RESOLVE] += total_pix;
    } else if (desc.use_graph) {
        // the whole render as one graph: clears, first wavefront, a while-loop node whose body is two
        // bounce iterations (the bookkeeping kernel clears the condition when the wavefront drains
        // or the iteration bound is reached), the last shadow rays and the resolve; each iteration
        // traces its extend rays and the previous iteration's shadow rays in one launch
        cudaGraph_t g = nullptr, gp = nullptr, gs = nullptr;
        cudaGraphExec_t ex = nullptr;
        auto cleanup = [&]() {
            if (ex) cudaGraphExecDestroy(ex);
            if (g) cudaGraphDestroy(g);
            if (gp) cudaGraphDestroy(gp);
            if (gs) cudaGraphDestroy(gs);
        };
        try {
            WR_CUDA(cudaGraphCreate(&g, 0));
            cudaGraphConditionalHandle h{};
            if (trace) {   // a handle must belong to a conditional node of the graph
                WR_CUDA(cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault));
                r.cond = h;
                r.has_cond = 1;
            }
            WR_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            clear();
            if (trace) wrk::launch_prime_fused(s.dev, b, r, st);
            WR_CUDA(cudaStreamEndCapture(st, &gp));
            cudaGraphNode_t np, nw, ns;
            WR_CUDA(cudaGraphAddChildGraphNode(&np, g, nullptr, 0, gp));
            cudaGraphNode_t last = np;
            if (trace) {
                cudaGraphNodeParams cp{};
                cp.type = cudaGraphNodeTypeConditional;
                cp.conditional.handle = h;
                cp.conditional.type = cudaGraphCondTypeWhile;
                cp.conditional.size = 1;
                WR_CUDA(cudaGraphAddNode(&nw, g, &np, 1, &cp));
                cudaGraph_t body = cp.conditional.phGraph_out[0];
                WR_CUDA(cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
                wrk::launch_iteration_fused(s.dev, b, r, 0, st);
                wrk::launch_iteration_fused(s.dev, b, r, 1, st);
                WR_CUDA(cudaStreamEndCapture(st, &body));
                last = nw;
            }
            WR_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            if (trace) wrk::launch_shadow_flush(s.dev, b, r, st);
            wrk::launch_resolve(b.film, dst, r, st);
            WR_CUDA(cudaStreamEndCapture(st, &gs));
            WR_CUDA(cudaGraphAddChildGraphNode(&ns, g, &last, 1, gs));
            WR_CUDA(cudaGraphInstantiate(&ex, g, 0));
            WR_CUDA(cudaEventRecord(s.ev0, st));
            WR_CUDA(cudaGraphLaunch(ex, st));
            launches += 1;
        } catch (...) {
            cudaStreamCaptureStatus cs;
            if (cudaStreamIsCapturing(st, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) {
                cudaGraph_t junk = nullptr;
                cudaStreamEndCapture(st, &junk);
                if (junk) cudaGraphDestroy(junk);
            }
            cleanup();
            throw;
        }
        WR_CUDA(cudaEventRecord(s.ev1, st));
        WR_CUDA(cudaMemcpyAsync(s.pinned, b.ctr, wrd::CTR_COUNT * 4, cudaMemcpyDeviceToHost, st));
        const cudaError_t e = cudaStreamSynchronize(st);
        cleanup();
        if (e != cudaSuccess) throw Error(WR_ERR_CUDA, std::string("render graph: ") + cudaGetErrorString(e));
    } else {
        clear();
        WR_CUDA(cudaEventRecord(s.ev0, st));
        if (trace) {
            wrk::launch_prime_fused(s.dev, b, r, st);
            WR_CUDA(cudaGetLastError());
            while (true) {
                wrk::launch_iteration_fused(s.dev, b, r, 0, st);
                wrk::launch_iteration_fused(s.dev, b, r, 1, st);
                WR_CUDA(cudaGetLastError());
                WR_CUDA(cudaMemcpyAsync(s.pinned, b.ctr, wrd::CTR_COUNT * 4, cudaMemcpyDeviceToHost, st));
                WR_CUDA(cudaStreamSynchronize(st));
                if (s.pinned[wrd::CTR_DONE]) break;
            }
            wrk::launch_shadow_flush(s.dev, b, r, st);
            WR_CUDA(cudaGetLastError());
        }
        wrk::launch_resolve(b.film, dst, r, st);
        WR_CUDA(cudaGetLastError());
        launches += 1;
    }
    if (!desc.use_graph || profile) WR_CUDA(cudaEventRecord(s.ev1, st));
    WR_CUDA(cudaMemcpyAsync(s.pinned, b.ctr, wrd::CTR_COUNT * 4, cudaMemcpyDeviceToHost, st));
    if (out_on_host && out) WR_CUDA(cudaMemcpyAsync(out, dst, total_pix * 3 * 8, cudaMemcpyDeviceToHost, st));
    if (po.record) WR_CUDA(cudaMemcpyAsync(s.pinned + 12, b.rec_count, 4, cudaMemcpyDeviceToHost, st));
    WR_CUDA(cudaStreamSynchronize(st));
    if (trace && s.pinned[wrd::CTR_TIMEOUT]) throw Error(WR_ERR_TIMEOUT, "wavefront did not drain within the iteration bound");
    if (trace && s.pinned[wrd::CTR_OVERFLOW]) throw Error(WR_ERR_CUDA, "shadow queue overflow");
    float ms = 0.f;
    WR_CUDA(cudaEventElapsedTime(&ms, s.ev0, s.ev1));
    if (profile >= 2) {
        unsigned long long prof[16];
        WR_CUDA(cudaMemcpy(prof, s.w_prof.p, sizeof(prof), cudaMemcpyDeviceToHost));
        for (int k = 0; k < 4; ++k) s.stats.kernel_items[k] = prof[k];
        s.stats.extend_node_visits = prof[6];
        s.stats.extend_tri_tests = prof[7];
        s.stats.shadow_node_visits = prof[8];
        s.stats.shadow_tri_tests = prof[9];
    }
    s.stats.render_ms = ms;
    s.stats.paths = total;
    s.stats.iterations = trace ? s.pinned[wrd::CTR_ITER] : 0;
    // kernels per render (a graph launch runs the same kernels). CTR_ITER counts the bookkeeping
    // launches, the first wavefront's included. Separate kernels (profile 1 / 2): prime 3 + 5 (6
    // with guiding) per further iteration + resolve; fused schedule: prime 2 + 4 (5) per further
    // iteration + the last shadow rays + resolve
    const unsigned long long iters = s.pinned[wrd::CTR_ITER] > 0 ? s.pinned[wrd::CTR_ITER] - 1ull : 0ull;
    if (profile == 1 || profile == 2)
        s.stats.kernel_launches = trace ? 3ull + (po.guide ? 6ull : 5ull) * iters + 1ull : 1ull;
    else
        s.stats.kernel_launches = trace ? 2ull + (po.guide ? 5ull : 4ull) * iters + 2ull : 1ull;
    s.stats.max_shadow_queue = s.pinned[wrd::CTR_SHADOW_MAX];
    s.stats.queue_capacity = capacity;
    s.stats.grid_trace = r.grid_trace;
    s.stats.grid_shade = r.grid_shade;
    s.stats.trace_block = r.trace_block;
    (void)launches;
}

HostJob scene_job(const wr::Scene &h, const wr_render_desc &desc) {
    if (!h.has_camera) throw Error(WR_ERR_INVALID_ARGUMENT, "scene has no camera");
    if (desc.render_index < 0) throw Error(WR_ERR_INVALID_ARGUMENT, "render_index must be >= 0");
    wr::RenderEntry re;
    if (size_t(desc.render_index) < h.renders.size()) re = h.renders[desc.render_index];
    HostJob j;
    j.cam = h.camera;
    j.spp = desc.num_spp > 0 ? desc.num_spp : re.num_spp;
    j.nverts = desc.num_path_vertices > 0 ? desc.num_path_vertices : re.num_path_vertices;
    j.seed = desc.seed;
    j.integrator = desc.integrator == 1 ? wrd::INTEGRATOR_NEE
                 : desc.integrator == 2 ? wrd::INTEGRATOR_PRIMITIVE
                 : desc.integrator == 3 ? wrd::INTEGRATOR_LIGHT
                                        : integrator_of(re.integrator);
    return j;
}

// ------------------------------------------------------------ guiding ----
constexpr float kGuideLr = 1e-3f;          // default Adam learning rate (wr_render_desc.guide_lr = 0)
constexpr double kGuideTimeShare = 0.18;   // default training budget: share of the render's device time
constexpr double kGuideStepMsGuess = 0.035; // Adam step time assumed before the first one is measured

int sm_count(const wr_scene &s) {
    int sms = 148;
    WR_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s.device));
    return sms;
}

void ensure_guide(wr_scene &s) {
    if (s.guide_ready) return;
    wrg::GuideNet g{};
    for (int k = 0; k < 3; ++k) {
        g.box_lo[k] = s.box_lo[k];
        g.box_inv[k] = s.box_inv[k];
    }
    try {
        wrg::guide_alloc(g);
        wrg::guide_init(g, 0x9E3779B9u, s.stream);
        WR_CUDA(cudaStreamSynchronize(s.stream));
    } catch (...) {
        wrg::guide_free(g);
        throw;
    }
    s.guide = g;
    s.guide_ready = true;
    s.guide_step = 0;
}

void check_guide_status(wr_scene &s) {
    uint32_t err = 0;
    WR_CUDA(cudaMemcpyAsync(&err, s.guide.err, 4, cudaMemcpyDeviceToHost, s.stream));
    WR_CUDA(cudaStreamSynchronize(s.stream));
    if (err) {
        WR_CUDA(cudaMemsetAsync(s.guide.err, 0, 4, s.stream));
        throw Error(WR_ERR_TIMEOUT, "guiding network: a tensor-core completion wait timed out");
    }
}

// a stride coprime with n (a fixed shuffle of the records: i -> i * stride mod n)
uint32_t shuffle_stride(uint32_t n) {
    if (n <= 2) return 1u;
    uint64_t c = uint64_t(double(n) * 0.6180339887) | 1u;
    auto gcd = [](uint64_t a, uint64_t b) { while (b) { const uint64_t t = a % b; a = b; b = t; } return a; };
    while (gcd(c, n) != 1) c += 2;
    return uint32_t(c % n);
}

// Adam steps over minibatches of records [0, n) in device memory; returns the summed loss
double train_records(wr_scene &s, const float4 *records, uint32_t n, uint32_t batch, int max_steps, float lr,
                     float c_max, std::vector<double> *per_step, unsigned long long *steps_out) {
    cudaStream_t st = s.stream;
    s.g_loss.alloc(8 * 2);
    const uint32_t stride = shuffle_stride(n);
    const int steps = max_steps > 0 ? max_steps : int((n + batch - 1) / batch);
    double total = 0.0;
    WR_CUDA(cudaMemsetAsync(s.g_loss.p, 0, 8, st));
    for (int k = 0; k < steps && n > 0; ++k) {
        const uint32_t first = uint32_t((uint64_t(k) * batch) % n);
        const uint32_t cnt = std::min(batch, n - first);
        if (per_step) WR_CUDA(cudaMemsetAsync(s.g_loss.p, 0, 8, st));
        // each kernel may be scheduled while the one before it ends (its set-up and the first
        // records' gather overlap that kernel); it waits for it before reading its results
        const int nslots = wrg::guide_gradient(s.guide, records, first + cnt, first, n, stride, c_max,
                                               s.g_loss.as<double>(), st, k > 0 && !per_step);
        wrg::guide_adam(s.guide, lr, 1.f / float(cnt), ++s.guide_step, nslots, st, true);
        if (per_step) {
            double l = 0.0;
            WR_CUDA(cudaMemcpyAsync(&l, s.g_loss.p, 8, cudaMemcpyDeviceToHost, st));
            WR_CUDA(cudaStreamSynchronize(st));
            per_step->push_back(l / double(cnt));
            total += l;
        }
        if (steps_out) ++*steps_out;
    }
    if (!per_step) {
        WR_CUDA(cudaMemcpyAsync(&total, s.g_loss.p, 8, cudaMemcpyDeviceToHost, st));
        WR_CUDA(cudaStreamSynchronize(st));
    }
    check_guide_status(s);
    return total;
}

void add_stats(wr_render_stats &a, const wr_render_stats &b) {
    a.render_ms += b.render_ms;
    a.paths += b.paths;
    a.iterations += b.iterations;
    a.max_shadow_queue = std::max(a.max_shadow_queue, b.max_shadow_queue);
    a.queue_capacity = b.queue_capacity;
    a.grid_trace = b.grid_trace;
    a.grid_shade = b.grid_shade;
    a.trace_block = b.trace_block;
    a.kernel_launches += b.kernel_launches;
    for (int k = 0; k < 8; ++k) {
        a.kernel_ms[k] += b.kernel_ms[k];
        a.kernel_count[k] += b.kernel_count[k];
        a.kernel_items[k] += b.kernel_items[k];
    }
    a.extend_node_visits += b.extend_node_visits;
    a.extend_tri_tests += b.extend_tri_tests;
    a.shadow_node_visits += b.shadow_node_visits;
    a.shadow_tri_tests += b.shadow_tri_tests;
}

// Guided render: training passes (records collected, Adam after each pass; the first pass
// samples the BSDF only), then one pass with the trained network for the remaining samples.
// All passes add to one film, normalised by the total spp, so the image is the same
// unbiased estimator as the plain render with a different sampling density.
void render_guided(wr_scene &s, const wr_render_desc &desc, double *out, bool out_on_host) {
    HostJob base = scene_job(s.host, desc);
    if (base.integrator != wrd::INTEGRATOR_NEE)
        throw Error(WR_ERR_UNSUPPORTED, "guiding applies to nextevent_path_tracer only");
    if (desc.guiding != 1 && desc.guiding != 2) throw Error(WR_ERR_INVALID_ARGUMENT, "guiding must be 0, 1 or 2");
    if (!(desc.guide_lr >= 0.f) || !std::isfinite(desc.guide_lr))
        throw Error(WR_ERR_INVALID_ARGUMENT, "guide_lr must be a finite value >= 0");
    const float lr = desc.guide_lr > 0.f ? desc.guide_lr : kGuideLr;
    if (base.spp <= 0) throw Error(WR_ERR_INVALID_ARGUMENT, "num_spp must be positive");
    ensure_guide(s);
    cudaStream_t st = s.stream;
    const int total = base.spp;
    const size_t npix = size_t(std::max(base.cam.width, 0)) * size_t(std::max(base.cam.height, 0));
    if (npix == 0) throw Error(WR_ERR_INVALID_ARGUMENT, "resolution must be positive");
    const int train = desc.guiding == 1 ? std::min(desc.guide_train_spp > 0 ? desc.guide_train_spp : 32, total) : 0;
    // training passes of about 2^22 paths, at least four of them
    const int pass = desc.guide_pass_spp > 0
                         ? desc.guide_pass_spp
                         : int(std::max<size_t>(1, std::min<size_t>(size_t(std::max(train / 4, 1)),
                                                                    (size_t(1) << 22) / npix)));
    const uint32_t batch = desc.guide_batch > 0 ? uint32_t(desc.guide_batch) : 16384u;
    const int n_train_passes = train > 0 ? (train + pass - 1) / pass : 0;
    // Adam step budget: fixed (desc.guide_steps) or kGuideTimeShare of the render's estimated
    // device time, estimated from the first (unguided) pass and the measured time per step
    int planned_steps = desc.guide_steps > 0 ? desc.guide_steps : 0;
    double budget_ms = 0.0;
    const uint64_t per_pass = uint64_t(npix) * uint64_t(pass) * uint64_t(std::max(1, base.nverts - 2));
    const uint32_t rec_cap = uint32_t(std::min<uint64_t>(per_pass, uint64_t(1) << 24));
    if (desc.guiding == 1) {
        wrg::guide_init(s.guide, desc.seed * 0x85EBCA6Bu + 0x6A09E667u, st);
        s.guide_step = 0;
    }
    wr_render_stats agg{};
    bool trained = desc.guiding == 2;
    double train_ms = 0.0, last_loss = 0.0;
    unsigned long long records = 0, steps = 0;
    int done = 0, passes = 0;
    const int sms = sm_count(s);
    while (done < train) {
        const int k = std::min(pass, train - done);
        HostJob j = base;
        j.spp = k;
        j.sample_offset = uint32_t(done);
        j.spp_norm = total;
        PassOpts po;
        po.guide = trained ? &s.guide : nullptr;
        po.record = true;
        po.keep_film = done > 0;
        po.record_capacity = rec_cap;
        const bool last = done + k == total;
        render_jobs(s, {j}, desc, last ? out : nullptr, out_on_host, po);
        add_stats(agg, s.stats);
        ++passes;
        const uint32_t n = std::min(s.pinned[12], s.w_record_capacity);
        records += n;
        // loss weight clamp: 20 x the mean c of the pass's records
        s.g_scratch2.alloc(16);
        wrg::guide_cstats(s.w_records.as<float4>(), n, s.g_scratch2.as<double>(), sms, st);
        double cs[2] = {0.0, 0.0};
        WR_CUDA(cudaMemcpyAsync(cs, s.g_scratch2.p, 16, cudaMemcpyDeviceToHost, st));
        WR_CUDA(cudaStreamSynchronize(st));
        const double clamp = desc.guide_clamp > 0.f ? double(desc.guide_clamp) : 1000.0;
        const float c_max = desc.guide_clamp < 0.f ? INFINITY
                          : cs[1] > 0.0 ? float(clamp * cs[0] / cs[1]) : wrg::kCMax;
        if (desc.guide_steps <= 0 && passes == 1) {
            const double est_ms = s.stats.render_ms / double(k) * double(total) * 1.1;   // guided passes ~10 % slower
            budget_ms = kGuideTimeShare * est_ms;
            planned_steps = int(std::min(8192.0, std::max(256.0, budget_ms / kGuideStepMsGuess)));
        }
        // the remaining step budget spread evenly over the remaining training passes
        int pass_steps = 0;
        {
            const int passes_left = n_train_passes - (passes - 1);
            int steps_left = planned_steps - int(steps);
            if (desc.guide_steps <= 0 && steps > 0) {   // re-plan with the measured time per step
                const double per_step = train_ms / double(steps);
                steps_left = int(std::max(0.0, (budget_ms - train_ms) / per_step));
                steps_left = std::min(steps_left, 8192 - int(steps));
                steps_left = std::max(steps_left, 256 - int(steps));
            }
            pass_steps = passes_left > 0 ? std::max(steps_left, 0) / passes_left : 0;
        }
        WR_CUDA(cudaEventRecord(s.ev0, st));
        const double loss = pass_steps > 0 ? train_records(s, s.w_records.as<float4>(), n, batch, pass_steps, lr,
                                                          c_max, nullptr, &steps)
                                           : 0.0;
        WR_CUDA(cudaEventRecord(s.ev1, st));
        WR_CUDA(cudaEventSynchronize(s.ev1));
        float ms = 0.f;
        WR_CUDA(cudaEventElapsedTime(&ms, s.ev0, s.ev1));
        train_ms += ms;
        if (pass_steps > 0 && n > 0) last_loss = loss / (double(pass_steps) * double(std::min(batch, n)));
        trained = trained || (n > 0 && steps > 0);
        done += k;
    }
    if (done < total) {
        HostJob j = base;
        j.spp = total - done;
        j.sample_offset = uint32_t(done);
        j.spp_norm = total;
        PassOpts po;
        po.guide = trained ? &s.guide : nullptr;
        po.keep_film = done > 0;
        render_jobs(s, {j}, desc, out, out_on_host, po);
        add_stats(agg, s.stats);
        ++passes;
    }
    check_guide_status(s);
    agg.render_ms += train_ms;
    agg.kernel_ms[WR_K_TRAIN] += train_ms;
    agg.kernel_count[WR_K_TRAIN] += steps;
    agg.kernel_items[WR_K_TRAIN] += records;
    agg.guide_records = records;
    agg.guide_steps = steps;
    agg.guide_train_ms = train_ms;
    agg.guide_loss = last_loss;
    agg.guide_passes = passes;
    s.stats = agg;
}

void render(wr_scene &s, const wr_render_desc *desc_in, double *out, bool out_on_host) {
    wr_render_desc desc{};
    if (desc_in) desc = *desc_in;
    if (desc.guiding) {
        render_guided(s, desc, out, out_on_host);
        return;
    }
    render_jobs(s, {scene_job(s.host, desc)}, desc, out, out_on_host);
}

void render_batch(wr_scene &s, const wr_job *jobs, int n, const wr_render_desc *desc_in, double *out, bool on_host) {
    if (n <= 0 || !jobs) throw Error(WR_ERR_INVALID_ARGUMENT, "empty job list");
    wr_render_desc desc{};
    if (desc_in) desc = *desc_in;
    std::vector<HostJob> hj;
    hj.reserve(size_t(n));
    for (int i = 0; i < n; ++i) {
        wr_render_desc d = desc;
        d.num_spp = jobs[i].num_spp;
        d.num_path_vertices = jobs[i].num_path_vertices;
        d.seed = jobs[i].seed;
        HostJob j = scene_job(s.host, d);
        if (jobs[i].camera_json) j.cam = wr::parse_camera_json(jobs[i].camera_json);
        hj.push_back(j);
    }
    render_jobs(s, hj, desc, out, on_host);
}

wrd::DevScene scene_for_queries(wr_scene &s) { return s.dev; }

void trace_batch(wr_scene &s, const float *rays, int n, int any_hit, std::vector<float> &out, unsigned long long *nv,
                 unsigned long long *nt) {
    if (n < 0 || (n > 0 && !rays)) throw Error(WR_ERR_INVALID_ARGUMENT, "bad ray batch");
    out.assign(size_t(n) * 12, 0.f);
    if (n == 0) return;
    DevBuf dr, dout, dvis;
    dr.alloc(size_t(n) * 32);
    dout.alloc(size_t(n) * 48);
    dvis.alloc(8);
    cudaStream_t st = s.stream;
    WR_CUDA(cudaMemcpyAsync(dr.p, rays, size_t(n) * 32, cudaMemcpyHostToDevice, st));
    WR_CUDA(cudaMemsetAsync(dvis.p, 0, 8, st));
    int sms = 148;
    WR_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s.device));
    const int grid = std::max(1, std::min(sms * 8, (n + wrd::kTraceBlock - 1) / wrd::kTraceBlock));
    wrk::launch_trace_batch(scene_for_queries(s), dr.as<float4>(), uint32_t(n), any_hit, dout.as<float4>(),
                            (nv || nt) ? dvis.as<uint32_t>() : nullptr, grid, st);
    WR_CUDA(cudaGetLastError());
    WR_CUDA(cudaMemcpyAsync(out.data(), dout.p, size_t(n) * 48, cudaMemcpyDeviceToHost, st));
    uint32_t vis[2] = {0, 0};
    WR_CUDA(cudaMemcpyAsync(vis, dvis.p, 8, cudaMemcpyDeviceToHost, st));
    WR_CUDA(cudaStreamSynchronize(st));
    if (nv) *nv = vis[0];
    if (nt) *nt = vis[1];
}

// build options checked, bvh_width 0 replaced by the default
wr_scene_options checked_options(const wr_scene_options *opts) {
    wr_scene_options o{};
    if (opts) o = *opts;
    if (o.bvh_builder != WR_BVH_HOST_SAH && o.bvh_builder != WR_BVH_DEVICE_LBVH)
        throw Error(WR_ERR_INVALID_ARGUMENT, "unknown bvh_builder");
    if (o.bvh_width == 0) o.bvh_width = WR_BVH_WIDTH_DEFAULT;
    if (o.bvh_width != 2 && o.bvh_width != 8) throw Error(WR_ERR_INVALID_ARGUMENT, "bvh_width must be 2 or 8");
    if (o.max_leaf < 0 || o.max_leaf > 16) throw Error(WR_ERR_INVALID_ARGUMENT, "max_leaf must be in 0..16");
    if (o.sah_trav_cost_milli < 0 || o.sah_trav_cost_milli > 100000)
        throw Error(WR_ERR_INVALID_ARGUMENT, "sah_trav_cost_milli must be in 0..100000");
    if (o.sah_patch_cost_milli < 0 || o.sah_patch_cost_milli > 1000000)
        throw Error(WR_ERR_INVALID_ARGUMENT, "sah_patch_cost_milli must be in 0..1000000");
    return o;
}

std::unique_ptr<wr_scene> create(wr::Scene &&host, const wr_scene_options *opts = nullptr) {
    std::unique_ptr<wr_scene> s(new wr_scene());
    s->opts = checked_options(opts);
    s->host = std::move(host);
    build_device_scene(*s);
    return s;
}

void run_scene(wr_scene &s) {
    const wr::Scene &h = s.host;
    for (size_t i = 0; i < h.renders.size(); ++i) {
        const wr::RenderEntry &re = h.renders[i];
        integrator_of(re.integrator);   // nextevent_path_tracer, primitive_path_tracer or light_splatting
        wr_render_desc d{};
        d.render_index = int(i);
        d.use_graph = 1;
        std::vector<double> img(size_t(h.camera.width) * h.camera.height * 3);
        render(s, &d, img.data(), true);
        if (!re.output.empty()) {
            const std::string out = re.output[0] == '/' ? re.output : h.base_dir + "/" + re.output;
            wr::write_pfm(out, img.data(), h.camera.width, h.camera.height);
        }
    }
}

}  // namespace

extern "C" {

const char *wr_last_error(void) { return g_last_error.c_str(); }

int wr_set_device(int device) {
    const cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) {
        g_last_error = std::string("cudaSetDevice: ") + cudaGetErrorString(e);
        return WR_ERR_CUDA;
    }
    return WR_OK;
}
int wr_abi_version(void) { return WR_ABI_VERSION; }

int wr_scene_create(const char *path, wr_scene **out) {
    if (!path || !out) { g_last_error = "null argument"; return WR_ERR_INVALID_ARGUMENT; }
    *out = nullptr;
    try {
        *out = create(wr::load_simple2_file(path)).release();
        return WR_OK;
    } catch (const Error &e) {
        return fail(e);
    } catch (const std::exception &e) {
        g_last_error = e.what();
        return WR_ERR_INVALID_ARGUMENT;
    }
}

int wr_scene_create_ex(const char *path, const wr_scene_options *opts, wr_scene **out) {
    if (!path || !out) { g_last_error = "null argument"; return WR_ERR_INVALID_ARGUMENT; }
    *out = nullptr;
    try {
        *out = create(wr::load_simple2_file(path), opts).release();
        return WR_OK;
    } catch (const Error &e) {
        return fail(e);
    } catch (const std::exception &e) {
        g_last_error = e.what();
        return WR_ERR_INVALID_ARGUMENT;
    }
}

int wr_scene_create_from_json(const char *json_text, const char *base_dir, wr_scene **out) {
    if (!json_text || !out) { g_last_error = "null argument"; return WR_ERR_INVALID_ARGUMENT; }
    *out = nullptr;
    try {
        *out = create(wr::load_simple2_text(json_text, base_dir ? base_dir : ".")).release();
        return WR_OK;
    } catch (const Error &e) {
        return fail(e);
    } catch (const std::exception &e) {
        g_last_error = e.what();
        return WR_ERR_INVALID_ARGUMENT;
    }
}

void wr_scene_destroy(wr_scene *s) { delete s; }

int wr_scene_inspect(const char *path, wr_scene_info *info) { return wr_scene_inspect_ex(path, nullptr, info); }

int wr_scene_inspect_ex(const char *path, const wr_scene_options *opts, wr_scene_info *info) {
    if (!path || !info) { g_last_error = "null argument"; return WR_ERR_INVALID_ARGUMENT; }
    try {
        const wr_scene_options o = checked_options(opts);
        if (o.bvh_builder != WR_BVH_HOST_SAH)
            throw Error(WR_ERR_UNSUPPORTED, "inspect builds the host SAH tree only (the LBVH is built on the device)");
        const auto t0 = std::chrono::steady_clock::now();
        wr::Scene h = wr::load_simple2_file(path);
        std::vector<float> verts;
        verts.reserve(size_t(h.num_triangles()) * 9);
        for (const wr::Mesh &m : h.meshes)
            for (uint32_t i : m.indices)
                for (int k = 0; k < 3; ++k) verts.push_back(m.positions[3 * size_t(i) + k]);
        const bool wide = o.bvh_width == 8;
        const int ml = o.max_leaf > 0 ? o.max_leaf : WR_MAX_LEAF_DEFAULT;
        const double ct = o.sah_trav_cost_milli > 0 ? o.sah_trav_cost_milli * 1e-3 : 1.0;
        wr::BvhBuildResult bvh = wr::build_bvh_sah(verts, wide ? std::min(ml, 3) : ml, 0, ct);
        int nodes = int(bvh.nodes.size() / 16);
        if (wide) {
            const wr::WideBvh wb = wr::build_wide8(bvh);
            nodes = int(wb.nodes.size() / 20);
            bvh.depth = wb.depth;
        }
        memset(info, 0, sizeof(*info));
        info->width = h.has_camera ? h.camera.width : 0;
        info->height = h.has_camera ? h.camera.height : 0;
        info->num_spp = h.renders.empty() ? 16 : h.renders[0].num_spp;
        info->num_path_vertices = h.renders.empty() ? 10 : h.renders[0].num_path_vertices;
        info->num_triangles = h.num_triangles();
        info->num_meshes = int(h.meshes.size());
        info->num_lights = int(h.lights.size());
        info->has_envmap = h.has_env ? 1 : 0;
        info->bvh_nodes = nodes;
        info->bvh_depth = bvh.depth;
        info->bvh_sah_cost = bvh.sah_cost;
        info->num_renders = int(h.renders.size());
        info->build_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        if (bvh.depth > wrd::kMaxStack) throw Error(WR_ERR_UNSUPPORTED, "BVH deeper than the traversal stack");
        return WR_OK;
    } catch (const Error &e) {
        return fail(e);
    } catch (const std::exception &e) {
        g_last_error = e.what();
        return WR_ERR_INVALID_ARGUMENT;
    }
}

int wr_scene_get_info(const wr_scene *s, wr_scene_info *info) {
    if (!s || !info) { g_last_error = "null argument"; return WR_ERR_INVALID_ARGUMENT; }
    memset(info, 0, sizeof(*info));
    const wr::Scene &h = s->host;
    info->width = h.has_camera ? h.camera.width : 0;
    info->height = h.has_camera ? h.camera.height : 0;
    info->num_spp = h.renders.empty() ? 16 : h.renders[0].num_spp;
    info->num_path_vertices = h.renders.empty() ? 10 : h.renders[0].num_path_vertices;
    info->num_triangles = h.num_triangles();
    info->num_meshes = int(h.meshes.size());
    info->num_lights = int(h.lights.size());
    info->has_envmap = h.has_env ? 1 : 0;
    info->bvh_nodes = s->bvh_nodes;
    info->bvh_depth = s->bvh_depth;
    info->bvh_sah_cost = s->sah_cost;
    info->build_ms = s->build_ms;
    info->num_renders = int(h.renders.size());
    info->bvh_builder = s->opts.bvh_builder;
    info->bvh_ms = s->bvh_ms;
    return WR_OK;
}

int wr_scene_set_camera_json(wr_scene *s, const char *camera_json) {
    if (!s || !camera_json) { g_last_error = "null argument"; return WR_ERR_INVALID_ARGUMENT; }
    try {
        s->host.camera = wr::parse_camera_json(camera_json);
        s->host.has_camera = true;
        return WR_OK;
    } catch (const Error &e) {
        return fail(e);
    }
}

int wr_render(wr_scene *s, const wr_render_desc *desc, double *out_rgb) {
    if (!s || !out_rgb) { g_last_error = "null argument"; return WR_ERR_INVALID_ARGUMENT; }
    try {
        render(*s, desc, out_rgb, true);
        return WR_OK;
    } catch (const Error &e) {
        return fail(e);
    }
}

int wr_render_device(wr_scene *s, const wr_render_desc *desc, double *out_rgb_device) {
    if (!s || !out_rgb_device) { g_last_error = "null argument"; return WR_ERR_INVALID_ARGUMENT; }
    try {
        render(*s, desc, out_rgb_device, false);
        return WR_OK;
    } catch (const Error &e) {
        return fail(e);
    }
}

int wr_render_batch(wr_scene *s, const wr_job *jobs, int n, const wr_render_desc *desc, double *out_rgb) {
    if (!s || !out_rgb) { g_last_error = "null argument"; return WR_ERR_INVALID_ARGUMENT; }
    try {
        render_batch(*s, jobs, n, desc, out_rgb, true);
        return WR_OK;
    } catch (const Error &e) {
        return fail(e);
    }
}

int wr_render_batch_device(wr_scene *s, const wr_job *jobs, int n, const wr_render_desc *desc, double *out_rgb_device) {
    if (!s || !out_rgb_device) { g_last_error = "null argument"; return WR_ERR_INVALID_ARGUMENT; }
    try {
        render_batch(*s, jobs, n, desc, out_rgb_device, false);
        return WR_OK;
    } catch (const Error &e) {
        return fail(e);
    }
}

}  // extern "C"

namespace {

// Coordinate descent over the wavefront knobs: traversal block size, wavefront capacity,
// persistent-CTA counts of the traversal and shading kernels, dynamic-fetch threshold. `probe`
// renders once with a candidate and returns its device time (ms); each candidate is scored by
// the mean of two probes after a warm-up probe. A setting replaces the current one only when it
// is 2 % faster: smaller differences are within the run-to-run spread of a probe render.
template <class Probe>
wr_render_desc tune_knobs(wr_scene &s, wr_render_desc cur, Probe probe, double *best_ms) {
    constexpr double kTuneMargin = 0.98;
    int sms = 148;
    WR_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s.device));
    auto trial = [&](const wr_render_desc &d) {
        probe(d);   // warm (allocations, caches)
        return 0.5 * (probe(d) + probe(d));
    };
    double bt = trial(cur);
    // 1) traversal block size (its persistent grid follows the occupancy of that size)
    for (int blk : {64, 128, 256}) {
        wr_render_desc d = cur;
        d.trace_block = blk;
        d.grid_trace = 0;
        const double t = trial(d);
        if (t < bt * kTuneMargin) { bt = t; cur = d; }
    }
    // 2) wavefront capacity
    for (int cap : {1 << 19, 1 << 20, 1 << 21, 1 << 22}) {
        wr_render_desc d = cur;
        d.queue_capacity = cap;
        const double t = trial(d);
        if (t < bt * kTuneMargin) { bt = t; cur = d; }
    }
    // 3) persistent-CTA count of the traversal and shading kernels
    const int blk = (cur.trace_block == 64 || cur.trace_block == 256) ? cur.trace_block : 128;
    const int occ_t = sms * std::max(1, wrk::occupancy_blocks(0, blk, s.dev.patches != nullptr, s.dev.wnodes != nullptr));
    const int occ_s = sms * std::max(1, wrk::occupancy_blocks(1));
    for (double f : {0.5, 1.0}) {
        wr_render_desc d = cur;
        d.grid_trace = std::max(sms, int(occ_t * f));
        const double t = trial(d);
        if (t < bt * kTuneMargin) { bt = t; cur = d; }
    }
    for (double f : {0.5, 1.0}) {
        wr_render_desc d = cur;
        d.grid_shade = std::max(sms, int(occ_s * f));
        const double t = trial(d);
        if (t < bt * kTuneMargin) { bt = t; cur = d; }
    }
    // 4) dynamic ray fetching threshold
    for (int th : {12, 16, 24, 28}) {
        wr_render_desc d = cur;
        d.fetch_threshold = th;
        const double t = trial(d);
        if (t < bt * kTuneMargin) { bt = t; cur = d; }
    }
    if (best_ms) *best_ms = bt;
    return cur;
}

}  // namespace

extern "C" {

int wr_autotune(wr_scene *s, const wr_render_desc *base, int probe_spp, wr_render_desc *best, double *best_ms) {
    if (!s || !best) { g_last_error = "null argument"; return WR_ERR_INVALID_ARGUMENT; }
    try {
        wr_render_desc cur{};
        if (base) cur = *base;
        cur.num_spp = probe_spp > 0 ? probe_spp : 4;
        cur.profile = 0;
        const wr::Camera &c = s->host.camera;
        if (!s->host.has_camera) throw Error(WR_ERR_INVALID_ARGUMENT, "scene has no camera");
        DevBuf out;
        out.alloc(size_t(c.width) * c.height * 3 * 8);
        auto probe = [&](const wr_render_desc &d) {
            render(*s, &d, out.as<double>(), false);
            return s->stats.render_ms;
        };
        *best = tune_knobs(*s, cur, probe, best_ms);
        if (base) { best->num_spp = base->num_spp; best->profile = base->profile; }
        else { best->num_spp = 0; }
        return WR_OK;
    } catch (const Error &e) {
        return fail(e);
    }
}

int wr_autotune_batch(wr_scene *s, const wr_job *jobs, int n, const wr_render_desc *base, wr_render_desc *best,
                      double *best_ms) {
    if (!s || !best || !jobs || n <= 0) { g_last_error = "null argument or empty job list"; return WR_ERR_INVALID_ARGUMENT; }
    try {
        wr_render_desc cur{};
        if (base) cur = *base;
        cur.profile = 0;
        size_t pix = 0;
        for (int i = 0; i < n; ++i) {
            const wr::Camera c = jobs[i].camera_json ? wr::parse_camera_json(jobs[i].camera_json) : s->host.camera;
            pix += size_t(c.width) * size_t(c.height);
        }
        DevBuf out;
        out.alloc(pix * 3 * 8);
        auto probe = [&](const wr_render_desc &d) {
            render_batch(*s, jobs, n, &d, out.as<double>(), false);
            return s->stats.render_ms;
        };
        *best = tune_knobs(*s, cur, probe, best_ms);
        if (base) best->profile = base->profile;
        return WR_OK;
    } catch (const Error &e) {
        return fail(e);
    }
}

int wr_get_render_stats(const wr_scene *s, wr_render_stats *st) {
    if (!s || !st) { g_last_error = "null argument"; return WR_ERR_INVALID_ARGUMENT; }
    *st = s->stats;
    return WR_OK;
}

// ---- learned guiding proposal ----
int wr_guide_reset(wr_scene *s, unsigned int seed) {
    if (!s) { g_last_error = "null argument"; return WR_ERR_INVALID_ARGUMENT; }
    try {
        ensure_guide(*s);
        wrg::guide_init(s->guide, seed, s->stream);
        s->guide_step = 0;
        WR_CUDA(cudaStreamSynchronize(s->stream));
        return WR_OK;
    } catch (const Error &e) {
        return fail(e);
    }
}

int wr_guide_get_params(wr_scene *s, float *params) {
    if (!s || !params) { g_last_error = "null argument"; return WR_ERR_INVALID_ARGUMENT; }
    try {
        ensure_guide(*s);
        wrg::guide_get_master(s->guide, params, s->stream);
        return WR_OK;
    } catch (const Error &e) {
        return fail(e);
    }
}

int wr_guide_set_params(wr_scene *s, const float *params) {
    if (!s || !params) { g_last_error = "null argument"; return WR_ERR_INVALID_ARGUMENT; }
    try {
        ensure_guide(*s);
        wrg::guide_set_master(s->guide, params, s->stream);
        WR_CUDA(cudaStreamSynchronize(s->stream));
        return WR_OK;
    } catch (const Error &e) {
        return fail(e);
    }
}

int wr_guide_box(const wr_scene *s, float lo[3], float inv_extent[3]) {
    if (!s || !lo || !inv_extent) { g_last_error = "null argument"; return WR_ERR_INVALID_ARGUMENT; }
    for (int k = 0; k < 3; ++k) {
        lo[k] = s->box_lo[k];
        inv_extent[k] = s->box_inv[k];
    }
    return WR_OK;
}

int wr_guide_eval(wr_scene *s, const float *rows, int n, float *lobes) {
    if (!s || n < 0 || (n > 0 && (!rows || !lobes))) { g_last_error = "null argument"; return WR_ERR_INVALID_ARGUMENT; }
    if (n == 0) return WR_OK;
    try {
        ensure_guide(*s);
        cudaStream_t st = s->stream;
        s->g_scratch.alloc(size_t(n) * 9 * 4);
        s->g_scratch2.alloc(size_t(n) * wrg::kLobeFloat4 * 16);
        WR_CUDA(cudaMemcpyAsync(s->g_scratch.p, rows, size_t(n) * 9 * 4, cudaMemcpyHostToDevice, st));
        wrg::guide_infer_rows(s->guide, s->g_scratch.as<float>(), uint32_t(n), s->g_scratch2.as<float4>(), sm_count(*s),
                              st);
        std::vector<float4> out(size_t(n) * wrg::kLobeFloat4);
        WR_CUDA(cudaMemcpyAsync(out.data(), s->g_scratch2.p, out.size() * 16, cudaMemcpyDeviceToHost, st));
        WR_CUDA(cudaStreamSynchronize(st));
        check_guide_status(*s);
        for (int i = 0; i < n; ++i) {
            const float4 *L = &out[size_t(i) * wrg::kLobeFloat4];
            float *o = lobes + 40 * size_t(i);
            for (int k = 0; k < 8; ++k) {
                o[4 * k + 0] = L[k].x;
                o[4 * k + 1] = L[k].y;
                o[4 * k + 2] = L[k].z;
                o[4 * k + 3] = L[k].w;
            }
            const float w[8] = {L[8].x, L[8].y, L[8].z, L[8].w, L[9].x, L[9].y, L[9].z, L[9].w};
            for (int k = 0; k < 8; ++k) o[32 + k] = w[k];
        }
        return WR_OK;
    } catch (const Error &e) {
        return fail(e);
    }
}

int wr_guide_gradient(wr_scene *s, const float *records, int n, float c_max, float *grad, double *loss) {
    if (!s || !grad || n < 0 || (n > 0 && !records)) { g_last_error = "null argument"; return WR_ERR_INVALID_ARGUMENT; }
    try {
        ensure_guide(*s);
        cudaStream_t st = s->stream;
        s->g_scratch.alloc(std::max<size_t>(size_t(n), 1) * wrg::kRecordFloat4 * 16);
        s->g_loss.alloc(16);
        if (n) WR_CUDA(cudaMemcpyAsync(s->g_scratch.p, records, size_t(n) * 80, cudaMemcpyHostToDevice, st));
        WR_CUDA(cudaMemsetAsync(s->g_loss.p, 0, 8, st));
        const int nslots = wrg::guide_gradient(s->guide, s->g_scratch.as<float4>(), uint32_t(n), 0, uint32_t(n), 1u,
                                               c_max, s->g_loss.as<double>(), st);
        wrg::guide_sum_gradient(s->guide, nslots, st);
        WR_CUDA(cudaMemcpyAsync(grad, s->guide.grad, size_t(wrg::kGuideParams) * 4, cudaMemcpyDeviceToHost, st));
        double l = 0.0;
        WR_CUDA(cudaMemcpyAsync(&l, s->g_loss.p, 8, cudaMemcpyDeviceToHost, st));
        WR_CUDA(cudaStreamSynchronize(st));
        check_guide_status(*s);
        if (loss) *loss = l;
        return WR_OK;
    } catch (const Error &e) {
        return fail(e);
    }
}

int wr_guide_train(wr_scene *s, const float *records, int n, int steps, int batch, float lr, double *loss_per_step) {
    if (!s || n < 0 || (n > 0 && !records) || steps < 0 || batch <= 0) {
        g_last_error = "invalid argument";
        return WR_ERR_INVALID_ARGUMENT;
    }
    if (n == 0 || steps == 0) return WR_OK;
    try {
        ensure_guide(*s);
        cudaStream_t st = s->stream;
        s->g_scratch.alloc(size_t(n) * wrg::kRecordFloat4 * 16);
        WR_CUDA(cudaMemcpyAsync(s->g_scratch.p, records, size_t(n) * 80, cudaMemcpyHostToDevice, st));
        std::vector<double> per;
        train_records(*s, s->g_scratch.as<float4>(), uint32_t(n), uint32_t(batch), steps, lr, wrg::kCMax, &per,
                      nullptr);
        if (loss_per_step)
            for (int k = 0; k < steps && k < int(per.size()); ++k) loss_per_step[k] = per[size_t(k)];
        return WR_OK;
    } catch (const Error &e) {
        return fail(e);
    }
}

int wr_trace_closest(wr_scene *s, const float *rays, int n, int *geom_id, int *prim_id, float *t, float *uv) {
    if (!s || (n > 0 && (!geom_id || !prim_id || !t))) { g_last_error = "null argument"; return WR_ERR_INVALID_ARGUMENT; }
    try {
        std::vector<float> out;
        trace_batch(*s, rays, n, 0, out, nullptr, nullptr);
        for (int i = 0; i < n; ++i) {
            const float *o = &out[12 * size_t(i)];
            uint32_t g, p;
            memcpy(&g, &o[0], 4);
            memcpy(&p, &o[1], 4);
            geom_id[i] = g == wrd::MISS ? -1 : int(g);
            prim_id[i] = p == wrd::MISS ? -1 : int(p);
            t[i] = o[2];
            if (uv) { uv[2 * i] = o[4]; uv[2 * i + 1] = o[5]; }
        }
        return WR_OK;
    } catch (const Error &e) {
        return fail(e);
    }
}

int wr_trace_hits(wr_scene *s, const float *rays, int n, int *geom_id, int *prim_id, float *t, float *normal) {
    if (!s || (n > 0 && (!geom_id || !prim_id || !t || !normal))) {
        g_last_error = "null argument";
        return WR_ERR_INVALID_ARGUMENT;
    }
    try {
        std::vector<float> out;
        trace_batch(*s, rays, n, 0, out, nullptr, nullptr);
        for (int i = 0; i < n; ++i) {
            const float *o = &out[12 * size_t(i)];
            uint32_t g, p;
            memcpy(&g, &o[0], 4);
            memcpy(&p, &o[1], 4);
            geom_id[i] = g == wrd::MISS ? -1 : int(g);
            prim_id[i] = p == wrd::MISS ? -1 : int(p);
            t[i] = o[2];
            for (int k = 0; k < 3; ++k) normal[3 * i + k] = o[8 + k];
        }
        return WR_OK;
    } catch (const Error &e) {
        return fail(e);
    }
}

int wr_trace_occluded(wr_scene *s, const float *rays, int n, int *occluded) {
    if (!s || (n > 0 && !occluded)) { g_last_error = "null argument"; return WR_ERR_INVALID_ARGUMENT; }
    try {
        std::vector<float> out;
        trace_batch(*s, rays, n, 1, out, nullptr, nullptr);
        for (int i = 0; i < n; ++i) {
            uint32_t g;
            memcpy(&g, &out[12 * size_t(i)], 4);
            occluded[i] = g == wrd::MISS ? 0 : 1;
        }
        return WR_OK;
    } catch (const Error &e) {
        return fail(e);
    }
}

int wr_trace_stats(wr_scene *s, const float *rays, int n, int any_hit, unsigned long long *node_visits,
                   unsigned long long *tri_tests) {
    if (!s || !node_visits || !tri_tests) { g_last_error = "null argument"; return WR_ERR_INVALID_ARGUMENT; }
    try {
        std::vector<float> out;
        trace_batch(*s, rays, n, any_hit, out, node_visits, tri_tests);
        return WR_OK;
    } catch (const Error &e) {
        return fail(e);
    }
}

int wr_write_pfm(const char *path, const double *rgb, int width, int height) {
    if (!path || !rgb || width <= 0 || height <= 0) { g_last_error = "bad argument"; return WR_ERR_INVALID_ARGUMENT; }
    try {
        wr::write_pfm(path, rgb, width, height);
        return WR_OK;
    } catch (const Error &e) {
        return fail(e);
    }
}

int wr_read_image(const char *path, int *width, int *height, float *rgb) {
    if (!path || !width || !height) { g_last_error = "null argument"; return WR_ERR_INVALID_ARGUMENT; }
    try {
        int w = 0, h = 0;
        const std::vector<float> img = wr::read_image(path, &w, &h);
        *width = w;
        *height = h;
        if (rgb) memcpy(rgb, img.data(), img.size() * sizeof(float));
        return WR_OK;
    } catch (const Error &e) {
        return fail(e);
    }
}

int wr_run_simple2(const char *path) {
    wr_scene *s = nullptr;
    int rc = wr_scene_create(path, &s);
    if (rc != WR_OK) return rc;
    try {
        run_scene(*s);
        wr_scene_destroy(s);
        return WR_OK;
    } catch (const Error &e) {
        wr_scene_destroy(s);
        return fail(e);
    }
}

int wr_run_jsimple2(const char *json_text) {
    wr_scene *s = nullptr;
    int rc = wr_scene_create_from_json(json_text, ".", &s);
    if (rc != WR_OK) return rc;
    try {
        run_scene(*s);
        wr_scene_destroy(s);
        return WR_OK;
    } catch (const Error &e) {
        wr_scene_destroy(s);
        return fail(e);
    }
}

}  // extern "C"

// ------------------------------------------------------------------------------------------
// Read-only view of a scene handle for other translation units of this library.
namespace wr_internal {

struct SceneView {
    wrd::DevScene dev;
    cudaStream_t stream;
    int device;
    uint32_t *pinned;
    cudaEvent_t ev0, ev1;
    const wr::Scene *host;
    wr_render_stats *stats;
};

bool scene_view(wr_scene *s, SceneView *v) {
    if (!s || !v) return false;
    v->dev = s->dev;
    v->stream = s->stream;
    v->device = s->device;
    v->pinned = s->pinned;
    v->ev0 = s->ev0;
    v->ev1 = s->ev1;
    v->host = &s->host;
    v->stats = &s->stats;
    return true;
}

wrd::DevCamera camera_constants(const wr::Camera &c) { return make_camera(c); }

int resolve_request(const wr::Scene &h, const wr_render_desc &desc, int *spp, int *nverts, int *integrator) {
    try {
        const HostJob j = scene_job(h, desc);
        *spp = j.spp;
        *nverts = j.nverts;
        *integrator = j.integrator;
        return WR_OK;
    } catch (const Error &e) {
        return fail(e);
    }
}

void set_last_error(const std::string &m) { g_last_error = m; }

}  // namespace wr_internal
