// Test infrastructure only: drives the reference's own `nextevent_path_tracer`
// code, compiled from its sources, so that the oracle can be checked against
// the reference itself. Built by oracle/Makefile into oracle/_ref/wurst_ref.
//
// It reproduces Simple2Parser::Parse / ParseScene (src/sceneio/simple2parser.h:
// 27-68,102-223) with the reference's own classes -- ThinlensCamera,
// PathNeeRenderer, PrimitivePathRenderer, EmbreeAccel, TriangleMeshGeometry, DiffuseAreaLight,
// EnvmapLight/EquiRectRep, the Lambert/Oren-Nayar/Phong/Mixed/TwoSided BSDFs,
// Film, FimageIo -- and only replaces the two third-party libraries that
// need cmake to build:
//   * Assimp's OBJ import: meshes come from the oracle's OBJ/MTL reader
//     (oracle/oracle_scene.h) and are turned into BSDFs and lights with the
//     mapping of AssimpInOut::LoadFromObj (src/sceneio/meshio/assimpio.h:79-150),
//     "mitsuba_srgb" converting Kd and Ks through the reference's own
//     SpectrumConvertUtil::SpectrumFromSrgb as AimatToTexture does (:287-337);
//     the "oren_nayar_sigma" mesh key selects OrenNayarBsdf for the diffuse part;
//   * Embree: see embree_shim.cpp.
//
// Usage:
//   wurst_ref render <scene.json> <out.pfm> [--spp N] [--vertices V] [--salt S]
//            [--crop x0 y0 x1 y1] [--serial] [--threads T] [--raw out.f64] [--camera '<json>']
//   wurst_ref trace <scene.json> <rays.f32> <hits.bin>
//   wurst_ref trace2 <scene.json> <rays.f32> <hits.bin>   (any geometry type; 8 words per ray)
//   wurst_ref imgload <image.pfm|.hdr|.exr> <out.bin>     (the reference's FimageIo::Load)
// `render` without --crop/--serial calls PathNeeRenderer::render() itself
// (all hardware threads). --serial/--crop run the same per-tile loop as
// render() (pathnextevent.h:152-191) over the selected tiles on --threads
// threads (default one), calling the reference's evalContribution and Film.
// Prints one JSON line: {"seconds": render time, "paths": samples traced, ...}.

#include "common/wurst.h"
#include "common/util/json.h"
#include "renderer/pathnextevent.h"
#include "renderer/primitivepath.h"
#include "renderer/lightsplatting.h"
#include "camera/thinlens.h"
#include "bsdf/lambertdiffuse.h"
#include "bsdf/orennayar.h"
#include "bsdf/phong.h"
#include "bsdf/mixed.h"
#include "bsdf/twosided.h"
#include "geometry/phongmesh.h"
#include "light/diffusearealight.h"
#include "light/envmap.h"
#include "sphericalrepresentation/equirectangular.h"
#include "texture/constanttexture.h"
#include "sampler/randomsampler.h"

#include <chrono>
#include <cstdio>

#include "../oracle_scene.h"

namespace {

struct SaltedSampler : public RandomSampler {
    explicit SaltedSampler(unsigned salt) : RandomSampler(0), mSalt(salt) {}
    shared_ptr<Sampler> clone(const int seed) const override {
        shared_ptr<RandomSampler> r = make_shared<RandomSampler>(seed);
        r->mRng.mGenerator64.seed(uint64_t(unsigned(seed) + mSalt * 0x9E3779B1u));
        return r;
    }
    unsigned mSalt;
};

struct Loaded {
    shared_ptr<const Scene> scene;
    shared_ptr<const Camera> camera;
    json root;
    filesystem::path dir;
};

shared_ptr<const Scene> parse_scene(const json &meshesJson, const shared_ptr<EnvmapLight> &envmap, const filesystem::path &dir) {
    shared_ptr<EmbreeAccel> accel = make_shared<EmbreeAccel>();
    std::vector<shared_ptr<const Geometry>> geometries, lightGeometries;
    for (const json &mj : meshesJson) {
        const std::string rel = Util::Json::GetValue<std::string>(mj, "path", "");
        const bool doUsePhongTessellation = Util::Json::GetValue<bool>(mj, "phong_tessellation", false);
        const bool doSrgbConversionTheMitsubaWay = Util::Json::GetValue<bool>(mj, "mitsuba_srgb", false);
        oracle::ObjFile of = oracle::load_obj((dir / rel).string(), doUsePhongTessellation);
        std::map<std::string, double> sigma;
        if (mj.find("oren_nayar_sigma") != mj.end())
            for (auto it = mj["oren_nayar_sigma"].begin(); it != mj["oren_nayar_sigma"].end(); ++it)
                sigma[it.key()] = it.value().get<double>();
        std::vector<shared_ptr<const Bsdf>> bsdfs;
        std::vector<shared_ptr<Light>> areaLights;
        for (const oracle::ObjMaterial &om : of.materials) {
            // AimatToTexture (assimpio.h:287-337): Kd and Ks through the reference's own
            // SpectrumFromSrgb when the entry asks for it, Ke never
            auto color = [&](const double *c) {
                return doSrgbConversionTheMitsubaWay ? SpectrumConvertUtil::SpectrumFromSrgb(c[0], c[1], c[2])
                                                     : SpectrumConvertUtil::SpectrumFromRgb(c[0], c[1], c[2]);
            };
            auto kdT = make_shared<ConstantTexture<Spectrum>>(color(om.kd));
            auto ksT = make_shared<ConstantTexture<Spectrum>>(color(om.ks));
            auto keT = make_shared<ConstantTexture<Spectrum>>(SpectrumConvertUtil::SpectrumFromRgb(om.ke[0], om.ke[1], om.ke[2]));
            auto nT = make_shared<ConstantTexture<double>>(om.ns / 4.0);
            if (!Math::IsZero(keT->average())) {
                if (nT->average() != 0.0) throw std::runtime_error("SimpleMetal area light is out of scope");
                areaLights.push_back(make_shared<DiffuseAreaLight>(keT));
            } else {
                areaLights.push_back(nullptr);
            }
            shared_ptr<const Bsdf> diffuse;
            auto sit = sigma.find(om.name);
            if (sit != sigma.end())
                diffuse = make_shared<const OrenNayarBsdf>(kdT, make_shared<ConstantTexture<Spectrum>>(Spectrum(sit->second)));
            else
                diffuse = make_shared<const LambertDiffuseBsdf>(kdT);
            shared_ptr<const Bsdf> glossy = make_shared<const PhongBsdf>(ksT, nT);
            if (Math::IsZero(kdT->average())) bsdfs.push_back(make_shared<const TwoSidedBsdf>(glossy));
            else if (Math::IsZero(ksT->average())) bsdfs.push_back(make_shared<const TwoSidedBsdf>(diffuse));
            else {
                std::vector<shared_ptr<const Bsdf>> two{diffuse, glossy};
                bsdfs.push_back(make_shared<const TwoSidedBsdf>(make_shared<const MixedBsdf>(two)));
            }
        }
        std::vector<shared_ptr<TriangleMeshGeometry>> geoms, lights;
        for (const oracle::ObjMesh &om : of.meshes) {
            if (doUsePhongTessellation && om.missing_normals && areaLights[om.material] == nullptr)
                throw std::runtime_error("phong_tessellation mesh without per-vertex normals");
            auto tm = make_shared<TriangleMeshGeometry>();
            const size_t nv = om.positions.size() / 3;
            for (size_t k = 0; k < nv; ++k) {
                tm->mPositions.emplace_back(om.positions[3 * k], om.positions[3 * k + 1], om.positions[3 * k + 2]);
                tm->mTextureCoords.emplace_back(0, 0);
                if (!om.normals.empty()) {   // assimpio.h:211-223
                    const float x = om.normals[3 * k], y = om.normals[3 * k + 1], z = om.normals[3 * k + 2];
                    if (Math::IsApprox(Math::Length(Vec3(x, y, z)), 0.0)) tm->mNormals.emplace_back(Vec3(0.0, 0.0, 0.0));
                    else tm->mNormals.emplace_back(Math::Normalize(Vec3(x, y, z)));
                }
            }
            for (size_t t = 0; t < om.triangles.size(); t += 3)
                tm->mTriangles.emplace_back(om.triangles[t], om.triangles[t + 1], om.triangles[t + 2]);
            if (areaLights[om.material] != nullptr) {
                tm->mAreaLight = areaLights[om.material];
                tm->precomputeForSampling();
                lights.push_back(tm);
            } else {
                tm->mBsdf = bsdfs[om.material];
                tm->mAlpha = nullptr;
                geoms.push_back(tm);
            }
        }
        // Simple2Parser::ParseScene (simple2parser.h:37-58): surfaces of a phong_tessellation
        // entry become PhongMeshGeometry user geometry, emitters stay triangle meshes
        for (auto &p : geoms) {
            if (doUsePhongTessellation) {
                shared_ptr<PhongMeshGeometry> q = make_shared<PhongMeshGeometry>();
                std::swap(q->mPositions, p->mPositions);
                std::swap(q->mNormals, p->mNormals);
                std::swap(q->mTextureCoords, p->mTextureCoords);
                std::swap(q->mTriangles, p->mTriangles);
                q->mAlpha = p->mAlpha;
                q->mBsdf = p->mBsdf;
                q->mMediumBackface = p->mMediumBackface;
                q->mMediumFrontface = p->mMediumFrontface;
                accel->addUserGeometry(q);
            } else {
                accel->addGeometry(p);
            }
        }
        for (auto &p : lights) accel->addGeometry(p);
        geometries.insert(geometries.end(), geoms.begin(), geoms.end());
        lightGeometries.insert(lightGeometries.end(), lights.begin(), lights.end());
    }
    accel->commit();
    return make_shared<const Scene>(accel, geometries, lightGeometries, envmap);
}

Loaded load(const std::string &path, const std::string &camera_override) {
    Loaded L;
    filesystem::path full = Util::File::MakeAbsolutePath(filesystem::path(path));
    std::ifstream ifs(full);
    if (!ifs.is_open()) throw std::runtime_error("file not found " + full.string());
    ifs >> L.root;
    L.dir = full.parent_path();
    shared_ptr<EnvmapLight> envmapLight = nullptr;
    const std::string envmapPath = Util::Json::GetValue<std::string>(L.root, "envmap", "");
    if (envmapPath != "") {
        Fimage<Spectrum> img = FimageIo::Load(L.dir / envmapPath);
        shared_ptr<const SphRep<Spectrum>> rep = make_shared<const EquiRectRep<Spectrum>>(img, true);
        envmapLight = make_shared<EnvmapLight>(rep);
    }
    L.scene = parse_scene(L.root["meshes"], envmapLight, L.dir);
    json camJson = camera_override.empty() ? L.root["camera"] : json::parse(camera_override);
    L.camera = ThinlensCamera::FromSimple2ParseJson(camJson);
    return L;
}

struct TileB { Ivec2 lo, hi; };

void gen_blocks(const Ivec2 &start, const Ivec2 &end, std::vector<TileB> &out) {
    // the block list of Parallel::Split2d (parallel.h:72-104), collected instead of enqueued
    const int B = int(Parallel::DefaultBlock2dSize);
    const Ivec2 size = end - start;
    const int maxE = std::max(size[0], size[1]);
    if (maxE <= B) { if (std::min(size[0], size[1]) != 0) out.push_back({start, end}); }
    else if (maxE == size[0]) {
        const int hx = start[0] + std::min(Math::DivAndCeil(size[0], B) / 2 * B, size[0]);
        gen_blocks(start, Ivec2(hx, end[1]), out); gen_blocks(Ivec2(hx, start[1]), end, out);
    } else {
        const int hy = start[1] + std::min(Math::DivAndCeil(size[1], B) / 2 * B, size[1]);
        gen_blocks(start, Ivec2(end[0], hy), out); gen_blocks(Ivec2(start[0], hy), end, out);
    }
}

int cmd_render(int argc, char **argv) {
    const std::string scenePath = argv[2], outPath = argv[3];
    int spp = -1, nverts = -1, renderIndex = 0;
    unsigned salt = 0;
    bool serial = false, crop = false;
    int threads = 1;
    int cx0 = 0, cy0 = 0, cx1 = 0, cy1 = 0;
    std::string raw, cam;
    for (int i = 4; i < argc; ++i) {
        std::string a = argv[i];
        if (a == "--spp") spp = atoi(argv[++i]);
        else if (a == "--vertices") nverts = atoi(argv[++i]);
        else if (a == "--salt") salt = unsigned(strtoul(argv[++i], nullptr, 10));
        else if (a == "--serial") serial = true;
        else if (a == "--raw") raw = argv[++i];
        else if (a == "--camera") cam = argv[++i];
        else if (a == "--render-index") renderIndex = atoi(argv[++i]);
        else if (a == "--threads") threads = std::max(1, atoi(argv[++i]));
        else if (a == "--crop") { crop = true; cx0 = atoi(argv[++i]); cy0 = atoi(argv[++i]); cx1 = atoi(argv[++i]); cy1 = atoi(argv[++i]); }
        else throw std::runtime_error("unknown option " + a);
    }
    auto tl0 = std::chrono::steady_clock::now();
    Loaded L = load(scenePath, cam);
    const double loadSeconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - tl0).count();
    json rj = L.root["render"][renderIndex];
    const bool primitive = rj["integrator"] == "primitive_path_tracer";
    const bool splatting = rj["integrator"] == "light_splatting";
    if (rj["integrator"] != "nextevent_path_tracer" && !primitive && !splatting)
        throw std::runtime_error("integrator is not nextevent_path_tracer, primitive_path_tracer or light_splatting");
    if (splatting && (serial || crop))
        throw std::runtime_error("light_splatting runs through LightSplattingRenderer::render() only (no --serial/--crop)");
    if (spp > 0) rj["num_spp"] = spp;
    if (nverts > 0) rj["num_path_vertices"] = nverts;
    shared_ptr<Sampler> sampler = make_shared<SaltedSampler>(salt);
    shared_ptr<const Camera> camera = L.camera;
    shared_ptr<const Scene> scene = L.scene;
    shared_ptr<PathNeeRenderer> r;
    shared_ptr<PrimitivePathRenderer> rp;
    shared_ptr<LightSplattingRenderer> rs;
    if (primitive) rp = PrimitivePathRenderer::FromSimple2Json(camera, scene, sampler, rj, L.dir);
    else if (splatting) rs = LightSplattingRenderer::FromSimple2Json(camera, scene, sampler, rj, L.dir);
    else r = PathNeeRenderer::FromSimple2Json(camera, scene, sampler, rj, L.dir);
    const int numSpp = primitive ? rp->mNumSpp : splatting ? rs->mNumSamples : r->mNumSpp;
    const int numVerts = primitive ? rp->mNumPathVertices : splatting ? rs->mNumPathVertices : r->mNumPathVertices;
    const Ivec2 res = camera->mFilm->mResolution;
    const int W = res[0], H = res[1];
    long long paths = 0;
    auto t0 = std::chrono::steady_clock::now();
    std::vector<double> img(size_t(W) * H * 3);
    if (!serial && !crop) {
        if (primitive) rp->render(); else if (splatting) rs->render(); else r->render();
        paths = (long long)W * H * numSpp;
        Fimage<Spectrum> im = camera->mFilm->getImage();
        for (int y = 0; y < H; ++y)
            for (int x = 0; x < W; ++x)
                for (int c = 0; c < 3; ++c) img[3 * (size_t(y) * W + x) + c] = im.at(x, y)[c];
    } else {
        if (!crop) { cx0 = 0; cy0 = 0; cx1 = W; cy1 = H; }
        Film &film = *camera->mFilm;
        if (!primitive) film.requestAtomicBuffer();
        film.requestBaseBuffer();
        std::vector<TileB> blocks, sel;
        gen_blocks(Ivec2(0, 0), res, blocks);
        long long npix = 0;
        for (const TileB &b : blocks)
            if (b.lo[0] < cx1 && b.hi[0] > cx0 && b.lo[1] < cy1 && b.hi[1] > cy0) {
                sel.push_back(b);
                npix += (long long)(b.hi[0] - b.lo[0]) * (b.hi[1] - b.lo[1]);
            }
        film.mBaseScalingFactor = 1.0 / double(numSpp);
        film.mAtomicScalingFactor = 1.0 / double(numSpp) / double(npix);
        if (primitive || numVerts > 1) {
            std::atomic<size_t> next(0);
            auto worker = [&]() {
                for (size_t ti = next++; ti < sel.size(); ti = next++) {
                    const TileB &b = sel[ti];
                    const Ibound2 bound(b.lo, b.hi);
                    const int tileSeed = bound.pMin[0] * H + bound.pMin[1];
                    shared_ptr<Sampler> ts = sampler->clone(tileSeed);
                    for (const Ivec2 pixel : bound) {
                        ts->setPixel(pixel);
                        for (int i = 0; i < numSpp; ++i) {
                            if (primitive) {
                                Splat sp;
                                rp->evalContribution(&sp, ts.get(), pixel);
                                film.addSample(sp.mRaster, sp.mContrib);
                            } else {
                                Splat splats[2];
                                r->evalContribution(splats, ts.get(), pixel);
                                film.addSample(splats[0].mRaster, splats[0].mContrib);
                                film.atomicAddSample(splats[1].mRaster, splats[1].mContrib);
                                ts->nextSample();
                            }
                        }
                    }
                }
            };
            std::vector<std::thread> pool;
            for (int t = 1; t < threads; ++t) pool.emplace_back(worker);
            worker();
            for (auto &th : pool) th.join();
        }
        paths = npix * numSpp;
        for (int y = 0; y < H; ++y)
            for (int x = 0; x < W; ++x) {
                Spectrum c = film.getPixel(Ivec2(x, y));
                for (int k = 0; k < 3; ++k) img[3 * (size_t(y) * W + x) + k] = c[k];
            }
    }
    const double seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    oracle::write_pfm(outPath, img.data(), W, H);
    if (!raw.empty()) {
        FILE *f = fopen(raw.c_str(), "wb");
        fwrite(img.data(), 8, img.size(), f);
        fclose(f);
    }
    printf("{\"seconds\": %.6f, \"paths\": %lld, \"load_seconds\": %.6f, \"threads\": %d, \"width\": %d, \"height\": %d}\n",
           seconds, paths, loadSeconds, (serial || crop) ? threads : Parallel::NumThreads(), W, H);
    return 0;
}

int cmd_trace(int argc, char **argv) {
    Loaded L = load(argv[2], "");
    std::string bytes = oracle::read_file(argv[3]);
    const size_t n = bytes.size() / 32;
    const float *r = reinterpret_cast<const float *>(bytes.data());
    std::vector<int32_t> out(4 * n);
    const EmbreeAccel &accel = *L.scene->mAccel;
    for (size_t i = 0; i < n; ++i) {
        const float *q = r + 8 * i;
        Ray3 ray(Vec3(q[0], q[1], q[2]), Vec3(q[4], q[5], q[6]), q[3], q[7]);
        TriangleInfoVertex tv;
        const bool hit = accel.intersectTriangleInfo(&tv, &ray);
        float t = hit ? float(ray.tMax) : INFINITY;
        out[4 * i + 0] = hit ? tv.mGeometryId : -1;
        out[4 * i + 1] = hit ? tv.mTriangleId : -1;
        memcpy(&out[4 * i + 2], &t, 4);
        out[4 * i + 3] = 0;
    }
    FILE *f = fopen(argv[4], "wb");
    fwrite(out.data(), 4, out.size(), f);
    fclose(f);
    printf("{\"rays\": %zu}\n", n);
    return 0;
}

// Closest hits through rtcIntersect1 on the accel's scene, for every geometry type (user
// geometry included, which intersectTriangleInfo does not report): per ray geomID, primID,
// tfar and the hit's Ng as the reference's intersect() reads them (embreeaccel.h:353-422).
int cmd_trace2(int argc, char **argv) {
    Loaded L = load(argv[2], "");
    std::string bytes = oracle::read_file(argv[3]);
    const size_t n = bytes.size() / 32;
    const float *r = reinterpret_cast<const float *>(bytes.data());
    std::vector<float> out(8 * n);
    const EmbreeAccel &accel = *L.scene->mAccel;
    for (size_t i = 0; i < n; ++i) {
        const float *q = r + 8 * i;
        RTCRayHit query;
        query.ray.org_x = q[0]; query.ray.org_y = q[1]; query.ray.org_z = q[2]; query.ray.tnear = q[3];
        query.ray.dir_x = q[4]; query.ray.dir_y = q[5]; query.ray.dir_z = q[6]; query.ray.tfar = q[7];
        query.ray.time = 0.f;
        query.hit.geomID = RTC_INVALID_GEOMETRY_ID;
        query.hit.primID = RTC_INVALID_GEOMETRY_ID;
        RTCIntersectContext ctx;
        rtcInitIntersectContext(&ctx);
        rtcIntersect1(accel.mRtcScene, &ctx, &query);
        const bool hit = query.hit.geomID != RTC_INVALID_GEOMETRY_ID;
        int32_t gid = hit ? int32_t(query.hit.geomID) : -1, pid = hit ? int32_t(query.hit.primID) : -1;
        memcpy(&out[8 * i + 0], &gid, 4);
        memcpy(&out[8 * i + 1], &pid, 4);
        out[8 * i + 2] = hit ? query.ray.tfar : INFINITY;
        out[8 * i + 3] = hit ? query.hit.Ng_x : 0.f;
        out[8 * i + 4] = hit ? query.hit.Ng_y : 0.f;
        out[8 * i + 5] = hit ? query.hit.Ng_z : 0.f;
        RTCRay occ;
        occ.org_x = q[0]; occ.org_y = q[1]; occ.org_z = q[2]; occ.tnear = q[3];
        occ.dir_x = q[4]; occ.dir_y = q[5]; occ.dir_z = q[6]; occ.tfar = q[7];
        occ.time = 0.f;
        rtcOccluded1(accel.mRtcScene, &ctx, &occ);
        out[8 * i + 6] = occ.tfar < 0.f ? 1.f : 0.f;
        out[8 * i + 7] = 0.f;
    }
    FILE *f = fopen(argv[4], "wb");
    fwrite(out.data(), 4, out.size(), f);
    fclose(f);
    printf("{\"rays\": %zu}\n", n);
    return 0;
}

// The reference's own image input (FimageIo::Load, src/common/floatimage.h:379-404: PFM, HDR via
// stb_image, EXR via tinyexr): writes width, height (int32) and W*H*3 floats, row 0 = top.
int cmd_imgload(int argc, char **argv) {
    (void)argc;
    Fimage<Spectrum> img = FimageIo::Load(filesystem::path(argv[2]));
    const int W = img.mSize[0], H = img.mSize[1];
    std::vector<float> out(size_t(W) * H * 3);
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x)
            for (int c = 0; c < 3; ++c) out[3 * (size_t(y) * W + x) + c] = float(img.at(x, y)[c]);
    FILE *f = fopen(argv[3], "wb");
    if (!f) throw std::runtime_error("cannot write " + std::string(argv[3]));
    const int32_t wh[2] = {W, H};
    fwrite(wh, 4, 2, f);
    fwrite(out.data(), 4, out.size(), f);
    fclose(f);
    printf("{\"width\": %d, \"height\": %d}\n", W, H);
    return 0;
}

}  // namespace

int main(int argc, char **argv) {
    try {
        if (argc >= 4 && std::string(argv[1]) == "render") return cmd_render(argc, argv);
        if (argc >= 5 && std::string(argv[1]) == "trace") return cmd_trace(argc, argv);
        if (argc >= 5 && std::string(argv[1]) == "trace2") return cmd_trace2(argc, argv);
        if (argc >= 4 && std::string(argv[1]) == "imgload") return cmd_imgload(argc, argv);
        fprintf(stderr, "usage: wurst_ref render <scene.json> <out.pfm> [options] | trace <scene.json> <rays> <hits>\n");
        return 2;
    } catch (const std::exception &e) {
        fprintf(stderr, "wurst_ref: %s\n", e.what());
        return 1;
    }
}
