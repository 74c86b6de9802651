// Test infrastructure only: FP64 CPU restatement of the reference's
// `nextevent_path_tracer` (PathNeeRenderer), used by tests/, the smoke check
// and the benchmark's CPU baseline as the checker. Nothing in the product
// links or calls it.
//
// It follows the reference operation by operation, in double precision and in
// the same evaluation order, with the same random-number streams
// (std::mt19937_64 per 32x32 tile seeded with pMin.x*H + pMin.y, values drawn
// through std::uniform_real_distribution<double>), so that, given the same
// ray caster, its image matches the reference's bit for bit:
//   integrator     src/renderer/pathnextevent.h:41-191
//   subpaths       src/pathsampler/generalsubpathsampler.h:13-337
//   vertex algebra src/common/path.h:47-76,175-417
//   scene queries  src/common/scene.h:82-147, src/accel/embreeaccel.h:336-422
//   camera         src/camera/thinlens.h:13-165, src/common/camera.h:7-35
//   BSDFs          src/bsdf/{twosided,lambertdiffuse,orennayar,phong,mixed}.h
//   lights         src/light/diffusearealight.h:21-82, src/light/envmap.h:22-101,
//                  src/sphericalrepresentation/equirectangular.h:33-123
//   sampling       src/common/cdftable.h:10-44, src/common/mapping.h:21-96,302-323,
//                  src/geometry/trianglemesh.h:110-159, src/common/math/coordframe.h:50-60
//   film           src/common/film.h:35-90, src/common/parallel.h:65-115
// Scene loading restates src/sceneio/simple2parser.h:27-68,102-223 and
// src/sceneio/meshio/assimpio.h:61-153 (see oracle_scene.h); the ray queries
// restate Embree's (see oracle_raycast.h).
//
// Compile with -ffp-contract=off and without -ffast-math: the reference's
// AVX2 double arithmetic performs no fused multiply-adds.

#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <mutex>
#include <random>
#include <thread>

#include "oracle_phong.h"
#include "oracle_raycast.h"
#include "oracle_scene.h"

namespace oracle {

static const double Pi = 3.141592653589793238462643383279502884197169399375105820974;
static const double InvPi = 0.318309886183790671537767526745028724068919291480912897495;
static const double SmallValue = 1e-12;
static const double RayEpsilon = 1e-4;   // Ray<Vec>::Epsilon, src/common/math/ray.h:8

// ------------------------------------------------------------- vectors ----
struct V3 {
    double x = 0, y = 0, z = 0;
    V3() {}
    V3(double a, double b, double c) : x(a), y(b), z(c) {}
    explicit V3(double a) : x(a), y(a), z(a) {}
    double operator[](int i) const { return i == 0 ? x : i == 1 ? y : z; }
};
static inline V3 operator+(V3 a, V3 b) { return V3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline V3 operator-(V3 a, V3 b) { return V3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline V3 operator-(V3 a) { return V3(-a.x, -a.y, -a.z); }
static inline V3 operator*(V3 a, V3 b) { return V3(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline V3 operator*(V3 a, double s) { return V3(a.x * s, a.y * s, a.z * s); }
static inline V3 operator*(double s, V3 a) { return V3(s * a.x, s * a.y, s * a.z); }
static inline V3 operator/(V3 a, double s) { return V3(a.x / s, a.y / s, a.z / s); }
static inline V3 operator/(V3 a, V3 b) { return V3(a.x / b.x, a.y / b.y, a.z / b.z); }
static inline double Dot(V3 u, V3 v) { double s = u.x * v.x; s += u.y * v.y; s += u.z * v.z; return s; }
static inline double AbsDot(V3 u, V3 v) { return std::abs(Dot(u, v)); }
static inline V3 Cross(V3 u, V3 v) { return V3(u.y * v.z - u.z * v.y, u.z * v.x - u.x * v.z, u.x * v.y - u.y * v.x); }
static inline double Length2(V3 v) { return Dot(v, v); }
static inline double Length(V3 v) { return std::sqrt(Length2(v)); }
static inline V3 Normalize(V3 v) { return v / Length(v); }
static inline bool IsZero(V3 v) { return v.x == 0.0 && v.y == 0.0 && v.z == 0.0; }
// SpectrumConvertUtil::FromSrgb (src/common/math/spectrum.h:13-17): the sRGB transfer curve
static inline double FromSrgb(double v) {
    if (v <= 0.04045) return v * (1.0 / 12.92);
    return std::pow((v + 0.055) * (1.0 / 1.055), 2.4);
}
static inline V3 FlipY(V3 v) { return V3(v.x, -v.y, v.z); }
static inline double Clamp(double v, double a, double b) { return std::max(std::min(v, b), a); }
static inline bool IsApprox(double a, double b) {
    const double absA = std::abs(a), absB = std::abs(b);
    const double larger = absA < absB ? absB : absA;
    return std::abs(a - b) <= std::max(larger * SmallValue, SmallValue);
}
typedef V3 Spectrum;

struct Frame {   // CoordFrame3, y = normal (Duff et al. 2017)
    V3 x = V3(1, 0, 0), y = V3(0, 1, 0), z = V3(0, 0, 1);
    Frame() {}
    explicit Frame(V3 n) {
        y = n;
        double sign = std::copysign(1.0, n.y);
        const double a = -1.0 / (sign + n.y);
        const double b = n.z * n.x * a;
        x = V3(sign + n.x * n.x * a, -n.x, b);
        z = V3(sign * b, -sign * n.z, 1.0 + sign * n.z * n.z * a);
    }
    V3 toLocal(V3 g) const { return V3(Dot(g, x), Dot(g, y), Dot(g, z)); }
    V3 toWorld(V3 l) const { return l.x * x + l.y * y + l.z * z; }
};

// Local3 helpers (src/common/math/local.h:32-106)
static inline double Cos(V3 v) { return v.y; }
static inline double Sin2(V3 v) { return Clamp(1.0 - v.y * v.y, 0.0, 1.0); }
static inline double Sin(V3 v) { return std::sqrt(Sin2(v)); }
static inline double SinAboutY(V3 v) { return v.z / Sin(v); }
static inline double CosAboutY(V3 v) { return v.x / Sin(v); }
static inline bool IsFront(V3 v) { return v.y > 0.0; }
static inline V3 Reflect(V3 v) { return V3(v.x, -v.y, v.z); }

static inline V3 CosineHemisphere(double s0, double s1) {
    const double sinPhi = std::sqrt(1.0 - s0);
    const double theta = Pi * 2.0 * s1;
    return V3(std::cos(theta) * sinPhi, std::sqrt(s0), std::sin(theta) * sinPhi);
}

// ----------------------------------------------------------- cdf table ----
struct CdfTable {
    std::vector<double> pdfs, cdfs;
    CdfTable() {}
    explicit CdfTable(const std::vector<double> &w) {
        if (w.empty()) return;
        pdfs.resize(w.size()); cdfs.resize(w.size());
        double sum = 0.0;
        for (size_t i = 0; i < w.size(); ++i) sum += std::abs(w[i]);
        for (size_t i = 0; i < w.size(); ++i) pdfs[i] = std::abs(w[i]) / sum;
        cdfs[0] = pdfs[0];
        cdfs[w.size() - 1] = 1.0;
        for (size_t i = 1; i + 1 < w.size(); ++i) cdfs[i] = cdfs[i - 1] + pdfs[i];
    }
    bool empty() const { return pdfs.empty(); }
    int sample(double *pdf, double *remapped, double u) const {
        int index = int(std::lower_bound(cdfs.begin(), cdfs.end(), u) - cdfs.begin());
        if (pdf) *pdf = pdfs[index];
        if (remapped) *remapped = std::min(index == 0 ? u / pdfs[index] : (u - cdfs[index - 1]) / pdfs[index], 1.0 - SmallValue);
        return index;
    }
};

// --------------------------------------------------------------- BSDFs ----
enum Comp { LAMBERT = 0, OREN_NAYAR = 1, PHONG = 2 };

struct Component {
    int kind = LAMBERT;
    Spectrum refl;       // Kd for Lambert/Oren-Nayar, Ks for Phong
    double param = 0.0;  // Oren-Nayar sigma or Phong exponent
};

static Spectrum comp_eval(const Component &c, V3 in, V3 out) {
    if (c.kind == LAMBERT) {
        if (Cos(in) <= 0.0) return Spectrum(0.0);
        if (Cos(out) <= 0.0) return Spectrum(0.0);
        return c.refl * InvPi;
    }
    if (c.kind == OREN_NAYAR) {
        if ((Cos(in) <= 0.0) || (Cos(out) <= 0.0)) return Spectrum(0.0);
        double sinPhiI = Sin(in), sinPhiO = Sin(out);
        double maxCos = 0.0, sinAlpha = 0.0, tanBeta = 0.0;
        if ((Sin(in) > 1e-4) && (Sin(out) > 1e-4)) {
            double sinThetaI = SinAboutY(in), cosThetaI = CosAboutY(in);
            double sinThetaO = SinAboutY(out), cosThetaO = CosAboutY(out);
            double dCos = cosThetaI * cosThetaO + sinThetaI * sinThetaO;
            maxCos = std::max(0.0, dCos);
            if (std::abs(Cos(in)) > std::abs(Cos(out))) { sinAlpha = sinPhiO; tanBeta = sinPhiI / Cos(in); }
            else { sinAlpha = sinPhiI; tanBeta = sinPhiO / Cos(out); }
        }
        const double s = c.param, s2 = s * s;
        const double A = 1.0 - s2 / (2 * (s2 + 0.33));
        const double B = 0.45 * s2 / (s2 + 0.09);
        return c.refl * InvPi * (A + B * maxCos * sinAlpha * tanBeta);
    }
    // modified Phong
    if ((Cos(in) <= 0.0) || (Cos(out) <= 0.0)) return Spectrum(0.0);
    const V3 reflect = Reflect(-in);
    if (Cos(reflect) <= 0.0f) return Spectrum(0.0);
    const double cosReflect = Dot(reflect, out);
    if (cosReflect <= 0.0) return Spectrum(0.0);
    const double n = c.param;
    return c.refl * ((n + 2.0) * std::pow(cosReflect, n) * InvPi * 0.5);
}

static double comp_pdf(const Component &c, V3 in, V3 out) {
    if (c.kind == LAMBERT) {
        if (Cos(in) <= 0.0) return 0.0;
        if (Cos(out) <= 0.0) return 0.0;
        return Cos(out) * InvPi;
    }
    if (c.kind == OREN_NAYAR) {
        if (Cos(out) <= 0.0) return 0.0;
        if (Cos(in) <= 0.0) return 0.0;
        return Cos(out) * InvPi;
    }
    if ((Cos(in) <= 0.0) && (Cos(out) <= 0.0)) return 0.0;
    const V3 reflect = Reflect(-in);
    const double cosReflect = Dot(reflect, out);
    if (cosReflect <= 0.0) return 0.0;
    const double n = c.param;
    return (n + 1.0) * std::pow(cosReflect, n) * InvPi * 0.5;
}

// returns bsdf*cos/pdf; `out` and `pdfW` are written exactly when the reference writes them
static Spectrum comp_sample(const Component &c, V3 *out, double *pdfW, V3 in, double s0, double s1) {
    if (c.kind == LAMBERT) {
        if (Cos(in) <= 0.0) return Spectrum(0.0);
        V3 o = CosineHemisphere(s0, s1);
        const double cosine = Cos(o);
        if (out) *out = o;
        if (pdfW) *pdfW = std::max(cosine, 0.0) * InvPi;
        if (cosine <= 0.0) return Spectrum(0.0);
        return c.refl;
    }
    if (c.kind == OREN_NAYAR) {
        if (Cos(in) < 0.0) { if (pdfW) *pdfW = 0.0; return Spectrum(0.0); }
        V3 o = CosineHemisphere(s0, s1);
        if (out) *out = o;
        if (pdfW) *pdfW = Cos(o) * InvPi;
        return comp_eval(c, o, in) * Pi;
    }
    if (Cos(in) <= 0.0) return Spectrum(0.0);
    const double n = c.param;
    const V3 reflect = Reflect(-in);
    const double cosTheta = std::pow(s0, 1.0f / (n + 1.0f));
    const double sinTheta = std::sqrt(1.0f - cosTheta * cosTheta);
    const double phi = 2.0f * Pi * s1;
    const double cosPhi = std::cos(phi), sinPhi = std::sin(phi);
    const V3 localOut(sinTheta * cosPhi, cosTheta, sinTheta * sinPhi);
    const Frame rb(reflect);
    const V3 o = rb.toWorld(localOut);
    const double cosReflect = Dot(o, reflect);
    if (out) *out = o;
    if (pdfW) *pdfW = (n + 1.0f) * 0.5f * InvPi * std::pow(cosReflect, n);
    if (Cos(reflect) <= 0.0 || Cos(o) <= 0.0 || cosReflect <= 0.0) return Spectrum(0.0);
    return c.refl * ((n + 2.0f) / (n + 1.0f) * Cos(o));
}

// TwoSided(inner) where inner = one component or Mixed(components)
struct Material {
    std::vector<Component> comps;   // size 1: plain BSDF; size 2: MixedBsdf
};

static Spectrum inner_eval(const Material &m, V3 in, V3 out) {
    if (m.comps.size() == 1) return comp_eval(m.comps[0], in, out);
    Spectrum r(0.0);
    for (auto &c : m.comps) r = r + comp_eval(c, in, out);
    return r;
}
static double inner_pdf(const Material &m, V3 in, V3 out) {
    if (m.comps.size() == 1) return comp_pdf(m.comps[0], in, out);
    double r = 0.0;
    for (auto &c : m.comps) r += comp_pdf(c, in, out);
    return r / double(m.comps.size());
}
static Spectrum inner_sample(const Material &m, V3 *out, double *pdfW, V3 in, double s0, double s1) {
    if (m.comps.size() == 1) return comp_sample(m.comps[0], out, pdfW, in, s0, s1);
    const unsigned numComps = unsigned(m.comps.size());
    const unsigned k = std::min((unsigned)std::floor(s0 * numComps), numComps - 1);
    const double r0 = std::min(s0 * numComps - k, 1.0 - SmallValue);
    V3 o;   // zero when the component declines to sample, as a default-constructed Vec3
    comp_sample(m.comps[k], &o, nullptr, in, r0, s1);
    if (out) *out = o;
    Spectrum bsdf = inner_eval(m, in, o);
    double pdf = inner_pdf(m, in, o);
    if (pdfW) *pdfW = pdf;
    if (pdf == 0.0) return Spectrum(0.0);
    return bsdf / pdf * Cos(o);
}

static Spectrum bsdf_eval(const Material &m, V3 in, V3 out) {
    if (IsFront(in) && IsFront(out)) return inner_eval(m, in, out);
    if (!IsFront(in) && !IsFront(out)) return inner_eval(m, FlipY(in), FlipY(out));
    return Spectrum(0.0);
}
static double bsdf_pdf(const Material &m, V3 in, V3 out) {
    if (IsFront(in) && IsFront(out)) return inner_pdf(m, in, out);
    if (!IsFront(in) && !IsFront(out)) return inner_pdf(m, FlipY(in), FlipY(out));
    return 0.0;
}
static Spectrum bsdf_sample(const Material &m, V3 *out, double *pdfW, V3 in, double s0, double s1) {
    if (IsFront(in)) return inner_sample(m, out, pdfW, in, s0, s1);
    Spectrum r = inner_sample(m, out, pdfW, FlipY(in), s0, s1);
    if (out) *out = FlipY(*out);
    return r;
}

// --------------------------------------------------------------- scene ----
struct Geometry {               // one reference TriangleMeshGeometry (or PhongMeshGeometry)
    std::vector<V3> pos;
    std::vector<int> tri;       // 3 per triangle
    std::vector<phong::Patch> patches;   // Phong tessellation surfaces: one patch per triangle
    int material = -1;          // index into Scene::materials (surfaces)
    int light = -1;             // index into Scene::lights (emitters)
    int geom_id = -1;           // Embree geomID (attach order)
    double area = 0.0, inv_area = 0.0;
    CdfTable tri_cdf;
};

struct AreaLight { Spectrum intensity; int geometry; };

struct EnvMap {
    int w = 0, h = 0;
    std::vector<Spectrum> texels;   // row 0 = top
    CdfTable cdf;
    V3 center; double radius = 0.0;
    Spectrum texel(int x, int y) const {
        x = ((x % w) + w) % w;
        y = std::min(std::max(y, 0), h - 1);
        return texels[size_t(y) * w + x];
    }
    static void panorama(V3 dir, double *u, double *v) {
        *u = std::atan2(-dir.z, -dir.x) * InvPi * 0.5f + 0.5f;
        *v = std::acos(dir.y) * InvPi;
    }
    Spectrum eval(V3 dir) const {
        double u, v; panorama(dir, &u, &v);
        const double su = u * double(w) - 0.5, sv = v * double(h) - 0.5;
        const int xp = int(std::floor(su)), yp = int(std::floor(sv));
        const double dx1 = su - xp, dy1 = sv - yp, dx2 = 1.0 - dx1, dy2 = 1.0 - dy1;
        return texel(xp, yp) * dx2 * dy2 + texel(xp, yp + 1) * dx2 * dy1 + texel(xp + 1, yp) * dx1 * dy2 +
               texel(xp + 1, yp + 1) * dx1 * dy1;
    }
    double pdfA(V3 dir) const {
        double u, v; panorama(dir, &u, &v);
        const int px = int(u * double(w)), py = int(v * double(h));
        const int idx = w * py + px;
        const double sine = Sin(dir);
        if (IsApprox(sine, 0.0)) return 0.0;
        return cdf.pdfs[idx] * double(size_t(w) * h) / sine * InvPi * InvPi * 0.5;
    }
    Spectrum sample(V3 *dir, double *pdfW, double s0, double s1) const {
        double pdf;
        double r0 = s0;
        unsigned idx = unsigned(cdf.sample(&pdf, &r0, r0));
        unsigned x = idx % unsigned(w), y = idx / unsigned(w);
        const double u = ((double)x + r0) / double(w), v = ((double)y + s1) / double(h);
        const double theta = u * Pi * 2.0, phi = v * Pi;
        const double sp = std::sin(phi), cp = std::cos(phi), st = std::sin(theta), ct = std::cos(theta);
        const V3 d(ct * sp, cp, st * sp);
        const double sine = Sin(d);
        pdf = IsApprox(sine, 0.0) ? 0.0 : pdf * double(size_t(w) * h) / sine * InvPi * InvPi * 0.5;
        *dir = d; *pdfW = pdf;
        return eval(d) / pdf;
    }
};

struct Camera {   // ThinlensCamera
    V3 origin; Frame frame;
    int W = 0, H = 0;
    double filmW = 0, filmH = 0, dist = 0, perFilm = 0, perPixel = 0, lensArea = 0, focal = 1, aperture = 0;
    void init(V3 from, V3 at, V3 up, double fovyDeg, int w, int h, double aperture_, double focal_) {
        origin = from; W = w; H = h;
        const double fov = fovyDeg * Pi / 180.0;
        if (fov > Pi) throw std::runtime_error("Thinlens camera doesn't support when fov > Pi radians");
        filmW = double(w); filmH = double(h);
        dist = filmH * 0.5 / std::tan(fov * 0.5);
        frame.z = Normalize(at - from);
        frame.x = Normalize(Cross(up, frame.z));
        frame.y = Normalize(Cross(frame.z, frame.x));
        aperture = aperture_; focal = focal_;
        lensArea = Pi * aperture * aperture;
        perPixel = dist * dist / (filmW * filmH);
        perFilm = dist * dist / (1.0 * 1.0);
    }
};

struct Scene {
    std::vector<Geometry> geoms;        // surfaces then lights per OBJ file, in attach order
    std::vector<int> surface_of_geom;   // geomID -> index in geoms
    std::vector<Material> materials;
    std::vector<AreaLight> lights;      // the reference's mLightGeometries order
    std::unique_ptr<EnvMap> env;
    CdfTable light_cdf;                 // area lights, then the environment (weight 1.23)
    RayCaster rc;
    Camera cam;
    int spp = 16, nverts = 10;
    int integrator = 0;   // 0 nextevent_path_tracer, 1 primitive_path_tracer, 2 light_splatting
    std::string output;
};

// ------------------------------------------------------------- vertices ----
enum VType { V_LIGHT = 2, V_ENV = 2 | 4, V_SURFACE = 8, V_CAMERA = 32 };

struct Vertex {
    int type = 0;
    V3 pos, normal;
    Frame frame;
    Spectrum contrib;      // mPathContrib
    int geom = -1;         // index into Scene::geoms (surface / light hits and light samples)
};

// Vertex::operator- (to - from) with the environment rules
static inline V3 diff(const Vertex &to, const Vertex &from) {
    if (from.type == V_ENV) return -from.pos;
    if (to.type == V_ENV) return to.pos;
    return to.pos - from.pos;
}

static double ConvertToArea(const Vertex &from, const Vertex &to) {
    double result = 1.0;
    V3 uv = diff(to, from);
    double length2 = Length2(uv);
    V3 nuv = uv / std::sqrt(length2);
    if (to.type != V_ENV) result *= AbsDot(to.normal, nuv);
    result /= length2;
    return result;
}

static double GeometryTerm(const Vertex &u, const Vertex &v) {
    double result = 1.0;
    V3 uv = diff(v, u);
    double length2 = Length2(uv);
    V3 nuv = uv / std::sqrt(length2);
    if (u.type != V_ENV) result *= AbsDot(u.normal, nuv);
    if (v.type != V_ENV) result *= AbsDot(v.normal, nuv);
    result /= length2;
    return result;
}

// -------------------------------------------------------------- queries ----
struct Ray { V3 o, d; double tmin = RayEpsilon, tmax = std::numeric_limits<double>::max(); };

static bool occluded(const Scene &s, const Ray &r) {
    const float o[3] = {float(r.o.x), float(r.o.y), float(r.o.z)};
    const float d[3] = {float(r.d.x), float(r.d.y), float(r.d.z)};
    return s.rc.occluded(o, d, float(r.tmin), float(r.tmax));
}

// Scene::intersect: closest hit, environment fallback; false when nothing is hit
static bool intersect(const Scene &s, Ray *r, Vertex *v) {
    const float o[3] = {float(r->o.x), float(r->o.y), float(r->o.z)};
    const float d[3] = {float(r->d.x), float(r->d.y), float(r->d.z)};
    RcHit h;
    if (s.rc.closest(o, d, float(r->tmin), float(r->tmax), &h)) {
        r->tmax = double(h.t);
        const int gi = s.surface_of_geom[h.geom];
        v->geom = gi;
        v->type = s.geoms[gi].light >= 0 ? V_LIGHT : V_SURFACE;
        v->pos = r->o + r->d * r->tmax;
        v->normal = Normalize(V3(double(h.ng[0]), double(h.ng[1]), double(h.ng[2])));
        v->frame = Frame(v->normal);
        return true;
    }
    if (s.env) {
        v->type = V_ENV;
        v->geom = -1;
        v->frame = Frame();
        v->pos = r->d;
        v->normal = V3();
        return true;
    }
    return false;
}

static V3 transmittance(const Scene &s, const Vertex &p1, const Vertex &p2) {
    if (p1.type == V_ENV) { Ray r; r.o = p2.pos; r.d = p1.pos; return V3(occluded(s, r) ? 0.0 : 1.0); }
    if (p2.type == V_ENV) { Ray r; r.o = p1.pos; r.d = p2.pos; return V3(occluded(s, r) ? 0.0 : 1.0); }
    const V3 uv = p2.pos - p1.pos;
    const double length = Length(uv);
    Spectrum tr(1.0);
    const V3 nuv = uv / length;
    Ray r; r.o = p1.pos; r.d = nuv; r.tmin = RayEpsilon; r.tmax = length - RayEpsilon;
    const double vis = occluded(s, r) ? 0.0 : 1.0;
    return tr * vis;
}

// ------------------------------------------------------------ lights ----
static double light_pdfA(const Scene &s, const Vertex &lv) {   // evalLightPdfA
    if (lv.type == V_ENV) return s.light_cdf.pdfs[s.lights.size()] * s.env->pdfA(lv.pos);
    const Geometry &g = s.geoms[lv.geom];
    return s.light_cdf.pdfs[g.light] * g.inv_area;
}

// LightVertex::scatter toward `to` (evalLe1)
static double light_le1(const Vertex &lv, const Vertex &to) {
    if (lv.type == V_ENV) return 1.0;
    const V3 w = Normalize(diff(to, lv));
    if (Cos(lv.frame.toLocal(w)) < 0.0) return 0.0;
    return InvPi;
}

static Spectrum light_le0(const Scene &s, const Vertex &lv) {   // source()
    if (lv.type == V_ENV) return s.env->eval(lv.pos);
    return s.lights[s.geoms[lv.geom].light].intensity * Pi;
}

// ------------------------------------------------------------ sampler ----
struct Sampler {
    std::mt19937_64 g;
    explicit Sampler(unsigned seed) : g(seed) {}
    double next() { return std::uniform_real_distribution<double>(0, 1)(g); }
    // RandomSampler::get2d builds Vec2(next(), next()); GCC evaluates those
    // constructor arguments right to left, so the second draw is component 0.
    void get2d(double *a, double *b) { *b = next(); *a = next(); }
};

struct Splat { double rx = 0.0, ry = 0.0; Spectrum c; };

// PathNeeRenderer::evalContribution
static void eval_contribution(const Scene &s, Sampler &smp, int px, int py, Splat sp[2]) {
    // ---- light subpath, one vertex (createLightSubpath)
    Vertex l;
    double lPdfA = 1.0;
    {
        double u0, u1; smp.get2d(&u0, &u1);
        double pdfLight;
        const int li = s.light_cdf.sample(&pdfLight, &u0, u0);
        if (li >= int(s.lights.size())) {
            V3 dir; double pdfDir;
            Spectrum r = s.env->sample(&dir, &pdfDir, u0, u1);
            l.type = V_ENV; l.geom = -1; l.frame = Frame(); l.pos = dir;
            l.contrib = r / pdfLight;
            lPdfA = pdfLight * pdfDir;
            double d0, d1; smp.get2d(&d0, &d1);   // light-tracing disk sample (sampleLe1CosByPdf)
        } else {
            const AreaLight &al = s.lights[li];
            const Geometry &g = s.geoms[al.geometry];
            double ls0 = u0;
            const int ti = g.tri_cdf.sample(nullptr, &ls0, ls0);
            const double sq = std::sqrt(ls0);
            const double b1 = sq * (1.0 - u1), b2 = u1 * sq;
            const V3 p0 = g.pos[g.tri[3 * ti]], p1 = g.pos[g.tri[3 * ti + 1]], p2 = g.pos[g.tri[3 * ti + 2]];
            const V3 w0 = V3(1.0 - b1 - b2);
            l.type = V_LIGHT; l.geom = al.geometry;
            l.pos = w0 * p0 + b1 * p1 + b2 * p2;
            l.normal = Normalize(Cross(p1 - p0, p2 - p0));
            l.frame = Frame(l.normal);
            const double pdfPos = g.inv_area;
            l.contrib = al.intensity * Pi / pdfPos / pdfLight;
            lPdfA = pdfLight * pdfPos;
        }
    }

    // ---- camera vertex (createCameraSubpath)
    const Camera &cam = s.cam;
    Vertex c0;
    {
        double a, b; smp.get2d(&a, &b);
        double lx = 0.0, ly = 0.0;   // DiskFromSquare(sample) * aperture
        double abx = a * 2.0 - 1.0, aby = b * 2.0 - 1.0;
        if (!(abx == 0 && aby == 0)) {
            double r, phi;
            if (abx * abx > aby * aby) { r = abx; phi = (Pi / 4.0) * (aby / abx); }
            else { r = aby; phi = (Pi / 2.0) - (Pi / 4.0) * (abx / aby); }
            lx = r * std::cos(phi); ly = r * std::sin(phi);
        }
        lx = lx * cam.aperture; ly = ly * cam.aperture;
        c0.type = V_CAMERA;
        c0.normal = cam.frame.z;
        c0.pos = cam.frame.toWorld(V3(lx, ly, 0.0)) + cam.origin;
        c0.contrib = Spectrum(1.0);
    }

    // ---- strategy C: light vertex connected to the camera (splat)
    do {
        const double G = GeometryTerm(l, c0);
        if (G == 0.0) break;
        const V3 w = Normalize(diff(l, c0));
        const V3 position = cam.frame.toLocal(c0.pos - cam.origin);
        const V3 direction = cam.frame.toLocal(w);
        const double cosTheta = direction.z;
        if (Dot(w, cam.frame.z) < 0.0) break;
        const V3 fpp = direction / cosTheta * cam.focal + position;
        const V3 film = -fpp / cam.focal * cam.dist;
        const double rx = (film.x / cam.filmW + 0.5) * double(cam.W);
        const double ry = (film.y / cam.filmH + 0.5) * double(cam.H);
        if (rx < 0.0 || rx >= double(cam.W) || ry < 0.0 || ry >= double(cam.H)) break;
        const double cos4 = (cosTheta * cosTheta) * (cosTheta * cosTheta);
        const Spectrum c0scatter(cam.perFilm / cos4);
        if (IsZero(c0scatter)) break;
        const Spectrum lscatter(light_le1(l, c0));
        if (IsZero(lscatter)) break;
        const Spectrum T = transmittance(s, l, c0);
        if (IsZero(T)) break;
        const double camPdfW = cam.perPixel / (cosTheta * cosTheta * cosTheta);
        const double camPdfA = camPdfW * ConvertToArea(c0, l);
        const double mis = lPdfA / (lPdfA + camPdfA);
        sp[1].rx = rx; sp[1].ry = ry;
        sp[1].c = mis * c0.contrib * c0scatter * G * T * lscatter * l.contrib;
    } while (false);

    // ---- camera ray (samplePerPixelWe1CosByPdf)
    Ray ray;
    double prevPdfW;
    {
        double a, b; smp.get2d(&a, &b);
        const double nsx = (double(px) + a) * (1.0 / double(cam.W)), nsy = (double(py) + b) * (1.0 / double(cam.H));
        const V3 camPos = cam.frame.toLocal(c0.pos - cam.origin);
        const V3 film((nsx - 0.5) * cam.filmW, (nsy - 0.5) * cam.filmH, -cam.dist);
        sp[0].rx = nsx * double(cam.W); sp[0].ry = nsy * double(cam.H);
        const V3 fpp = cam.focal * film / film.z;
        const V3 dir = Normalize(fpp - camPos);
        const double cosTheta = dir.z;
        ray.o = c0.pos;
        ray.d = cam.frame.toWorld(dir);
        prevPdfW = cam.perFilm / (cosTheta * cosTheta * cosTheta);
        prevPdfW = prevPdfW * ((1.0 / double(cam.W)) * (1.0 / double(cam.H)));
    }

    // ---- random walk with the NEE / emitter-hit callbacks
    Spectrum prevContrib(1.0);
    Vertex prev = c0;
    int countVertices = 0, cNumVertices = 1;
    const int numVertices = s.nverts - 1;
    if (numVertices == 0) return;
    while (true) {
        Vertex v;
        const bool hit = intersect(s, &ray, &v);
        double du0, du1; smp.get2d(&du0, &du1);   // doVolumetric consumes a sample per segment
        if (!hit) break;
        v.contrib = prevContrib * prev.contrib;
        double pdf = prevPdfW;
        pdf *= ConvertToArea(prev, v);
        // callback
        cNumVertices += 1;
        bool cont = true;
        if (v.type == V_SURFACE && cNumVertices != s.nverts) {
            const Material &m = s.materials[s.geoms[v.geom].material];
            do {
                const double G = GeometryTerm(v, l);
                if (G == 0.0) break;
                const Spectrum T = transmittance(s, v, l);
                if (IsZero(T)) break;
                const V3 wi = Normalize(diff(prev, v)), wo = Normalize(diff(l, v));
                const Spectrum scatter1 = bsdf_eval(m, v.frame.toLocal(wi), v.frame.toLocal(wo));
                if (IsZero(scatter1)) break;
                const Spectrum scatter2(light_le1(l, v));
                if (IsZero(scatter2)) break;
                const double bsdfPdfA = bsdf_pdf(m, v.frame.toLocal(wi), v.frame.toLocal(wo)) * ConvertToArea(v, l);
                const double mis = lPdfA / (lPdfA + bsdfPdfA);
                sp[0].c = sp[0].c + mis * v.contrib * scatter1 * scatter2 * T * G * l.contrib;
            } while (false);
        } else if (v.type == V_LIGHT || v.type == V_ENV) {
            const double bsdfPdfA = pdf;
            const double lightPdfA = light_pdfA(s, v);
            const double mis = bsdfPdfA / (lightPdfA + bsdfPdfA);
            sp[0].c = sp[0].c + mis * v.contrib * Spectrum(light_le1(v, prev)) * light_le0(s, v);
        } else {
            cont = false;
        }
        if (!cont) break;
        if (++countVertices == numVertices) break;
        if (v.type != V_SURFACE) break;
        const Material &m = s.materials[s.geoms[v.geom].material];
        const V3 inLocal = v.frame.toLocal(-ray.d);
        V3 outLocal;
        double pdfW = 0.0;
        double b0, b1; smp.get2d(&b0, &b1);
        const Spectrum w = bsdf_sample(m, &outLocal, &pdfW, inLocal, b0, b1);
        if (IsZero(w)) break;
        prevContrib = w;
        prevPdfW = pdfW;
        ray = Ray();
        ray.o = v.pos;
        ray.d = v.frame.toWorld(outLocal);
        prev = v;
    }
}

// PrimitivePathRenderer::evalContribution (src/renderer/primitivepath.h:43-58): camera subpath
// only, BSDF sampling, an emitter (or the environment) hit ends the path and contributes
// pathContrib * Le1 * Le0 without MIS. Same sample consumption as createCameraSubpath +
// randomWalk with the volumetric sample per segment (generalsubpathsampler.h:34-53).
static void eval_primitive(const Scene &s, Sampler &smp, int px, int py, Splat *sp) {
    const Camera &cam = s.cam;
    Vertex c0;
    {
        double a, b; smp.get2d(&a, &b);
        double lx = 0.0, ly = 0.0;
        double abx = a * 2.0 - 1.0, aby = b * 2.0 - 1.0;
        if (!(abx == 0 && aby == 0)) {
            double r, phi;
            if (abx * abx > aby * aby) { r = abx; phi = (Pi / 4.0) * (aby / abx); }
            else { r = aby; phi = (Pi / 2.0) - (Pi / 4.0) * (abx / aby); }
            lx = r * std::cos(phi); ly = r * std::sin(phi);
        }
        lx = lx * cam.aperture; ly = ly * cam.aperture;
        c0.type = V_CAMERA;
        c0.normal = cam.frame.z;
        c0.pos = cam.frame.toWorld(V3(lx, ly, 0.0)) + cam.origin;
        c0.contrib = Spectrum(1.0);
    }
    Ray ray;
    {
        double a, b; smp.get2d(&a, &b);
        const double nsx = (double(px) + a) * (1.0 / double(cam.W)), nsy = (double(py) + b) * (1.0 / double(cam.H));
        const V3 camPos = cam.frame.toLocal(c0.pos - cam.origin);
        const V3 film((nsx - 0.5) * cam.filmW, (nsy - 0.5) * cam.filmH, -cam.dist);
        sp->rx = nsx * double(cam.W); sp->ry = nsy * double(cam.H);
        const V3 fpp = cam.focal * film / film.z;
        const V3 dir = Normalize(fpp - camPos);
        ray.o = c0.pos;
        ray.d = cam.frame.toWorld(dir);
    }
    Spectrum prevContrib(1.0);
    Vertex prev = c0;
    int countVertices = 0;
    const int numVertices = s.nverts - 1;
    if (numVertices == 0) return;
    while (true) {
        Vertex v;
        const bool hit = intersect(s, &ray, &v);
        double du0, du1; smp.get2d(&du0, &du1);
        if (!hit) break;
        v.contrib = prevContrib * prev.contrib;
        if (v.type == V_LIGHT || v.type == V_ENV) {
            sp->c = v.contrib * Spectrum(light_le1(v, prev)) * light_le0(s, v);
            break;
        }
        if (++countVertices == numVertices) break;
        const Material &m = s.materials[s.geoms[v.geom].material];
        const V3 inLocal = v.frame.toLocal(-ray.d);
        V3 outLocal;
        double b0, b1; smp.get2d(&b0, &b1);
        const Spectrum w = bsdf_sample(m, &outLocal, nullptr, inLocal, b0, b1);
        if (IsZero(w)) break;
        prevContrib = w;
        ray = Ray();
        ray.o = v.pos;
        ray.d = v.frame.toWorld(outLocal);
        prev = v;
    }
}

// LightSplattingRenderer::render's per-sample body (src/renderer/lightsplatting.h:47-108) with
// GeneralSubpathSampler(scene, false): no camera stratification, no volumetric sample per
// segment. A lens vertex c0 is sampled (createCameraSubpath with one vertex, which still draws
// the direction sample, generalsubpathsampler.h:286-304), then a light subpath of
// num_path_vertices - 1 vertices (createLightSubpath + randomWalk, :185-268, :13-160); the light
// vertex and every surface vertex of it are connected to c0 and splatted with weight
// 1 / (spp * W * H) (`inv`). Splats are appended to `out`.
struct CameraConnection { double rx = 0.0, ry = 0.0; Spectrum c; bool ok = false; };

// c0->mPathContrib * c0->scatter(raster, CameraImaginary, v) * G(v, c0) * transmittance(v, c0) * lscatter
static CameraConnection connect_camera(const Scene &s, const Vertex &c0, const Vertex &v, const Spectrum &lscatter) {
    CameraConnection r;
    const Camera &cam = s.cam;
    const double G = GeometryTerm(v, c0);
    if (G == 0.0) return r;
    // evalWe1 (thinlens.h:63-80) toward v
    const V3 w = Normalize(diff(v, c0));
    const V3 position = cam.frame.toLocal(c0.pos - cam.origin);
    const V3 direction = cam.frame.toLocal(w);
    const double cosTheta = direction.z;
    if (Dot(w, cam.frame.z) < 0.0) return r;
    const V3 fpp = direction / cosTheta * cam.focal + position;
    const V3 film = -fpp / cam.focal * cam.dist;
    const double rx = (film.x / cam.filmW + 0.5) * double(cam.W);
    const double ry = (film.y / cam.filmH + 0.5) * double(cam.H);
    if (rx < 0.0 || rx >= double(cam.W) || ry < 0.0 || ry >= double(cam.H)) return r;
    const double cos4 = (cosTheta * cosTheta) * (cosTheta * cosTheta);
    const Spectrum c0scatter(cam.perFilm / cos4);
    if (IsZero(c0scatter)) return r;
    if (IsZero(lscatter)) return r;
    const Spectrum T = transmittance(s, v, c0);
    if (IsZero(T)) return r;
    r.rx = rx; r.ry = ry;
    r.c = c0.contrib * c0scatter * G * T * lscatter * v.contrib;
    r.ok = true;
    return r;
}

static void eval_light_splat(const Scene &s, Sampler &smp, double inv, std::vector<Splat> &out) {
    if (s.nverts < 2) return;
    const Camera &cam = s.cam;
    // ---- camera vertex: sampleWe0ByPdf, then the unused sampleWe1CosByPdf draw
    Vertex c0;
    {
        double a, b; smp.get2d(&a, &b);
        double lx = 0.0, ly = 0.0;
        double abx = a * 2.0 - 1.0, aby = b * 2.0 - 1.0;
        if (!(abx == 0 && aby == 0)) {
            double r, phi;
            if (abx * abx > aby * aby) { r = abx; phi = (Pi / 4.0) * (aby / abx); }
            else { r = aby; phi = (Pi / 2.0) - (Pi / 4.0) * (abx / aby); }
            lx = r * std::cos(phi); ly = r * std::sin(phi);
        }
        lx = lx * cam.aperture; ly = ly * cam.aperture;
        c0.type = V_CAMERA;
        c0.normal = cam.frame.z;
        c0.pos = cam.frame.toWorld(V3(lx, ly, 0.0)) + cam.origin;
        c0.contrib = Spectrum(1.0);
        double d0, d1; smp.get2d(&d0, &d1);
    }
    auto splat = [&](const CameraConnection &cc) {
        if (!cc.ok) return;
        Splat sp; sp.rx = cc.rx; sp.ry = cc.ry; sp.c = cc.c * inv;
        out.push_back(sp);
    };
    // ---- light vertex
    const int numVertices = s.nverts - 1;
    Vertex l;
    Ray ray;
    Spectrum contrib1(1.0);
    {
        double u0, u1; smp.get2d(&u0, &u1);
        double pdfLight;
        const int li = s.light_cdf.sample(&pdfLight, &u0, u0);
        if (li >= int(s.lights.size())) {
            V3 dir; double pdfDir;
            Spectrum r = s.env->sample(&dir, &pdfDir, u0, u1);
            l.type = V_ENV; l.geom = -1; l.frame = Frame(); l.pos = dir;
            l.contrib = r / pdfLight;
            splat(connect_camera(s, c0, l, Spectrum(1.0)));
            // sampleLe1CosByPdf: a point on the disk of the scene's bounding sphere (envmap.h:83-101)
            double a, b; smp.get2d(&a, &b);
            double px = 0.0, py = 0.0;
            const double abx = a * 2.0 - 1.0, aby = b * 2.0 - 1.0;
            if (!(abx == 0 && aby == 0)) {
                double r2, phi;
                if (abx * abx > aby * aby) { r2 = abx; phi = (Pi / 4.0) * (aby / abx); }
                else { r2 = aby; phi = (Pi / 2.0) - (Pi / 4.0) * (abx / aby); }
                px = r2 * std::cos(phi); py = r2 * std::sin(phi);
            }
            px = px * s.env->radius; py = py * s.env->radius;
            const V3 q(px, -s.env->radius, py);
            const Frame frame(-l.pos);
            const double area = Pi * (s.env->radius * s.env->radius);
            ray.o = frame.toWorld(q) + s.env->center;
            ray.d = -l.pos;
            contrib1 = Spectrum(area);
        } else {
            const AreaLight &al = s.lights[li];
            const Geometry &g = s.geoms[al.geometry];
            double ls0 = u0;
            const int ti = g.tri_cdf.sample(nullptr, &ls0, ls0);
            const double sq = std::sqrt(ls0);
            const double b1 = sq * (1.0 - u1), b2 = u1 * sq;
            const V3 p0 = g.pos[g.tri[3 * ti]], p1 = g.pos[g.tri[3 * ti + 1]], p2 = g.pos[g.tri[3 * ti + 2]];
            const V3 w0 = V3(1.0 - b1 - b2);
            l.type = V_LIGHT; l.geom = al.geometry;
            l.pos = w0 * p0 + b1 * p1 + b2 * p2;
            l.normal = Normalize(Cross(p1 - p0, p2 - p0));
            l.frame = Frame(l.normal);
            l.contrib = al.intensity * Pi / g.inv_area / pdfLight;
            splat(connect_camera(s, c0, l, Spectrum(light_le1(l, c0))));
            if (numVertices == 1) return;
            double a, b; smp.get2d(&a, &b);   // sampleLe1CosByPdf: cosine-weighted about the normal
            const V3 outLocal = CosineHemisphere(a, b);
            ray.o = l.pos;
            ray.d = l.frame.toWorld(outLocal);
        }
    }
    // ---- randomWalk(numVertices - 1) with the camera-connection callback
    const int walkVertices = numVertices - 1;
    if (walkVertices == 0) return;
    Spectrum prevContrib = contrib1;
    Vertex prev = l;
    int countVertices = 0;
    while (true) {
        Vertex v;
        if (!intersect(s, &ray, &v)) break;
        v.contrib = prevContrib * prev.contrib;
        if (v.type == V_SURFACE) {
            const Material &m = s.materials[s.geoms[v.geom].material];
            const V3 wi = Normalize(diff(prev, v)), wo = Normalize(diff(c0, v));
            splat(connect_camera(s, c0, v, bsdf_eval(m, v.frame.toLocal(wi), v.frame.toLocal(wo))));
        }
        if (++countVertices == walkVertices) break;
        if (v.type != V_SURFACE) break;
        const Material &m = s.materials[s.geoms[v.geom].material];
        const V3 inLocal = v.frame.toLocal(-ray.d);
        V3 outLocal;
        double b0, b1; smp.get2d(&b0, &b1);
        const Spectrum w = bsdf_sample(m, &outLocal, nullptr, inLocal, b0, b1);
        if (IsZero(w)) break;
        prevContrib = w;
        ray = Ray();
        ray.o = v.pos;
        ray.d = v.frame.toWorld(outLocal);
        prev = v;
    }
}

// -------------------------------------------------------------- loading ----
static V3 vec3_of(const Json &j) {
    if (j.type == Json::Arr && j.arr.size() == 3) return V3(j.arr[0].number(), j.arr[1].number(), j.arr[2].number());
    if (j.type == Json::Arr && j.arr.size() == 1) return V3(j.arr[0].number());
    if (j.type == Json::Num) return V3(j.num);
    throw std::runtime_error("can't parse vec3");
}

static void set_camera(Scene &s, const Json &cj) {
    const Json &res = cj.at("resolution");
    if (res.arr.size() != 2) throw std::runtime_error("can't parse resolution");
    s.cam.init(vec3_of(cj.at("pos")), vec3_of(cj.at("lookat")), vec3_of(cj.at("up")), cj.get("fovy", 90.0),
               int(res.arr[0].number()), int(res.arr[1].number()), cj.get("radius", 0.0), cj.get("radius", 1.0));
}

static Scene *load_scene(const std::string &json_path, int render_index) {
    std::unique_ptr<Scene> s(new Scene());
    const Json root = JsonParser::parse(read_file(json_path));
    const std::string dir = dir_of(json_path);
    std::vector<int> surface_geoms, light_geoms;
    if (root.has("envmap") && !root.at("envmap").str.empty()) {
        int w, h;
        std::vector<float> px = read_pfm(dir + "/" + root.at("envmap").str, &w, &h);
        if (w != 2 * h) throw std::runtime_error("envmap has wrong size");
        s->env.reset(new EnvMap());
        EnvMap &e = *s->env;
        e.w = w; e.h = h;
        e.texels.resize(size_t(w) * h);
        for (size_t i = 0; i < e.texels.size(); ++i)
            e.texels[i] = V3(double(px[3 * i]), double(px[3 * i + 1]), double(px[3 * i + 2]));
        std::vector<double> weights(size_t(w) * h);
        for (int y = 0; y < h; ++y) {
            const double v = (double(y) + 0.5) / double(h);
            const double sine = std::sin(v * Pi);
            for (int x = 0; x < w; ++x) weights[size_t(y) * w + x] = sine * Length(e.texels[size_t(y) * w + x]);
        }
        e.cdf = CdfTable(weights);
    }
    int next_geom_id = 0;
    if (root.has("meshes")) {
        for (const Json &mj : root.at("meshes").arr) {
            const bool phong_file = mj.getb("phong_tessellation", false);
            // "mitsuba_srgb" (simple2parser.h:36): Kd and Ks go through FromSrgb, Ke and Ns do not
            // (assimpio.h:178-181, 317-325)
            const bool srgb = mj.getb("mitsuba_srgb", false);
            ObjFile of = load_obj(dir + "/" + mj.get("path", std::string("")), phong_file);
            std::map<std::string, double> sigma;
            if (mj.has("oren_nayar_sigma"))
                for (auto &kv : mj.at("oren_nayar_sigma").obj) sigma[kv.first] = kv.second.number();
            // materials -> (light | BSDF), assimpio.h:79-121
            std::vector<int> mat_index(of.materials.size(), -1), light_of_mat(of.materials.size(), -1);
            std::vector<Spectrum> ke(of.materials.size());
            for (size_t i = 0; i < of.materials.size(); ++i) {
                const ObjMaterial &om = of.materials[i];
                const V3 kd = srgb ? V3(FromSrgb(om.kd[0]), FromSrgb(om.kd[1]), FromSrgb(om.kd[2]))
                                   : V3(om.kd[0], om.kd[1], om.kd[2]);
                const V3 ks = srgb ? V3(FromSrgb(om.ks[0]), FromSrgb(om.ks[1]), FromSrgb(om.ks[2]))
                                   : V3(om.ks[0], om.ks[1], om.ks[2]);
                ke[i] = V3(om.ke[0], om.ke[1], om.ke[2]);
                if (!IsZero(ke[i])) {
                    if (om.ns / 4.0 != 0.0) throw std::runtime_error("emitter with Ns != 0 (SimpleMetal light) is not supported");
                    light_of_mat[i] = 1;
                }
                Material m;
                Component diffuse;
                diffuse.refl = kd;
                auto it = sigma.find(om.name);
                if (it != sigma.end()) { diffuse.kind = OREN_NAYAR; diffuse.param = it->second; }
                Component glossy;
                glossy.kind = PHONG; glossy.refl = ks; glossy.param = om.ns / 4.0;
                if (IsZero(kd)) m.comps = {glossy};
                else if (IsZero(ks)) m.comps = {diffuse};
                else m.comps = {diffuse, glossy};
                mat_index[i] = int(s->materials.size());
                s->materials.push_back(m);
            }
            std::vector<int> file_surfaces, file_lights;
            for (ObjMesh &om : of.meshes) {
                Geometry g;
                g.pos.resize(om.positions.size() / 3);
                for (size_t k = 0; k < g.pos.size(); ++k)
                    g.pos[k] = V3(double(om.positions[3 * k]), double(om.positions[3 * k + 1]), double(om.positions[3 * k + 2]));
                g.tri = om.triangles;
                const int gi = int(s->geoms.size());
                if (light_of_mat[om.material] >= 0) {
                    AreaLight al; al.intensity = ke[om.material]; al.geometry = gi;
                    g.light = int(s->lights.size());
                    s->lights.push_back(al);
                    // precomputeForSampling (trianglemesh.h:110-129)
                    std::vector<double> areas(g.tri.size() / 3);
                    double sumArea = 0.0;
                    for (size_t t = 0; t < areas.size(); ++t) {
                        const V3 a = g.pos[g.tri[3 * t]], b = g.pos[g.tri[3 * t + 1]], c = g.pos[g.tri[3 * t + 2]];
                        const double area = Length(Cross(b - a, c - a)) / 2.0;
                        sumArea += area;
                        areas[t] = area;
                    }
                    g.area = sumArea; g.inv_area = 1.0 / sumArea;
                    g.tri_cdf = CdfTable(areas);
                    file_lights.push_back(gi);
                } else {
                    g.material = mat_index[om.material];
                    file_surfaces.push_back(gi);
                    if (phong_file) {
                        // PhongMeshGeometry from the Assimp mesh (simple2parser.h:41-52); normals as
                        // AssimpInOut stores them (assimpio.h:211-223): zero when of ~zero length,
                        // else normalised in FP64
                        if (om.missing_normals)
                            throw std::runtime_error("phong_tessellation mesh without per-vertex normals");
                        std::vector<phong::D3> nrm(g.pos.size());
                        for (size_t k = 0; k < nrm.size(); ++k) {
                            const phong::D3 n = phong::d3(om.normals[3 * k], om.normals[3 * k + 1], om.normals[3 * k + 2]);
                            nrm[k] = phong::is_approx_zero(phong::length(n)) ? phong::D3() : phong::normalize(n);
                        }
                        for (size_t t = 0; t < g.tri.size(); t += 3) {
                            phong::Patch P;
                            for (int c = 0; c < 3; ++c) {
                                const V3 &q = g.pos[g.tri[t + c]];
                                P.p[c] = phong::d3(q.x, q.y, q.z);
                                P.n[c] = nrm[g.tri[t + c]];
                            }
                            g.patches.push_back(P);
                        }
                    }
                }
                s->geoms.push_back(std::move(g));
            }
            // Embree attach order: this file's surfaces, then its lights
            for (int gi : file_surfaces) s->geoms[gi].geom_id = next_geom_id++;
            for (int gi : file_lights) s->geoms[gi].geom_id = next_geom_id++;
        }
    }
    s->surface_of_geom.assign(next_geom_id, -1);
    for (size_t gi = 0; gi < s->geoms.size(); ++gi) s->surface_of_geom[s->geoms[gi].geom_id] = int(gi);
    for (int id = 0; id < next_geom_id; ++id) {
        const int gi = s->surface_of_geom[id];
        const Geometry &g = s->geoms[gi];
        if (!g.patches.empty()) {
            // user geometry: Embree keeps the float-rounded patch bounds (embreeaccel.h:63-75)
            for (size_t t = 0; t < g.patches.size(); ++t) {
                double lo[3], hi[3];
                phong::bound(g.patches[t], lo, hi);
                RcUser u;
                for (int k = 0; k < 3; ++k) { u.lo[k] = float(lo[k]); u.hi[k] = float(hi[k]); }
                u.geom = id;
                u.prim = int(t);
                u.ref = gi;
                s->rc.add_user(u);
            }
            continue;
        }
        std::vector<float> pf(g.pos.size() * 3);
        for (size_t k = 0; k < g.pos.size(); ++k) { pf[3 * k] = float(g.pos[k].x); pf[3 * k + 1] = float(g.pos[k].y); pf[3 * k + 2] = float(g.pos[k].z); }
        s->rc.add_mesh(pf.data(), g.tri.data(), int(g.tri.size() / 3), id);
    }
    {
        // the user intersect / occluded callbacks (embreeaccel.h:77-180) around PhongMeshGeometry::intersect
        const Scene *sc = s.get();
        s->rc.user_closest = [sc](const RcUser &u, const float o[3], const float d[3], float tnear, float tfar, RcHit *h) {
            double tmax = tfar;
            phong::D3 n;
            if (!phong::intersect(sc->geoms[u.ref].patches[u.prim], o, d, tnear, &tmax, &n)) return false;
            h->t = float(tmax);
            h->u = 0.f; h->v = 0.f;   // the patch leaves the texture coordinate at zero
            h->ng[0] = float(n.x); h->ng[1] = float(n.y); h->ng[2] = float(n.z);
            h->geom = u.geom; h->prim = u.prim;
            return true;
        };
        s->rc.user_any = [sc](const RcUser &u, const float o[3], const float d[3], float tnear, float tfar) {
            double tmax = tfar;
            phong::D3 n;
            return phong::intersect(sc->geoms[u.ref].patches[u.prim], o, d, tnear, &tmax, &n);
        };
    }
    s->rc.build();
    if (s->env) {   // Scene ctor: envmap->updateSceneRadius(bounding sphere of the accel)
        V3 lo(s->rc.scene_lo[0], s->rc.scene_lo[1], s->rc.scene_lo[2]), hi(s->rc.scene_hi[0], s->rc.scene_hi[1], s->rc.scene_hi[2]);
        s->env->center = (lo + hi) * 0.5;
        s->env->radius = std::sqrt(Length2(lo - hi)) * 0.5;
    }
    // GeneralSubpathSampler ctor: light CDF over |average intensity|, then the environment
    std::vector<double> weights;
    for (const AreaLight &al : s->lights) weights.push_back(Length(al.intensity));
    if (s->env) weights.push_back(1.23);
    s->light_cdf = CdfTable(weights);
    if (root.has("camera")) set_camera(*s, root.at("camera"));
    if (root.has("render") && render_index >= 0 && render_index < int(root.at("render").arr.size())) {
        const Json &rj = root.at("render").arr[render_index];
        s->nverts = int(rj.get("num_path_vertices", 10.0));
        s->spp = int(rj.get("num_spp", 16.0));
        s->output = rj.get("output", std::string(""));
        const std::string integ = rj.get("integrator", std::string("nextevent_path_tracer"));
        if (integ == "primitive_path_tracer") s->integrator = 1;
        else if (integ == "light_splatting") s->integrator = 2;
        else if (integ != "nextevent_path_tracer") throw std::runtime_error("integrator not restated by the oracle: " + integ);
    }
    return s.release();
}

// ------------------------------------------------------------- rendering ----
struct Tile { int x0, y0, x1, y1; };

// Parallel::Split2d's recursive 32x32 block generation (parallel.h:65-115)
static void gen_tiles(int sx, int sy, int ex, int ey, std::vector<Tile> &out) {
    const int bx = ex - sx, by = ey - sy, maxE = std::max(bx, by);
    const int B = 32;
    if (maxE <= B) { if (std::min(bx, by) != 0) out.push_back({sx, sy, ex, ey}); }
    else if (maxE == bx) { const int half = ((bx + B - 1) / B) / 2; const int hx = sx + std::min(half * B, bx); gen_tiles(sx, sy, hx, ey, out); gen_tiles(hx, sy, ex, ey, out); }
    else { const int half = ((by + B - 1) / B) / 2; const int hy = sy + std::min(half * B, by); gen_tiles(sx, sy, ex, hy, out); gen_tiles(sx, hy, ex, ey, out); }
}

struct RenderStats { double seconds = 0.0; long long paths = 0; };

// Renders the tiles that intersect [cx0,cx1) x [cy0,cy1) (the whole film when
// the crop is empty) and writes W*H*3 doubles: base/spp + splat*scale, where
// scale = 1/(spp * number of pixels rendered).
static RenderStats render(const Scene &s, int spp, int nverts, unsigned salt, int cx0, int cy0, int cx1, int cy1,
                          int nthreads, double *out) {
    const int W = s.cam.W, H = s.cam.H;
    Scene &ms = const_cast<Scene &>(s);
    ms.spp = spp; ms.nverts = nverts;
    if (cx1 <= cx0 || cy1 <= cy0) { cx0 = 0; cy0 = 0; cx1 = W; cy1 = H; }
    std::vector<Tile> all, tiles;
    gen_tiles(0, 0, W, H, all);
    for (const Tile &t : all)
        if (t.x0 < cx1 && t.x1 > cx0 && t.y0 < cy1 && t.y1 > cy0) tiles.push_back(t);
    std::vector<double> base(size_t(W) * H * 3, 0.0);
    std::vector<std::atomic<double>> splat(size_t(W) * H * 3);
    for (auto &a : splat) a.store(0.0);
    long long npix = 0;
    for (const Tile &t : tiles) npix += (long long)(t.x1 - t.x0) * (t.y1 - t.y0);
    // light splatting weights every splat by 1/(spp * W * H) (lightsplatting.h:42); over a crop the
    // pixels rendered take the place of W * H
    const double lsInv = 1.0 / double(spp) / double(npix);
    std::atomic<int> next(0);
    auto t0 = std::chrono::steady_clock::now();
    auto worker = [&]() {
        for (;;) {
            const int ti = next++;
            if (ti >= int(tiles.size())) return;
            const Tile &t = tiles[ti];
            const int tileSeed = t.x0 * H + t.y0;
            Sampler smp(unsigned(tileSeed) + salt * 0x9E3779B1u);
            std::vector<Splat> ls;
            for (int y = t.y0; y < t.y1; ++y)
                for (int x = t.x0; x < t.x1; ++x)
                    for (int i = 0; i < spp; ++i) {
                        if (s.integrator == 2) {   // light splatting: only atomic splats, already scaled
                            ls.clear();
                            eval_light_splat(s, smp, lsInv, ls);
                            for (const Splat &sp : ls) {
                                std::atomic<double> *a = &splat[3 * (size_t(int(sp.ry)) * W + int(sp.rx))];
                                const double c[3] = {sp.c.x, sp.c.y, sp.c.z};
                                for (int k = 0; k < 3; ++k) {
                                    double prev = a[k].load();
                                    while (!a[k].compare_exchange_weak(prev, prev + c[k])) {}
                                }
                            }
                            continue;
                        }
                        Splat sp[2];
                        if (s.integrator == 1) eval_primitive(s, smp, x, y, sp);
                        else if (nverts > 1) eval_contribution(s, smp, x, y, sp);
                        const int bx = int(sp[0].rx), by = int(sp[0].ry);
                        double *b = &base[3 * (size_t(by) * W + bx)];
                        b[0] += sp[0].c.x; b[1] += sp[0].c.y; b[2] += sp[0].c.z;
                        const int ax = int(sp[1].rx), ay = int(sp[1].ry);
                        std::atomic<double> *a = &splat[3 * (size_t(ay) * W + ax)];
                        const double c[3] = {sp[1].c.x, sp[1].c.y, sp[1].c.z};
                        for (int k = 0; k < 3; ++k) {
                            double prev = a[k].load();
                            while (!a[k].compare_exchange_weak(prev, prev + c[k])) {}
                        }
                    }
        }
    };
    if (nthreads <= 0) nthreads = int(std::thread::hardware_concurrency());
    std::vector<std::thread> th;
    for (int i = 1; i < nthreads; ++i) th.emplace_back(worker);
    worker();
    for (auto &x : th) x.join();
    RenderStats st;
    st.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    st.paths = npix * spp;
    const double baseScale = 1.0 / double(spp);
    const double atomicScale = s.integrator == 2 ? 1.0 : 1.0 / double(spp) / double(npix);
    for (size_t i = 0; i < base.size(); ++i) {
        double c = 0.0;
        c += base[i] * baseScale;
        c += splat[i].load() * atomicScale;
        out[i] = c;
    }
    return st;
}

}  // namespace oracle

// ------------------------------------------------------------------ C API ----
extern "C" {

static thread_local std::string g_err;

const char *oracle_last_error(void) { return g_err.c_str(); }

void *oracle_scene_load(const char *json_path, int render_index) {
    try {
        return oracle::load_scene(json_path, render_index);
    } catch (const std::exception &e) {
        g_err = e.what();
        return nullptr;
    }
}

void oracle_scene_free(void *s) { delete static_cast<oracle::Scene *>(s); }

// width, height, spp, num_path_vertices of the loaded render entry
void oracle_scene_info(void *sp, int *info4, double *bbox6, int *counts3) {
    auto *s = static_cast<oracle::Scene *>(sp);
    info4[0] = s->cam.W; info4[1] = s->cam.H; info4[2] = s->spp; info4[3] = s->nverts;
    for (int k = 0; k < 3; ++k) { bbox6[k] = s->rc.scene_lo[k]; bbox6[3 + k] = s->rc.scene_hi[k]; }
    counts3[0] = int(s->rc.tris.size() + s->rc.users.size()); counts3[1] = int(s->geoms.size()); counts3[2] = int(s->lights.size());
}

// Overrides the camera with a simple2 camera JSON object (used for batched jobs).
int oracle_set_camera_json(void *sp, const char *camera_json) {
    try {
        auto *s = static_cast<oracle::Scene *>(sp);
        oracle::set_camera(*s, oracle::JsonParser::parse(camera_json));
        return 0;
    } catch (const std::exception &e) {
        g_err = e.what();
        return 1;
    }
}

// Renders W*H*3 doubles into out_rgb (row 0 = top). Returns seconds spent in the render loop.
double oracle_render(void *sp, int spp, int num_path_vertices, unsigned salt, int cx0, int cy0, int cx1, int cy1,
                     int nthreads, double *out_rgb, long long *paths_out) {
    auto *s = static_cast<oracle::Scene *>(sp);
    oracle::RenderStats st = oracle::render(*s, spp, num_path_vertices, salt, cx0, cy0, cx1, cy1, nthreads, out_rgb);
    if (paths_out) *paths_out = st.paths;
    return st.seconds;
}

// Closest-hit queries: rays are n x 8 floats (ox, oy, oz, tnear, dx, dy, dz, tfar).
void oracle_trace_closest(void *sp, const float *rays, int n, int *geom_id, int *prim_id, float *t, float *uv) {
    auto *s = static_cast<oracle::Scene *>(sp);
    for (int i = 0; i < n; ++i) {
        const float *r = rays + 8 * size_t(i);
        oracle::RcHit h;
        const bool hit = s->rc.closest(r, r + 4, r[3], r[7], &h);
        geom_id[i] = hit ? h.geom : -1;
        prim_id[i] = hit ? h.prim : -1;
        t[i] = hit ? h.t : INFINITY;
        uv[2 * i] = h.u; uv[2 * i + 1] = h.v;
    }
}

// Closest hits with the hit's geometry normal as the reference receives it from Embree
// (Ng: unnormalised for triangles, the float-rounded unit patch normal for Phong patches).
void oracle_trace_hits(void *sp, const float *rays, int n, int *geom_id, int *prim_id, float *t, float *ng) {
    auto *s = static_cast<oracle::Scene *>(sp);
    for (int i = 0; i < n; ++i) {
        const float *r = rays + 8 * size_t(i);
        oracle::RcHit h;
        const bool hit = s->rc.closest(r, r + 4, r[3], r[7], &h);
        geom_id[i] = hit ? h.geom : -1;
        prim_id[i] = hit ? h.prim : -1;
        t[i] = hit ? h.t : INFINITY;
        for (int k = 0; k < 3; ++k) ng[3 * i + k] = hit ? h.ng[k] : 0.f;
    }
}

void oracle_trace_occluded(void *sp, const float *rays, int n, int *occluded) {
    auto *s = static_cast<oracle::Scene *>(sp);
    for (int i = 0; i < n; ++i) {
        const float *r = rays + 8 * size_t(i);
        occluded[i] = s->rc.occluded(r, r + 4, r[3], r[7]) ? 1 : 0;
    }
}

// Occlusion bounds per ray (RayCaster::occluded_bracket): lo[i] = blocked beyond doubt,
// hi[i] = possibly blocked, with tolerance eps (barycentric, and relative on the segment ends).
void oracle_trace_occluded_bracket(void *sp, const float *rays, int n, double eps, int *lo, int *hi) {
    auto *s = static_cast<oracle::Scene *>(sp);
    for (int i = 0; i < n; ++i) {
        const float *r = rays + 8 * size_t(i);
        bool l = false, h = false;
        s->rc.occluded_bracket(r, r + 4, r[3], r[7], eps, &l, &h);
        lo[i] = l ? 1 : 0;
        hi[i] = h ? 1 : 0;
    }
}

int oracle_write_pfm(const char *path, const double *rgb, int w, int h) {
    try { oracle::write_pfm(path, rgb, w, h); return 0; }
    catch (const std::exception &e) { g_err = e.what(); return 1; }
}

}  // extern "C"
