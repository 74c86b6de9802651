// simple2 scene loading for the B200 renderer: scene JSON, OBJ/MTL meshes,
// PFM environment maps and PFM output.
//
// Drop-in semantics, following the reference:
//   * JSON keys and defaults of Simple2Parser::Parse/ParseScene
//     (src/sceneio/simple2parser.h:27-68,102-223), ThinlensCamera::FromSimple2ParseJson
//     (src/camera/thinlens.h:13-26; aperture and focal distance both read "radius")
//     and PathNeeRenderer::FromSimple2Json (src/renderer/pathnextevent.h:17-26);
//   * the OBJ/MTL reading the reference gets from Assimp 4.1.0 (one mesh per
//     object x material in file order, material defaults Kd 0.6 / Ks 0 / Ke 0 /
//     Ns 0, DefaultMaterial for faces without usemtl) and the material mapping of
//     AssimpInOut::LoadFromObj (src/sceneio/meshio/assimpio.h:79-150);
//   * the extension key "oren_nayar_sigma" {material: sigma} on a mesh entry
//     selects an Oren-Nayar diffuse lobe (src/bsdf/orennayar.h), which the
//     reference's OBJ path cannot express and its JSON reader ignores;
//   * PFM layout of FimageIo::LoadPfm/SavePfmColor (src/common/floatimage.h:238-277,
//     435-462): "PF\n W H\n-1\n", little-endian float RGB, rows bottom to top.
// Errors are reported as wr::Error with a status code (the reference throws
// std::runtime_error for the same conditions).

#include <cctype>
#include <cerrno>
#include <charconv>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <unordered_map>

#include "wr_host.h"

namespace wr {

// ------------------------------------------------------------------ JSON ----
namespace {

struct JNode {
    enum Kind : uint8_t { NUL, BOOL, NUM, STR, ARR, OBJ } kind = NUL;
    double n = 0.0;
    std::string s;
    std::vector<JNode> items;                       // array items or object values
    std::vector<std::string> keys;                  // object keys (parallel to items)

    const JNode *find(const char *k) const {
        if (kind != OBJ) return nullptr;
        for (size_t i = 0; i < keys.size(); ++i) if (keys[i] == k) return &items[i];
        return nullptr;
    }
    double num(const char *k, double def) const {
        const JNode *v = find(k);
        if (!v) return def;
        if (v->kind == NUM || v->kind == BOOL) return v->n;
        throw Error(WR_ERR_PARSE, std::string("scene json: key '") + k + "' is not a number");
    }
    std::string str(const char *k, const std::string &def) const {
        const JNode *v = find(k);
        if (!v) return def;
        if (v->kind != STR) throw Error(WR_ERR_PARSE, std::string("scene json: key '") + k + "' is not a string");
        return v->s;
    }
};

class JReader {
  public:
    explicit JReader(const std::string &t) : s_(t.c_str()), end_(t.c_str() + t.size()) {}
    JNode parse() {
        JNode v = value();
        skip();
        if (s_ != end_) fail("trailing characters");
        return v;
    }

  private:
    const char *s_, *end_;
    [[noreturn]] void fail(const char *what) { throw Error(WR_ERR_PARSE, std::string("scene json: ") + what); }
    void skip() {
        while (s_ < end_ && (*s_ == ' ' || *s_ == '\t' || *s_ == '\n' || *s_ == '\r')) ++s_;
    }
    bool lit(const char *w) {
        size_t n = strlen(w);
        if (size_t(end_ - s_) >= n && !memcmp(s_, w, n)) { s_ += n; return true; }
        return false;
    }
    std::string string_body() {
        std::string out;
        ++s_;
        while (s_ < end_ && *s_ != '"') {
            if (*s_ == '\\') {
                if (++s_ >= end_) fail("bad escape");
                switch (*s_) {
                    case 'n': out += '\n'; break;
                    case 't': out += '\t'; break;
                    case 'r': out += '\r'; break;
                    case 'b': out += '\b'; break;
                    case 'f': out += '\f'; break;
                    case 'u': {
                        if (end_ - s_ < 5) fail("bad unicode escape");
                        unsigned cp = unsigned(strtoul(std::string(s_ + 1, 4).c_str(), nullptr, 16));
                        if (cp < 0x80) out += char(cp);
                        else if (cp < 0x800) { out += char(0xC0 | (cp >> 6)); out += char(0x80 | (cp & 63)); }
                        else { out += char(0xE0 | (cp >> 12)); out += char(0x80 | ((cp >> 6) & 63)); out += char(0x80 | (cp & 63)); }
                        s_ += 4;
                        break;
                    }
                    default: out += *s_;
                }
                ++s_;
            } else {
                out += *s_++;
            }
        }
        if (s_ >= end_) fail("unterminated string");
        ++s_;
        return out;
    }
    JNode value() {
        skip();
        if (s_ >= end_) fail("unexpected end of input");
        JNode v;
        const char c = *s_;
        if (c == '{') {
            v.kind = JNode::OBJ;
            ++s_;
            skip();
            if (s_ < end_ && *s_ == '}') { ++s_; return v; }
            while (true) {
                skip();
                if (s_ >= end_ || *s_ != '"') fail("expected key");
                v.keys.push_back(string_body());
                skip();
                if (s_ >= end_ || *s_ != ':') fail("expected ':'");
                ++s_;
                v.items.push_back(value());
                skip();
                if (s_ < end_ && *s_ == ',') { ++s_; continue; }
                if (s_ < end_ && *s_ == '}') { ++s_; return v; }
                fail("expected ',' or '}'");
            }
        }
        if (c == '[') {
            v.kind = JNode::ARR;
            ++s_;
            skip();
            if (s_ < end_ && *s_ == ']') { ++s_; return v; }
            while (true) {
                v.items.push_back(value());
                skip();
                if (s_ < end_ && *s_ == ',') { ++s_; continue; }
                if (s_ < end_ && *s_ == ']') { ++s_; return v; }
                fail("expected ',' or ']'");
            }
        }
        if (c == '"') { v.kind = JNode::STR; v.s = string_body(); return v; }
        if (lit("true")) { v.kind = JNode::BOOL; v.n = 1; return v; }
        if (lit("false")) { v.kind = JNode::BOOL; v.n = 0; return v; }
        if (lit("null")) return v;
        char *e = nullptr;
        errno = 0;
        v.n = strtod(s_, &e);
        if (e == s_) fail("unexpected character");
        v.kind = JNode::NUM;
        s_ = e;
        return v;
    }
};

std::string slurp(const std::string &path) {
    FILE *f = fopen(path.c_str(), "rb");
    if (!f) throw Error(WR_ERR_IO, "file not found: " + path);
    std::string data;
    fseek(f, 0, SEEK_END);
    long n = ftell(f);
    fseek(f, 0, SEEK_SET);
    data.resize(size_t(n > 0 ? n : 0));
    if (n > 0 && fread(&data[0], 1, size_t(n), f) != size_t(n)) { fclose(f); throw Error(WR_ERR_IO, "read failed: " + path); }
    fclose(f);
    return data;
}

std::string parent_dir(const std::string &p) {
    size_t k = p.find_last_of('/');
    if (k == std::string::npos) return ".";
    if (k == 0) return "/";
    return p.substr(0, k);
}

std::string join_path(const std::string &dir, const std::string &rel) {
    if (!rel.empty() && rel[0] == '/') return rel;
    return dir + "/" + rel;
}

void vec3_of(const JNode *n, const char *key, double out[3]) {
    // Util::Json::Vec3FromJson: one element -> splat, three -> vector
    if (!n) throw Error(WR_ERR_PARSE, std::string("can't parse ") + key);
    if (n->kind == JNode::NUM) { out[0] = out[1] = out[2] = n->n; return; }
    if (n->kind == JNode::ARR && n->items.size() == 1) { out[0] = out[1] = out[2] = n->items[0].n; return; }
    if (n->kind == JNode::ARR && n->items.size() == 3) { for (int k = 0; k < 3; ++k) out[k] = n->items[k].n; return; }
    throw Error(WR_ERR_PARSE, std::string("can't parse ") + key);
}

Camera camera_of(const JNode &cj) {
    Camera c;
    vec3_of(cj.find("pos"), "pos", c.pos);
    vec3_of(cj.find("lookat"), "lookat", c.lookat);
    vec3_of(cj.find("up"), "up", c.up);
    c.fovy_deg = cj.num("fovy", 90.0);
    if (c.fovy_deg * 3.141592653589793 / 180.0 > 3.141592653589793)
        throw Error(WR_ERR_UNSUPPORTED, "Thinlens camera doesn't support when fov > Pi radians");
    const JNode *res = cj.find("resolution");
    if (!res || res->kind != JNode::ARR || res->items.size() != 2) throw Error(WR_ERR_PARSE, "can't parse resolution");
    c.width = int(res->items[0].n);
    c.height = int(res->items[1].n);
    if (c.width <= 0 || c.height <= 0) throw Error(WR_ERR_INVALID_ARGUMENT, "resolution must be positive");
    c.aperture = cj.num("radius", 0.0);
    c.focal = cj.num("radius", 1.0);
    return c;
}

// ---------------------------------------------------------------- OBJ/MTL ----
struct MtlEntry {
    std::string name;
    float kd[3] = {0.6f, 0.6f, 0.6f};
    float ks[3] = {0.f, 0.f, 0.f};
    float ke[3] = {0.f, 0.f, 0.f};
    float ns = 0.f;
};

inline const char *skip_ws(const char *p, const char *e) {
    while (p < e && (*p == ' ' || *p == '\t' || *p == '\r')) ++p;
    return p;
}
inline const char *token_end(const char *p, const char *e) {
    while (p < e && *p != ' ' && *p != '\t' && *p != '\r' && *p != '\n') ++p;
    return p;
}

// Numbers of the vertex and face lines: std::from_chars after the line's spaces and an optional
// '+' (correctly rounded like strtof, without the locale, several times faster); whatever it does
// not take as a whole (hex floats, out of range, no number) is read by strtol / strtof from the
// same position as before.
inline float read_float(char *&p, const char *le) {
    const char *s = p;
    while (s < le && (*s == ' ' || *s == '\t')) ++s;
    if (s < le && *s == '+') ++s;
    float v = 0.f;
    const auto r = std::from_chars(s, le, v);
    // a letter right after the digits: a hex float ("0x1p3") that only strtof reads whole
    if (r.ec == std::errc() && !(r.ptr < le && isalpha(static_cast<unsigned char>(*r.ptr)))) {
        p = const_cast<char *>(r.ptr);
        return v;
    }
    return strtof(p, &p);
}

inline long read_long(const char *p, const char *le, char **end) {
    const char *s = p;
    if (s < le && *s == '+') ++s;
    long v = 0;
    const auto r = std::from_chars(s, le, v);
    if (r.ec == std::errc()) {
        *end = const_cast<char *>(r.ptr);
        return v;
    }
    return strtol(p, end, 10);
}

void parse_mtl(const std::string &path, std::vector<MtlEntry> &mats, std::unordered_map<std::string, int> &idx) {
    FILE *f = fopen(path.c_str(), "rb");
    if (!f) return;  // a missing library leaves named materials at their defaults
    fclose(f);
    const std::string data = slurp(path);
    const char *p = data.data(), *end = p + data.size();
    MtlEntry *cur = nullptr;
    while (p < end) {
        const char *le = static_cast<const char *>(memchr(p, '\n', size_t(end - p)));
        if (!le) le = end;
        const char *q = skip_ws(p, le);
        const char *te = token_end(q, le);
        std::string key(q, te);
        q = skip_ws(te, le);
        if (key == "newmtl") {
            MtlEntry m;
            m.name = std::string(q, token_end(q, le));
            idx[m.name] = int(mats.size());
            mats.push_back(m);
            cur = &mats.back();
        } else if (cur && (key == "Kd" || key == "Ks" || key == "Ke")) {
            float *dst = key == "Kd" ? cur->kd : key == "Ks" ? cur->ks : cur->ke;
            char *e2 = const_cast<char *>(q);
            for (int k = 0; k < 3; ++k) dst[k] = strtof(e2, &e2);
        } else if (cur && key == "Ns") {
            cur->ns = strtof(q, nullptr);
        }
        p = le + 1;
    }
}

struct ObjMeshRaw {
    std::string name;
    int mtl = 0;
    std::vector<uint32_t> gidx;   // global vertex indices, 3 per triangle
    std::vector<int32_t> nidx;    // global `vn` indices per corner (-1: none)
};

// `phong`: the mesh entry's "phong_tessellation" flag. Its surface meshes become Phong
// tessellation patches (Simple2Parser::ParseScene, src/sceneio/simple2parser.h:37-55) with one
// vertex per distinct (position, normal) pair, as Assimp's JoinIdenticalVertices leaves them;
// its emitters stay triangle meshes (simple2parser.h:58).
// sRGB-encoded reflectance to linear (IEC 61966-2-1 transfer curve), in FP64 as the reference
// converts it (SpectrumConvertUtil::FromSrgb, src/common/math/spectrum.h:13-17)
double srgb_to_linear(double v) {
    if (v <= 0.04045) return v * (1.0 / 12.92);
    return std::pow((v + 0.055) * (1.0 / 1.055), 2.4);
}

// srgb: the mesh entry's "mitsuba_srgb" -- Kd and Ks are sRGB-encoded (assimpio.h:178-181, 317-325)
void load_obj(const std::string &path, const std::map<std::string, double> &sigma, bool phong, bool srgb,
              Scene &scene) {
    const std::string data = slurp(path);
    std::vector<MtlEntry> mats(1);
    mats[0].name = "DefaultMaterial";
    std::unordered_map<std::string, int> mat_idx{{"DefaultMaterial", 0}};
    std::vector<float> verts, norms;
    std::vector<ObjMeshRaw> meshes;
    int cur_mtl = 0;
    auto start_mesh = [&](const std::string &name) {
        meshes.push_back(ObjMeshRaw());
        meshes.back().name = name;
        meshes.back().mtl = cur_mtl;
    };
    const char *p = data.data(), *end = p + data.size();
    std::vector<long> poly, npoly;
    while (p < end) {
        const char *le = static_cast<const char *>(memchr(p, '\n', size_t(end - p)));
        if (!le) le = end;
        const char *q = skip_ws(p, le);
        if (q + 1 < le && q[0] == 'v' && (q[1] == ' ' || q[1] == '\t')) {
            char *e2 = const_cast<char *>(q + 1);
            for (int k = 0; k < 3; ++k) verts.push_back(read_float(e2, le));
        } else if (q + 2 < le && q[0] == 'v' && q[1] == 'n' && (q[2] == ' ' || q[2] == '\t')) {
            char *e2 = const_cast<char *>(q + 2);
            for (int k = 0; k < 3; ++k) norms.push_back(read_float(e2, le));
        } else if (q + 1 < le && q[0] == 'f' && (q[1] == ' ' || q[1] == '\t')) {
            if (meshes.empty()) start_mesh("defaultobject");
            poly.clear();
            npoly.clear();
            const char *r = q + 1;
            const long nv = long(verts.size() / 3), nn = long(norms.size() / 3);
            while (true) {
                r = skip_ws(r, le);
                if (r >= le) break;
                char *e2;
                long v = read_long(r, le, &e2);
                if (e2 == r) break;
                long gi = v < 0 ? nv + v : v - 1;
                if (gi < 0 || gi >= nv) throw Error(WR_ERR_PARSE, "obj: vertex index out of range in " + path);
                poly.push_back(gi);
                long ni = -1;   // v, v/vt, v//vn or v/vt/vn
                if (e2 < le && *e2 == '/') {
                    char *e3 = e2 + 1;
                    if (e3 < le && *e3 != '/') read_long(e3, le, &e3);
                    if (e3 < le && *e3 == '/') {
                        char *e4 = e3 + 1;
                        const long n = read_long(e4, le, &e3);
                        if (e3 != e4) {
                            ni = n < 0 ? nn + n : n - 1;
                            if (ni < 0 || ni >= nn) throw Error(WR_ERR_PARSE, "obj: normal index out of range in " + path);
                        }
                    }
                    e2 = e3;
                }
                npoly.push_back(ni);
                r = token_end(e2, le);
            }
            for (size_t k = 1; k + 1 < poly.size(); ++k) {
                for (size_t c : {size_t(0), k, k + 1}) {
                    meshes.back().gidx.push_back(uint32_t(poly[c]));
                    meshes.back().nidx.push_back(int32_t(npoly[c]));
                }
            }
        } else if (q + 1 < le && (q[0] == 'o' || q[0] == 'g') && (q[1] == ' ' || q[1] == '\t')) {
            const char *n0 = skip_ws(q + 1, le);
            const char *n1 = le;
            while (n1 > n0 && (n1[-1] == ' ' || n1[-1] == '\r' || n1[-1] == '\t')) --n1;
            start_mesh(std::string(n0, n1));
        } else if (le - q > 6 && !strncmp(q, "usemtl", 6)) {
            const char *n0 = skip_ws(q + 6, le);
            std::string name(n0, token_end(n0, le));
            auto it = mat_idx.find(name);
            int id;
            if (it == mat_idx.end()) {
                MtlEntry m;
                m.name = name;
                id = mat_idx[name] = int(mats.size());
                mats.push_back(m);
            } else {
                id = it->second;
            }
            if (id != cur_mtl) {
                cur_mtl = id;
                if (meshes.empty() || !meshes.back().gidx.empty())
                    start_mesh(meshes.empty() ? std::string("defaultobject") : meshes.back().name);
                meshes.back().mtl = cur_mtl;
            }
        } else if (le - q > 6 && !strncmp(q, "mtllib", 6)) {
            const char *n0 = skip_ws(q + 6, le);
            parse_mtl(join_path(parent_dir(path), std::string(n0, token_end(n0, le))), mats, mat_idx);
        }
        p = le + 1;
    }

    // material mapping (assimpio.h:79-121)
    std::vector<int> surface_mat(mats.size(), -1);
    std::vector<bool> emitter(mats.size(), false);
    for (size_t i = 0; i < mats.size(); ++i) {
        const MtlEntry &m = mats[i];
        const bool ke_nonzero = m.ke[0] != 0.f || m.ke[1] != 0.f || m.ke[2] != 0.f;
        if (ke_nonzero) {
            if (double(m.ns) / 4.0 != 0.0)
                throw Error(WR_ERR_UNSUPPORTED, "material '" + m.name + "': emitters with Ns != 0 (SimpleMetal area light) are not supported");
            emitter[i] = true;
        }
        Material mat;
        double kd[3], ks[3];
        for (int k = 0; k < 3; ++k) {
            kd[k] = srgb ? srgb_to_linear(double(m.kd[k])) : double(m.kd[k]);
            ks[k] = srgb ? srgb_to_linear(double(m.ks[k])) : double(m.ks[k]);
            mat.kd[k] = float(kd[k]);
            mat.ks[k] = float(ks[k]);
        }
        mat.exponent = float(double(m.ns) / 4.0);
        // the component choice sees the FP64 reflectances, as the reference's does
        const bool kd_zero = kd[0] == 0.0 && kd[1] == 0.0 && kd[2] == 0.0;
        const bool ks_zero = ks[0] == 0.0 && ks[1] == 0.0 && ks[2] == 0.0;
        if (kd_zero) { mat.has_glossy = true; }
        else if (ks_zero) { mat.has_diffuse = true; }
        else { mat.has_diffuse = true; mat.has_glossy = true; }
        auto s = sigma.find(m.name);
        if (s != sigma.end()) mat.sigma = float(s->second);
        surface_mat[i] = int(scene.materials.size());
        scene.materials.push_back(mat);
    }

    // per-file attach order: surfaces, then emitters (simple2parser.h:38-61)
    std::vector<Mesh> surfaces, emitters;
    std::vector<int32_t> local(verts.size() / 3, -1);
    for (ObjMeshRaw &om : meshes) {
        if (om.gidx.empty()) continue;
        Mesh m;
        m.name = om.name;
        m.indices.resize(om.gidx.size());
        if (phong && !emitter[om.mtl]) {
            // one vertex per distinct (position, normal) pair
            std::unordered_map<uint64_t, uint32_t> pair_idx;
            for (size_t k = 0; k < om.gidx.size(); ++k) {
                if (om.nidx[k] < 0)
                    throw Error(WR_ERR_UNSUPPORTED, "phong_tessellation mesh '" + om.name + "' in " + path +
                                                        " has a face corner without a vertex normal (vn)");
                const uint64_t key = (uint64_t(om.gidx[k]) << 32) | uint32_t(om.nidx[k]);
                auto it = pair_idx.find(key);
                uint32_t li;
                if (it == pair_idx.end()) {
                    li = uint32_t(pair_idx.size());
                    pair_idx.emplace(key, li);
                    for (int c = 0; c < 3; ++c) {
                        m.positions.push_back(verts[3 * size_t(om.gidx[k]) + c]);
                        m.normals.push_back(norms[3 * size_t(om.nidx[k]) + c]);
                    }
                } else {
                    li = it->second;
                }
                m.indices[k] = li;
            }
            m.phong = true;
        } else {
            std::vector<uint32_t> used;
            for (size_t k = 0; k < om.gidx.size(); ++k) {
                const uint32_t g = om.gidx[k];
                if (local[g] < 0) { local[g] = int32_t(used.size()); used.push_back(g); }
                m.indices[k] = uint32_t(local[g]);
            }
            m.positions.resize(used.size() * 3);
            for (size_t k = 0; k < used.size(); ++k) {
                for (int c = 0; c < 3; ++c) m.positions[3 * k + c] = verts[3 * size_t(used[k]) + c];
                local[used[k]] = -1;
            }
        }
        if (emitter[om.mtl]) {
            m.light = int(om.mtl);   // temporarily the material index; resolved below
            emitters.push_back(std::move(m));
        } else {
            m.material = surface_mat[om.mtl];
            surfaces.push_back(std::move(m));
        }
    }
    for (Mesh &m : surfaces) scene.meshes.push_back(std::move(m));
    for (Mesh &m : emitters) {
        const MtlEntry &mt = mats[size_t(m.light)];
        AreaLight al;
        for (int k = 0; k < 3; ++k) al.intensity[k] = mt.ke[k];
        al.mesh = int(scene.meshes.size());
        m.light = int(scene.lights.size());
        scene.lights.push_back(al);
        scene.meshes.push_back(std::move(m));
    }
}

Scene load_from_node(const JNode &root, const std::string &base_dir) {
    if (root.kind != JNode::OBJ) throw Error(WR_ERR_PARSE, "scene json: top level must be an object");
    Scene s;
    s.base_dir = base_dir;
    s.comment = root.str("comment", "");
    const std::string envmap = root.str("envmap", "");
    if (!envmap.empty()) {
        int w = 0, h = 0;
        s.env.rgb = read_image(join_path(base_dir, envmap), &w, &h);
        if (w != 2 * h) throw Error(WR_ERR_INVALID_ARGUMENT, "envmap has wrong size");
        s.env.width = w;
        s.env.height = h;
        s.has_env = true;
    }
    if (const JNode *meshes = root.find("meshes")) {
        if (meshes->kind != JNode::ARR) throw Error(WR_ERR_PARSE, "scene json: 'meshes' must be an array");
        for (const JNode &mj : meshes->items) {
            const bool phong = mj.num("phong_tessellation", 0.0) != 0.0;
            std::map<std::string, double> sigma;
            if (const JNode *sj = mj.find("oren_nayar_sigma")) {
                for (size_t i = 0; i < sj->keys.size(); ++i) sigma[sj->keys[i]] = sj->items[i].n;
            }
            const bool srgb = mj.num("mitsuba_srgb", 0.0) != 0.0;
            load_obj(join_path(base_dir, mj.str("path", "")), sigma, phong, srgb, s);
        }
    }
    if (const JNode *cj = root.find("camera")) {
        s.camera = camera_of(*cj);
        s.has_camera = true;
    }
    if (root.find("medium")) throw Error(WR_ERR_UNSUPPORTED, "participating media are not supported");
    if (const JNode *rs = root.find("render")) {
        for (const JNode &rj : rs->items) {
            RenderEntry r;
            r.integrator = rj.str("integrator", "");
            r.output = rj.str("output", "");
            r.num_spp = int(rj.num("num_spp", 16));
            r.num_path_vertices = int(rj.num("num_path_vertices", 10));
            s.renders.push_back(r);
        }
    }
    return s;
}

}  // namespace

Scene load_simple2_file(const std::string &json_path) {
    const std::string text = slurp(json_path);
    JNode root = JReader(text).parse();
    return load_from_node(root, parent_dir(json_path));
}

Scene load_simple2_text(const std::string &json_text, const std::string &base_dir) {
    JNode root = JReader(json_text).parse();
    return load_from_node(root, base_dir.empty() ? std::string(".") : base_dir);
}

Camera parse_camera_json(const std::string &camera_json) {
    JNode n = JReader(camera_json).parse();
    return camera_of(n);
}

// ------------------------------------------------------------------- PFM ----
void write_pfm(const std::string &path, const double *rgb, int width, int height) {
    FILE *f = fopen(path.c_str(), "wb");
    if (!f) throw Error(WR_ERR_IO, "cannot open file " + path);
    fprintf(f, "PF\n%d %d\n-1\n", width, height);
    std::vector<float> row(size_t(width) * 3);
    for (int y = height - 1; y >= 0; --y) {
        const double *src = rgb + size_t(y) * width * 3;
        for (size_t i = 0; i < row.size(); ++i) row[i] = float(src[i]);
        if (fwrite(row.data(), 4, row.size(), f) != row.size()) { fclose(f); throw Error(WR_ERR_IO, "write failed " + path); }
    }
    fclose(f);
}

std::vector<float> read_pfm(const std::string &path, int *width, int *height) {
    std::ifstream is(path, std::ios::binary);
    if (!is) throw Error(WR_ERR_IO, "cannot find specified PFM file " + path);
    std::string magic, scale;
    is >> magic >> *width >> *height >> scale;
    char c = char(is.get());
    if (c == '\r') is.get();
    if (magic != "PF" && magic != "Pf") throw Error(WR_ERR_PARSE, "not a PFM file: " + path);
    if (*width <= 0 || *height <= 0) throw Error(WR_ERR_PARSE, "bad PFM size: " + path);
    const int nc = magic == "PF" ? 3 : 1;
    std::vector<float> out(size_t(*width) * *height * 3);
    std::vector<float> row(size_t(*width) * nc);
    for (int y = *height - 1; y >= 0; --y) {
        is.read(reinterpret_cast<char *>(row.data()), std::streamsize(row.size() * 4));
        if (!is) throw Error(WR_ERR_PARSE, "truncated PFM file " + path);
        for (int x = 0; x < *width; ++x)
            for (int k = 0; k < 3; ++k) out[(size_t(y) * *width + x) * 3 + k] = row[size_t(x) * nc + (nc == 3 ? k : 0)];
    }
    return out;
}

}  // namespace wr
