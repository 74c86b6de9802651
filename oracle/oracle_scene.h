// Test infrastructure only: the CPU oracle's scene input (JSON, OBJ/MTL, PFM).
//
// This header is part of the oracle, the FP64 CPU restatement of the
// reference's `nextevent_path_tracer` that the tests and the benchmark's CPU
// baseline use as a checker. Nothing in the product links it.
//
// It restates the input semantics the reference depends on:
//   * simple2 scene JSON keys (src/sceneio/simple2parser.h:27-68,102-223,
//     src/camera/thinlens.h:13-26, src/renderer/pathnextevent.h:17-26);
//   * Assimp 4.1.0's OBJ/MTL import as the reference consumes it
//     (src/sceneio/meshio/assimpio.h:61-153,155-279,287-337; Assimp's material
//     defaults Kd 0.6, Ks 0, Ke 0, Ns 0 from dependencies/assimp/code/ObjFileData.h:187-193;
//     one mesh per object x material, dependencies/assimp/code/ObjFileParser.cpp:543-600);
//   * PFM read/write (src/common/floatimage.h:238-277,435-462).
// Numbers are parsed with strtof/strtod (Assimp's fast_atof may differ by one
// ulp on some inputs; the scene writers emit %.9g so both agree).
#pragma once

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace oracle {

// ---------------------------------------------------------------- JSON ----
struct Json {
    enum Type { Null, Bool, Num, Str, Arr, Obj } type = Null;
    bool b = false;
    double num = 0.0;
    std::string str;
    std::vector<Json> arr;
    std::vector<std::pair<std::string, Json>> obj;

    bool has(const std::string &k) const {
        if (type != Obj) return false;
        for (auto &kv : obj) if (kv.first == k) return true;
        return false;
    }
    const Json &at(const std::string &k) const {
        for (auto &kv : obj) if (kv.first == k) return kv.second;
        throw std::runtime_error("json: missing key " + k);
    }
    double number() const {
        if (type == Num) return num;
        if (type == Bool) return b ? 1.0 : 0.0;
        throw std::runtime_error("json: not a number");
    }
    double get(const std::string &k, double def) const { return has(k) ? at(k).number() : def; }
    std::string get(const std::string &k, const std::string &def) const {
        return has(k) ? at(k).str : def;
    }
    bool getb(const std::string &k, bool def) const { return has(k) ? at(k).number() != 0.0 : def; }
};

struct JsonParser {
    const char *p, *e;
    void ws() { while (p < e && (*p == ' ' || *p == '\n' || *p == '\r' || *p == '\t')) ++p; }
    [[noreturn]] void fail(const char *m) { throw std::runtime_error(std::string("json: ") + m); }
    Json value() {
        ws();
        if (p >= e) fail("unexpected end");
        Json j;
        if (*p == '{') {
            j.type = Json::Obj; ++p; ws();
            if (p < e && *p == '}') { ++p; return j; }
            for (;;) {
                ws(); Json k = value(); if (k.type != Json::Str) fail("key");
                ws(); if (p >= e || *p != ':') fail("colon"); ++p;
                j.obj.emplace_back(k.str, value()); ws();
                if (p < e && *p == ',') { ++p; continue; }
                if (p < e && *p == '}') { ++p; return j; }
                fail("object");
            }
        }
        if (*p == '[') {
            j.type = Json::Arr; ++p; ws();
            if (p < e && *p == ']') { ++p; return j; }
            for (;;) {
                j.arr.push_back(value()); ws();
                if (p < e && *p == ',') { ++p; continue; }
                if (p < e && *p == ']') { ++p; return j; }
                fail("array");
            }
        }
        if (*p == '"') {
            j.type = Json::Str; ++p;
            while (p < e && *p != '"') {
                if (*p == '\\' && p + 1 < e) {
                    ++p;
                    char c = *p;
                    j.str.push_back(c == 'n' ? '\n' : c == 't' ? '\t' : c);
                } else j.str.push_back(*p);
                ++p;
            }
            if (p >= e) fail("string");
            ++p; return j;
        }
        if (!strncmp(p, "true", 4)) { j.type = Json::Bool; j.b = true; p += 4; return j; }
        if (!strncmp(p, "false", 5)) { j.type = Json::Bool; j.b = false; p += 5; return j; }
        if (!strncmp(p, "null", 4)) { p += 4; return j; }
        char *end = nullptr;
        j.num = strtod(p, &end);
        if (end == p) fail("value");
        j.type = Json::Num; p = end; return j;
    }
    static Json parse(const std::string &s) {
        JsonParser jp{s.data(), s.data() + s.size()};
        return jp.value();
    }
};

inline std::string read_file(const std::string &path) {
    std::ifstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("file not found: " + path);
    std::stringstream ss; ss << f.rdbuf(); return ss.str();
}

inline std::string dir_of(const std::string &path) {
    size_t k = path.find_last_of('/');
    return k == std::string::npos ? std::string(".") : path.substr(0, k);
}

// ------------------------------------------------------------- OBJ/MTL ----
struct ObjMaterial {
    std::string name;
    double kd[3] = {0.6, 0.6, 0.6};   // Assimp ObjFile::Material default diffuse
    double ks[3] = {0.0, 0.0, 0.0};
    double ke[3] = {0.0, 0.0, 0.0};
    double ns = 0.0;                  // raw MTL shininess; the exponent is ns / 4
};

struct ObjMesh {
    std::string name;
    int material = 0;                   // index into ObjFile::materials
    std::vector<float> positions;       // 3 floats per vertex (local to the mesh)
    std::vector<int> triangles;         // 3 local indices per triangle
    // with load_obj(path, true): one vertex per distinct (position, normal) pair and the `vn`
    // normal of each vertex as read (zero where a face corner has none)
    std::vector<float> normals;
    bool missing_normals = false;       // some face corner has no `vn`
};

struct ObjFile {
    std::vector<ObjMaterial> materials; // [0] = Assimp's DefaultMaterial
    std::vector<ObjMesh> meshes;        // Assimp mesh order: objects in file order
};

inline void load_mtl(const std::string &path, ObjFile &of, std::map<std::string, int> &byname) {
    std::ifstream f(path);
    if (!f) return;  // Assimp continues without the library
    std::string line;
    ObjMaterial *cur = nullptr;
    while (std::getline(f, line)) {
        std::istringstream ls(line);
        std::string k; ls >> k;
        if (k == "newmtl") {
            std::string n; ls >> n;
            of.materials.push_back(ObjMaterial());
            of.materials.back().name = n;
            byname[n] = int(of.materials.size()) - 1;
            cur = &of.materials.back();
        } else if (cur && (k == "Kd" || k == "Ks" || k == "Ke")) {
            double *dst = k == "Kd" ? cur->kd : k == "Ks" ? cur->ks : cur->ke;
            std::string t[3]; ls >> t[0] >> t[1] >> t[2];
            for (int i = 0; i < 3; ++i) dst[i] = double(strtof(t[i].c_str(), nullptr));
        } else if (cur && k == "Ns") {
            std::string t; ls >> t; cur->ns = double(strtof(t.c_str(), nullptr));
        }
    }
}

// `pairs`: key vertices by (position, normal) pair, as Assimp's JoinIdenticalVertices does
// for meshes that carry normals (the Phong tessellation input); otherwise by position.
inline ObjFile load_obj(const std::string &path, bool pairs = false) {
    std::ifstream f(path);
    if (!f) throw std::runtime_error("cannot open file " + path);
    ObjFile of;
    of.materials.push_back(ObjMaterial());
    of.materials[0].name = "DefaultMaterial";
    std::map<std::string, int> byname;
    byname["DefaultMaterial"] = 0;
    std::vector<float> v, vn;          // global vertex and normal lists
    int cur_mat = 0;
    ObjMesh *mesh = nullptr;
    std::map<std::pair<int, int>, int> remap;   // global (vertex, normal) -> local index of the current mesh
    auto new_mesh = [&](const std::string &name) {
        of.meshes.push_back(ObjMesh());
        of.meshes.back().name = name;
        of.meshes.back().material = cur_mat;
        mesh = &of.meshes.back();
        remap.clear();
    };
    std::string line;
    while (std::getline(f, line)) {
        const char *s = line.c_str();
        while (*s == ' ' || *s == '\t') ++s;
        if (s[0] == 'v' && (s[1] == ' ' || s[1] == '\t')) {
            char *end = const_cast<char *>(s + 1);
            for (int i = 0; i < 3; ++i) v.push_back(strtof(end, &end));
        } else if (s[0] == 'v' && s[1] == 'n' && (s[2] == ' ' || s[2] == '\t')) {
            char *end = const_cast<char *>(s + 2);
            for (int i = 0; i < 3; ++i) vn.push_back(strtof(end, &end));
        } else if ((s[0] == 'o' || s[0] == 'g') && (s[1] == ' ' || s[1] == '\t')) {
            std::string name(s + 2);
            new_mesh(name);
        } else if (!strncmp(s, "usemtl", 6)) {
            std::istringstream ls(s + 6);
            std::string n; ls >> n;
            int id;
            auto it = byname.find(n);
            if (it == byname.end()) {
                of.materials.push_back(ObjMaterial());
                of.materials.back().name = n;
                id = byname[n] = int(of.materials.size()) - 1;
            } else id = it->second;
            if (id == cur_mat) continue;
            cur_mat = id;
            if (!mesh || !mesh->triangles.empty()) new_mesh(mesh ? mesh->name : std::string("defaultobject"));
            mesh->material = cur_mat;
        } else if (!strncmp(s, "mtllib", 6)) {
            std::istringstream ls(s + 6);
            std::string n; ls >> n;
            load_mtl(dir_of(path) + "/" + n, of, byname);
        } else if (s[0] == 'f' && (s[1] == ' ' || s[1] == '\t')) {
            if (!mesh) new_mesh("defaultobject");
            std::istringstream ls(s + 1);
            std::string tok;
            std::vector<int> poly;
            const int nv = int(v.size() / 3), nn = int(vn.size() / 3);
            while (ls >> tok) {
                int gi = atoi(tok.c_str());
                gi = gi < 0 ? nv + gi : gi - 1;
                if (gi < 0 || gi >= nv) throw std::runtime_error("obj: bad vertex index");
                int ni = -1;   // v, v/vt, v//vn, v/vt/vn
                const size_t s1 = tok.find('/');
                if (s1 != std::string::npos) {
                    const size_t s2 = tok.find('/', s1 + 1);
                    if (s2 != std::string::npos && s2 + 1 < tok.size()) {
                        ni = atoi(tok.c_str() + s2 + 1);
                        ni = ni < 0 ? nn + ni : ni - 1;
                        if (ni < 0 || ni >= nn) throw std::runtime_error("obj: bad normal index");
                    }
                }
                const std::pair<int, int> key(gi, pairs ? ni : -1);
                auto it = remap.find(key);
                int li;
                if (it == remap.end()) {
                    li = int(mesh->positions.size() / 3);
                    remap[key] = li;
                    for (int k = 0; k < 3; ++k) mesh->positions.push_back(v[3 * gi + k]);
                    if (pairs) {
                        for (int k = 0; k < 3; ++k) mesh->normals.push_back(ni >= 0 ? vn[3 * ni + k] : 0.f);
                        if (ni < 0) mesh->missing_normals = true;
                    }
                } else li = it->second;
                poly.push_back(li);
            }
            for (size_t k = 1; k + 1 < poly.size(); ++k) {
                mesh->triangles.push_back(poly[0]);
                mesh->triangles.push_back(poly[k]);
                mesh->triangles.push_back(poly[k + 1]);
            }
        }
    }
    std::vector<ObjMesh> kept;
    for (auto &m : of.meshes) if (!m.triangles.empty()) kept.push_back(std::move(m));
    of.meshes.swap(kept);
    return of;
}

// ----------------------------------------------------------------- PFM ----
// Rows are stored bottom-to-top; image row 0 is the top row.
inline void write_pfm(const std::string &path, const double *rgb, int w, int h) {
    std::ofstream os(path, std::ios::binary);
    if (!os) throw std::runtime_error("cannot open file " + path);
    os << "PF\n" << w << " " << h << "\n-1\n";
    for (int y = h; y >= 1; --y)
        for (int x = 0; x < w; ++x)
            for (int c = 0; c < 3; ++c) {
                float f = float(rgb[3 * (size_t(y - 1) * w + x) + c]);
                os.write(reinterpret_cast<const char *>(&f), 4);
            }
}

inline std::vector<float> read_pfm(const std::string &path, int *w, int *h) {
    std::ifstream is(path, std::ios::binary);
    if (!is) throw std::runtime_error("cannot find PFM file " + path);
    std::string pf, scale;
    is >> pf >> *w >> *h >> scale;
    char c = char(is.get());
    if (c == '\r') is.get();
    if (pf != "PF" && pf != "Pf") throw std::runtime_error("not a PFM file");
    const int nc = pf == "PF" ? 3 : 1;
    std::vector<float> out(size_t(*w) * *h * 3);
    std::vector<float> row(size_t(*w) * nc);
    for (int y = *h; y > 0; --y) {
        is.read(reinterpret_cast<char *>(row.data()), row.size() * 4);
        for (int x = 0; x < *w; ++x)
            for (int k = 0; k < 3; ++k)
                out[3 * (size_t(y - 1) * *w + x) + k] = row[size_t(x) * nc + (nc == 3 ? k : 0)];
    }
    return out;
}

}  // namespace oracle
