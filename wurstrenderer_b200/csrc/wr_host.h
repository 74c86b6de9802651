// Host-side scene model of the B200 renderer: what the simple2 scene loader
// produces and what the device upload consumes.
//
// The model mirrors the objects the reference builds in
// Simple2Parser::ParseScene (src/sceneio/simple2parser.h:27-68):
//   * meshes in Embree attach order -- per OBJ file its surfaces, then its
//     emitters (geomID = position in that order);
//   * one BSDF per surface mesh, from AssimpInOut::LoadFromObj's material
//     mapping (src/sceneio/meshio/assimpio.h:79-121): TwoSided(Lambert | Oren-Nayar
//     | Phong | Mixed(diffuse, Phong)), Phong exponent = Ns / 4;
//   * one diffuse area light per emitter mesh (Ke != 0, Ns == 0);
//   * an optional equirectangular environment light (src/light/envmap.h);
//   * the thin-lens camera of src/camera/thinlens.h:13-26 and the render list.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/wurst_b200.h"

namespace wr {

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

// status codes are the WR_* values of include/wurst_b200.h
struct Material {          // TwoSided(inner) material of one surface mesh
    float kd[3] = {0, 0, 0};
    float ks[3] = {0, 0, 0};
    float exponent = 0.f;  // Phong exponent n
    float sigma = -1.f;    // Oren-Nayar sigma (radians); < 0: Lambert diffuse part
    bool has_diffuse = false, has_glossy = false;
};

struct Mesh {
    std::string name;
    std::vector<float> positions;   // xyz per vertex
    std::vector<uint32_t> indices;  // 3 per triangle
    std::vector<float> normals;     // phong meshes: the OBJ's `vn` per vertex, as read (float xyz)
    bool phong = false;             // Phong tessellation patches instead of flat triangles
    int material = -1;              // surfaces: index into Scene::materials
    int light = -1;                 // emitters: index into Scene::lights
    uint32_t num_triangles() const { return uint32_t(indices.size() / 3); }
};

struct AreaLight {
    float intensity[3];
    int mesh;                       // index into Scene::meshes
};

struct EnvMap {
    int width = 0, height = 0;
    std::vector<float> rgb;         // row 0 = top, 3 floats per texel
};

struct Camera {
    double pos[3], lookat[3], up[3];
    double fovy_deg = 90.0;
    int width = 0, height = 0;
    double aperture = 0.0, focal = 1.0;   // both read from "radius" (thinlens.h:22-23)
};

struct RenderEntry {
    std::string integrator, output;
    int num_spp = 16, num_path_vertices = 10;
};

struct Scene {
    std::vector<Mesh> meshes;       // Embree attach order
    std::vector<Material> materials;
    std::vector<AreaLight> lights;  // mLightGeometries order
    EnvMap env;
    bool has_env = false;
    bool has_camera = false;
    Camera camera;
    std::vector<RenderEntry> renders;
    std::string base_dir;
    std::string comment;
    uint64_t num_triangles() const {
        uint64_t n = 0;
        for (auto &m : meshes) n += m.num_triangles();
        return n;
    }
};

// simple2 loading (wr_scene_io.cpp)
Scene load_simple2_file(const std::string &json_path);
Scene load_simple2_text(const std::string &json_text, const std::string &base_dir);
Camera parse_camera_json(const std::string &camera_json);
void write_pfm(const std::string &path, const double *rgb, int width, int height);
std::vector<float> read_pfm(const std::string &path, int *width, int *height);
// .pfm / .hdr / .exr by extension (FimageIo::LoadAny, src/common/floatimage.h:379-396); RGB, row 0 = top
std::vector<float> read_image(const std::string &path, int *width, int *height);

// BVH (wr_bvh.cpp): binary BVH over all triangles, device node layout
struct BvhBuildResult {
    std::vector<float> nodes;        // 16 floats per node (see wr_device.cuh)
    std::vector<uint32_t> tri_order; // leaf order -> global triangle index
    int depth = 0;
    double sah_cost = 0.0;
};
// Binned-SAH BVH over triangles (9 floats each). trav_cost: SAH cost of a traversal step;
// prim_cost: SAH cost of each primitive's test (null: 1 each), both relative to one triangle test.
BvhBuildResult build_bvh_sah(const std::vector<float> &tri_vertices, int max_leaf, int threads,
                             double trav_cost = 1.0, const std::vector<float> *prim_cost = nullptr);

// Compressed 8-wide BVH collapsed from a binary one whose leaves hold at most 3 triangles
// (layout in wr_bvh.cpp); `order` is the new leaf order -> global triangle index.
struct WideBvh {
    std::vector<uint32_t> nodes;     // 20 words (80 bytes) per node
    std::vector<uint32_t> order;
    int depth = 0;
};
WideBvh build_wide8(const BvhBuildResult &binary);

}  // namespace wr
