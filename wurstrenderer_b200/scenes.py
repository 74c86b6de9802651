"""Seeded procedural scene writers for the benchmark workloads.

Every scene is written in the reference's own input format -- a simple2 scene
JSON (``camera``/``meshes``/``render`` keys, ``src/sceneio/simple2parser.h:102-223``)
plus OBJ/MTL meshes (read through Assimp's OBJ importer in the reference,
``src/sceneio/meshio/assimpio.h:61-153``) -- so the reference renderer, the
oracle and this framework all read the same files.

Conventions the writers follow so that the reference's loader semantics apply:

* one ``o``/``usemtl`` pair per mesh, triangles only (Assimp's triangulation of
  polygons is never exercised);
* ``Ns`` is written as ``4 * exponent`` because the reference divides the
  Assimp shininess by 4 (``assimpio.h:310-315``);
* emitters carry ``Ke`` and ``Ns 0`` so they become diffuse area lights
  (``assimpio.h:84-91``); their front face (``cross(p1-p0, p2-p0)``) points into
  the scene;
* Oren-Nayar materials, which the reference only builds programmatically
  (``src/bsdf/orennayar.h:10-12``), are requested with the extension key
  ``"oren_nayar_sigma": {material name: sigma in radians}`` on a mesh entry;
  the reference's ``Util::Json::GetValue`` ignores unknown keys.

Numbers are written with ``%.9g`` so every float32 survives the text round trip.
"""
from __future__ import annotations

import json
import math
import os
from dataclasses import dataclass, field

import numpy as np


# --------------------------------------------------------------------------
# mesh building blocks
# --------------------------------------------------------------------------

@dataclass
class Material:
    name: str
    kd: tuple = (0.0, 0.0, 0.0)
    ks: tuple = (0.0, 0.0, 0.0)
    exponent: float = 0.0          # modified-Phong exponent n (written as Ns = 4n)
    ke: tuple = (0.0, 0.0, 0.0)
    sigma: float | None = None     # Oren-Nayar roughness in radians (extension)


@dataclass
class Mesh:
    name: str
    material: str
    positions: np.ndarray          # (V, 3) float32
    triangles: np.ndarray          # (T, 3) int, 0-based, local to this mesh
    normals: np.ndarray | None = None   # (V, 3) float32 vertex normals, written as `vn`


@dataclass
class SceneSpec:
    meshes: list = field(default_factory=list)
    materials: dict = field(default_factory=dict)

    def add(self, name, material, positions, triangles, normals=None):
        self.meshes.append(Mesh(name, material.name,
                                np.asarray(positions, np.float32),
                                np.asarray(triangles, np.int64),
                                None if normals is None else np.asarray(normals, np.float32)))
        self.materials.setdefault(material.name, material)

    @property
    def num_triangles(self):
        return int(sum(m.triangles.shape[0] for m in self.meshes))


def quad(p0, p1, p2, p3):
    """Two triangles (p0,p1,p2), (p0,p2,p3); front face = cross(p1-p0, p2-p0)."""
    return np.array([p0, p1, p2, p3], np.float64), np.array([[0, 1, 2], [0, 2, 3]])


def grid_quad(origin, du, dv, n_u, n_v):
    """A parallelogram origin + s*du + t*dv tessellated into n_u x n_v quads."""
    origin, du, dv = (np.asarray(a, np.float64) for a in (origin, du, dv))
    s = np.linspace(0.0, 1.0, n_u + 1)
    t = np.linspace(0.0, 1.0, n_v + 1)
    ss, tt = np.meshgrid(s, t, indexing="ij")
    pos = origin + ss[..., None] * du + tt[..., None] * dv
    pos = pos.reshape(-1, 3)
    i, j = np.meshgrid(np.arange(n_u), np.arange(n_v), indexing="ij")
    v00 = (i * (n_v + 1) + j).ravel()
    v10 = ((i + 1) * (n_v + 1) + j).ravel()
    v11 = ((i + 1) * (n_v + 1) + j + 1).ravel()
    v01 = (i * (n_v + 1) + j + 1).ravel()
    tris = np.concatenate([np.stack([v00, v10, v11], 1), np.stack([v00, v11, v01], 1)])
    return pos, tris


def box(center, size, angle_y=0.0, tess=1):
    """Closed box: 6 faces, each tess x tess quads (12 * tess^2 triangles)."""
    c = np.asarray(center, np.float64)
    h = np.asarray(size, np.float64) * 0.5
    ca, sa = math.cos(angle_y), math.sin(angle_y)
    rot = np.array([[ca, 0.0, sa], [0.0, 1.0, 0.0], [-sa, 0.0, ca]])
    faces = []
    for axis in range(3):
        for sign in (-1.0, 1.0):
            u_axis, v_axis = (axis + 1) % 3, (axis + 2) % 3
            if sign < 0:
                u_axis, v_axis = v_axis, u_axis
            o = np.zeros(3)
            o[axis] = sign * h[axis]
            o[u_axis] = -h[u_axis]
            o[v_axis] = -h[v_axis]
            du = np.zeros(3); du[u_axis] = 2 * h[u_axis]
            dv = np.zeros(3); dv[v_axis] = 2 * h[v_axis]
            faces.append(grid_quad(o, du, dv, tess, tess))
    pos, tris, off = [], [], 0
    for p, t in faces:
        pos.append(p); tris.append(t + off); off += p.shape[0]
    pos = np.concatenate(pos) @ rot.T + c
    return pos, np.concatenate(tris)


def icosphere(center, radius, subdivisions):
    """Icosahedron subdivided `subdivisions` times: 20 * 4**subdivisions faces."""
    t = (1.0 + math.sqrt(5.0)) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0),
             (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
             (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11),
             (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6), (7, 1, 8),
             (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9),
             (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    v = np.array(verts, np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    f = np.array(faces, np.int64)
    for _ in range(subdivisions):
        edges = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
        edges.sort(axis=1)
        uniq, inv = np.unique(edges, axis=0, return_inverse=True)
        mids = v[uniq[:, 0]] + v[uniq[:, 1]]
        mids /= np.linalg.norm(mids, axis=1, keepdims=True)
        base = v.shape[0]
        v = np.concatenate([v, mids])
        nf = f.shape[0]
        m01 = base + inv[:nf]; m12 = base + inv[nf:2 * nf]; m20 = base + inv[2 * nf:]
        f = np.concatenate([np.stack([f[:, 0], m01, m20], 1),
                            np.stack([f[:, 1], m12, m01], 1),
                            np.stack([f[:, 2], m20, m12], 1),
                            np.stack([m01, m12, m20], 1)])
    return v * radius + np.asarray(center, np.float64), f


def fbm_heightfield(n, extent, amplitude, octaves, rng):
    """n x n heights over [-extent, extent]^2 from seeded value-noise fBm."""
    xs = np.linspace(0.0, 1.0, n)
    h = np.zeros((n, n))
    amp, freq = 1.0, 4.0
    total = 0.0
    for _ in range(octaves):
        g = int(math.ceil(freq)) + 2
        lattice = rng.uniform(-1.0, 1.0, size=(g, g))
        x = xs * freq
        i0 = np.floor(x).astype(np.int64)
        fx = x - i0
        fx = fx * fx * (3.0 - 2.0 * fx)
        a = lattice[i0[:, None], i0[None, :]]
        b = lattice[i0[:, None] + 1, i0[None, :]]
        c = lattice[i0[:, None], i0[None, :] + 1]
        d = lattice[i0[:, None] + 1, i0[None, :] + 1]
        wx = fx[:, None]; wy = fx[None, :]
        h += amp * ((a * (1 - wx) + b * wx) * (1 - wy) + (c * (1 - wx) + d * wx) * wy)
        total += amp
        amp *= 0.5
        freq *= 2.0
    h *= amplitude / total
    gx, gz = np.meshgrid(np.linspace(-extent, extent, n), np.linspace(-extent, extent, n), indexing="ij")
    pos = np.stack([gx, h, gz], -1).reshape(-1, 3)
    i, j = np.meshgrid(np.arange(n - 1), np.arange(n - 1), indexing="ij")
    v00 = (i * n + j).ravel(); v10 = ((i + 1) * n + j).ravel()
    v11 = ((i + 1) * n + j + 1).ravel(); v01 = (i * n + j + 1).ravel()
    # front faces point up (+y): cross(p1-p0, p2-p0) with p1 along +z first
    tris = np.concatenate([np.stack([v00, v01, v11], 1), np.stack([v00, v11, v10], 1)])
    return pos, tris, h


# --------------------------------------------------------------------------
# writers
# --------------------------------------------------------------------------

def _fmt3(v):
    return "%.9g %.9g %.9g" % tuple(float(np.float32(x)) for x in v)


def write_obj(spec: SceneSpec, obj_path: str, mtl_name: str):
    """Writes one OBJ (global 1-based vertex indices) and its MTL. Meshes with normals get
    one `vn` per vertex and `f v//vn` faces (normal index = vertex index)."""
    with open(obj_path, "w") as f:
        f.write("mtllib %s\n" % mtl_name)
        base = 1
        nbase = 1
        for m in spec.meshes:
            f.write("o %s\nusemtl %s\n" % (m.name, m.material))
            np.savetxt(f, m.positions.astype(np.float32), fmt="v %.9g %.9g %.9g")
            if m.normals is not None:
                np.savetxt(f, m.normals.astype(np.float32), fmt="vn %.9g %.9g %.9g")
                idx = m.triangles + base
                nidx = m.triangles + nbase
                np.savetxt(f, np.stack([idx[:, 0], nidx[:, 0], idx[:, 1], nidx[:, 1], idx[:, 2], nidx[:, 2]], 1),
                           fmt="f %d//%d %d//%d %d//%d")
                nbase += m.normals.shape[0]
            else:
                np.savetxt(f, m.triangles + base, fmt="f %d %d %d")
            base += m.positions.shape[0]
    mtl_path = os.path.join(os.path.dirname(obj_path), mtl_name)
    with open(mtl_path, "w") as f:
        for mat in spec.materials.values():
            f.write("newmtl %s\n" % mat.name)
            f.write("Kd %s\n" % _fmt3(mat.kd))
            f.write("Ks %s\n" % _fmt3(mat.ks))
            f.write("Ns %.9g\n" % float(np.float32(4.0 * mat.exponent)))
            f.write("Ke %s\n" % _fmt3(mat.ke))
            f.write("\n")


def write_scene(out_dir, name, spec, camera, renders, envmap=None, extra=None):
    """Writes `<name>.obj`, `<name>.mtl` and `<name>.json`; returns the JSON path."""
    os.makedirs(out_dir, exist_ok=True)
    obj_name = name + ".obj"
    write_obj(spec, os.path.join(out_dir, obj_name), name + ".mtl")
    mesh_entry = {"path": obj_name}
    sig = {m.name: float(m.sigma) for m in spec.materials.values() if m.sigma is not None}
    if sig:
        mesh_entry["oren_nayar_sigma"] = sig
    scene = {"comment": name, "camera": camera, "meshes": [mesh_entry], "render": renders}
    if envmap is not None:
        scene["envmap"] = envmap
    if extra:
        scene.update(extra)
    path = os.path.join(out_dir, name + ".json")
    with open(path, "w") as f:
        json.dump(scene, f, indent=1)
    return path


def write_scene_entries(out_dir, name, entries, camera, renders, envmap=None):
    """Writes a scene with several mesh entries: `entries` is a list of (suffix, spec, extra
    mesh-entry keys); each spec goes to `<name>_<suffix>.obj/.mtl`. Returns the JSON path."""
    os.makedirs(out_dir, exist_ok=True)
    meshes = []
    for suffix, spec, extra in entries:
        base = "%s_%s" % (name, suffix)
        write_obj(spec, os.path.join(out_dir, base + ".obj"), base + ".mtl")
        entry = {"path": base + ".obj"}
        sig = {m.name: float(m.sigma) for m in spec.materials.values() if m.sigma is not None}
        if sig:
            entry["oren_nayar_sigma"] = sig
        entry.update(extra or {})
        meshes.append(entry)
    scene = {"comment": name, "camera": camera, "meshes": meshes, "render": renders}
    if envmap is not None:
        scene["envmap"] = envmap
    path = os.path.join(out_dir, name + ".json")
    with open(path, "w") as f:
        json.dump(scene, f, indent=1)
    return path


def vertex_normals(positions, triangles):
    """Area-weighted vertex normals (unit, float32) of an indexed triangle mesh."""
    p = np.asarray(positions, np.float64)
    t = np.asarray(triangles, np.int64)
    fn = np.cross(p[t[:, 1]] - p[t[:, 0]], p[t[:, 2]] - p[t[:, 0]])
    n = np.zeros_like(p)
    for c in range(3):
        np.add.at(n, t[:, c], fn)
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    return n.astype(np.float32)


def nee_render(output, spp, num_path_vertices):
    return {"integrator": "nextevent_path_tracer", "output": output,
            "num_spp": int(spp), "num_path_vertices": int(num_path_vertices)}


# --------------------------------------------------------------------------
# workloads
# --------------------------------------------------------------------------

# rotation about y of the two boxes in the Cornell-box test fixtures (tests/golden/scenes): turned
# boxes exercise faces that no axis slab bounds tightly; the workloads keep them axis-aligned
FIXTURE_BOX_ANGLE = 0.3


def cornell_spec(seed=1001, light_ke=(17.0, 12.0, 4.0), box_angle=0.0):
    """Procedural Cornell box: 5 walls (10 tris) + 2 boxes (24) + light (2) = 36 tris. The boxes are
    axis-aligned (workload C1) unless box_angle turns them about y (by -box_angle and +box_angle)."""
    rng = np.random.default_rng(seed)
    alb = lambda: tuple(rng.uniform(0.2, 0.8, 3))
    spec = SceneSpec()
    walls = {
        "floor": quad((-1, 0, -1), (-1, 0, 1), (1, 0, 1), (1, 0, -1)),
        "ceiling": quad((-1, 2, -1), (1, 2, -1), (1, 2, 1), (-1, 2, 1)),
        "back": quad((-1, 0, -1), (1, 0, -1), (1, 2, -1), (-1, 2, -1)),
        "left": quad((-1, 0, -1), (-1, 2, -1), (-1, 2, 1), (-1, 0, 1)),
        "right": quad((1, 0, -1), (1, 0, 1), (1, 2, 1), (1, 2, -1)),
    }
    colors = {"floor": alb(), "ceiling": alb(), "back": alb(),
              "left": (rng.uniform(0.6, 0.8), 0.2, 0.2),
              "right": (0.2, rng.uniform(0.6, 0.8), 0.2)}
    for name, (p, t) in walls.items():
        spec.add(name, Material("m_" + name, kd=colors[name]), p, t)
    p, t = box((0.35, 0.3, 0.3), (0.6, 0.6, 0.6), angle_y=-box_angle)
    spec.add("short_box", Material("m_short_box", kd=alb()), p, t)
    p, t = box((-0.35, 0.6, -0.35), (0.6, 1.2, 0.6), angle_y=box_angle)
    spec.add("tall_box", Material("m_tall_box", kd=alb()), p, t)
    y = 2.0 - 1e-3
    p, t = quad((-0.25, y, -0.25), (0.25, y, -0.25), (0.25, y, 0.25), (-0.25, y, 0.25))
    spec.add("light", Material("m_light", kd=(0, 0, 0), ke=light_ke), p, t)
    return spec


CORNELL_CAMERA = {"pos": [0.0, 1.0, 3.6], "lookat": [0.0, 1.0, 0.0], "up": [0.0, 1.0, 0.0],
                  "fovy": 40.0, "resolution": [256, 256]}


def write_cornell(out_dir, name="cornell", resolution=(256, 256), spp=16,
                  num_path_vertices=10, seed=1001, spec=None, output=None):
    """Workload C1: 256x256, 16 spp, max depth 8 (num_path_vertices 10)."""
    spec = spec or cornell_spec(seed)
    cam = dict(CORNELL_CAMERA, resolution=list(resolution))
    return write_scene(out_dir, name, spec, cam,
                       [nee_render(output or name + ".pfm", spp, num_path_vertices)])


def write_cornell_lens(out_dir, name="lens", resolution=(48, 48), spp=4, num_path_vertices=10, radius=0.1):
    """The Cornell box (fixture variant, turned boxes) seen through a thin lens: the simple2
    camera's "radius" key is both the aperture radius and the focal distance
    (src/camera/thinlens.h:22-23)."""
    cam = dict(CORNELL_CAMERA, resolution=list(resolution), radius=float(radius))
    return write_scene(out_dir, name, cornell_spec(box_angle=FIXTURE_BOX_ANGLE), cam,
                       [nee_render(name + ".pfm", spp, num_path_vertices)])


def write_srgb_zoo(out_dir, name="srgb", resolution=(48, 40), spp=4, num_path_vertices=10):
    """The material zoo in one mesh entry with "mitsuba_srgb": true: its Kd and Ks are read as
    sRGB-encoded and linearised, its Ke and Ns are not (src/sceneio/meshio/assimpio.h:178-181)."""
    cam = dict(CORNELL_CAMERA, resolution=list(resolution))
    return write_scene_entries(out_dir, name, [("zoo", material_zoo_spec(), {"mitsuba_srgb": True})], cam,
                               [nee_render(name + ".pfm", spp, num_path_vertices)])


def phong_objects_spec(seed=1007, n_objects=5):
    """Smooth low-poly objects for Phong tessellation: icospheres (1-2 subdivisions) and
    radially perturbed blobs, each with area-weighted vertex normals; diffuse, glossy
    and mixed materials."""
    rng = np.random.default_rng(seed)
    spec = SceneSpec()
    centers = [(-0.5, 0.32, 0.25), (0.45, 0.3, 0.35), (0.0, 0.9, -0.4), (-0.45, 1.35, -0.2), (0.5, 1.0, -0.35)]
    radii = [0.3, 0.28, 0.33, 0.25, 0.22]
    for i in range(n_objects):
        p, t = icosphere(centers[i], radii[i], 1 + (i % 2))
        if i >= 3:   # a blob: radius varies smoothly with direction
            d = (p - np.asarray(centers[i])) / radii[i]
            r = radii[i] * (1.0 + 0.18 * d[:, 0] * d[:, 1] + 0.12 * d[:, 2] ** 2)
            p = np.asarray(centers[i]) + d * r[:, None]
        n = vertex_normals(p, t)
        kind = i % 3
        if kind == 0:
            mat = Material("m_phong%d" % i, kd=tuple(rng.uniform(0.3, 0.8, 3)))
        elif kind == 1:
            mat = Material("m_phong%d" % i, ks=tuple(rng.uniform(0.5, 0.8, 3)), exponent=float(rng.uniform(20, 80)))
        else:
            mat = Material("m_phong%d" % i, kd=tuple(rng.uniform(0.2, 0.5, 3)), ks=(0.3, 0.3, 0.3), exponent=30.0)
        spec.add("phong%d" % i, mat, p, t, normals=n)
    return spec


def write_phong_cornell(out_dir, name="phong_cornell", resolution=(128, 128), spp=16,
                        num_path_vertices=8, integrator="nextevent_path_tracer"):
    """Cornell walls and light as triangles (first entry) plus the smooth objects of
    `phong_objects_spec` as a "phong_tessellation": true entry."""
    walls = cornell_spec()
    walls.meshes = [m for m in walls.meshes if m.name not in ("short_box", "tall_box")]
    cam = dict(CORNELL_CAMERA, resolution=list(resolution))
    render = nee_render(name + ".pfm", spp, num_path_vertices)
    render["integrator"] = integrator
    return write_scene_entries(out_dir, name, [("walls", walls, None),
                                               ("objects", phong_objects_spec(), {"phong_tessellation": True})],
                               cam, [render])


def material_zoo_spec(seed=7):
    """Cornell box (fixture variant, turned boxes) whose boxes exercise every BSDF: Oren-Nayar,
    Phong-only, Lambert+Phong."""
    rng = np.random.default_rng(seed)
    spec = cornell_spec(seed, box_angle=FIXTURE_BOX_ANGLE)
    spec.materials["m_short_box"] = Material("m_short_box", kd=(0.6, 0.5, 0.4), sigma=0.4)
    spec.materials["m_tall_box"] = Material("m_tall_box", kd=(0.3, 0.35, 0.4), ks=(0.45, 0.4, 0.35),
                                            exponent=30.0)
    spec.materials["m_back"] = Material("m_back", ks=(0.7, 0.7, 0.7), exponent=200.0)
    spec.materials["m_floor"] = Material("m_floor", kd=tuple(rng.uniform(0.3, 0.6, 3)), sigma=0.25)
    return spec


def heightfield_spheres_spec(seed=1002, n_grid=512, n_spheres=2000, sphere_subdiv=2,
                             extent=8.0, n_lights=4, light_ke=(60.0, 55.0, 50.0)):
    """Workload C2: 512^2-vertex fBm floor + 2000 icospheres (320 faces) + 4 lights.

    Materials: 50% Oren-Nayar (sigma ~ U[0, 0.5]) and 50% Lambert+modified-Phong
    (exponent log-uniform in [10, 1000], kd + ks <= 0.9).
    """
    rng = np.random.default_rng(seed)
    spec = SceneSpec()
    pos, tris, h = fbm_heightfield(n_grid, extent, 0.3, 6, rng)
    spec.add("floor", Material("m_floor", kd=(0.45, 0.42, 0.38), sigma=0.3), pos, tris)

    def height_at(x, z):
        u = (x + extent) / (2 * extent) * (n_grid - 1)
        v = (z + extent) / (2 * extent) * (n_grid - 1)
        return h[int(np.clip(round(u), 0, n_grid - 1)), int(np.clip(round(v), 0, n_grid - 1))]

    for i in range(n_spheres):
        r = math.exp(rng.uniform(math.log(0.05), math.log(0.5)))
        x, z = rng.uniform(-extent * 0.95, extent * 0.95, 2)
        cy = height_at(x, z) + r * rng.uniform(0.6, 1.4)
        name = "m_s%04d" % i
        if rng.uniform() < 0.5:
            mat = Material(name, kd=tuple(rng.uniform(0.2, 0.8, 3)), sigma=float(rng.uniform(0.0, 0.5)))
        else:
            kd = rng.uniform(0.05, 0.6, 3)
            ks_scalar = rng.uniform(0.1, 0.9 - kd.max())
            ks = np.clip(ks_scalar * rng.uniform(0.8, 1.0, 3), 0.0, 0.9 - kd)
            n = math.exp(rng.uniform(math.log(10.0), math.log(1000.0)))
            mat = Material(name, kd=tuple(kd), ks=tuple(ks), exponent=n)
        p, t = icosphere((x, cy, z), r, sphere_subdiv)
        spec.add("sphere%04d" % i, mat, p, t)

    for i in range(n_lights):
        a = 2 * math.pi * (i + 0.5) / n_lights
        cx, cz = 0.55 * extent * math.cos(a), 0.55 * extent * math.sin(a)
        y = 4.0 + 0.5 * i
        s = 0.75
        p, t = quad((cx - s, y, cz - s), (cx + s, y, cz - s), (cx + s, y, cz + s), (cx - s, y, cz + s))
        spec.add("light%d" % i, Material("m_light%d" % i, ke=tuple(np.array(light_ke) * (0.8 + 0.1 * i))), p, t)
    return spec


HEIGHTFIELD_CAMERA = {"pos": [0.0, 3.2, 9.5], "lookat": [0.0, 0.0, 0.0], "up": [0.0, 1.0, 0.0],
                      "fovy": 45.0, "resolution": [1024, 512]}


def write_heightfield_spheres(out_dir, name="heightfield_spheres", resolution=(1024, 512), spp=64,
                              num_path_vertices=18, seed=1002, **kw):
    """Workload C2 at its full size: 1024x512, 64 spp, max depth 16 (18 vertices)."""
    spec = heightfield_spheres_spec(seed, **kw)
    cam = dict(HEIGHTFIELD_CAMERA, resolution=list(resolution))
    return write_scene(out_dir, name, spec, cam, [nee_render(name + ".pfm", spp, num_path_vertices)])


def write_heightfield_phong(out_dir, name="heightfield_phong", resolution=(1024, 512), spp=16,
                            num_path_vertices=18, seed=1002, n_spheres=2000):
    """The heightfield workload with its spheres as Phong tessellation patches: the fBm floor
    and the lights stay triangles (first mesh entry); the 2000 spheres are 80-face icospheres
    with their exact (radial) vertex normals in a "phong_tessellation": true entry."""
    spec = heightfield_spheres_spec(seed, sphere_subdiv=1, n_spheres=n_spheres)
    base, smooth = SceneSpec(), SceneSpec()
    for m in spec.meshes:
        mat = spec.materials[m.material]
        if m.name.startswith("sphere"):
            c = m.positions.astype(np.float64).mean(axis=0)
            n = m.positions.astype(np.float64) - c
            n /= np.linalg.norm(n, axis=1, keepdims=True)
            smooth.add(m.name, mat, m.positions, m.triangles, normals=n.astype(np.float32))
        else:
            base.add(m.name, mat, m.positions, m.triangles)
    cam = dict(HEIGHTFIELD_CAMERA, resolution=list(resolution))
    return write_scene_entries(out_dir, name, [("base", base, None), ("spheres", smooth, {"phong_tessellation": True})],
                               cam, [nee_render(name + ".pfm", spp, num_path_vertices)])


def batch_jobs(seed=1003, n_jobs=128, num_path_vertices=14):
    """Workload C3 job table: random cameras inside the Cornell box looking at a box centre."""
    rng = np.random.default_rng(seed)
    targets = [(0.35, 0.3, 0.3), (-0.35, 0.6, -0.35)]
    jobs = []
    for i in range(n_jobs):
        pos = rng.uniform([-0.9, 0.1, -0.9], [0.9, 1.9, 0.9])
        tgt = np.array(targets[int(rng.integers(0, 2))])
        if np.linalg.norm(tgt - pos) < 0.2:
            pos = pos + np.array([0.0, 0.0, 0.5])
        res = int(rng.choice([64, 128, 256, 512]))
        spp = int(round(math.exp(rng.uniform(math.log(4), math.log(256)))))
        jobs.append({"camera": {"pos": [float(x) for x in pos], "lookat": [float(x) for x in tgt],
                                "up": [0.0, 1.0, 0.0], "fovy": 60.0, "resolution": [res, res]},
                     "num_spp": spp, "num_path_vertices": num_path_vertices,
                     "output": "job%03d.pfm" % i})
    return jobs


def door_room_spec(seed=1004, n_boxes=300, wall_tess=70, box_tess=6):
    """Workload C4: closed room, emitter hidden behind a wall with a 0.2 m door gap."""
    rng = np.random.default_rng(seed)
    spec = SceneSpec()
    W, H, D = 6.0, 3.0, 6.0
    wall = Material("m_wall", kd=(0.6, 0.6, 0.6), sigma=0.2)
    faces = {
        "floor": ((-W / 2, 0, -D / 2), (0, 0, D), (W, 0, 0)),
        "ceiling": ((-W / 2, H, -D / 2), (W, 0, 0), (0, 0, D)),
        "wall_n": ((-W / 2, 0, -D / 2), (W, 0, 0), (0, H, 0)),
        "wall_s": ((-W / 2, 0, D / 2), (0, H, 0), (W, 0, 0)),
        "wall_w": ((-W / 2, 0, -D / 2), (0, H, 0), (0, 0, D)),
        "wall_e": ((W / 2, 0, -D / 2), (0, 0, D), (0, H, 0)),
    }
    for name, (o, du, dv) in faces.items():
        p, t = grid_quad(o, du, dv, wall_tess, wall_tess)
        spec.add(name, wall, p, t)
    # partition at z = -1.5 with a 0.2 m wide full-height door gap at x in [0.9, 1.1]
    zp = -1.5
    for k, (x0, x1) in enumerate([(-W / 2, 0.9), (1.1, W / 2)]):
        n_u = max(2, int(wall_tess * (x1 - x0) / W))
        p, t = grid_quad((x0, 0, zp), (x1 - x0, 0, 0), (0, H, 0), n_u, wall_tess // 2)
        spec.add("partition%d" % k, wall, p, t)
        p, t = grid_quad((x0, 0, zp - 0.02), (0, H, 0), (x1 - x0, 0, 0), wall_tess // 2, n_u)
        spec.add("partition%db" % k, wall, p, t)
    # emitter behind the partition, facing +z (toward the door), 1 x 1
    zl = -2.6
    p, t = quad((-0.5, 1.0, zl), (0.5, 1.0, zl), (0.5, 2.0, zl), (-0.5, 2.0, zl))
    spec.add("light", Material("m_light", ke=(40.0, 38.0, 34.0)), p, t)
    for i in range(n_boxes):
        s = rng.uniform(0.08, 0.4, 3)
        c = (rng.uniform(-W / 2 + 0.3, W / 2 - 0.3), s[1] / 2 + rng.uniform(0.0, 1.5) * (rng.uniform() < 0.3),
             rng.uniform(zp + 0.4, D / 2 - 0.3))
        name = "m_b%03d" % i
        if rng.uniform() < 0.5:
            mat = Material(name, kd=tuple(rng.uniform(0.2, 0.8, 3)), sigma=float(rng.uniform(0.0, 0.5)))
        else:
            kd = rng.uniform(0.05, 0.5, 3)
            ks = np.minimum(rng.uniform(0.1, 0.4, 3), 0.9 - kd)
            mat = Material(name, kd=tuple(kd), ks=tuple(ks), exponent=math.exp(rng.uniform(math.log(10), math.log(500))))
        p, t = box(c, s, angle_y=rng.uniform(0, math.pi), tess=box_tess)
        spec.add("box%03d" % i, mat, p, t)
    return spec


DOOR_ROOM_CAMERA = {"pos": [0.0, 1.5, 2.9], "lookat": [0.5, 1.2, -1.5], "up": [0.0, 1.0, 0.0],
                    "fovy": 60.0, "resolution": [1024, 1024]}


def envmap_image(width, height, seed=1005, n_suns=3):
    """Equirectangular HDR sky: vertical gradient plus Gaussian suns (row 0 = top)."""
    rng = np.random.default_rng(seed)
    v = (np.arange(height) + 0.5) / height
    u = (np.arange(width) + 0.5) / width
    theta = u * 2 * math.pi
    phi = v * math.pi
    # direction of each texel, the inverse of the reference's PanoramaFromWorld
    d = np.stack([np.cos(theta)[None, :] * np.sin(phi)[:, None],
                  np.broadcast_to(np.cos(phi)[:, None], (height, width)),
                  np.sin(theta)[None, :] * np.sin(phi)[:, None]], -1)
    up = np.clip(d[..., 1], -1, 1)
    sky = np.stack([0.25 + 0.35 * (up > 0) * up, 0.35 + 0.35 * (up > 0) * up, 0.6 + 0.5 * (up > 0) * up], -1)
    sky = np.where((up < 0)[..., None], np.array([0.08, 0.07, 0.06]), sky)
    img = sky.copy()
    for _ in range(n_suns):
        el = rng.uniform(0.15, 1.2)
        az = rng.uniform(0, 2 * math.pi)
        s = np.array([math.cos(az) * math.cos(el), math.sin(el), math.sin(az) * math.cos(el)])
        width_rad = rng.uniform(0.02, 0.08)
        cosang = np.clip((d * s).sum(-1), -1, 1)
        ang = np.arccos(cosang)
        power = rng.uniform(200.0, 800.0) * np.array([1.0, rng.uniform(0.8, 1.0), rng.uniform(0.6, 0.9)])
        img += np.exp(-0.5 * (ang / width_rad) ** 2)[..., None] * power
    return img.astype(np.float32)


def write_pfm(path, img):
    """PFM writer (little endian, rows bottom-to-top; img row 0 = top)."""
    img = np.asarray(img, np.float32)
    h, w = img.shape[:2]
    with open(path, "wb") as f:
        f.write(b"PF\n%d %d\n-1\n" % (w, h))
        f.write(np.ascontiguousarray(img[::-1]).astype("<f4").tobytes())


def env_scene_spec(seed=1006):
    """Open scene for the environment light: ground, boxes, spheres and one area light."""
    rng = np.random.default_rng(seed)
    spec = SceneSpec()
    p, t = grid_quad((-4, 0, -4), (0, 0, 8), (8, 0, 0), 4, 4)
    spec.add("ground", Material("m_ground", kd=(0.5, 0.5, 0.45), sigma=0.35), p, t)
    for i in range(6):
        c = (rng.uniform(-2, 2), 0.0, rng.uniform(-2, 2))
        s = rng.uniform(0.3, 0.9, 3)
        mat = Material("m_box%d" % i, kd=tuple(rng.uniform(0.1, 0.5, 3)), ks=tuple(rng.uniform(0.1, 0.4, 3)),
                       exponent=float(rng.uniform(20, 400))) if i % 2 else \
            Material("m_box%d" % i, kd=tuple(rng.uniform(0.2, 0.8, 3)))
        p, t = box((c[0], s[1] / 2, c[2]), s, angle_y=rng.uniform(0, 3))
        spec.add("box%d" % i, mat, p, t)
    for i in range(4):
        r = rng.uniform(0.2, 0.5)
        p, t = icosphere((rng.uniform(-2.5, 2.5), r, rng.uniform(-2.5, 2.5)), r, 2)
        spec.add("sphere%d" % i, Material("m_sphere%d" % i, ks=(0.8, 0.8, 0.8), exponent=float(rng.uniform(50, 2000))), p, t)
    p, t = quad((-0.4, 2.5, -0.4), (0.4, 2.5, -0.4), (0.4, 2.5, 0.4), (-0.4, 2.5, 0.4))
    spec.add("light", Material("m_light", ke=(20.0, 18.0, 15.0)), p, t)
    return spec


ENV_CAMERA = {"pos": [0.0, 2.0, 6.0], "lookat": [0.0, 0.5, 0.0], "up": [0.0, 1.0, 0.0],
              "fovy": 50.0, "resolution": [128, 96]}


def write_env_scene(out_dir, name="env_scene", resolution=(128, 96), spp=8, num_path_vertices=8,
                    env_size=(128, 64), seed=1006):
    os.makedirs(out_dir, exist_ok=True)
    env_name = name + "_sky.pfm"
    write_pfm(os.path.join(out_dir, env_name), envmap_image(env_size[0], env_size[1], seed))
    cam = dict(ENV_CAMERA, resolution=list(resolution))
    return write_scene(out_dir, name, env_scene_spec(seed), cam,
                       [nee_render(name + ".pfm", spp, num_path_vertices)], envmap=env_name)


def write_spec(out_dir, name, spec, camera, resolution, spp, num_path_vertices):
    cam = dict(camera, resolution=list(resolution))
    return write_scene(out_dir, name, spec, cam, [nee_render(name + ".pfm", spp, num_path_vertices)])


def full_combination_spec(seed=1005, n_grid=2048, n_spheres=20000, sphere_subdiv=1, extent=24.0, n_lights=16):
    """Workload C5: 2048^2-vertex fBm floor (8,380,418 triangles) + 20000 icospheres of 80 faces
    (1,600,000) + 16 area lights (32): 9,980,450 triangles. Materials: 50 % Oren-Nayar, 50 %
    Lambert + modified Phong with exponents log-uniform in [10, 2000]. Lit by the equirectangular
    sky of `full_combination_envmap` as well."""
    rng = np.random.default_rng(seed)
    spec = SceneSpec()
    pos, tris, h = fbm_heightfield(n_grid, extent, 0.6, 6, rng)
    spec.add("floor", Material("m_floor", kd=(0.42, 0.40, 0.36), sigma=0.25), pos, tris)

    def height_at(x, z):
        u = (x + extent) / (2 * extent) * (n_grid - 1)
        v = (z + extent) / (2 * extent) * (n_grid - 1)
        return h[int(np.clip(round(u), 0, n_grid - 1)), int(np.clip(round(v), 0, n_grid - 1))]

    n_mat = 256      # spheres share a pool of materials (one mesh per object, as the reference loads it)
    mats = []
    for i in range(n_mat):
        name = "m_s%03d" % i
        if i % 2 == 0:
            mats.append(Material(name, kd=tuple(rng.uniform(0.2, 0.8, 3)), sigma=float(rng.uniform(0.0, 0.5))))
        else:
            kd = rng.uniform(0.05, 0.5, 3)
            ks_scalar = rng.uniform(0.1, 0.9 - kd.max())
            ks = np.clip(ks_scalar * rng.uniform(0.8, 1.0, 3), 0.0, 0.9 - kd)
            n = math.exp(rng.uniform(math.log(10.0), math.log(2000.0)))
            mats.append(Material(name, kd=tuple(kd), ks=tuple(ks), exponent=n))
    for i in range(n_spheres):
        r = math.exp(rng.uniform(math.log(0.05), math.log(0.5)))
        x, z = rng.uniform(-extent * 0.95, extent * 0.95, 2)
        cy = height_at(x, z) + r * rng.uniform(0.6, 1.4)
        p, t = icosphere((x, cy, z), r, sphere_subdiv)
        spec.add("sphere%05d" % i, mats[int(rng.integers(n_mat))], p, t)

    for i in range(n_lights):
        a = 2 * math.pi * (i + 0.5) / n_lights
        rad = (0.3 + 0.4 * (i % 4) / 3.0) * extent
        cx, cz = rad * math.cos(a), rad * math.sin(a)
        y = 5.0 + 0.5 * (i % 3)
        s = 0.6
        p, t = quad((cx - s, y, cz - s), (cx + s, y, cz - s), (cx + s, y, cz + s), (cx - s, y, cz + s))
        spec.add("light%02d" % i, Material("m_light%02d" % i, ke=(40.0, 36.0, 30.0)), p, t)
    return spec


FULL_COMBINATION_CAMERA = {"pos": [0.0, 4.5, 20.0], "lookat": [0.0, 0.5, 0.0], "up": [0.0, 1.0, 0.0],
                           "fovy": 50.0, "resolution": [3840, 2160]}


def write_full_combination(out_dir, name="full_combination", resolution=(3840, 2160), spp=1024,
                           num_path_vertices=26, env_size=(2048, 1024), seed=1005, **kw):
    """Workload C5 at its full size: 3840x2160, 1024 spp, max depth 24 (26 vertices), a
    2048x1024 FP32 sky (3 Gaussian suns + gradient) plus 16 area lights, ~10M triangles."""
    os.makedirs(out_dir, exist_ok=True)
    env_name = name + "_sky.pfm"
    write_pfm(os.path.join(out_dir, env_name), envmap_image(env_size[0], env_size[1], seed))
    cam = dict(FULL_COMBINATION_CAMERA, resolution=list(resolution))
    return write_scene(out_dir, name, full_combination_spec(seed, **kw), cam,
                       [nee_render(name + ".pfm", spp, num_path_vertices)], envmap=env_name)


# the full-size plain NEE+MIS workloads whose FP64 reference crops live in tests/golden:
# c1, the whole 256^2 frame of the procedural Cornell box (36 triangles, 10 vertices); c2 and c2h,
# two crops (spheres in the middle distance, the horizon) of the 1024x512 frame of the
# 1,162,250-triangle heightfield-and-spheres scene (18 vertices)
PLAIN_WORKLOADS = {
    "c1": {"resolution": (256, 256), "num_path_vertices": 10, "crop": (0, 0, 256, 256)},
    "c2": {"resolution": (1024, 512), "num_path_vertices": 18, "crop": (448, 288, 576, 352)},
    "c2h": {"resolution": (1024, 512), "num_path_vertices": 18, "crop": (768, 160, 896, 224)},
}


def write_plain_workload(name, out_dir, spp=64):
    """Writes the Cornell box (c1) or the heightfield-and-spheres scene (c2, c2h) at full size."""
    w = PLAIN_WORKLOADS[name]
    if name == "c1":
        return write_cornell(out_dir, resolution=w["resolution"], spp=spp, num_path_vertices=w["num_path_vertices"])
    return write_heightfield_spheres(out_dir, resolution=w["resolution"], spp=spp,
                                     num_path_vertices=w["num_path_vertices"])


# the full-size guided-vs-plain workloads whose FP64 reference crops live in tests/golden
GUIDED_WORKLOADS = {
    "door": {"resolution": (1024, 1024), "num_path_vertices": 10, "crop": (448, 448, 576, 576)},
    "c5": {"resolution": (3840, 2160), "num_path_vertices": 26, "crop": (1856, 1056, 1984, 1120)},
}


def write_guided_workload(name, out_dir, spp=64):
    """Writes the door-gap room (config 4) or the full combination (config 5) at full size."""
    w = GUIDED_WORKLOADS[name]
    if name == "door":
        cam = dict(DOOR_ROOM_CAMERA, resolution=list(w["resolution"]))
        return write_spec(out_dir, "door", door_room_spec(seed=1004), cam, w["resolution"], spp,
                          w["num_path_vertices"])
    return write_full_combination(out_dir, resolution=w["resolution"], spp=spp,
                                  num_path_vertices=w["num_path_vertices"], seed=1005)
