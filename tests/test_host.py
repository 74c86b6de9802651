"""Host-side logic of the B200 library, exercised without a GPU.

Covers: the C ABI library loads and exports every function include/wurst_b200.h
declares; scene loading (simple2 JSON, OBJ/MTL, PFM) and the BVH build agree
with the oracle's reading of the same files; error statuses; the CLI flags.
"""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import FIXTURES, GOLDEN, ROOT, golden_scene


def declared_functions():
    text = open(os.path.join(ROOT, "include", "wurst_b200.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|void|const char \*)\s*(wr_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol(wr_lib):
    L = wr_lib.load_library()
    names = declared_functions()
    assert len(names) >= 15
    for n in names:
        assert hasattr(L, n), n
    assert set(names) == set(wr_lib.EXPORTS)
    assert L.wr_abi_version() == 1


def test_symbols_visible_in_dynamic_table(wr_lib):
    out = subprocess.run(["nm", "-D", "--defined-only", wr_lib.LIB_PATH], capture_output=True, text=True).stdout
    for n in declared_functions():
        assert re.search(r"\bT %s\b" % n, out), n


@pytest.mark.parametrize("name", FIXTURES)
def test_inspect_matches_oracle_scene(wr_lib, oracle_lib, name):
    path, _ = golden_scene(name)
    info = wr_lib.inspect_scene(path)
    sc = oracle_lib.OracleScene(path)
    assert info["num_triangles"] == sc.num_triangles
    assert info["num_meshes"] == sc.num_meshes
    assert info["num_lights"] == sc.num_lights
    assert (info["width"], info["height"]) == (sc.width, sc.height)
    assert info["num_path_vertices"] == sc.num_path_vertices
    assert 0 < info["bvh_depth"] <= 64
    assert info["bvh_nodes"] >= 1
    assert info["has_envmap"] == (1 if name.startswith("env") else 0)


def test_pfm_roundtrip_layout(wr_lib, tmp_path):
    img = np.random.default_rng(1).uniform(size=(5, 7, 3))
    p = str(tmp_path / "x.pfm")
    wr_lib.write_pfm(p, img)
    raw = open(p, "rb").read()
    assert raw.startswith(b"PF\n7 5\n-1\n")
    back = wr_lib.read_pfm(p)
    assert np.array_equal(back, img.astype(np.float32))
    # rows are stored bottom-to-top: the first stored row is the last image row
    first = np.frombuffer(raw[len(b"PF\n7 5\n-1\n"):][:7 * 12], "<f4").reshape(7, 3)
    assert np.array_equal(first, img[-1].astype(np.float32))


def test_error_statuses(wr_lib, tmp_path):
    with pytest.raises(wr_lib.WurstError) as e:
        wr_lib.inspect_scene(str(tmp_path / "missing.json"))
    assert e.value.status == 2
    bad = tmp_path / "bad.json"
    bad.write_text('{"camera": [1, 2,')
    with pytest.raises(wr_lib.WurstError) as e:
        wr_lib.inspect_scene(str(bad))
    assert e.value.status == 3
    # emitters with Ns != 0 are SimpleMetal lights in the reference (assimpio.h:84-91): unsupported here
    (tmp_path / "m.obj").write_text("mtllib m.mtl\no a\nusemtl e\nv 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 3\n")
    (tmp_path / "m.mtl").write_text("newmtl e\nKe 1 1 1\nNs 10\n")
    (tmp_path / "s.json").write_text('{"meshes": [{"path": "m.obj"}]}')
    with pytest.raises(wr_lib.WurstError) as e:
        wr_lib.inspect_scene(str(tmp_path / "s.json"))
    assert e.value.status == 4


def test_obj_semantics(wr_lib, oracle_lib, tmp_path):
    """Assimp-style reading: one mesh per object x material, a new object keeps the
    current material (ObjFileParser::createObject), polygon fans, emitters attached
    after the surfaces of their file."""
    (tmp_path / "m.mtl").write_text("newmtl a\nKd 0.5 0.5 0.5\nnewmtl l\nKe 5 5 5\n")
    (tmp_path / "m.obj").write_text(
        "mtllib m.mtl\n"
        "v 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nv 0 0 1\n"
        "o light\nusemtl l\nf 1 2 3\n"
        "o quad\nusemtl a\nf 1 2 3 4\n"
        "usemtl l\nf -1 -2 -3\n"
        "o nomat\nf 1 3 5\n")
    (tmp_path / "s.json").write_text(
        '{"camera": {"pos": [0,0,5], "lookat": [0,0,0], "up": [0,1,0], "resolution": [8, 6]},'
        ' "meshes": [{"path": "m.obj"}], "render": [{"integrator": "nextevent_path_tracer"}]}')
    info = wr_lib.inspect_scene(str(tmp_path / "s.json"))
    assert info["num_triangles"] == 1 + 2 + 1 + 1
    assert info["num_meshes"] == 4
    assert info["num_lights"] == 3
    assert (info["num_spp"], info["num_path_vertices"]) == (16, 10)
    sc = oracle_lib.OracleScene(str(tmp_path / "s.json"))
    assert (sc.num_triangles, sc.num_meshes, sc.num_lights) == (5, 4, 3)


def test_phong_mesh_entries(wr_lib, oracle_lib, tmp_path):
    """"phong_tessellation": true turns the entry's surfaces into patches with one vertex per
    (position, normal) pair (v//vn, v/vt/vn and negative indices); its emitters stay triangles;
    a patch corner without a normal is rejected."""
    (tmp_path / "m.mtl").write_text("newmtl a\nKd 0.5 0.5 0.5\nnewmtl l\nKe 5 5 5\n")
    (tmp_path / "m.obj").write_text(
        "mtllib m.mtl\n"
        "v 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\n"
        "vn 0 0 1\nvn 0.1 0 1\nvn 0 0.1 1\nvt 0 0\n"
        "o smooth\nusemtl a\nf 1//1 2//2 3//3\nf 1/1/1 3/1/3 4/1/-3\n"
        "o light\nusemtl l\nf 1 2 4\n")
    scene = ('{"camera": {"pos": [0,0,5], "lookat": [0,0,0], "up": [0,1,0], "resolution": [8, 6]},'
             ' "meshes": [{"path": "m.obj", "phong_tessellation": true}],'
             ' "render": [{"integrator": "nextevent_path_tracer"}]}')
    (tmp_path / "s.json").write_text(scene)
    info = wr_lib.inspect_scene(str(tmp_path / "s.json"))
    assert (info["num_triangles"], info["num_meshes"], info["num_lights"]) == (3, 2, 1)
    sc = oracle_lib.OracleScene(str(tmp_path / "s.json"))
    assert (sc.num_triangles, sc.num_meshes, sc.num_lights) == (3, 2, 1)
    (tmp_path / "n.obj").write_text("v 0 0 0\nv 1 0 0\nv 1 1 0\nvn 0 0 1\nf 1//1 2 3//1\n")
    (tmp_path / "n.json").write_text(scene.replace("m.obj", "n.obj"))
    with pytest.raises(wr_lib.WurstError, match="vertex normal"):
        wr_lib.inspect_scene(str(tmp_path / "n.json"))


def test_cli_reports_errors(wr_lib, tmp_path):
    r = subprocess.run([wr_lib.CLI_PATH, "--simple2parse", str(tmp_path / "nope.json")], capture_output=True,
                       text=True, cwd=str(tmp_path))
    assert r.returncode == 1
    assert "file not found" in r.stderr


def test_cli_default_txt_created(wr_lib, tmp_path):
    r = subprocess.run([wr_lib.CLI_PATH], capture_output=True, text=True, cwd=str(tmp_path))
    assert r.returncode == 0
    assert (tmp_path / "default.txt").exists()


def test_heightfield_workload_size(wr_lib, tmp_path):
    """The 1M-triangle workload: 511^2*2 floor + 2000 x 320-face spheres + 4 quad lights."""
    from wurstrenderer_b200 import scenes
    path = scenes.write_heightfield_spheres(str(tmp_path), spp=64)
    info = wr_lib.inspect_scene(path)
    assert info["num_triangles"] == 511 * 511 * 2 + 2000 * 320 + 4 * 2
    assert info["num_lights"] == 4
    assert (info["width"], info["height"], info["num_spp"], info["num_path_vertices"]) == (1024, 512, 64, 18)
    assert info["bvh_depth"] <= 64


def test_inspect_build_options(wr_lib):
    """Leaf size, SAH traversal cost and BVH width through the host-only inspect: one triangle per
    leaf gives n - 1 inner nodes; a dearer traversal step gives fewer nodes; the 8-wide tree is
    shallower; bad options fail with WR_ERR_INVALID_ARGUMENT, the device LBVH with UNSUPPORTED."""
    path, _ = golden_scene("hf")
    base = wr_lib.inspect_scene(path)
    n = base["num_triangles"]
    assert wr_lib.inspect_scene(path, max_leaf=1)["bvh_nodes"] == n - 1
    leaf4 = wr_lib.inspect_scene(path, max_leaf=4)
    assert leaf4["bvh_nodes"] <= base["bvh_nodes"] < n - 1          # default: 2 per leaf
    dear = wr_lib.inspect_scene(path, max_leaf=8, sah_trav_cost=4.0)
    assert dear["bvh_nodes"] < leaf4["bvh_nodes"]
    wide = wr_lib.inspect_scene(path, bvh_width=8)
    assert wide["bvh_depth"] < base["bvh_depth"] and wide["bvh_nodes"] < base["bvh_nodes"]
    for bad in (dict(max_leaf=17), dict(max_leaf=-1), dict(bvh_width=4), dict(sah_trav_cost=-1.0),
                dict(sah_trav_cost=200.0)):
        with pytest.raises(wr_lib.WurstError) as e:
            wr_lib.inspect_scene(path, **bad)
        assert e.value.status == 1, bad
    L = wr_lib.load_library()
    opts = wr_lib.SceneOptions()
    opts.bvh_builder = wr_lib.BVH_DEVICE_LBVH
    info = wr_lib.SceneInfo()
    assert L.wr_scene_inspect_ex(path.encode(), ctypes.byref(opts), ctypes.byref(info)) == 4   # WR_ERR_UNSUPPORTED


def test_obj_number_formats_parse_alike(wr_lib, tmp_path):
    """The same float32 vertices written plainly and in the other forms strtof reads (hex floats,
    '+' signs, exponents, tabs, CRLF, relative and '+' face indices) give the same scene: same
    triangle count and a BVH with the same SAH cost, nodes and depth."""
    import json
    rng = np.random.default_rng(11)
    pts = rng.normal(0.0, 3.0, (300, 3)).astype(np.float32)
    tris = rng.integers(0, len(pts), (400, 3))

    def fancy(x, k):
        x = float(x)
        forms = [x.hex(), ("+%.9g" % x) if x >= 0 else "%.9g" % x, "%.8e" % x, repr(x)]
        return forms[k % len(forms)]

    plain = ["mtllib m.mtl", "o a", "usemtl w"] + ["v %.9g %.9g %.9g" % tuple(p) for p in pts]
    plain += ["f %d %d %d" % tuple(t + 1) for t in tris]
    odd = ["mtllib m.mtl", "o a", "usemtl w"]
    odd += ["v\t" + "\t ".join(fancy(c, 3 * i + k) for k, c in enumerate(p)) for i, p in enumerate(pts)]
    odd += ["f %d +%d %d" % (t[0] - len(pts), t[1] + 1, t[2] + 1) for t in tris]   # relative and '+' indices
    scene = json.load(open(golden_scene("cornell")[0]))
    infos = []
    for name, lines, eol in (("plain", plain, "\n"), ("odd", odd, "\r\n")):
        d = tmp_path / name
        d.mkdir()
        (d / "a.obj").write_bytes(eol.join(lines).encode() + eol.encode())
        (d / "m.mtl").write_text("newmtl w\nKd 0.5 0.5 0.5\n")
        (d / "s.json").write_text(json.dumps(dict(scene, meshes=[{"path": "a.obj"}])))
        infos.append(wr_lib.inspect_scene(str(d / "s.json")))
    a, b = infos
    assert a["num_triangles"] == b["num_triangles"] == len(tris)
    assert (a["bvh_sah_cost"], a["bvh_nodes"], a["bvh_depth"]) == (b["bvh_sah_cost"], b["bvh_nodes"], b["bvh_depth"])
