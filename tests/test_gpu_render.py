"""Image parity of the B200 NEE+MIS renderer against the reference.

Reference: two independent renders of the reference's own PathNeeRenderer at
4096 spp (tests/golden/*_ref_hi_{a,b}.npy). The GPU renders the same scene at
the same total spp as K independent seeds. Tolerances (FP32 GPU vs FP64
reference, different random streams):
  * relMSE(gpu, ref_a) <= 2 x relMSE(ref_b, ref_a)  -- within the reference's own
    noise floor (expected ratio ~1 for an unbiased estimator of equal variance);
  * every 8x8 block: |z| < 4 with z = (mean_gpu - mean_ref) / sqrt(2 var_gpu),
    var_gpu the variance of the GPU block mean estimated from the K seeds.
relMSE = mean over pixels and channels of (x - ref)^2 / (ref^2 + 1e-2).
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import FIXTURES, GOLDEN, golden_scene

pytestmark = pytest.mark.gpu

K = 8


def relmse(x, ref, eps=1e-2):
    return float(np.mean((x - ref) ** 2 / (ref ** 2 + eps)))


def block_z(runs, ref, block=8, ref_pair=None, ref_var=None):
    """z scores of 8x8 block means; runs: K x H x W x 3 independent renders.

    Without ref_pair the reference's variance is taken equal to the GPU's (same spp, same
    estimator): z = (gpu - ref) / sqrt(2 var_gpu). With ref_pair = (ref_a, ref_b), two independent
    halves whose mean is `ref`, the reference's own variance is estimated from them per pixel,
    (a - b)^2 / 4, and z = (gpu - ref) / sqrt(var_gpu + var_ref) -- needed when the GPU estimator
    is much less noisy than the reference (the learned proposal).

    ref_var (H x W x 3): a second per-pixel estimate of the variance of `ref`, from more samples of
    the reference's own estimator; each block then takes the larger of the two. Two halves give
    one degree of freedom per pixel, and for path-traced light through a narrow gap their sample
    variance is often well below the true one (rare high-contribution paths are missing from
    both halves), which would make the test reject a correct renderer whose own noise is low."""
    k, h, w, _ = runs.shape
    hb, wb = h // block, w // block
    r = runs[:, :hb * block, :wb * block].reshape(k, hb, block, wb, block, 3)
    ref_b = ref[:hb * block, :wb * block].reshape(hb, block, wb, block, 3).mean(axis=(1, 3))
    pix_var = runs[:, :hb * block, :wb * block].var(axis=0, ddof=1) / k      # variance of the K-run mean, per pixel
    var_b = pix_var.reshape(hb, block, wb, block, 3).sum(axis=(1, 3)) / (block * block) ** 2
    mean_b = r.mean(axis=0).mean(axis=(1, 3))
    if ref_pair is None:
        return (mean_b - ref_b) / np.sqrt(2.0 * var_b + 1e-30)
    a, b = ref_pair
    pair_var = ((a - b) ** 2 / 4.0)[:hb * block, :wb * block]
    var_r = pair_var.reshape(hb, block, wb, block, 3).sum(axis=(1, 3)) / (block * block) ** 2
    if ref_var is not None:
        other = ref_var[:hb * block, :wb * block].reshape(hb, block, wb, block, 3).sum(axis=(1, 3)) / (block * block) ** 2
        var_r = np.maximum(var_r, other)
    return (mean_b - ref_b) / np.sqrt(var_b + var_r + 1e-30)


@pytest.mark.parametrize("name", FIXTURES)
def test_image_matches_reference(wr_lib, name):
    path, meta = golden_scene(name)
    ref_a = np.load("%s/%s_ref_hi_a.npy" % (GOLDEN, name)).astype(np.float64)
    ref_b = np.load("%s/%s_ref_hi_b.npy" % (GOLDEN, name)).astype(np.float64)
    spp = meta["hi_spp"] // K
    with wr_lib.Scene.from_file(path) as sc:
        runs = np.stack([sc.render(spp=spp, seed=1000 + i) for i in range(K)])
    assert np.isfinite(runs).all()
    img = runs.mean(axis=0)
    floor = relmse(ref_b, ref_a)
    err = relmse(img, ref_a)
    assert err <= 2.0 * floor + 1e-6, "relMSE %.3g vs reference noise floor %.3g" % (err, floor)
    z = block_z(runs, ref_a)
    assert np.abs(z).max() < 4.0, "max |z| %.2f" % np.abs(z).max()
    # image mean within 1% (fluxes agree)
    assert abs(img.mean() / ref_a.mean() - 1.0) < 0.01


@pytest.mark.parametrize("name", ["hf", "phong"])
def test_wide_bvh_image_matches_reference(wr_lib, name):
    """Renders through the compressed 8-wide BVH pass the same image bar."""
    path, meta = golden_scene(name)
    ref_a = np.load("%s/%s_ref_hi_a.npy" % (GOLDEN, name)).astype(np.float64)
    ref_b = np.load("%s/%s_ref_hi_b.npy" % (GOLDEN, name)).astype(np.float64)
    spp = meta["hi_spp"] // K
    with wr_lib.Scene.from_file(path, bvh_width=8) as sc:
        runs = np.stack([sc.render(spp=spp, seed=2000 + i) for i in range(K)])
    img = runs.mean(axis=0)
    floor = relmse(ref_b, ref_a)
    err = relmse(img, ref_a)
    assert err <= 2.0 * floor + 1e-6, "relMSE %.3g vs reference noise floor %.3g" % (err, floor)
    z = block_z(runs, ref_a)
    assert np.abs(z).max() < 4.0, "max |z| %.2f" % np.abs(z).max()


def test_exr_and_hdr_envmaps_render_like_pfm(wr_lib, tmp_path):
    """The env fixture with its sky stored losslessly as OpenEXR (FLOAT, ZIP) renders as with the
    PFM; stored as Radiance HDR it renders as the PFM of the HDR's decoded values."""
    import json
    import shutil
    import sys
    sys.path.insert(0, GOLDEN)
    from image_writers import write_exr, write_hdr
    path, _ = golden_scene("env")
    d = os.path.dirname(path)
    for f in os.listdir(d):
        shutil.copy(os.path.join(d, f), tmp_path / f)
    scene = json.load(open(path))
    env = wr_lib.read_image(os.path.join(d, scene["envmap"]))
    write_exr(str(tmp_path / "sky.exr"), {c: env[..., k] for k, c in enumerate("RGB")}, "zip", "float")
    write_hdr(str(tmp_path / "sky.hdr"), env, rle=True)
    wr_lib.write_pfm(str(tmp_path / "sky_hdr.pfm"), wr_lib.read_image(str(tmp_path / "sky.hdr")))
    images = {}
    for name in ("sky.exr", "sky.hdr", "sky_hdr.pfm", scene["envmap"]):
        scene_v = dict(scene, envmap=name)
        p = tmp_path / ("scene_" + name.replace(".", "_") + ".json")
        p.write_text(json.dumps(scene_v))
        with wr_lib.Scene.from_file(str(p)) as sc:
            images[name] = sc.render(spp=16, seed=7)
    # same random streams and the same environment; only the FP64 atomic summation order may differ
    assert np.allclose(images["sky.exr"], images[scene["envmap"]], rtol=1e-9, atol=1e-12)
    assert np.allclose(images["sky.hdr"], images["sky_hdr.pfm"], rtol=1e-9, atol=1e-12)
    assert np.isfinite(images["sky.hdr"]).all()


def test_graph_and_plain_launches_agree(wr_lib):
    path, _ = golden_scene("zoo")
    with wr_lib.Scene.from_file(path) as sc:
        a = sc.render(spp=64, seed=3, use_graph=True)
        b = sc.render(spp=64, seed=3, use_graph=False)
    # same random streams; only the FP64 atomic summation order may differ
    assert np.allclose(a, b, rtol=1e-9, atol=1e-12)


def test_small_wavefront_regeneration(wr_lib):
    """A wavefront far smaller than the sample count forces path regeneration every iteration."""
    path, _ = golden_scene("cornell")
    with wr_lib.Scene.from_file(path) as sc:
        a = sc.render(spp=16, seed=9, queue_capacity=1024)
        st = sc.stats
        b = sc.render(spp=16, seed=9)
    assert st["queue_capacity"] == 1024 and st["iterations"] > 100
    assert np.allclose(a, b, rtol=1e-9, atol=1e-12)


@pytest.mark.parametrize("nverts", [1, 2, 3])
def test_short_paths_match_oracle(wr_lib, oracle_lib, nverts):
    """num_path_vertices 1: nothing is traced; 2: direct emission + light splats; 3: one bounce."""
    path, _ = golden_scene("cornell")
    with wr_lib.Scene.from_file(path) as sc:
        img = np.mean([sc.render(spp=256, num_path_vertices=nverts, seed=s) for s in range(4)], axis=0)
    ref, _, _ = oracle_lib.OracleScene(path).render(spp=256, num_path_vertices=nverts, threads=0)
    if nverts == 1:
        assert not img.any()
        return
    assert abs(img.mean() / ref.mean() - 1.0) < 0.03


def test_resolutions_and_spp_edges(wr_lib):
    path, _ = golden_scene("cornell")
    with wr_lib.Scene.from_file(path) as sc:
        for res in ([1, 1], [7, 3], [33, 65]):
            sc.set_camera('{"pos": [0,1,3.6], "lookat": [0,1,0], "up": [0,1,0], "fovy": 40, "resolution": %s}' % res)
            img = sc.render(spp=1)
            assert img.shape == (res[1], res[0], 3) and np.isfinite(img).all()


def test_cli_simple2parse_writes_pfm(wr_lib, tmp_path):
    from wurstrenderer_b200 import scenes
    p = scenes.write_cornell(str(tmp_path), resolution=(32, 32), spp=64)
    r = subprocess.run([wr_lib.CLI_PATH, "--simple2parse", p], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    img = wr_lib.read_pfm(os.path.join(str(tmp_path), "cornell.pfm"))
    assert img.shape == (32, 32, 3) and np.isfinite(img).all() and img.mean() > 0


def test_light_splatting_under_sky_matches_reference(wr_lib):
    """light_splatting under the sky (env_ls): light tracing there is dominated by rare bright
    splats, so its reference is rendered at 2 x 65536 spp. GPU: 8 seeds x 8192 spp (65536 in
    total) within 2 x the reference's own noise floor, every 8x8 block |z| < 4 with both
    estimators' variances, image flux within 2 %."""
    path, meta = golden_scene("env_ls")
    assert meta["hi_spp"] >= 65536
    ref_a = np.load("%s/env_ls_ref_hi_a.npy" % GOLDEN).astype(np.float64)
    ref_b = np.load("%s/env_ls_ref_hi_b.npy" % GOLDEN).astype(np.float64)
    ref = 0.5 * (ref_a + ref_b)
    with wr_lib.Scene.from_file(path) as sc:
        runs = np.stack([sc.render(spp=meta["hi_spp"] // 8, seed=500 + i) for i in range(8)])
    assert np.isfinite(runs).all()
    img = runs.mean(axis=0)
    floor = relmse(ref_a, ref_b)
    err = relmse(img, ref)
    assert err <= 2.0 * floor, "relMSE %.3g vs reference noise floor %.3g" % (err, floor)
    z = block_z(runs, ref, ref_pair=(ref_a, ref_b))
    assert np.abs(z).max() < 4.0, "max |z| %.2f" % np.abs(z).max()
    assert abs(img.mean() / ref.mean() - 1.0) < 0.02, (img.mean(), ref.mean())


def test_profiled_schedules_agree(wr_lib):
    """The separate-kernel schedule (profile 1 / 2) and the fused one (unprofiled renders and
    profile 3: each iteration's extend rays traced with the previous iteration's shadow rays) add
    the same contributions; only the FP64 atomic order may differ."""
    path, _ = golden_scene("zoo")
    with wr_lib.Scene.from_file(path) as sc:
        a = sc.render(spp=32, seed=5)
        fused = sc.stats
        b = sc.render(spp=32, seed=5, profile=2)
        sep = sc.stats
        c = sc.render(spp=32, seed=5, profile=3)
        p3 = sc.stats
    assert np.allclose(a, b, rtol=1e-9, atol=1e-12)
    assert np.allclose(a, c, rtol=1e-9, atol=1e-12)
    k = wr_lib.KERNELS
    n2, n3 = dict(zip(k, sep["kernel_count"])), dict(zip(k, p3["kernel_count"]))
    i2, i3 = dict(zip(k, sep["kernel_items"])), dict(zip(k, p3["kernel_items"]))
    # "iterations" counts the bookkeeping launches, the first wavefront's included
    assert n3["extend"] == p3["iterations"] - 1 and n3["shadow"] == 1      # pair launches + the last shadow rays
    assert n2["extend"] == sep["iterations"] - 1 and n2["shadow"] == sep["iterations"]
    assert i3["extend"] == i2["extend"] and i3["shadow"] == i2["shadow"]   # the same rays either way
    # node visits and triangle tests depend slightly on which rays share a warp (a lane holding a
    # postponed leaf keeps descending until the warp's other lanes hold one too), not the hits
    for key in ("extend_node_visits", "extend_tri_tests", "shadow_node_visits", "shadow_tri_tests"):
        assert abs(p3[key] / sep[key] - 1.0) < 0.01, key
    assert fused["kernel_launches"] == 2 + 4 * (fused["iterations"] - 1) + 2
    assert sep["kernel_launches"] == 3 + 5 * (sep["iterations"] - 1) + 1


@pytest.mark.parametrize("mode", ["graph", "launches", "guided"])
def test_iteration_bound_reports_timeout_and_handle_recovers(wr_lib, mode):
    """The wavefront's iteration bound (the device-side loop limit of every render) stops a render
    that has not drained and reports WR_ERR_TIMEOUT; nothing is left in flight, so the next render
    on the same handle is the right image. The bound is lowered through the debugging field
    max_iterations to make it trip."""
    path, _ = golden_scene("zoo")
    use_graph = mode != "launches"
    guiding = 1 if mode == "guided" else 0
    with wr_lib.Scene.from_file(path) as sc:
        ref = sc.render(spp=32, seed=11, use_graph=use_graph)
        with pytest.raises(wr_lib.WurstError) as e:
            sc.render(spp=32, seed=11, use_graph=use_graph, guiding=guiding, max_iterations=3)
        assert e.value.status == 7          # WR_ERR_TIMEOUT
        again = sc.render(spp=32, seed=11, use_graph=use_graph)
        assert sc.stats["iterations"] > 3
    assert np.allclose(again, ref, rtol=1e-9, atol=1e-12)


@pytest.mark.parametrize("res", [[37, 23], [8, 5], [5, 4], [64, 3]])
def test_tile_order_covers_every_pixel(wr_lib, oracle_lib, res):
    """New samples are issued in 8x4 pixel tiles, with the pixels outside the whole tiles in
    scanline order: every pixel of an odd-sized film gets its samples (from a camera inside the
    Cornell box every camera ray sees lit geometry, so no pixel may stay black), and the image
    mean matches the oracle's."""
    path, _ = golden_scene("cornell")
    cam = '{"pos": [0,1,0.95], "lookat": [0,1,0], "up": [0,1,0], "fovy": 40, "resolution": %s}' % res
    spp = max(64, 100000 // (res[0] * res[1]))      # about 400k GPU samples over the film
    with wr_lib.Scene.from_file(path) as sc:
        sc.set_camera(cam)
        img = np.mean([sc.render(spp=spp, seed=70 + i) for i in range(4)], axis=0)
    assert img.shape == (res[1], res[0], 3)
    assert (img.max(axis=2) > 0).all()
    osc = oracle_lib.OracleScene(path)
    osc.set_camera(__import__("json").loads(cam))
    ref, _, _ = osc.render(spp=4 * spp, threads=0)
    assert abs(img.mean() / ref.mean() - 1.0) < 0.03


def test_environment_only_scene_matches_oracle(wr_lib, oracle_lib, tmp_path):
    """A scene with no meshes, lit by the sky alone: every camera ray misses and picks the sky up
    directly (strategy B), the sky's light samples reach the lens (strategy C); the image matches
    the oracle's (the reference renders this scene too)."""
    import json
    import shutil
    src, _ = golden_scene("env")
    scene = json.load(open(src))
    shutil.copy(os.path.join(os.path.dirname(src), scene["envmap"]), tmp_path / "sky.pfm")
    doc = {"camera": {"pos": [0, 1, 3], "lookat": [0, 1, 0], "up": [0, 1, 0], "fovy": 60, "resolution": [32, 16]},
           "envmap": "sky.pfm", "meshes": [],
           "render": [{"integrator": "nextevent_path_tracer", "output": "o.pfm", "num_spp": 64, "num_path_vertices": 6}]}
    p = tmp_path / "sky_only.json"
    p.write_text(json.dumps(doc))
    with wr_lib.Scene.from_file(str(p)) as sc:
        assert sc.info["num_triangles"] == 0 and sc.info["has_envmap"] == 1
        img = np.mean([sc.render(spp=1024, seed=40 + i) for i in range(4)], axis=0)
    ref, _, _ = oracle_lib.OracleScene(str(p)).render(spp=4096, threads=0)
    assert np.isfinite(img).all()
    assert abs(img.mean() / ref.mean() - 1.0) < 0.01
    assert relmse(img, ref) < 0.01


@pytest.mark.parametrize("integrator", ["nextevent_path_tracer", "primitive_path_tracer", "light_splatting"])
def test_scene_without_any_emitter_renders_black(wr_lib, tmp_path, integrator):
    """No emitter and no sky: nothing to connect to and nothing to hit, so every integrator returns
    an all-zero image and no error. (The reference's light-selection CDF over zero lights is
    undefined there: its renderer crashes on such a scene.)"""
    from wurstrenderer_b200 import scenes
    spec = scenes.cornell_spec()
    spec.meshes = [m for m in spec.meshes if m.name != "light"]
    p = scenes.write_scene(str(tmp_path), "dark", spec, dict(scenes.CORNELL_CAMERA, resolution=[24, 16]),
                           [scenes.nee_render("o.pfm", 16, 8)])
    with wr_lib.Scene.from_file(p) as sc:
        assert sc.info["num_lights"] == 0 and sc.info["has_envmap"] == 0
        img = sc.render(spp=16, seed=3, integrator=integrator)
    assert img.shape == (16, 24, 3) and np.isfinite(img).all() and not img.any()
