"""Batched render jobs (many cameras, resolutions and sample counts over one scene) in one wavefront.

Each job is an independent PathNeeRenderer::render with its own camera
(src/renderer/pathnextevent.h:152-191). Job j of a batch uses the random
streams of a single render whose seed is seed_j + j * 0x9E3779B9, so a batch must
reproduce the single renders up to FP64 summation order.
"""
import json

import numpy as np
import pytest

from conftest import golden_scene

pytestmark = pytest.mark.gpu

GOLDEN_RATIO32 = 0x9E3779B9


def jobs_for_test():
    from wurstrenderer_b200 import scenes
    jobs = scenes.batch_jobs(seed=1003, n_jobs=6, num_path_vertices=14)
    for k, j in enumerate(jobs):
        r = [32, 48, 17, 64, 40, 8][k]
        j["camera"]["resolution"] = [r, max(1, r * 3 // 4)]
        j["num_spp"] = [4, 16, 1, 8, 32, 64][k]
        j["seed"] = 100 + k
    return jobs


@pytest.mark.parametrize("use_graph", [True, False])
def test_batch_reproduces_single_renders(wr_lib, use_graph):
    path, _ = golden_scene("cornell")
    jobs = jobs_for_test()
    with wr_lib.Scene.from_file(path) as sc:
        imgs = sc.render_batch(jobs, use_graph=use_graph, queue_capacity=4096)
        st = sc.stats
        assert st["paths"] == sum(j["camera"]["resolution"][0] * j["camera"]["resolution"][1] * j["num_spp"]
                                  for j in jobs)
        for k, (j, img) in enumerate(zip(jobs, imgs)):
            sc.set_camera(json.dumps(j["camera"]))
            single = sc.render(spp=j["num_spp"], num_path_vertices=j["num_path_vertices"],
                               seed=(j["seed"] + k * GOLDEN_RATIO32) & 0xFFFFFFFF)
            assert img.shape == single.shape
            assert np.allclose(img, single, rtol=1e-9, atol=1e-12), "job %d max diff %g" % (k, np.abs(img - single).max())


def test_batch_job_matches_oracle(wr_lib, oracle_lib):
    """One job of a batch against the oracle rendering the same camera."""
    path, _ = golden_scene("cornell")
    jobs = jobs_for_test()[:3]
    jobs[1]["num_spp"] = 1024
    jobs[1]["camera"]["resolution"] = [24, 18]
    with wr_lib.Scene.from_file(path) as sc:
        imgs = sc.render_batch(jobs)
    osc = oracle_lib.OracleScene(path)
    osc.set_camera(jobs[1]["camera"])
    ref, _, _ = osc.render(spp=1024, num_path_vertices=14, threads=0)
    assert abs(imgs[1].mean() / ref.mean() - 1.0) < 0.03


def test_autotune_returns_valid_settings(wr_lib):
    path, _ = golden_scene("zoo")
    with wr_lib.Scene.from_file(path) as sc:
        best, ms = sc.autotune(probe_spp=2)
        assert best["trace_block"] in (0, 64, 128, 256)
        assert ms > 0
        a = sc.render(spp=32, seed=5, **{k: v for k, v in best.items() if k != "use_graph"})
        b = sc.render(spp=32, seed=5)
    assert np.allclose(a, b, rtol=1e-9, atol=1e-12)


@pytest.mark.parametrize("block", [64, 256])
def test_traversal_block_sizes_agree(wr_lib, block):
    path, _ = golden_scene("hf")
    with wr_lib.Scene.from_file(path) as sc:
        a = sc.render(spp=16, seed=2, trace_block=block)
        b = sc.render(spp=16, seed=2)
    assert np.allclose(a, b, rtol=1e-9, atol=1e-12)


def test_batch_jobs_pass_the_reference_image_bar(wr_lib):
    """Eight jobs of one batch render the cornell fixture's own camera with different seeds,
    between jobs of other cameras and resolutions; together they are K = 8 independent renders
    and must pass the image bar of the single renders against the reference's 4096-spp images
    (relMSE within 2 x the reference noise floor, every 8x8 block |z| < 4, mean within 1 %)."""
    from conftest import GOLDEN
    from test_gpu_render import block_z, relmse
    path, meta = golden_scene("cornell")
    cam = json.load(open(path))["camera"]
    ref_a = np.load("%s/cornell_ref_hi_a.npy" % GOLDEN).astype(np.float64)
    ref_b = np.load("%s/cornell_ref_hi_b.npy" % GOLDEN).astype(np.float64)
    others = jobs_for_test()
    jobs = []
    for k in range(8):
        jobs.append({"camera": cam, "num_spp": meta["hi_spp"] // 8, "num_path_vertices": 10, "seed": 3000 + 7 * k})
        jobs.append(others[k % len(others)])
    with wr_lib.Scene.from_file(path) as sc:
        imgs = sc.render_batch(jobs)
    runs = np.stack(imgs[0::2])
    assert runs.shape[1:] == ref_a.shape and np.isfinite(runs).all()
    img = runs.mean(axis=0)
    floor = relmse(ref_b, ref_a)
    err = relmse(img, ref_a)
    assert err <= 2.0 * floor + 1e-6, "relMSE %.3g vs reference noise floor %.3g" % (err, floor)
    z = block_z(runs, ref_a)
    assert np.abs(z).max() < 4.0, "max |z| %.2f" % np.abs(z).max()
    assert abs(img.mean() / ref_a.mean() - 1.0) < 0.01


def test_batch_autotuner_returns_valid_settings(wr_lib):
    """wr_autotune_batch times probe batches; its settings change the schedule, not the images."""
    path, _ = golden_scene("cornell")
    jobs = jobs_for_test()
    with wr_lib.Scene.from_file(path) as sc:
        best, ms = sc.autotune_batch(jobs[:3])
        assert best["trace_block"] in (0, 64, 128, 256) and ms > 0
        assert best["queue_capacity"] in (0, 1 << 19, 1 << 20, 1 << 21, 1 << 22)
        a = sc.render_batch(jobs, **{k: v for k, v in best.items() if k != "use_graph"})
        b = sc.render_batch(jobs)
    for x, y in zip(a, b):
        assert np.allclose(x, y, rtol=1e-9, atol=1e-12)
