"""The oracle (FP64 CPU restatement) pinned against the reference's own renderer.

The golden fixtures were produced by the reference's PathNeeRenderer and
EmbreeAccel code compiled from its sources (tests/golden/make_golden.py).
The oracle follows the same random streams and arithmetic order, so its
images must match bit for bit and its ray queries exactly.
"""
import numpy as np
import pytest

from conftest import FIXTURES, GOLDEN, golden_scene


@pytest.mark.parametrize("name", FIXTURES + ["env_ls"])
def test_oracle_render_matches_reference_bit_exact(oracle_lib, name):
    path, meta = golden_scene(name)
    ref = np.load("%s/%s_ref_spp4.npy" % (GOLDEN, name))
    sc = oracle_lib.OracleScene(path)
    img, _, paths = sc.render(threads=1)
    assert paths == sc.width * sc.height * 4
    assert img.shape == ref.shape
    if name.endswith("_ls"):
        # the reference's light_splatting render is multi-threaded: exact up to the order of the
        # FP64 atomic splat sums
        assert np.allclose(img, ref, rtol=1e-12, atol=1e-15), "max abs diff %g" % np.abs(img - ref).max()
    else:
        assert np.array_equal(img, ref), "max abs diff %g" % np.abs(img - ref).max()


@pytest.mark.parametrize("name", FIXTURES)
def test_oracle_trace_matches_reference(oracle_lib, name):
    path, _ = golden_scene(name)
    rays = np.load("%s/%s_rays.npy" % (GOLDEN, name))
    hits = np.load("%s/%s_hits.npy" % (GOLDEN, name))
    sc = oracle_lib.OracleScene(path)
    g, p, t, _ = sc.trace_closest(rays)
    assert np.array_equal(g, hits[:, 0])
    assert np.array_equal(p, hits[:, 1])
    hit = g >= 0
    assert np.array_equal(t[hit].view(np.int32), hits[hit, 2])
    assert 0.2 < hit.mean() <= 1.0


def test_oracle_patch_normals_and_occlusion_match_reference(oracle_lib):
    """Phong tessellation patches: the oracle's FP64 restatement of PhongMeshGeometry gives the
    reference's own Ng (the float-rounded unit patch normal) and occlusion answers bit for bit."""
    path, _ = golden_scene("phong")
    rays = np.load("%s/phong_rays.npy" % GOLDEN)
    hng = np.load("%s/phong_hits_ng.npy" % GOLDEN)
    sc = oracle_lib.OracleScene(path)
    g, p, t, ng = sc.trace_hits(rays)
    hit = g >= 0
    assert np.array_equal(ng[hit], hng[hit, 1:4])
    assert np.array_equal(t[hit], hng[hit, 0])
    occ = sc.trace_occluded(rays)
    assert np.array_equal(occ.astype(bool), hng[:, 4] > 0.5)


def test_oracle_patch_bounds_contain_the_surface(oracle_lib):
    """The patch bound (phongmesh.h:61-164) gates the patch test, so it must enclose the patch:
    a short ray aimed along the interpolated normal at a point sampled on the Phong surface of
    each patch of the fixture's objects hits it (the box could only cut such hits off)."""
    from wurstrenderer_b200 import scenes
    path, _ = golden_scene("phong")
    sc = oracle_lib.OracleScene(path)
    alpha = 0.75
    rng = np.random.default_rng(9)
    rays = []
    for m in scenes.phong_objects_spec().meshes:
        P = m.positions.astype(np.float64)
        N = m.normals.astype(np.float64)
        N /= np.linalg.norm(N, axis=1, keepdims=True)
        for a, b, c in m.triangles:
            for _ in range(2):
                u, v = rng.uniform(0.02, 0.96, 2)
                if u + v > 0.98:
                    u, v = 1 - u, 1 - v
                w = 1 - u - v
                puv = u * P[a] + v * P[b] + w * P[c]
                ps = sum(wt * (puv - np.dot(puv - P[i], N[i]) * N[i]) for wt, i in ((u, a), (v, b), (w, c)))
                q = (1 - alpha) * puv + alpha * ps
                nrm = u * N[a] + v * N[b] + w * N[c]
                nrm /= np.linalg.norm(nrm)
                rays.append([*(q + 0.05 * nrm), 0.0, *(-nrm), 0.1])
    rays = np.asarray(rays, np.float32)
    g, _, t, _ = sc.trace_closest(rays)
    assert (g >= 0).mean() > 0.995
    assert np.median(t[g >= 0]) == pytest.approx(0.05, rel=1e-3)


@pytest.mark.parametrize("name", FIXTURES)
def test_reference_noise_floor_is_small(name):
    a = np.load("%s/%s_ref_hi_a.npy" % (GOLDEN, name)).astype(np.float64)
    b = np.load("%s/%s_ref_hi_b.npy" % (GOLDEN, name)).astype(np.float64)
    rel = np.mean((a - b) ** 2 / (b ** 2 + 1e-2))
    assert np.isfinite(a).all() and np.isfinite(b).all()
    assert a.mean() > 0
    assert rel < 0.05


def test_oracle_threads_agree_to_summation_order(oracle_lib):
    path, _ = golden_scene("zoo")
    sc = oracle_lib.OracleScene(path)
    a, _, _ = sc.render(spp=2, threads=1, salt=3)
    b, _, _ = sc.render(spp=2, threads=4, salt=3)
    assert np.allclose(a, b, rtol=1e-12, atol=1e-15)


def test_oracle_salt_changes_streams(oracle_lib):
    path, _ = golden_scene("cornell")
    sc = oracle_lib.OracleScene(path)
    a, _, _ = sc.render(spp=1, threads=1, salt=0)
    b, _, _ = sc.render(spp=1, threads=1, salt=1)
    assert not np.array_equal(a, b)


def test_oracle_crop_scales_splats(oracle_lib):
    """A crop renders whole 32x32 tiles and rescales the splat film by the pixels rendered."""
    path, _ = golden_scene("cornell")
    sc = oracle_lib.OracleScene(path)
    img, _, paths = sc.render(spp=1, threads=1, crop=(0, 0, 8, 8))
    assert paths == 32 * 32
    assert img[:32, :32].mean() > 0


@pytest.mark.parametrize("nverts", [1, 2])
def test_oracle_short_paths(oracle_lib, nverts):
    path, _ = golden_scene("cornell")
    sc = oracle_lib.OracleScene(path)
    img, _, _ = sc.render(spp=2, num_path_vertices=nverts, threads=1)
    if nverts == 1:
        assert not img.any()   # PathNeeRenderer::render returns before sampling
    else:
        assert img.max() > 0   # emitter seen directly + light splats


def test_oracle_live_against_reference_binary(oracle_lib, tmp_path):
    """Where the reference was compiled here, check a fresh salted render end to end."""
    if not oracle_lib.reference_available():
        pytest.skip("reference binary not built in this environment")
    path, _ = golden_scene("env")
    raw = str(tmp_path / "r.f64")
    oracle_lib.run_reference(path, str(tmp_path / "r.pfm"), spp=3, salt=12345, serial=True, raw=raw)
    sc = oracle_lib.OracleScene(path)
    ref = np.fromfile(raw, np.float64).reshape(sc.height, sc.width, 3)
    img, _, _ = sc.render(spp=3, salt=12345, threads=1)
    assert np.array_equal(img, ref)
