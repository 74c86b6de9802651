"""Traversal parity on the GPU: closest-hit triangle ids against the reference.

The golden hits are the reference's own closest-hit answers
(EmbreeAccel::intersectTriangleInfo through the oracle's restatement of Embree's
triangle test). The B200 kernel uses a watertight test, so ids must agree
exactly except on rays whose two candidate hits tie in distance within
1e-5 relative, or that graze a triangle edge (barycentric within 1e-5 of an
edge), where the two tests may legitimately pick different triangles.

Any-hit answers are held to the same rule: every GPU answer must lie between the
oracle's FP64 bounds for the ray (occluded_bracket: triangles shrunk / grown by 1e-5
in barycentric coordinates, segment ends moved by 1e-5 relative, grazing rays
excused), so an answer may differ from the reference's only on an edge graze or an
end-point tie, and nowhere else.
"""
import numpy as np
import pytest

from conftest import FIXTURES, GOLDEN, golden_scene

pytestmark = pytest.mark.gpu


def _tie_or_edge(t_ref, t_gpu, uv_ref):
    with np.errstate(invalid="ignore"):
        tie = np.abs(t_ref - t_gpu) <= 1e-5 * np.maximum(np.abs(t_ref), 1.0)
    edge = (uv_ref[:, 0] < 1e-5) | (uv_ref[:, 1] < 1e-5) | (1.0 - uv_ref[:, 0] - uv_ref[:, 1] < 1e-5)
    # a Phong patch hit reports uv = (0, 0) (the reference's texture coordinate): no edge excuse
    patch = (uv_ref[:, 0] == 0.0) & (uv_ref[:, 1] == 0.0)
    return tie | (edge & ~patch)


@pytest.mark.parametrize("name", FIXTURES)
def test_closest_hit_ids_match_reference(wr_lib, oracle_lib, name):
    path, _ = golden_scene(name)
    rays = np.load("%s/%s_rays.npy" % (GOLDEN, name))
    hits = np.load("%s/%s_hits.npy" % (GOLDEN, name))
    with wr_lib.Scene.from_file(path) as sc:
        g, p, t, uv = sc.trace_closest(rays)
    _, _, _, uv_ref = oracle_lib.OracleScene(path).trace_closest(rays)
    t_ref = hits[:, 2].view(np.float32)
    same = (g == hits[:, 0]) & (p == hits[:, 1])
    excused = _tie_or_edge(t_ref, t, uv_ref)
    bad = ~same & ~excused
    assert bad.sum() == 0, "mismatching rays: %s" % np.nonzero(bad)[0][:10]
    assert same.mean() > 0.99
    hit = same & (g >= 0)
    assert np.allclose(t[hit], t_ref[hit], rtol=2e-5, atol=1e-6)
    assert np.allclose(uv[hit], uv_ref[hit], atol=2e-4)


@pytest.mark.parametrize("name", FIXTURES)
def test_wide_bvh_hits_match_reference(wr_lib, oracle_lib, name):
    """The compressed 8-wide BVH gives the same closest hits and occlusion answers as the binary
    one (the tree changes which boxes are visited, never the accepted hit)."""
    path, _ = golden_scene(name)
    rays = np.load("%s/%s_rays.npy" % (GOLDEN, name))
    hits = np.load("%s/%s_hits.npy" % (GOLDEN, name))
    with wr_lib.Scene.from_file(path, bvh_width=8) as sc:
        g, p, t, uv = sc.trace_closest(rays)
        occ = sc.trace_occluded(rays)
    with wr_lib.Scene.from_file(path, bvh_width=2) as sb:
        g2, p2, t2, uv2 = sb.trace_closest(rays)
        occ2 = sb.trace_occluded(rays)
    _, _, _, uv_ref = oracle_lib.OracleScene(path).trace_closest(rays)
    t_ref = hits[:, 2].view(np.float32)
    same = (g == hits[:, 0]) & (p == hits[:, 1])
    bad = ~same & ~_tie_or_edge(t_ref, t, uv_ref)
    assert bad.sum() == 0, "mismatching rays: %s" % np.nonzero(bad)[0][:10]
    both = (g == g2) & (p == p2)
    assert np.array_equal(t[both], t2[both])
    # the two trees test tied candidates (a ray through a shared edge) in different orders
    assert (~both & ~_tie_or_edge(t2, t, uv_ref)).sum() == 0
    lo, hi = oracle_lib.OracleScene(path).trace_occluded_bracket(rays)
    assert_within_bracket(occ, lo, hi)
    assert_within_bracket(occ2, lo, hi)


def assert_within_bracket(occ, lo, hi, max_ambiguous=0.005):
    """Any-hit answers against the oracle's bounds: blocked where it is blocked beyond doubt,
    free where nothing can block it."""
    occ = np.asarray(occ).astype(bool)
    bad = (occ & ~hi) | (~occ & lo)
    assert bad.sum() == 0, "any-hit answers outside the oracle's bounds: rays %s" % np.nonzero(bad)[0][:10]
    assert (hi & ~lo).mean() <= max_ambiguous, "too many ambiguous rays: %d" % (hi & ~lo).sum()


def shadow_segments(rays, hits, lo, hi, seed=5):
    """Three kinds of finite segments over a ray batch: ending halfway to the reference's closest
    hit, ending beyond it, and from the ray's origin to a random point of the scene box (the shape
    of a shadow ray toward a light sample, tmax = length - 1e-4)."""
    rng = np.random.default_rng(seed)
    t_ref = hits[:, 2].view(np.float32)
    n = len(rays)
    out = np.repeat(rays[None], 3, axis=0).reshape(3 * n, 8).copy()
    out[:n, 7] = np.where(hits[:, 0] >= 0, 0.5 * t_ref, 10.0)
    out[n:2 * n, 7] = np.where(hits[:, 0] >= 0, 1.5 * t_ref, 10.0)
    tgt = lo + rng.uniform(size=(n, 3)) * (hi - lo)
    d = tgt - rays[:, 0:3]
    ln = np.linalg.norm(d, axis=1)
    out[2 * n:, 4:7] = d / ln[:, None]
    out[2 * n:, 3] = 1e-4
    out[2 * n:, 7] = ln - 1e-4
    return out


@pytest.mark.parametrize("name", FIXTURES)
def test_occlusion_matches_oracle(wr_lib, oracle_lib, name):
    path, _ = golden_scene(name)
    rays = np.load("%s/%s_rays.npy" % (GOLDEN, name))
    hits = np.load("%s/%s_hits.npy" % (GOLDEN, name))
    osc = oracle_lib.OracleScene(path)
    segs = shadow_segments(rays, hits, osc.bbox_lo, osc.bbox_hi)
    with wr_lib.Scene.from_file(path) as sc:
        occ = sc.trace_occluded(segs)
    lo, hi = osc.trace_occluded_bracket(segs)
    assert_within_bracket(occ, lo, hi)
    # the reference's own answers lie inside the same bounds
    assert_within_bracket(osc.trace_occluded(segs), lo, hi)


def test_empty_and_tiny_batches(wr_lib, oracle_lib):
    path, _ = golden_scene("cornell")
    with wr_lib.Scene.from_file(path) as sc:
        g, p, t, uv = sc.trace_closest(np.zeros((0, 8), np.float32))
        assert g.shape == (0,)
        r = np.array([[0.6, 1.5, 3.5, 1e-4, 0, 0, -1, np.inf],      # over the short box to the back wall
                      [0, 1, 3.5, 1e-4, 0, 0, -1, np.inf],          # onto the tall box
                      [0, 1, 3.5, 1e-4, 0, 0, 1, np.inf],           # out of the open front: miss
                      [0, 1, 0.5, 1e-4, 0, 1, 0, 0.5]], np.float32)  # segment ending below the ceiling: miss
        g, p, t, uv = sc.trace_closest(r)
    go, po, to, _ = oracle_lib.OracleScene(path).trace_closest(r)
    assert g[0] >= 0 and abs(t[0] - 4.5) < 1e-4
    assert np.array_equal(g, go) and np.array_equal(p, po)
    assert (g[2], p[2], g[3]) == (-1, -1, -1)
    assert np.allclose(t[:2], to[:2], rtol=1e-5)


def test_traversal_statistics(wr_lib):
    path, _ = golden_scene("hf")
    rays = np.load("%s/hf_rays.npy" % GOLDEN)
    with wr_lib.Scene.from_file(path) as sc:
        nv, nt = sc.trace_stats(rays)
    assert nv >= len(rays) and nt > 0


@pytest.mark.parametrize("name", ["phong"])
def test_patch_hits_and_normals_match_reference(wr_lib, oracle_lib, name):
    """Phong tessellation patches: the FP64 patch test on the GPU against the reference's own
    PhongMeshGeometry::intersect (through Embree's user-geometry callbacks): ids exact except
    on distance ties, t within 1e-6 relative, the unit normal within 1e-5 of the reference's
    normalised Ng, and occlusion identical but for ties."""
    path, _ = golden_scene(name)
    rays = np.load("%s/%s_rays.npy" % (GOLDEN, name))
    hits = np.load("%s/%s_hits.npy" % (GOLDEN, name))
    hng = np.load("%s/%s_hits_ng.npy" % (GOLDEN, name))
    t_ref = hits[:, 2].view(np.float32)
    with wr_lib.Scene.from_file(path) as sc:
        g, p, t, nrm = sc.trace_hits(rays)
        occ = sc.trace_occluded(rays)
    _, _, _, uv_ref = oracle_lib.OracleScene(path).trace_closest(rays)
    patch = (hits[:, 0] >= 0) & (uv_ref[:, 0] == 0.0) & (uv_ref[:, 1] == 0.0)
    assert patch.sum() > 200, "the ray batch should hit many patches"
    same = (g == hits[:, 0]) & (p == hits[:, 1])
    with np.errstate(invalid="ignore"):
        tie = np.abs(t_ref - t) <= 1e-5 * np.maximum(np.abs(t_ref), 1.0)
    assert (~same & ~tie).sum() == 0, "mismatching rays: %s" % np.nonzero(~same & ~tie)[0][:10]
    m = same & patch
    assert np.allclose(t[m], t_ref[m], rtol=1e-6, atol=0.0), np.max(np.abs(t[m] / t_ref[m] - 1.0))
    ng_ref = hng[:, 1:4].astype(np.float64)
    ng_ref /= np.linalg.norm(ng_ref, axis=1, keepdims=True) + 1e-300
    assert np.abs(nrm[m] - ng_ref[m]).max() < 1e-5
    assert np.abs(np.linalg.norm(nrm[m], axis=1) - 1.0).max() < 1e-5
    occ_ref = hng[:, 4] > 0.5
    lo, hi = oracle_lib.OracleScene(path).trace_occluded_bracket(rays)
    assert_within_bracket(occ_ref, lo, hi)
    assert_within_bracket(occ, lo, hi)


@pytest.mark.parametrize("name", ["hf", "phong"])
@pytest.mark.parametrize("opts", [dict(max_leaf=1), dict(max_leaf=8, sah_trav_cost=3.0),
                                  dict(sah_patch_cost=1.0), dict(sah_patch_cost=200.0, bvh_width=8)],
                         ids=["leaf1", "leaf8_ct3", "patch1", "patch200_w8"])
def test_tree_shape_options_keep_the_hits(wr_lib, oracle_lib, name, opts):
    """Leaf size and the SAH's traversal / patch-test costs change the tree, never the accepted
    hit: the same closest hits as the reference (ties and edges excused) and the same hits as
    the default tree."""
    path, _ = golden_scene(name)
    rays = np.load("%s/%s_rays.npy" % (GOLDEN, name))
    hits = np.load("%s/%s_hits.npy" % (GOLDEN, name))
    with wr_lib.Scene.from_file(path, **opts) as sc:
        g, p, t, _ = sc.trace_closest(rays)
        occ = sc.trace_occluded(rays)
    with wr_lib.Scene.from_file(path) as sd:
        g2, p2, t2, _ = sd.trace_closest(rays)
        occ2 = sd.trace_occluded(rays)
    _, _, _, uv_ref = oracle_lib.OracleScene(path).trace_closest(rays)
    t_ref = hits[:, 2].view(np.float32)
    same = (g == hits[:, 0]) & (p == hits[:, 1])
    assert (~same & ~_tie_or_edge(t_ref, t, uv_ref)).sum() == 0
    both = (g == g2) & (p == p2)
    assert np.array_equal(t[both], t2[both])
    assert (~both & ~_tie_or_edge(t2, t, uv_ref)).sum() == 0
    lo, hi = oracle_lib.OracleScene(path).trace_occluded_bracket(rays)
    assert_within_bracket(occ, lo, hi)
    assert_within_bracket(occ2, lo, hi)


def test_tree_shape_option_errors(wr_lib):
    path, _ = golden_scene("cornell")
    for bad in (dict(sah_trav_cost=-1.0), dict(sah_trav_cost=101.0), dict(sah_patch_cost=-2.0),
                dict(sah_patch_cost=1001.0), dict(bvh_width=4)):
        with pytest.raises(wr_lib.WurstError) as e:
            wr_lib.Scene.from_file(path, **bad)
        assert e.value.status == 1     # WR_ERR_INVALID_ARGUMENT


def test_degenerate_and_coincident_triangles(wr_lib, oracle_lib, tmp_path):
    """Zero-area triangles (collinear and repeated vertices) and exact duplicates of the Cornell
    box's triangles in one scene: the build and traversal take them, closest hits match the oracle
    except on ties (a duplicate is a tie), and no ray reports a degenerate triangle."""
    from wurstrenderer_b200 import scenes
    spec = scenes.cornell_spec()
    dup = [m for m in spec.meshes if m.name in ("tall_box", "floor")]
    for m in dup:
        spec.add(m.name + "_copy", spec.materials[m.material], m.positions.copy(), m.triangles.copy())
    mat = spec.materials["m_floor"]
    spec.add("degenerate", mat, np.array([[0, 0.5, 0], [0.5, 0.5, 0], [1.0, 0.5, 0], [0.2, 1.0, 0.2]], np.float32),
             np.array([[0, 1, 2], [3, 3, 3], [0, 0, 1]], np.int64))
    path = scenes.write_scene(str(tmp_path), "degenerate", spec, dict(scenes.CORNELL_CAMERA, resolution=[16, 16]),
                              [scenes.nee_render("o.pfm", 4, 6)])
    rng = np.random.default_rng(11)
    n = 4096
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3] = rng.uniform([-0.95, 0.05, -0.95], [0.95, 1.95, 0.95], size=(n, 3))
    d = rng.normal(size=(n, 3))
    rays[:, 4:7] = d / np.linalg.norm(d, axis=1, keepdims=True)
    rays[:, 3] = 1e-4
    rays[:, 7] = np.inf
    osc = oracle_lib.OracleScene(path)
    go, po, to, uv_ref = osc.trace_closest(rays)
    with wr_lib.Scene.from_file(path) as sc:
        g, p, t, uv = sc.trace_closest(rays)
        occ = sc.trace_occluded(rays)
        img = sc.render(spp=16, seed=1)
    same = (g == go) & (p == po)
    assert (~same & ~_tie_or_edge(to, t, uv_ref)).sum() == 0
    assert np.isfinite(img).all() and img.mean() > 0
    lo, hi = osc.trace_occluded_bracket(rays)
    assert_within_bracket(occ, lo, hi)
