"""The seeded benchmark workloads (wurstrenderer_b200/scenes.py) against the shapes their configs
state: the Cornell box of config 1 (five walls and two axis-aligned boxes, a 0.5 x 0.5 ceiling
light of radiance (17, 12, 4), albedos in [0.2, 0.8] with red and green side walls), the about
1M-triangle heightfield-and-spheres scene of config 2, the 128-job table of config 3 and the
about 200k-triangle door-gap room of config 4. CPU only: the generators are numpy."""
import numpy as np
import pytest

from wurstrenderer_b200 import scenes


def _mesh(spec, name):
    return next(m for m in spec.meshes if m.name == name)


def test_cornell_box_of_config_1():
    spec = scenes.cornell_spec()
    walls = ["floor", "ceiling", "back", "left", "right"]
    assert sum(_mesh(spec, w).triangles.shape[0] for w in walls) + \
        sum(_mesh(spec, b).triangles.shape[0] for b in ("short_box", "tall_box")) == 34
    assert spec.num_triangles == 36   # with the two triangles of the light
    for b in ("short_box", "tall_box"):   # axis-aligned: two distinct values per coordinate
        p = _mesh(spec, b).positions
        for k in range(3):
            assert len(np.unique(np.round(p[:, k], 6))) == 2, (b, k)
    light = _mesh(spec, "light")
    ext = light.positions.max(axis=0) - light.positions.min(axis=0)
    assert np.allclose(sorted(ext)[1:], [0.5, 0.5]) and ext[1] < 1e-6
    assert spec.materials[light.material].ke == (17.0, 12.0, 4.0)
    for w in walls + ["short_box", "tall_box"]:
        kd = np.asarray(spec.materials[_mesh(spec, w).material].kd)
        assert ((kd >= 0.2 - 1e-9) & (kd <= 0.8 + 1e-9)).all(), w
    red, green = (np.asarray(spec.materials[_mesh(spec, w).material].kd) for w in ("left", "right"))
    assert red[0] > red[1] and red[0] > red[2] and green[1] > green[0] and green[1] > green[2]
    cam = scenes.CORNELL_CAMERA
    assert cam["fovy"] == 40.0 and cam["resolution"] == [256, 256]


def test_fixture_cornell_boxes_are_turned():
    p = _mesh(scenes.cornell_spec(box_angle=scenes.FIXTURE_BOX_ANGLE), "tall_box").positions
    assert len(np.unique(np.round(p[:, 0], 6))) > 2


def test_heightfield_spheres_of_config_2():
    spec = scenes.heightfield_spheres_spec()
    assert spec.num_triangles == 1162250
    lights = [m for m in spec.meshes if any(spec.materials[m.material].ke)]
    assert len(lights) == 4


def test_batch_jobs_of_config_3():
    jobs = scenes.batch_jobs()
    assert len(jobs) == 128
    res = {j["camera"]["resolution"][0] for j in jobs}
    assert res <= {64, 128, 256, 512} and len(res) == 4
    assert all(j["camera"]["resolution"][0] == j["camera"]["resolution"][1] for j in jobs)
    spp = np.array([j["num_spp"] for j in jobs])
    assert spp.min() >= 4 and spp.max() <= 256
    assert all(j["num_path_vertices"] == 14 for j in jobs)   # max depth 12


@pytest.mark.timeout(600)
def test_door_room_of_config_4():
    spec = scenes.door_room_spec(seed=1004)
    assert spec.num_triangles == 197782
    lights = [m for m in spec.meshes if any(spec.materials[m.material].ke)]
    assert len(lights) == 1
    ext = lights[0].positions.max(axis=0) - lights[0].positions.min(axis=0)
    assert np.allclose(sorted(ext)[1:], [1.0, 1.0], atol=1e-6)   # the 1 x 1 emitter


@pytest.mark.timeout(600)
def test_full_combination_of_config_5():
    spec = scenes.full_combination_spec()
    assert spec.num_triangles == 9980450   # about 10M
    lights = [m for m in spec.meshes if any(spec.materials[m.material].ke)]
    assert len(lights) == 16
    exps = [m.exponent for m in spec.materials.values() if m.exponent > 0]
    assert max(exps) <= 2000.0 and max(exps) > 1000.0   # glossy Phong up to exponent 2000
    sky = scenes.envmap_image(2048, 1024)
    assert sky.shape == (1024, 2048, 3) and sky.dtype == np.float32 and (sky > 0).all()
