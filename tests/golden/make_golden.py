"""Generates the golden fixtures under tests/golden/ from the reference itself.

Needs the reference renderer compiled by ``make -C oracle ref`` (the
reference's own ``PathNeeRenderer`` / ``EmbreeAccel`` code; see
oracle/ref/ref_harness.cpp). For each fixture scene it writes:

  scenes/<name>/...            the scene (simple2 JSON + OBJ/MTL [+ PFM envmap])
  <name>_ref_spp4.npy          reference render, 4 spp, one thread (light_splatting: all threads),
                               seed salt 0 (float64)
  <name>_ref_hi_a.npy/_b.npy   two independent reference renders at HI_SPP (float32)
  <name>_rays.npy              seeded ray batch (float32 n x 8)
  <name>_hits.npy              reference closest hits for the batch: geomID, primID, t bits (int32 n x 3)
  <name>_hits_ng.npy           the same hits with Embree's Ng and the occlusion answer
                               (float32 n x 5: t, Ng xyz, occluded), for every geometry type

Usage: python tests/golden/make_golden.py [--hi-spp 4096]
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from wurstrenderer_b200 import scenes  # noqa: E402

FIXTURES = ["cornell", "zoo", "env", "hf", "cornell_pt", "env_pt", "cornell_ls", "hf_ls", "phong", "phong_pt",
            "phong_ls", "srgb", "lens", "lens_ls"]


def with_integrator(path, integrator):
    with open(path) as f:
        scene = json.load(f)
    for r in scene["render"]:
        r["integrator"] = integrator
    with open(path, "w") as f:
        json.dump(scene, f, indent=1)
    return path


def write_fixture_scene(name, out_dir):
    if name.endswith("_pt"):   # the same scene rendered by primitive_path_tracer
        return with_integrator(write_fixture_scene(name[:-3], out_dir), "primitive_path_tracer")
    if name.endswith("_ls"):   # the same scene rendered by light_splatting
        return with_integrator(write_fixture_scene(name[:-3], out_dir), "light_splatting")
    if name == "cornell":
        return scenes.write_cornell(out_dir, name="cornell", resolution=(48, 48), spp=4, num_path_vertices=10,
                                    spec=scenes.cornell_spec(box_angle=scenes.FIXTURE_BOX_ANGLE))
    if name == "zoo":
        return scenes.write_spec(out_dir, "zoo", scenes.material_zoo_spec(), scenes.CORNELL_CAMERA, (48, 40), 4, 10)
    if name == "env":
        return scenes.write_env_scene(out_dir, name="env", resolution=(48, 36), spp=4, num_path_vertices=8,
                                      env_size=(64, 32))
    if name == "hf":
        spec = scenes.heightfield_spheres_spec(seed=1012, n_grid=33, n_spheres=24, sphere_subdiv=1, extent=3.0,
                                               n_lights=4, light_ke=(30.0, 28.0, 25.0))
        cam = dict(scenes.HEIGHTFIELD_CAMERA, pos=[0.0, 2.2, 5.5])
        return scenes.write_spec(out_dir, "hf", spec, cam, (48, 24), 4, 12)
    if name == "srgb":    # sRGB-encoded reflectances (a "mitsuba_srgb": true mesh entry)
        return scenes.write_srgb_zoo(out_dir, name="srgb", resolution=(48, 40), spp=4, num_path_vertices=10)
    if name == "lens":    # thin-lens camera: aperture radius and focal distance 0.1 ("radius")
        return scenes.write_cornell_lens(out_dir, name="lens", resolution=(48, 48), spp=4, num_path_vertices=10,
                                         radius=0.1)
    if name == "phong":   # Phong tessellation surfaces (a "phong_tessellation": true mesh entry)
        return scenes.write_phong_cornell(out_dir, name="phong", resolution=(48, 48), spp=4, num_path_vertices=8)
    raise KeyError(name)


def seeded_rays(json_path, n, seed):
    """Rays from random points inside the scene box toward random directions, plus
    rays from the camera region toward random scene points (hits and misses)."""
    sc = oracle.OracleScene(json_path)
    lo, hi = sc.bbox_lo, sc.bbox_hi
    ext = hi - lo
    rng = np.random.default_rng(seed)
    o = lo - 0.1 * ext + rng.uniform(size=(n, 3)) * ext * 1.2
    tgt = lo + rng.uniform(size=(n, 3)) * ext
    d = np.where(rng.uniform(size=(n, 1)) < 0.5, tgt - o, rng.normal(size=(n, 3)))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3] = o
    rays[:, 3] = 1e-4
    rays[:, 4:7] = d
    rays[:, 7] = np.inf
    return rays


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--hi-spp", type=int, default=4096)
    ap.add_argument("--only", default=None)
    args = ap.parse_args()
    if not oracle.reference_available():
        oracle.build(with_reference=True)
    # env_ls (light tracing under the sky: very noisy, kept for the oracle check and a flux test)
    for name in FIXTURES + ["env_ls"]:
        if args.only and name != args.only:
            continue
        sdir = os.path.join(HERE, "scenes", name)
        path = write_fixture_scene(name, sdir)
        tmp = os.path.join(sdir, "_tmp.pfm")
        raw = os.path.join(sdir, "_tmp.f64")
        sc = oracle.OracleScene(path)
        shape = (sc.height, sc.width, 3)
        # light_splatting runs through the reference's own multi-threaded render() only, so its
        # 4-spp fixture is exact up to the order of the FP64 atomic splat sums
        oracle.run_reference(path, tmp, serial=not name.endswith("_ls"), raw=raw)
        np.save(os.path.join(HERE, name + "_ref_spp4.npy"), np.fromfile(raw, np.float64).reshape(shape))
        for tag, salt in (("a", 11), ("b", 22)):
            rep = oracle.run_reference(path, tmp, spp=args.hi_spp, salt=salt, raw=raw)
            np.save(os.path.join(HERE, "%s_ref_hi_%s.npy" % (name, tag)),
                    np.fromfile(raw, np.float64).reshape(shape).astype(np.float32))
            print(name, tag, rep, flush=True)
        rays = seeded_rays(path, 2048, seed=77)
        rays_path = os.path.join(HERE, name + "_rays.npy")
        np.save(rays_path, rays)
        rays.tofile(os.path.join(sdir, "_rays.f32"))
        # rtcIntersect1 / rtcOccluded1 on the reference's accel (user geometry included)
        g, p, t, ng, occ = oracle.run_reference_trace(path, rays, sdir)
        hits = np.stack([g, p, t.view(np.int32)], 1).astype(np.int32)
        np.save(os.path.join(HERE, name + "_hits.npy"), hits)
        np.save(os.path.join(HERE, name + "_hits_ng.npy"),
                np.concatenate([t[:, None], ng, occ[:, None].astype(np.float32)], 1).astype(np.float32))
        for f in ("_tmp.pfm", "_tmp.f64", "_rays.f32", "trace2_rays.f32", "trace2_hits.bin"):
            if os.path.exists(os.path.join(sdir, f)):
                os.remove(os.path.join(sdir, f))
        with open(os.path.join(HERE, name + "_meta.json"), "w") as f:
            json.dump({"scene": os.path.relpath(path, HERE), "hi_spp": args.hi_spp, "salts": [11, 22],
                       "width": sc.width, "height": sc.height,
                       "integrator": json.load(open(path))["render"][0]["integrator"]}, f)


if __name__ == "__main__":
    main()
