"""Generates FP64 reference crops (and ray batches) for the full-size workloads.

The scenes are regenerated deterministically by wurstrenderer_b200.scenes wherever they are
needed (they are large), so only the reference image of a crop is stored:

  c1:   the procedural Cornell box (config 1; 36 triangles), 256 x 256, 10 vertices, the whole frame
  c2:   the heightfield-and-spheres scene (config 2; 512^2 fBm floor + 2000 icospheres + 4 area
        lights, 1,162,250 triangles), 1024 x 512, 18 vertices, crop 128 x 64 at (448, 288)
  c2h:  the same frame, crop 128 x 64 at (768, 160) (the horizon: distant small spheres)
  door: the door-gap room (config 4; closed 6 x 3 x 6 m room, 1 x 1 emitter behind a partition
        with a 0.2 m door gap, 300 seeded boxes, 197,782 triangles), 1024 x 1024, 10 vertices,
        crop 128 x 128 at (448, 448)
  c5:   the full combination (config 5; 2048^2 fBm floor + 20000 icospheres + 16 area lights +
        a 2048 x 1024 FP32 sky, 9,980,450 triangles), 3840 x 2160, 26 vertices,
        crop 128 x 64 at (1856, 1056)

For each, <name>_crop_ref_a.npy / _b.npy are two independent renders of the crop by the
reference's own PathNeeRenderer code (oracle/_ref) with salts 11 / 22, `--spp` each, and
<name>_crop_meta.json records the crop, spp and scene parameters.

With --rays N (c1, c2): a seeded batch of N rays over the workload's scene and the reference's
answers for it (EmbreeAccel::intersect / isIntersect through oracle/_ref):
  <name>_rays.npy   float32 (N, 8): origin, tnear, direction, tfar
  <name>_hits.npy   int32 (N, 4): geomID, primID, bits of the float hit distance, occluded (tfar = inf)

Usage: python tests/golden/make_crop_golden.py --workload c1|c2|c2h|door|c5 [--spp 8192] [--threads N]
                                              [--rays 65536] [--no-crop]
"""
from __future__ import annotations

import argparse
import json
import math
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

import oracle  # noqa: E402
from make_golden import seeded_rays  # noqa: E402
from wurstrenderer_b200 import scenes  # noqa: E402

WORKLOADS = {
    "c1": {"scene": "scenes.write_cornell(seed=1001)", "camera": scenes.CORNELL_CAMERA},
    "c2": {"scene": "scenes.write_heightfield_spheres(seed=1002)", "camera": scenes.HEIGHTFIELD_CAMERA},
    "c2h": {"scene": "scenes.write_heightfield_spheres(seed=1002)", "camera": scenes.HEIGHTFIELD_CAMERA},
    "door": {"scene": "scenes.door_room_spec(seed=1004)", "camera": scenes.DOOR_ROOM_CAMERA},
    "c5": {"scene": "scenes.write_full_combination(seed=1005)", "camera": scenes.FULL_COMBINATION_CAMERA},
}
for _name, _w in WORKLOADS.items():
    _w.update(scenes.PLAIN_WORKLOADS.get(_name) or scenes.GUIDED_WORKLOADS[_name])


def write_workload_scene(name, out_dir, spp=64):
    if name in scenes.PLAIN_WORKLOADS:
        return scenes.write_plain_workload(name, out_dir, spp)
    return scenes.write_guided_workload(name, out_dir, spp)


def camera_rays(camera, n, seed):
    """Pinhole primary rays of the workload's camera through uniformly random film points."""
    rng = np.random.default_rng(seed)
    pos, at, up = (np.asarray(camera[k], np.float64) for k in ("pos", "lookat", "up"))
    z = at - pos
    z /= np.linalg.norm(z)
    x = np.cross(up, z)
    x /= np.linalg.norm(x)
    y = np.cross(z, x)
    w, h = camera["resolution"]
    th = math.tan(math.radians(camera["fovy"]) / 2.0)
    sx = (rng.uniform(size=n) * 2.0 - 1.0) * th * w / h
    sy = (1.0 - rng.uniform(size=n) * 2.0) * th
    d = z[None] + sx[:, None] * x[None] + sy[:, None] * y[None]
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3] = pos
    rays[:, 3] = 1e-4
    rays[:, 4:7] = d
    rays[:, 7] = np.inf
    return rays


def make_rays(name, path, n, work_dir):
    """Half random rays through the scene box (make_golden.seeded_rays), half camera rays."""
    rays = np.concatenate([seeded_rays(path, n - n // 2, seed=177), camera_rays(WORKLOADS[name]["camera"], n // 2, 178)])
    g, p, t, _, occ = oracle.run_reference_trace(path, rays, work_dir)
    hits = np.stack([g, p, t.view(np.int32), occ.astype(np.int32)], 1).astype(np.int32)
    np.save(os.path.join(HERE, name + "_rays.npy"), rays)
    np.save(os.path.join(HERE, name + "_hits.npy"), hits)
    print("rays", name, n, "hit fraction %.3f" % (g >= 0).mean(), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="door", choices=sorted(WORKLOADS))
    ap.add_argument("--spp", type=int, default=8192)
    ap.add_argument("--threads", type=int, default=os.cpu_count())
    ap.add_argument("--rays", type=int, default=0)
    ap.add_argument("--no-crop", action="store_true")
    args = ap.parse_args()
    w = WORKLOADS[args.workload]
    if not oracle.reference_available():
        oracle.build(with_reference=True)
    with tempfile.TemporaryDirectory() as tmp:
        path = write_workload_scene(args.workload, tmp)
        if args.rays:
            make_rays(args.workload, path, args.rays, tmp)
        if args.no_crop:
            return
        x0, y0, x1, y1 = w["crop"]
        W, H = w["resolution"]
        reports = {}
        for tag, salt in (("a", 11), ("b", 22)):
            raw = os.path.join(tmp, "crop.f64")
            rep = oracle.run_reference(path, os.path.join(tmp, "crop.pfm"), spp=args.spp, salt=salt, crop=w["crop"],
                                       raw=raw, threads=args.threads)
            img = np.fromfile(raw, np.float64).reshape(H, W, 3)[y0:y1, x0:x1]
            np.save(os.path.join(HERE, "%s_crop_ref_%s.npy" % (args.workload, tag)), img.astype(np.float32))
            reports[tag] = rep
            print(tag, rep, flush=True)
    with open(os.path.join(HERE, "%s_crop_meta.json" % args.workload), "w") as f:
        json.dump({"crop": list(w["crop"]), "resolution": list(w["resolution"]),
                   "num_path_vertices": w["num_path_vertices"], "spp_each": args.spp, "salts": [11, 22],
                   "scene": w["scene"], "camera": w["camera"], "reports": reports}, f, indent=1)


if __name__ == "__main__":
    main()
