"""Generates the FP64 reference crop of the door-gap room (the guided-vs-plain workload).

The scene (closed 6 x 3 x 6 m room, 1 x 1 emitter behind a partition with a 0.2 m
door gap, 300 seeded Phong / Oren-Nayar boxes, about 200k triangles, 1024 x 1024,
10 path vertices) is written by wurstrenderer_b200.scenes.door_room_spec(seed=1004);
it is regenerated deterministically wherever it is needed, so only the reference
image of a 128 x 128 crop is stored:

  door_crop_ref_a.npy / door_crop_ref_b.npy   two independent renders of the crop by the
                                              reference's own PathNeeRenderer code
                                              (oracle/_ref), 8192 spp each, salts 11 / 22
  door_crop_meta.json                         crop rectangle, spp, salts, scene parameters

Usage: python tests/golden/make_door_golden.py [--spp 8192] [--threads N]
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from wurstrenderer_b200 import scenes  # noqa: E402

CROP = (448, 448, 576, 576)   # x0, y0, x1, y1 (whole 32 x 32 tiles)
RESOLUTION = (1024, 1024)
NUM_VERTICES = 10


def write_door_scene(out_dir, resolution=RESOLUTION, spp=64):
    cam = dict(scenes.DOOR_ROOM_CAMERA, resolution=list(resolution))
    return scenes.write_spec(out_dir, "door", scenes.door_room_spec(seed=1004), cam, resolution, spp, NUM_VERTICES)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--spp", type=int, default=8192)
    ap.add_argument("--threads", type=int, default=os.cpu_count())
    args = ap.parse_args()
    if not oracle.reference_available():
        oracle.build(with_reference=True)
    with tempfile.TemporaryDirectory() as tmp:
        path = write_door_scene(tmp)
        x0, y0, x1, y1 = CROP
        reports = {}
        for tag, salt in (("a", 11), ("b", 22)):
            raw = os.path.join(tmp, "crop.f64")
            rep = oracle.run_reference(path, os.path.join(tmp, "crop.pfm"), spp=args.spp, salt=salt, crop=CROP,
                                       raw=raw, threads=args.threads)
            img = np.fromfile(raw, np.float64).reshape(RESOLUTION[1], RESOLUTION[0], 3)[y0:y1, x0:x1]
            np.save(os.path.join(HERE, "door_crop_ref_%s.npy" % tag), img.astype(np.float32))
            reports[tag] = rep
            print(tag, rep, flush=True)
    with open(os.path.join(HERE, "door_crop_meta.json"), "w") as f:
        json.dump({"crop": list(CROP), "resolution": list(RESOLUTION), "num_path_vertices": NUM_VERTICES,
                   "spp_each": args.spp, "salts": [11, 22], "scene": "scenes.door_room_spec(seed=1004)",
                   "camera": scenes.DOOR_ROOM_CAMERA, "reports": reports}, f, indent=1)


if __name__ == "__main__":
    main()
