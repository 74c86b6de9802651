"""Generates FP64 reference crops for the full-size guided-vs-plain workloads.

The scenes are regenerated deterministically by wurstrenderer_b200.scenes wherever they are
needed (they are large), so only the reference image of a crop is stored:

  door: the door-gap room (config 4; closed 6 x 3 x 6 m room, 1 x 1 emitter behind a partition
        with a 0.2 m door gap, 300 seeded boxes, 197,782 triangles), 1024 x 1024, 10 vertices,
        crop 128 x 128 at (448, 448)
  c5:   the full combination (config 5; 2048^2 fBm floor + 20000 icospheres + 16 area lights +
        a 2048 x 1024 FP32 sky, 9,980,450 triangles), 3840 x 2160, 26 vertices,
        crop 128 x 64 at (1856, 1056)

For each, <name>_crop_ref_a.npy / _b.npy are two independent renders of the crop by the
reference's own PathNeeRenderer code (oracle/_ref) with salts 11 / 22, `--spp` each (16384 spp
in total by default), and <name>_crop_meta.json records the crop, spp and scene parameters.

Usage: python tests/golden/make_crop_golden.py --workload door|c5 [--spp 8192] [--threads N]
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

WORKLOADS = {
    "door": {"scene": "scenes.door_room_spec(seed=1004)", "camera": scenes.DOOR_ROOM_CAMERA},
    "c5": {"scene": "scenes.write_full_combination(seed=1005)", "camera": scenes.FULL_COMBINATION_CAMERA},
}
for _name, _w in WORKLOADS.items():
    _w.update(scenes.GUIDED_WORKLOADS[_name])


def write_workload_scene(name, out_dir, spp=64):
    return scenes.write_guided_workload(name, out_dir, spp)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="door", choices=sorted(WORKLOADS))
    ap.add_argument("--spp", type=int, default=8192)
    ap.add_argument("--threads", type=int, default=os.cpu_count())
    args = ap.parse_args()
    w = WORKLOADS[args.workload]
    if not oracle.reference_available():
        oracle.build(with_reference=True)
    with tempfile.TemporaryDirectory() as tmp:
        path = write_workload_scene(args.workload, tmp)
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
