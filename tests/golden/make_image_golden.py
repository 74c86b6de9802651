"""Writes the environment-map input fixtures under tests/golden/images/ and decodes each with the
reference's own image input (FimageIo::Load: stb_image for .hdr, tinyexr for .exr), through
``oracle/_ref/wurst_ref imgload``. For each image it saves <name>.npy: (H, W, 3) float32, row 0 =
top, as the reference reads it.

Usage: python tests/golden/make_image_golden.py   (needs ``make -C oracle ref``)
"""
from __future__ import annotations

import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, HERE)

import oracle  # noqa: E402
from image_writers import write_exr, write_hdr  # noqa: E402

OUT = os.path.join(HERE, "images")


def hdr_values(h, w, seed):
    """Sky-like radiance: a smooth gradient, a few very bright suns, some zeros and tiny values."""
    rng = np.random.default_rng(seed)
    y = np.linspace(0, 1, h)[:, None, None]
    x = np.linspace(0, 1, w)[None, :, None]
    img = 0.2 + 0.8 * y * np.array([0.5, 0.7, 1.0]) + 0.1 * x
    img = np.broadcast_to(img, (h, w, 3)).copy()
    for _ in range(3):
        cy, cx = rng.integers(0, h), rng.integers(0, w)
        img[cy, cx] = rng.uniform(200.0, 5000.0, 3)
    img[0, :3] = 0.0
    img[1, 1] = [3e-6, 6e-8, 1e-5]   # subnormal halves
    img *= rng.uniform(0.5, 1.5, (h, w, 1))
    return img


def cases():
    a = hdr_values(21, 37, 1)
    noise = np.random.default_rng(2).uniform(0, 10, (7, 19, 3))   # does not compress: blocks stored raw
    ch = lambda img, alpha=None: {**{c: img[..., k] for k, c in enumerate("RGB")}, **({"A": alpha} if alpha is not None else {})}
    return [
        ("zip_half_rgba.exr", lambda p: write_exr(p, ch(a, np.full(a.shape[:2], 0.5)), "zip", "half")),
        ("zips_float.exr", lambda p: write_exr(p, ch(a), "zips", "float")),
        ("rle_half.exr", lambda p: write_exr(p, ch(a), "rle", "half")),
        ("none_float_decreasing.exr", lambda p: write_exr(p, ch(a), "none", "float", line_order=1)),
        ("zip_float_raw_blocks.exr", lambda p: write_exr(p, ch(noise), "zip", "float")),
        ("grey_zip_half.exr", lambda p: write_exr(p, {"Y": a[..., 1]}, "zip", "half")),
        ("rle.hdr", lambda p: write_hdr(p, a, rle=True)),
        ("flat.hdr", lambda p: write_hdr(p, a, rle=False)),
        ("narrow.hdr", lambda p: write_hdr(p, a[:, :5], rle=False)),
    ]


def main():
    if not oracle.reference_available():
        oracle.build(with_reference=True)
    os.makedirs(OUT, exist_ok=True)
    for name, writer in cases():
        path = os.path.join(OUT, name)
        writer(path)
        tmp = os.path.join(OUT, "_decoded.bin")
        subprocess.run([oracle.REF_BIN, "imgload", path, tmp], check=True, capture_output=True)
        raw = np.fromfile(tmp, np.uint8)
        w, h = np.frombuffer(raw[:8].tobytes(), np.int32)
        img = np.frombuffer(raw[8:].tobytes(), np.float32).reshape(h, w, 3)
        np.save(os.path.join(OUT, os.path.splitext(name)[0] + "_" + os.path.splitext(name)[1][1:] + ".npy"), img)
        os.remove(tmp)
        print(name, img.shape, float(img.max()))


if __name__ == "__main__":
    main()
