"""Environment-map input: .pfm / .hdr / .exr read as the reference reads them.

The golden arrays under tests/golden/images/ are the reference's own decodes of each file
(FimageIo::Load with stb_image for Radiance HDR and tinyexr for OpenEXR, through
``oracle/_ref/wurst_ref imgload``; tests/golden/make_image_golden.py). The loader must return
them bit for bit: the decodes are exact (RGBE = mantissa x power of two, half -> float), so any
difference is a decoding error. Malformed and unsupported files fail with a status, not a crash.
"""
import glob
import json
import os
import struct
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, golden_scene

IMAGES = sorted(glob.glob(os.path.join(GOLDEN, "images", "*.exr")) + glob.glob(os.path.join(GOLDEN, "images", "*.hdr")))


def golden_of(path):
    base, ext = os.path.splitext(path)
    return np.load(base + "_" + ext[1:] + ".npy")


@pytest.mark.parametrize("path", IMAGES, ids=[os.path.basename(p) for p in IMAGES])
def test_image_matches_reference_decoder(wr_lib, path):
    assert np.array_equal(wr_lib.read_image(path), golden_of(path))


def test_image_fixture_set_covers_the_variants():
    names = {os.path.basename(p) for p in IMAGES}
    # EXR: ZIP, ZIPS, RLE, none, raw-stored blocks, one channel, decreasing line order; HDR: RLE and plain
    assert len(names) >= 9


def test_image_live_against_reference_binary(wr_lib, oracle_lib, tmp_path):
    if not oracle_lib.reference_available():
        pytest.skip("reference harness not built here")
    import sys
    sys.path.insert(0, GOLDEN)
    from image_writers import write_exr, write_hdr
    rng = np.random.default_rng(17)
    img = rng.lognormal(0.0, 2.0, (13, 29, 3))
    cases = {"a.exr": lambda p: write_exr(p, {c: img[..., k] for k, c in enumerate("RGB")}, "zip", "half"),
             "b.exr": lambda p: write_exr(p, {c: img[..., k] for k, c in enumerate("BGR")}, "rle", "float", 1),
             "c.hdr": lambda p: write_hdr(p, img, rle=True)}
    for name, writer in cases.items():
        p = str(tmp_path / name)
        writer(p)
        out = str(tmp_path / "dec.bin")
        subprocess.run([oracle_lib.REF_BIN, "imgload", p, out], check=True, capture_output=True)
        raw = np.fromfile(out, np.uint8)
        w, h = np.frombuffer(raw[:8].tobytes(), np.int32)
        ref = np.frombuffer(raw[8:].tobytes(), np.float32).reshape(h, w, 3)
        assert np.array_equal(wr_lib.read_image(p), ref), name


def test_pfm_through_read_image(wr_lib, tmp_path):
    img = np.random.default_rng(3).uniform(0, 5, (6, 11, 3))
    p = str(tmp_path / "x.pfm")
    wr_lib.write_pfm(p, img)
    assert np.array_equal(wr_lib.read_image(p), img.astype(np.float32))


def _exr_bytes():
    return open(os.path.join(GOLDEN, "images", "zip_half_rgba.exr"), "rb").read()


def test_image_errors(wr_lib, tmp_path):
    def status(path):
        with pytest.raises(wr_lib.WurstError) as e:
            wr_lib.read_image(path)
        return e.value.status

    data = _exr_bytes()
    (tmp_path / "trunc.exr").write_bytes(data[: len(data) - 100])
    assert status(str(tmp_path / "trunc.exr")) == 3                  # WR_ERR_PARSE
    i = data.index(b"compression\0compression\0") + len(b"compression\0compression\0") + 4
    (tmp_path / "piz.exr").write_bytes(data[:i] + bytes([4]) + data[i + 1:])
    assert status(str(tmp_path / "piz.exr")) == 4                    # WR_ERR_UNSUPPORTED
    (tmp_path / "tiled.exr").write_bytes(data[:4] + struct.pack("<I", 2 | 0x200) + data[8:])
    assert status(str(tmp_path / "tiled.exr")) == 4
    (tmp_path / "bad.exr").write_bytes(b"not an exr file at all")
    assert status(str(tmp_path / "bad.exr")) == 3
    (tmp_path / "x.png").write_bytes(b"\x89PNG")
    assert status(str(tmp_path / "x.png")) == 4
    assert status(str(tmp_path / "missing.exr")) == 2                # WR_ERR_IO
    hdr = open(os.path.join(GOLDEN, "images", "rle.hdr"), "rb").read()
    (tmp_path / "t.hdr").write_bytes(hdr[: len(hdr) // 2])
    assert status(str(tmp_path / "t.hdr")) == 3


def test_scene_with_exr_envmap_loads(wr_lib, tmp_path):
    """A scene whose "envmap" is an .exr holding the env fixture's PFM values exactly is read
    with the same environment (inspect: host only)."""
    import shutil
    import sys
    sys.path.insert(0, GOLDEN)
    from image_writers import write_exr
    path, _ = golden_scene("env")
    d = os.path.dirname(path)
    for f in os.listdir(d):
        shutil.copy(os.path.join(d, f), tmp_path / f)
    scene = json.load(open(path))
    env = wr_lib.read_image(os.path.join(d, scene["envmap"]))
    write_exr(str(tmp_path / "sky.exr"), {c: env[..., k] for k, c in enumerate("RGB")}, "zip", "float")
    assert np.array_equal(wr_lib.read_image(str(tmp_path / "sky.exr")), env)
    scene["envmap"] = "sky.exr"
    p = tmp_path / os.path.basename(path)
    p.write_text(json.dumps(scene))
    assert wr_lib.inspect_scene(str(p))["has_envmap"] == 1
