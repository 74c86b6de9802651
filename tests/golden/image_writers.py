"""Small writers of OpenEXR and Radiance HDR files for the image-input tests.

They produce the variants the loader must read (written from the published file formats, not
from any library): EXR one-part scanline images with HALF / FLOAT channels, NONE / RLE / ZIPS /
ZIP compression (a block that does not shrink is stored raw, as the format allows), increasing
or decreasing line order; HDR files with run-length or plain RGBE scanlines.
"""
from __future__ import annotations

import struct
import zlib

import numpy as np

COMPRESSION = {"none": 0, "rle": 1, "zips": 2, "zip": 3}
LINES = {"none": 1, "rle": 1, "zips": 1, "zip": 16}


def _attr(name, typ, payload):
    return name.encode() + b"\0" + typ.encode() + b"\0" + struct.pack("<i", len(payload)) + payload


def _predict(raw: bytes) -> bytes:
    """Interleave (even bytes, then odd bytes) and replace each byte by its difference + 128."""
    a = np.frombuffer(raw, np.uint8)
    t = np.concatenate([a[0::2], a[1::2]]).astype(np.int32)
    d = t.copy()
    d[1:] = (t[1:] - t[:-1] + 128) & 0xFF
    return d.astype(np.uint8).tobytes()


def _rle(data: bytes) -> bytes:
    out = bytearray()
    i, n = 0, len(data)
    while i < n:
        run = 1
        while i + run < n and run < 128 and data[i + run] == data[i]:
            run += 1
        if run >= 3:
            out += struct.pack("<b", run - 1) + bytes([data[i]])
            i += run
            continue
        j = i
        while j < n and j - i < 127:
            if j + 2 < n and data[j] == data[j + 1] == data[j + 2]:
                break
            j += 1
        out += struct.pack("<b", -(j - i)) + data[i:j]
        i = j
    return bytes(out)


def write_exr(path, channels: dict, compression="zip", pixel_type="half", line_order=0):
    """channels: name -> (H, W) float array; written in name order as the format requires."""
    names = sorted(channels)
    h, w = next(iter(channels.values())).shape
    pt = {"half": 1, "float": 2}[pixel_type]
    dtype = np.float16 if pt == 1 else np.float32
    chl = b"".join(n.encode() + b"\0" + struct.pack("<iB3xii", pt, 0, 1, 1) for n in names) + b"\0"
    header = b"".join([
        _attr("channels", "chlist", chl),
        _attr("compression", "compression", bytes([COMPRESSION[compression]])),
        _attr("dataWindow", "box2i", struct.pack("<4i", 0, 0, w - 1, h - 1)),
        _attr("displayWindow", "box2i", struct.pack("<4i", 0, 0, w - 1, h - 1)),
        _attr("lineOrder", "lineOrder", bytes([line_order])),
        _attr("pixelAspectRatio", "float", struct.pack("<f", 1.0)),
        _attr("screenWindowCenter", "v2f", struct.pack("<2f", 0.0, 0.0)),
        _attr("screenWindowWidth", "float", struct.pack("<f", 1.0)),
    ]) + b"\0"
    lines = LINES[compression]
    blocks = []
    for y0 in range(0, h, lines):
        raw = b"".join(np.ascontiguousarray(channels[n][y].astype(dtype)).tobytes()
                       for y in range(y0, min(h, y0 + lines)) for n in names)
        if compression == "none":
            data = raw
        elif compression == "rle":
            data = _rle(_predict(raw))
        else:
            data = zlib.compress(_predict(raw))
        if compression != "none" and len(data) >= len(raw):
            data = raw
        blocks.append((y0, data))
    if line_order == 1:
        blocks = blocks[::-1]
    start = 8 + len(header) + 8 * len(blocks)
    offsets, body, pos = [], bytearray(), start
    for y0, data in blocks:
        offsets.append(pos)
        chunk = struct.pack("<ii", y0, len(data)) + data
        body += chunk
        pos += len(chunk)
    # the offset table is indexed by block number (y order), whatever the line order of the data
    order = sorted(range(len(blocks)), key=lambda k: blocks[k][0])
    table = b"".join(struct.pack("<Q", offsets[k]) for k in order)
    with open(path, "wb") as f:
        f.write(struct.pack("<II", 20000630, 2) + header + table + bytes(body))


def _rgbe(rgb):
    out = np.zeros(rgb.shape[:-1] + (4,), np.uint8)
    v = rgb.max(axis=-1)
    ok = v >= 1e-32
    m, e = np.frexp(v[ok])
    scale = m * 256.0 / v[ok]
    out[ok, 0:3] = np.floor(rgb[ok] * scale[:, None]).astype(np.uint8)
    out[ok, 3] = (e + 128).astype(np.uint8)
    return out


def write_hdr(path, rgb, rle=True):
    h, w, _ = rgb.shape
    px = _rgbe(np.asarray(rgb, np.float64))
    with open(path, "wb") as f:
        f.write(b"#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n-Y %d +X %d\n" % (h, w))
        for y in range(h):
            if not rle:
                f.write(px[y].tobytes())
                continue
            f.write(bytes([2, 2, w >> 8, w & 0xFF]))
            for k in range(4):
                comp = px[y, :, k].tobytes()
                i = 0
                while i < w:
                    run = 1
                    while i + run < w and run < 127 and comp[i + run] == comp[i]:
                        run += 1
                    if run >= 3:
                        f.write(bytes([128 + run, comp[i]]))
                        i += run
                        continue
                    j = i
                    while j < w and j - i < 128:
                        if j + 2 < w and comp[j] == comp[j + 1] == comp[j + 2]:
                            break
                        j += 1
                    f.write(bytes([j - i]) + comp[i:j])
                    i = j
