// Float image input for environment maps: the formats FimageIo::LoadAny of the reference reads
// as floats (src/common/floatimage.h:238-345,379-396), dispatched on the extension as there
// (".pfm", ".hdr", ".exr"; the extension is compared as written).
//
//   * PFM: read_pfm in wr_scene_io.cpp (floatimage.h:238-277).
//   * Radiance HDR (the reference decodes it with stb_image's stbi_loadf, floatimage.h:283-305):
//     header lines up to an empty line ("#?RADIANCE" or "#?RGBE" first, FORMAT=32-bit_rle_rgbe),
//     the resolution line "-Y h +X w", then h scanlines of RGBE pixels, each either flat or in
//     the run-length form of the format (2, 2, width as 2 bytes, then the four components one
//     after another, each as runs (count > 128: count - 128 copies of one byte) and literals).
//     A pixel (r, g, b, e) decodes to (r, g, b) * 2^(e - 136) (zero when e = 0), exact in float.
//   * OpenEXR (the reference decodes it with tinyexr's LoadEXR, floatimage.h:308-345): one-part
//     scanline images with HALF or FLOAT channels, uncompressed or with RLE, ZIPS or ZIP
//     compression; R, G, B are taken by name (A is not used), a single-channel image is grey.
//     ZIP / ZIPS blocks are zlib streams of 16 / 1 scanlines; RLE and ZIP data are stored with
//     a byte predictor (each byte is the difference to the previous one, plus 128) over two
//     interleaved halves (even bytes, then odd bytes). A block whose stored size equals its raw
//     size is raw. As the reference's decoder does, an image whose line order is not increasing
//     comes out upside down. Tiled, multi-part, deep, PIZ / PXR24 / B44 / DWA images and UINT
//     channels are rejected with WR_ERR_UNSUPPORTED.
// Output: width x height x 3 floats, row 0 = top (the layout of every image here).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include <zlib.h>

#include "wr_host.h"

namespace wr {
namespace {

std::string slurp_binary(const std::string &path, const char *what) {
    std::ifstream f(path, std::ios::binary);
    if (!f) throw Error(WR_ERR_IO, std::string("cannot find specified ") + what + " file " + path);
    std::stringstream ss;
    ss << f.rdbuf();
    return ss.str();
}

std::string extension_of(const std::string &path) {
    const size_t slash = path.find_last_of('/');
    const size_t dot = path.find_last_of('.');
    if (dot == std::string::npos || (slash != std::string::npos && dot < slash)) return "";
    return path.substr(dot);
}

// ------------------------------------------------------------ Radiance HDR ----
void rgbe_to_float(const unsigned char *p, float *out) {
    if (p[3] != 0) {
        const float f = std::ldexp(1.0f, int(p[3]) - 136);
        out[0] = float(p[0]) * f;
        out[1] = float(p[1]) * f;
        out[2] = float(p[2]) * f;
    } else {
        out[0] = out[1] = out[2] = 0.f;
    }
}

std::vector<float> read_hdr(const std::string &path, int *width, int *height) {
    const std::string data = slurp_binary(path, "HDR");
    const unsigned char *p = reinterpret_cast<const unsigned char *>(data.data());
    const unsigned char *end = p + data.size();
    auto line = [&]() {
        std::string l;
        while (p < end && *p != '\n') l.push_back(char(*p++));
        if (p < end) ++p;
        return l;
    };
    const std::string magic = line();
    if (magic != "#?RADIANCE" && magic != "#?RGBE") throw Error(WR_ERR_PARSE, "not a Radiance HDR file: " + path);
    bool rgbe = false;
    while (true) {
        if (p >= end) throw Error(WR_ERR_PARSE, "truncated HDR header: " + path);
        const std::string l = line();
        if (l.empty()) break;
        if (l == "FORMAT=32-bit_rle_rgbe") rgbe = true;
    }
    if (!rgbe) throw Error(WR_ERR_UNSUPPORTED, "HDR file is not in the 32-bit_rle_rgbe format: " + path);
    const std::string res = line();
    int h = 0, w = 0;
    char ys[4] = {0}, xs[4] = {0};
    if (sscanf(res.c_str(), "%3s %d %3s %d", ys, &h, xs, &w) != 4 || std::string(ys) != "-Y" || std::string(xs) != "+X")
        throw Error(WR_ERR_UNSUPPORTED, "HDR orientation other than -Y h +X w: " + path);
    if (w <= 0 || h <= 0 || w > (1 << 24) / std::max(h, 1)) throw Error(WR_ERR_PARSE, "bad HDR size: " + path);
    *width = w;
    *height = h;
    std::vector<float> out(size_t(w) * h * 3);
    auto need = [&](size_t n) {
        if (size_t(end - p) < n) throw Error(WR_ERR_PARSE, "truncated HDR data: " + path);
    };
    std::vector<unsigned char> scan(size_t(w) * 4);
    bool all_flat = w < 8 || w >= 32768;
    for (int y = 0; y < h; ++y) {
        float *row = &out[size_t(y) * w * 3];
        bool flat = all_flat;
        if (!flat) {
            need(4);
            if (p[0] != 2 || p[1] != 2 || (p[2] & 0x80)) {
                // a first scanline that is not run-length encoded makes the whole image plain
                // RGBE; stb_image restarts at row 0 when a later one is not, so such files are refused
                if (y > 0) throw Error(WR_ERR_UNSUPPORTED, "HDR file mixes plain and run-length scanlines: " + path);
                all_flat = flat = true;
            }
        }
        if (flat) {   // plain RGBE pixels
            need(size_t(w) * 4);
            for (int x = 0; x < w; ++x, p += 4) rgbe_to_float(p, row + 3 * x);
            continue;
        }
        if ((int(p[2]) << 8 | p[3]) != w) throw Error(WR_ERR_PARSE, "HDR scanline width mismatch: " + path);
        p += 4;
        for (int k = 0; k < 4; ++k) {
            int x = 0;
            while (x < w) {
                need(1);
                int count = *p++;
                if (count > 128) {
                    count -= 128;
                    need(1);
                    const unsigned char v = *p++;
                    if (x + count > w) throw Error(WR_ERR_PARSE, "bad HDR run length: " + path);
                    for (int i = 0; i < count; ++i) scan[size_t(x++) * 4 + k] = v;
                } else {
                    if (count == 0 || x + count > w) throw Error(WR_ERR_PARSE, "bad HDR literal length: " + path);
                    need(size_t(count));
                    for (int i = 0; i < count; ++i) scan[size_t(x++) * 4 + k] = *p++;
                }
            }
        }
        for (int x = 0; x < w; ++x) rgbe_to_float(&scan[size_t(x) * 4], row + 3 * x);
    }
    return out;
}

// ----------------------------------------------------------------- OpenEXR ----
float half_to_float(uint16_t h) {
    const uint32_t sign = uint32_t(h >> 15) << 31;
    const uint32_t e = (h >> 10) & 0x1f, m = h & 0x3ff;
    uint32_t bits;
    if (e == 0) {
        if (m == 0) {
            bits = sign;
        } else {   // subnormal half: normalise
            int shift = 0;
            uint32_t mm = m;
            while (!(mm & 0x400)) { mm <<= 1; ++shift; }
            bits = sign | uint32_t(127 - 15 - shift + 1) << 23 | (mm & 0x3ff) << 13;
        }
    } else if (e == 31) {
        bits = sign | 0x7f800000u | m << 13;
    } else {
        bits = sign | (e - 15 + 127) << 23 | m << 13;
    }
    float f;
    memcpy(&f, &bits, 4);
    return f;
}

struct ExrChannel {
    std::string name;
    int type;   // 0 UINT, 1 HALF, 2 FLOAT
};

template <typename T> T get_le(const unsigned char *p) {
    T v;
    memcpy(&v, p, sizeof(T));
    return v;
}

// undo the predictor and the two-half interleave of RLE / ZIP blocks
void exr_unpredict(std::vector<unsigned char> &t) {
    for (size_t i = 1; i < t.size(); ++i) t[i] = static_cast<unsigned char>(int(t[i - 1]) + int(t[i]) - 128);
    std::vector<unsigned char> o(t.size());
    const size_t half = (t.size() + 1) / 2;
    for (size_t i = 0; i < t.size(); ++i) o[i] = (i & 1) ? t[half + i / 2] : t[i / 2];
    t.swap(o);
}

std::vector<float> read_exr(const std::string &path, int *width, int *height) {
    const std::string data = slurp_binary(path, "EXR");
    const unsigned char *b = reinterpret_cast<const unsigned char *>(data.data());
    const size_t n = data.size();
    auto need = [&](size_t off, size_t len) {
        if (off > n || len > n - off) throw Error(WR_ERR_PARSE, "truncated EXR file: " + path);
    };
    need(0, 8);
    if (get_le<uint32_t>(b) != 20000630u) throw Error(WR_ERR_PARSE, "not an OpenEXR file: " + path);
    const uint32_t version = get_le<uint32_t>(b + 4);
    if ((version & 0xff) != 2) throw Error(WR_ERR_UNSUPPORTED, "OpenEXR version other than 2: " + path);
    if (version & (0x200u | 0x800u | 0x1000u))
        throw Error(WR_ERR_UNSUPPORTED, "tiled, deep or multi-part OpenEXR files are not supported: " + path);
    size_t off = 8;
    std::vector<ExrChannel> chans;
    int compression = -1, line_order = 0;
    int32_t dw[4] = {0, 0, -1, -1};
    bool have_dw = false;
    auto cstring = [&]() {
        std::string s;
        while (true) {
            need(off, 1);
            const char c = char(b[off++]);
            if (!c) break;
            s.push_back(c);
        }
        return s;
    };
    while (true) {
        const std::string name = cstring();
        if (name.empty()) break;
        const std::string type = cstring();
        need(off, 4);
        const uint32_t size = get_le<uint32_t>(b + off);
        off += 4;
        need(off, size);
        const unsigned char *v = b + off;
        if (name == "channels" && type == "chlist") {
            size_t q = 0;
            while (q < size && v[q]) {
                std::string cn;
                while (q < size && v[q]) cn.push_back(char(v[q++]));
                ++q;
                if (q + 16 > size) throw Error(WR_ERR_PARSE, "bad EXR channel list: " + path);
                const int pt = int(get_le<int32_t>(v + q));
                const int xs = get_le<int32_t>(v + q + 8), ys = get_le<int32_t>(v + q + 12);
                if (xs != 1 || ys != 1) throw Error(WR_ERR_UNSUPPORTED, "subsampled EXR channels: " + path);
                chans.push_back(ExrChannel{cn, pt});
                q += 16;
            }
        } else if (name == "compression" && type == "compression" && size >= 1) {
            compression = v[0];
        } else if (name == "dataWindow" && type == "box2i" && size >= 16) {
            for (int k = 0; k < 4; ++k) dw[k] = get_le<int32_t>(v + 4 * k);
            have_dw = true;
        } else if (name == "lineOrder" && type == "lineOrder" && size >= 1) {
            line_order = v[0];
        }
        off += size;
    }
    if (chans.empty() || !have_dw || compression < 0) throw Error(WR_ERR_PARSE, "incomplete EXR header: " + path);
    if (compression > 3)
        throw Error(WR_ERR_UNSUPPORTED, "EXR compression other than none, RLE, ZIPS or ZIP: " + path);
    // Blocks carry their own y. The reference's decoder (tinyexr, as vendored with it) stores a
    // file whose line order is not increasing upside down -- scanline y goes to row h - 1 - y --
    // so that is done here too.
    const bool flip = line_order != 0;
    const int64_t w64 = int64_t(dw[2]) - dw[0] + 1, h64 = int64_t(dw[3]) - dw[1] + 1;
    if (w64 <= 0 || h64 <= 0 || w64 * h64 > (int64_t(1) << 28)) throw Error(WR_ERR_PARSE, "bad EXR data window: " + path);
    const int w = int(w64), h = int(h64);
    size_t pixel_bytes = 0;
    for (const ExrChannel &c : chans) {
        if (c.type != 1 && c.type != 2) throw Error(WR_ERR_UNSUPPORTED, "EXR channel type other than HALF or FLOAT: " + path);
        pixel_bytes += c.type == 1 ? 2 : 4;
    }
    int ir = -1, ig = -1, ib = -1;
    for (size_t c = 0; c < chans.size(); ++c) {
        if (chans[c].name == "R") ir = int(c);
        else if (chans[c].name == "G") ig = int(c);
        else if (chans[c].name == "B") ib = int(c);
    }
    if (chans.size() == 1) ir = ig = ib = 0;
    else if (ir < 0 || ig < 0 || ib < 0) throw Error(WR_ERR_PARSE, "EXR file without R, G and B channels: " + path);
    const int lines = compression == 3 ? 16 : 1;
    const int nblocks = (h + lines - 1) / lines;
    need(off, size_t(nblocks) * 8);
    std::vector<uint64_t> offsets(static_cast<size_t>(nblocks));
    for (int i = 0; i < nblocks; ++i) offsets[size_t(i)] = get_le<uint64_t>(b + off + 8 * size_t(i));
    *width = w;
    *height = h;
    std::vector<float> out(size_t(w) * h * 3, 0.f);
    std::vector<bool> seen(static_cast<size_t>(h), false);
    const size_t line_bytes = size_t(w) * pixel_bytes;
    std::vector<unsigned char> raw;
    for (int bi = 0; bi < nblocks; ++bi) {
        const uint64_t bo = offsets[size_t(bi)];
        need(size_t(bo), 8);
        const int32_t y0 = get_le<int32_t>(b + bo) - dw[1];
        const uint32_t stored = get_le<uint32_t>(b + bo + 4);
        need(size_t(bo) + 8, stored);
        if (y0 < 0 || y0 >= h || y0 % lines) throw Error(WR_ERR_PARSE, "bad EXR block position: " + path);
        const int nl = std::min(lines, h - y0);
        const size_t expect = line_bytes * size_t(nl);
        const unsigned char *src = b + bo + 8;
        if (compression == 0 || stored == expect) {
            if (stored != expect) throw Error(WR_ERR_PARSE, "bad EXR block size: " + path);
            raw.assign(src, src + expect);
        } else if (compression == 1) {   // RLE
            raw.clear();
            size_t q = 0;
            while (q < stored) {
                const int count = int(static_cast<signed char>(src[q++]));
                if (count < 0) {
                    if (q + size_t(-count) > stored) throw Error(WR_ERR_PARSE, "bad EXR RLE data: " + path);
                    raw.insert(raw.end(), src + q, src + q + size_t(-count));
                    q += size_t(-count);
                } else {
                    if (q >= stored) throw Error(WR_ERR_PARSE, "bad EXR RLE data: " + path);
                    raw.insert(raw.end(), size_t(count) + 1, src[q++]);
                }
                if (raw.size() > expect) throw Error(WR_ERR_PARSE, "bad EXR RLE data: " + path);
            }
            if (raw.size() != expect) throw Error(WR_ERR_PARSE, "bad EXR RLE block size: " + path);
            exr_unpredict(raw);
        } else {   // ZIPS / ZIP
            raw.assign(expect, 0);
            uLongf dlen = uLongf(expect);
            if (uncompress(raw.data(), &dlen, src, uLong(stored)) != Z_OK || dlen != expect)
                throw Error(WR_ERR_PARSE, "bad EXR ZIP block: " + path);
            exr_unpredict(raw);
        }
        for (int l = 0; l < nl; ++l) {
            const int y = flip ? h - 1 - (y0 + l) : y0 + l;
            seen[size_t(y)] = true;
            const unsigned char *line = raw.data() + size_t(l) * line_bytes;
            size_t co = 0;
            for (size_t c = 0; c < chans.size(); ++c) {
                const int sz = chans[c].type == 1 ? 2 : 4;
                for (int k = 0; k < 3; ++k) {
                    if (int(c) != (k == 0 ? ir : k == 1 ? ig : ib)) continue;
                    for (int x = 0; x < w; ++x) {
                        const unsigned char *v = line + co + size_t(x) * sz;
                        out[(size_t(y) * w + x) * 3 + k] =
                            sz == 2 ? half_to_float(get_le<uint16_t>(v)) : get_le<float>(v);
                    }
                }
                co += size_t(w) * sz;
            }
        }
    }
    for (int y = 0; y < h; ++y)
        if (!seen[size_t(y)]) throw Error(WR_ERR_PARSE, "EXR file misses scanlines: " + path);
    return out;
}

}  // namespace

std::vector<float> read_image(const std::string &path, int *width, int *height) {
    const std::string ext = extension_of(path);
    if (ext == ".pfm") return read_pfm(path, width, height);
    if (ext == ".hdr") return read_hdr(path, width, height);
    if (ext == ".exr") return read_exr(path, width, height);
    if (ext.empty()) throw Error(WR_ERR_UNSUPPORTED, "unknown file type: " + path);
    throw Error(WR_ERR_UNSUPPORTED, "unsupported image format '" + ext + "' (envmaps: .pfm, .hdr, .exr): " + path);
}

}  // namespace wr
