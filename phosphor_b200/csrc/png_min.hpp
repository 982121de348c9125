// png_min.hpp — PNG decoder for the glTF loader's textures: non-interlaced images of bit depth 8 or
// 16 in grey, grey+alpha, RGB, RGBA or palette colour, decompressed with zlib and unfiltered
// (None, Sub, Up, Average, Paeth), returned as 8-bit RGB the way the reference loads textures
// (3 channels requested: grey replicated, alpha dropped, 16-bit samples keep their high byte).
// Returns false, with a reason, for anything else (interlaced images, bit depths below 8) and for
// truncated or corrupt data; chunk CRCs are not checked.
#pragma once

#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include <zlib.h>

namespace phx {

inline bool png_decode_rgb8(const uint8_t *data, size_t size, std::vector<uint8_t> &rgb, uint32_t *w, uint32_t *h,
                            std::string &why) {
    static const uint8_t sig[8] = {0x89, 'P', 'N', 'G', '\r', '\n', 0x1A, '\n'};
    if (size < 8 || std::memcmp(data, sig, 8) != 0) {
        why = "not a PNG";
        return false;
    }
    auto be32 = [](const uint8_t *p) { return (uint32_t)p[0] << 24 | (uint32_t)p[1] << 16 | (uint32_t)p[2] << 8 | p[3]; };
    uint32_t width = 0, height = 0;
    int depth = 0, ctype = -1, interlace = 0;
    std::vector<uint8_t> idat, palette;
    size_t pos = 8;
    bool ended = false;
    while (pos + 8 <= size && !ended) {
        const uint32_t len = be32(data + pos);
        const uint8_t *type = data + pos + 4;
        if ((uint64_t)pos + 12 + len > size) {
            why = "truncated chunk";
            return false;
        }
        const uint8_t *body = data + pos + 8;
        if (!std::memcmp(type, "IHDR", 4) && len >= 13) {
            width = be32(body);
            height = be32(body + 4);
            depth = body[8];
            ctype = body[9];
            interlace = body[12];
        } else if (!std::memcmp(type, "PLTE", 4)) {
            palette.assign(body, body + len);
        } else if (!std::memcmp(type, "IDAT", 4)) {
            idat.insert(idat.end(), body, body + len);
        } else if (!std::memcmp(type, "IEND", 4)) {
            ended = true;
        }
        pos += 12 + (size_t)len;
    }
    if (!width || !height || width > (1u << 15) || height > (1u << 15)) {
        why = "bad image size";
        return false;
    }
    if (interlace != 0 || (depth != 8 && depth != 16)) {
        why = "interlaced or below 8 bits per sample (unsupported)";
        return false;
    }
    int chans;
    switch (ctype) {
    case 0: chans = 1; break;
    case 2: chans = 3; break;
    case 3: chans = 1; break;
    case 4: chans = 2; break;
    case 6: chans = 4; break;
    default: why = "unknown colour type"; return false;
    }
    if (ctype == 3 && depth != 8) {
        why = "16-bit palette";
        return false;
    }
    const size_t bpp = (size_t)chans * (depth / 8), stride = (size_t)width * bpp;
    std::vector<uint8_t> raw((stride + 1) * height);
    uLongf out_len = (uLongf)raw.size();
    if (uncompress(raw.data(), &out_len, idat.data(), (uLong)idat.size()) != Z_OK || out_len != raw.size()) {
        why = "zlib data does not inflate to the image size";
        return false;
    }
    std::vector<uint8_t> img(stride * height);
    for (uint32_t y = 0; y < height; y++) {
        const uint8_t f = raw[y * (stride + 1)];
        const uint8_t *src = raw.data() + y * (stride + 1) + 1;
        uint8_t *dst = img.data() + y * stride;
        const uint8_t *up = y ? img.data() + (y - 1) * stride : nullptr;
        for (size_t x = 0; x < stride; x++) {
            const int a = x >= bpp ? dst[x - bpp] : 0, b = up ? up[x] : 0, c = (up && x >= bpp) ? up[x - bpp] : 0;
            int v = src[x];
            switch (f) {
            case 0: break;
            case 1: v += a; break;
            case 2: v += b; break;
            case 3: v += (a + b) / 2; break;
            case 4: {
                const int p = a + b - c, pa = p > a ? p - a : a - p, pb = p > b ? p - b : b - p,
                          pc = p > c ? p - c : c - p;
                v += (pa <= pb && pa <= pc) ? a : (pb <= pc ? b : c);
                break;
            }
            default: why = "bad filter"; return false;
            }
            dst[x] = (uint8_t)v;
        }
    }
    rgb.resize((size_t)width * height * 3);
    const size_t step = depth / 8;
    for (size_t i = 0; i < (size_t)width * height; i++) {
        const uint8_t *px = img.data() + i * bpp;
        uint8_t r, g, b;
        if (ctype == 3) {
            const size_t k = (size_t)px[0] * 3;
            if (k + 3 > palette.size()) {
                why = "palette index out of range";
                return false;
            }
            r = palette[k];
            g = palette[k + 1];
            b = palette[k + 2];
        } else if (chans <= 2) {
            r = g = b = px[0];
        } else {
            r = px[0];
            g = px[step];
            b = px[2 * step];
        }
        rgb[3 * i] = r;
        rgb[3 * i + 1] = g;
        rgb[3 * i + 2] = b;
    }
    *w = width;
    *h = height;
    return true;
}

} // namespace phx
