// BMP and TGA input for the command line, written from the formats' specifications (Microsoft's
// BITMAPINFOHEADER family; Truevision TGA 2.0).  Output is RGBA8 like the reference's
// stbi_load(..., 4) (src/main.cpp:37-57): grey expands to R = G = B, a missing alpha becomes 255.
// The metrics ignore alpha, so only the colour bytes matter; for the lossless layouts read here
// they are the file's bytes.  Covered: BMP with 8-bit palettes, 24-bit and 32-bit pixels
// (BI_RGB, or BI_BITFIELDS with byte-aligned 8-bit masks), bottom-up or top-down rows; TGA types
// 1, 2, 3 and their run-length forms 9, 10, 11 with 8-, 24- or 32-bit pixels and 24- or 32-bit
// colour maps, either origin.  Other layouts are refused with a reason.
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "png_io.h"

namespace IQM {
namespace {

uint32_t le16(const std::vector<unsigned char> &f, size_t o) {
    if (o + 2 > f.size()) throw std::runtime_error("truncated");
    return uint32_t(f[o]) | uint32_t(f[o + 1]) << 8;
}
uint32_t le32(const std::vector<unsigned char> &f, size_t o) {
    if (o + 4 > f.size()) throw std::runtime_error("truncated");
    return le16(f, o) | le16(f, o + 2) << 16;
}

// Position (0-7, 8-bit lanes) of an 8-bit channel mask, -1 for an absent channel.
int mask_shift(uint32_t m) {
    if (m == 0) return -1;
    for (int s = 0; s < 32; s += 8)
        if (m == (0xffu << s)) return s;
    throw std::runtime_error("BMP channel masks other than whole bytes are not supported");
}

void check_size(int64_t w, int64_t h) {
    if (w <= 0 || h <= 0 || w > 65536 || h > 65536 || w * h >= (int64_t(1) << 31))
        throw std::runtime_error("image size out of range");
}

}  // namespace

InputImage decode_bmp(const std::vector<unsigned char> &f) {
    if (f.size() < 26 || f[0] != 'B' || f[1] != 'M') throw std::runtime_error("not a BMP file");
    const uint32_t data_off = le32(f, 10), hdr = le32(f, 14);
    if (hdr < 40) throw std::runtime_error("BMP core headers are not supported");
    const int32_t w = int32_t(le32(f, 18)), hs = int32_t(le32(f, 22));
    const uint32_t bpp = le16(f, 28), comp = le32(f, 30);
    const bool top_down = hs < 0;
    const int64_t h = top_down ? -int64_t(hs) : hs;
    check_size(w, h);
    uint32_t masks[4] = {0x00ff0000u, 0x0000ff00u, 0x000000ffu, 0u};  // R, G, B, A of BI_RGB 32-bit
    if (comp == 3) {
        if (bpp != 32) throw std::runtime_error("BMP bit fields other than 32-bit are not supported");
        const size_t mo = hdr >= 52 ? 54 : 14 + hdr;  // masks inside the header, or right after it
        for (int i = 0; i < (hdr >= 56 ? 4 : 3); i++) masks[i] = le32(f, mo + 4 * i);
    } else if (comp != 0) {
        throw std::runtime_error("compressed BMP is not supported");
    }
    if (bpp != 8 && bpp != 24 && bpp != 32) throw std::runtime_error("BMP bit depth " + std::to_string(bpp) + " is not supported");
    std::vector<unsigned char> pal;
    if (bpp == 8) {
        uint32_t ncol = le32(f, 46);
        if (ncol == 0 || ncol > 256) ncol = 256;
        const size_t po = 14 + hdr;
        if (po + 4 * size_t(ncol) > f.size()) throw std::runtime_error("truncated");
        pal.assign(f.begin() + po, f.begin() + po + 4 * ncol);  // B, G, R, reserved
    }
    const int sh[4] = {mask_shift(masks[0]), mask_shift(masks[1]), mask_shift(masks[2]), mask_shift(masks[3])};
    const size_t stride = (size_t(w) * bpp / 8 + 3) & ~size_t(3);
    if (data_off + stride * size_t(h) > f.size()) throw std::runtime_error("truncated");
    InputImage img;
    img.width = w;
    img.height = int(h);
    img.data.resize(size_t(w) * h * 4);
    for (int64_t y = 0; y < h; y++) {
        const unsigned char *row = f.data() + data_off + stride * size_t(top_down ? y : h - 1 - y);
        unsigned char *o = img.data.data() + size_t(y) * w * 4;
        for (int32_t x = 0; x < w; x++, o += 4) {
            if (bpp == 8) {
                const size_t i = size_t(row[x]) * 4;
                if (i + 3 > pal.size()) throw std::runtime_error("BMP palette index out of range");
                o[0] = pal[i + 2], o[1] = pal[i + 1], o[2] = pal[i], o[3] = 255;
            } else if (bpp == 24) {
                o[0] = row[3 * x + 2], o[1] = row[3 * x + 1], o[2] = row[3 * x], o[3] = 255;
            } else {
                const uint32_t v = uint32_t(row[4 * x]) | uint32_t(row[4 * x + 1]) << 8 | uint32_t(row[4 * x + 2]) << 16 |
                                   uint32_t(row[4 * x + 3]) << 24;
                for (int c = 0; c < 3; c++) o[c] = sh[c] < 0 ? 0 : (v >> sh[c]) & 0xffu;
                o[3] = sh[3] < 0 ? 255 : (v >> sh[3]) & 0xffu;
            }
        }
    }
    return img;
}

InputImage decode_tga(const std::vector<unsigned char> &f) {
    if (f.size() < 18) throw std::runtime_error("not a TGA file");
    const unsigned id_len = f[0], cmap_type = f[1], type = f[2];
    const uint32_t cmap_first = le16(f, 3), cmap_len = le16(f, 5), cmap_bits = f[7];
    const int32_t w = int32_t(le16(f, 12)), h = int32_t(le16(f, 14));
    const unsigned bpp = f[16], desc = f[17];
    const bool rle = type >= 9;
    const unsigned base = rle ? type - 8 : type;
    if (base < 1 || base > 3 || (type > 3 && type < 9) || type > 11) throw std::runtime_error("not a TGA file");
    check_size(w, h);
    const bool mapped = base == 1, grey = base == 3;
    if (mapped ? (bpp != 8 || cmap_type != 1 || (cmap_bits != 24 && cmap_bits != 32)) :
                 grey ? bpp != 8 : (bpp != 24 && bpp != 32))
        throw std::runtime_error("TGA pixel depth " + std::to_string(bpp) + " is not supported");
    size_t pos = 18 + id_len;
    std::vector<unsigned char> cmap;
    if (cmap_type == 1) {
        const size_t bytes = size_t(cmap_len) * ((cmap_bits + 7) / 8);
        if (pos + bytes > f.size()) throw std::runtime_error("truncated");
        if (mapped) cmap.assign(f.begin() + pos, f.begin() + pos + bytes);
        pos += bytes;
    }
    const unsigned pb = bpp / 8, cb = cmap_bits / 8;
    // decode to RGBA in file order (rows bottom-up unless descriptor bit 5 marks a top-left origin)
    std::vector<unsigned char> px(size_t(w) * h * 4);
    auto put = [&](size_t i, const unsigned char *p) {
        unsigned char *o = &px[4 * i];
        if (mapped) {
            const uint32_t idx = p[0];
            if (idx < cmap_first || idx - cmap_first >= cmap_len) throw std::runtime_error("TGA colour index out of range");
            const unsigned char *e = &cmap[size_t(idx - cmap_first) * cb];
            o[0] = e[2], o[1] = e[1], o[2] = e[0], o[3] = cb == 4 ? e[3] : 255;
        } else if (grey) {
            o[0] = o[1] = o[2] = p[0], o[3] = 255;
        } else {
            o[0] = p[2], o[1] = p[1], o[2] = p[0], o[3] = pb == 4 ? p[3] : 255;
        }
    };
    const size_t n = size_t(w) * h;
    for (size_t i = 0; i < n;) {
        if (!rle) {
            if (pos + pb > f.size()) throw std::runtime_error("truncated");
            put(i++, &f[pos]);
            pos += pb;
            continue;
        }
        if (pos >= f.size()) throw std::runtime_error("truncated");
        const unsigned head = f[pos++], count = (head & 0x7f) + 1;
        if (i + count > n) throw std::runtime_error("TGA run past the image");
        if (head & 0x80) {  // one pixel repeated
            if (pos + pb > f.size()) throw std::runtime_error("truncated");
            for (unsigned k = 0; k < count; k++) put(i++, &f[pos]);
            pos += pb;
        } else {            // count literal pixels
            if (pos + size_t(count) * pb > f.size()) throw std::runtime_error("truncated");
            for (unsigned k = 0; k < count; k++, pos += pb) put(i++, &f[pos]);
        }
    }
    InputImage img;
    img.width = w;
    img.height = h;
    img.data.resize(n * 4);
    const bool top_left = desc & 0x20, right_left = desc & 0x10;
    for (int32_t y = 0; y < h; y++)
        for (int32_t x = 0; x < w; x++) {
            const size_t src = size_t(top_left ? y : h - 1 - y) * w + (right_left ? w - 1 - x : x);
            for (int c = 0; c < 4; c++) img.data[(size_t(y) * w + x) * 4 + c] = px[src * 4 + c];
        }
    return img;
}

}  // namespace IQM
