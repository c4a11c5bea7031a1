// BMP, TGA, GIF, Radiance HDR, Photoshop PSD and Softimage PIC input for the command line, written
// from the formats' specifications (Microsoft's BITMAPINFOHEADER family; Truevision TGA 2.0;
// GIF89a; the Radiance RGBE picture format; Adobe's PSD file format; Softimage's PIC format).  Output is RGBA8 like the reference's
// stbi_load(..., 4) (src/main.cpp:37-57), including that loader's conversions where a format
// needs one (see each decoder).  Grey expands to R = G = B, a missing alpha becomes 255.
// Covered: BMP with the OS/2 core or Windows headers, 1/4/8-bit palettes, 16, 24 and 32-bit pixels
// (BI_RGB, or BI_BITFIELDS of up to 8 bits a channel), bottom-up or top-down rows; TGA types 1, 2, 3
// and their run-length forms 9, 10, 11 with 8, 15, 16, 24 or 32-bit pixels or 8/16-bit indices into
// 8, 15, 16, 24 or 32-bit colour maps; the first frame of a GIF; HDR with run-length or flat RGBE scanlines; RGB PSD, 8 or 16 bits, raw or
// PackBits; PIC with raw, pure or mixed run-length packets of 8-bit channels.  Other layouts are refused with a reason.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
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
uint32_t be16(const std::vector<unsigned char> &f, size_t o) {
    if (o + 2 > f.size()) throw std::runtime_error("truncated");
    return uint32_t(f[o]) << 8 | uint32_t(f[o + 1]);
}
uint32_t be32(const std::vector<unsigned char> &f, size_t o) {
    if (o + 4 > f.size()) throw std::runtime_error("truncated");
    return be16(f, o) << 16 | be16(f, o + 2);
}

void check_size(int64_t w, int64_t h) {
    if (w <= 0 || h <= 0 || w > 65536 || h > 65536 || w * h >= (int64_t(1) << 31))
        throw std::runtime_error("image size out of range");
}

// An n-bit channel value (1 <= n <= 8) widened to 8 bits by repeating its bit pattern (abc ->
// abcabcab): stb_image's expansion of BMP bit-field channels.
unsigned widen_bits(unsigned v, int n) {
    if (n <= 0) return 0;
    unsigned r = 0;
    int have = 0;
    while (have < 8) {
        r = r << n | v;
        have += n;
    }
    return (r >> (have - 8)) & 0xffu;
}

// One BMP bit-field channel: the mask's top bit lands on bit 7 of a byte, the byte keeps the mask's
// bit count (at most 8) from its top, and the value is widened to 8 bits (stb_image's reading; for a
// contiguous mask it is the field's value).
struct BmpField {
    uint32_t mask = 0;
    int high = 0, bits = 0;
    explicit BmpField(uint32_t m) : mask(m) {
        for (uint32_t t = m; t; t &= t - 1) bits++;
        for (int b = 31; b >= 0; b--)
            if (m >> b & 1u) {
                high = b;
                break;
            }
    }
    unsigned operator()(uint32_t px) const {
        uint32_t v = px & mask;
        v = high >= 7 ? v >> (high - 7) : v << (7 - high);
        return widen_bits((v & 0xffu) >> (8 - bits), bits);
    }
};

}  // namespace

// BMP as stb_image reads it: the OS/2 core header (12 bytes) and the 40, 56, 108 and 124-byte
// Windows headers; 1, 4 and 8-bit palettes (3-byte entries in the core header, 4-byte ones
// otherwise), 16-bit pixels (5-5-5 unless bit fields are given), 24-bit, 32-bit (B, G, R and an alpha
// byte that is used unless it is 0 everywhere, or bit fields); bit fields of at most 8 bits per
// channel, widened by repeating their bit pattern; no run-length or embedded JPEG/PNG compression.
// Rows are bottom-up unless the height is negative.  A palette index beyond the file's palette reads
// black (the reference's loader reads an unset table entry there).
InputImage decode_bmp(const std::vector<unsigned char> &f) {
    if (f.size() < 26 || f[0] != 'B' || f[1] != 'M') throw std::runtime_error("not a BMP file");
    const uint32_t data_off = le32(f, 10), hsz = le32(f, 14);
    if (hsz != 12 && hsz != 40 && hsz != 56 && hsz != 108 && hsz != 124)
        throw std::runtime_error("BMP header size " + std::to_string(hsz) + " is not supported");
    int64_t w, hs;
    uint32_t bpp, comp = 0;
    if (hsz == 12) {
        w = le16(f, 18);
        hs = le16(f, 20);
        if (le16(f, 22) != 1) throw std::runtime_error("bad BMP");
        bpp = le16(f, 24);
    } else {
        w = int32_t(le32(f, 18));
        hs = int32_t(le32(f, 22));
        if (le16(f, 26) != 1) throw std::runtime_error("bad BMP");
        bpp = le16(f, 28);
        comp = le32(f, 30);
    }
    if (comp == 1 || comp == 2) throw std::runtime_error("run-length BMP is not supported");
    if (comp > 3) throw std::runtime_error("compressed BMP is not supported");
    if (comp == 3 && bpp != 16 && bpp != 32) throw std::runtime_error("bad BMP");
    if (bpp != 1 && bpp != 4 && bpp != 8 && bpp != 16 && bpp != 24 && bpp != 32)
        throw std::runtime_error("BMP bit depth " + std::to_string(bpp) + " is not supported");
    const bool top_down = hs < 0;
    const int64_t h = top_down ? -hs : hs;
    check_size(w, h);
    // channel masks R, G, B, A; BI_RGB 32-bit pixels carry an alpha byte that counts only if some
    // pixel's alpha is not 0
    uint32_t m[4] = {0, 0, 0, 0};
    bool alpha_if_any = false;
    auto default_masks = [&]() {
        if (bpp == 16) {
            m[0] = 31u << 10, m[1] = 31u << 5, m[2] = 31u;
        } else if (bpp == 32) {
            m[0] = 0xffu << 16, m[1] = 0xffu << 8, m[2] = 0xffu, m[3] = 0xffu << 24;
            alpha_if_any = true;
        } else {
            m[0] = m[1] = m[2] = m[3] = 0;
        }
    };
    if (hsz == 40 || hsz == 56) {
        if (bpp == 16 || bpp == 32) {
            if (comp == 0) {
                default_masks();
            } else {  // R, G, B masks after the header
                for (int i = 0; i < 3; i++) m[i] = le32(f, 14 + hsz + 4 * i);
                if (m[0] == m[1] && m[1] == m[2]) throw std::runtime_error("bad BMP");
            }
        }
    } else if (hsz >= 108) {  // R, G, B, A masks in the header; BI_RGB replaces them by the defaults
        for (int i = 0; i < 4; i++) m[i] = le32(f, 54 + 4 * i);
        if (comp != 3) default_masks();
    }
    InputImage img;
    img.width = int(w);
    img.height = int(h);
    img.data.resize(size_t(w) * h * 4);
    const size_t row_bytes = (size_t(w) * bpp + 7) / 8, stride = (row_bytes + 3) & ~size_t(3);
    if (size_t(data_off) + stride * size_t(h) > f.size()) throw std::runtime_error("truncated");
    auto row_of = [&](int64_t y) { return f.data() + data_off + stride * size_t(top_down ? y : h - 1 - y); };
    if (bpp <= 8) {
        const size_t esz = hsz == 12 ? 3 : 4, pal_off = 14 + hsz;
        const size_t nent = data_off > pal_off ? (data_off - pal_off) / esz : 0;
        if (nent == 0 || nent > 256) throw std::runtime_error("bad BMP palette");
        for (int64_t y = 0; y < h; y++) {
            const unsigned char *row = row_of(y);
            unsigned char *o = img.data.data() + size_t(y) * w * 4;
            for (int64_t x = 0; x < w; x++, o += 4) {
                unsigned idx;
                if (bpp == 8) idx = row[x];
                else if (bpp == 4) idx = x & 1 ? row[x >> 1] & 15u : row[x >> 1] >> 4;
                else idx = row[x >> 3] >> (7 - (x & 7)) & 1u;
                if (idx < nent) {
                    const unsigned char *e = &f[pal_off + idx * esz];  // B, G, R
                    o[0] = e[2], o[1] = e[1], o[2] = e[0];
                } else {
                    o[0] = o[1] = o[2] = 0;
                }
                o[3] = 255;
            }
        }
        return img;
    }
    const bool plain32 = bpp == 32 && m[0] == 0xff0000u && m[1] == 0xff00u && m[2] == 0xffu && m[3] == 0xff000000u;
    if (bpp != 24 && !plain32) {
        if (!m[0] || !m[1] || !m[2]) throw std::runtime_error("bad BMP channel masks");
        for (uint32_t mk : m) {
            int bits = 0;
            for (uint32_t t = mk; t; t &= t - 1) bits++;
            if (bits > 8) throw std::runtime_error("BMP channel masks wider than 8 bits are not supported");
        }
    }
    const BmpField fr(m[0]), fg(m[1]), fb(m[2]), fa(m[3]);
    unsigned alpha_or = 0;
    for (int64_t y = 0; y < h; y++) {
        const unsigned char *row = row_of(y);
        unsigned char *o = img.data.data() + size_t(y) * w * 4;
        for (int64_t x = 0; x < w; x++, o += 4) {
            if (bpp == 24) {
                o[0] = row[3 * x + 2], o[1] = row[3 * x + 1], o[2] = row[3 * x], o[3] = 255;
                continue;
            }
            const unsigned char *p = row + (bpp == 16 ? 2 : 4) * x;
            const uint32_t v = bpp == 16 ? uint32_t(p[0]) | uint32_t(p[1]) << 8
                                         : uint32_t(p[0]) | uint32_t(p[1]) << 8 | uint32_t(p[2]) << 16 | uint32_t(p[3]) << 24;
            o[0] = (unsigned char)fr(v), o[1] = (unsigned char)fg(v), o[2] = (unsigned char)fb(v);
            o[3] = m[3] ? (unsigned char)fa(v) : 255;
            alpha_or |= o[3];
        }
    }
    if (alpha_if_any && alpha_or == 0)
        for (size_t i = 3; i < img.data.size(); i += 4) img.data[i] = 255;
    return img;
}

// TGA as stb_image reads it: types 1, 2, 3 and their run-length forms 9, 10, 11.  True colour of 15
// or 16 bits (5-5-5, each channel widened as v * 255 / 31, no alpha), 24 or 32 bits (B, G, R, A);
// grey of 8 bits, or 16 (grey and alpha); colour-mapped pixels of 8 or 16-bit indices into a map of
// 8-bit grey, 15/16, 24 or 32-bit entries, read after skipping as many bytes as the map's first-entry
// field holds, an index beyond the map taking entry 0.  Only the top-left-origin bit of the
// descriptor counts (rows are never mirrored left to right).
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
    auto depth_ok = [](unsigned b) { return b == 8 || b == 15 || b == 16 || b == 24 || b == 32; };
    if (mapped ? (cmap_type != 1 || (bpp != 8 && bpp != 16) || !depth_ok(cmap_bits) || cmap_len == 0)
               : grey ? (bpp != 8 && bpp != 16) : !depth_ok(bpp))
        throw std::runtime_error("TGA pixel depth " + std::to_string(bpp) + " is not supported");
    // one pixel (or map entry) of `bits` bits to RGBA; `as_grey`: 8 bits grey, 16 bits grey + alpha
    auto to_rgba = [](const unsigned char *p, unsigned bits, bool as_grey, unsigned char *o) {
        if (bits == 8 || (as_grey && bits == 16)) {
            o[0] = o[1] = o[2] = p[0];
            o[3] = bits == 16 ? p[1] : 255;
        } else if (bits == 15 || bits == 16) {
            const unsigned v = unsigned(p[0]) | unsigned(p[1]) << 8;
            o[0] = (unsigned char)(((v >> 10) & 31u) * 255 / 31);
            o[1] = (unsigned char)(((v >> 5) & 31u) * 255 / 31);
            o[2] = (unsigned char)((v & 31u) * 255 / 31);
            o[3] = 255;
        } else {
            o[0] = p[2], o[1] = p[1], o[2] = p[0], o[3] = bits == 32 ? p[3] : 255;
        }
    };
    size_t pos = 18 + id_len;
    std::vector<unsigned char> cmap;  // RGBA per entry
    if (mapped) {
        pos += cmap_first;
        const unsigned eb = (cmap_bits + 7) / 8;
        if (pos + size_t(cmap_len) * eb > f.size()) throw std::runtime_error("truncated");
        cmap.resize(size_t(cmap_len) * 4);
        for (uint32_t i = 0; i < cmap_len; i++) to_rgba(&f[pos + size_t(i) * eb], cmap_bits, false, &cmap[4 * i]);
        pos += size_t(cmap_len) * eb;
    } else if (cmap_type == 1) {  // a colour map on an unmapped image is skipped
        pos += size_t(cmap_len) * ((cmap_bits + 7) / 8);
    }
    const unsigned pb = (bpp + 7) / 8;
    // decode to RGBA in file order (rows bottom-up unless descriptor bit 5 marks a top-left origin)
    std::vector<unsigned char> px(size_t(w) * h * 4);
    auto put = [&](size_t i, const unsigned char *p) {
        unsigned char *o = &px[4 * i];
        if (mapped) {
            uint32_t idx = pb == 1 ? p[0] : uint32_t(p[0]) | uint32_t(p[1]) << 8;
            if (idx >= cmap_len) idx = 0;
            std::memcpy(o, &cmap[4 * size_t(idx)], 4);
        } else {
            to_rgba(p, bpp, grey, o);
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
        const unsigned head = f[pos++];
        const unsigned count = unsigned(std::min<size_t>((head & 0x7f) + 1, n - i));  // a run ends with the image
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
    const bool top_left = desc & 0x20;
    for (int32_t y = 0; y < h; y++)
        std::memcpy(&img.data[size_t(y) * w * 4], &px[size_t(top_left ? y : h - 1 - y) * w * 4], size_t(w) * 4);
    return img;
}

// First frame of a GIF, as stbi_load composes it: the canvas starts transparent black, the frame's
// pixels are drawn unless their palette entry is the transparent one, and when the screen's
// background index is not 0, every canvas pixel the frame's raster did not reach takes the global
// palette's background entry with alpha 255 -- copied in the loader's internal palette order
// (B, G, R), which the output keeps.  The LZW stream must start with a clear code.
InputImage decode_gif(const std::vector<unsigned char> &f) {
    if (f.size() < 13 || std::memcmp(f.data(), "GIF8", 4) != 0 || (f[4] != '7' && f[4] != '9') || f[5] != 'a')
        throw std::runtime_error("not a GIF file");
    const int w = int(le16(f, 6)), h = int(le16(f, 8));
    const unsigned flags = f[10], bgindex = f[11];
    check_size(w, h);
    size_t pos = 13;
    auto byte = [&]() -> unsigned {
        if (pos >= f.size()) throw std::runtime_error("truncated");
        return f[pos++];
    };
    unsigned char gpal[256][4] = {}, lpal[256][4] = {};  // r, g, b, a
    auto read_palette = [&](unsigned char (*pal)[4], int n, int transparent) {
        for (int i = 0; i < n; i++) {
            pal[i][0] = byte(), pal[i][1] = byte(), pal[i][2] = byte();
            pal[i][3] = i == transparent ? 0 : 255;
        }
    };
    if (flags & 0x80) read_palette(gpal, 2 << (flags & 7), -1);
    int transparent = -1;
    unsigned eflags = 0;
    for (;;) {
        const unsigned tag = byte();
        if (tag == 0x21) {  // extension
            const unsigned ext = byte();
            if (ext == 0xF9) {  // graphic control: disposal, delay, transparent index
                const unsigned len = byte();
                if (len == 4) {
                    eflags = byte();
                    byte(), byte();
                    const unsigned t = byte();
                    if (transparent >= 0) gpal[transparent][3] = 255;
                    transparent = (eflags & 1) ? int(t) : -1;
                    if (transparent >= 0) gpal[transparent][3] = 0;
                } else {
                    pos += len;
                }
            }
            for (unsigned len; (len = byte()) != 0;) pos += len;  // remaining sub-blocks
            continue;
        }
        if (tag == 0x3B) throw std::runtime_error("GIF has no image");
        if (tag != 0x2C) throw std::runtime_error("corrupt GIF");
        // image descriptor
        const int x0 = int(le16(f, pos)), y0 = int(le16(f, pos + 2));
        const int fw = int(le16(f, pos + 4)), fh = int(le16(f, pos + 6));
        pos += 8;
        if (x0 + fw > w || y0 + fh > h) throw std::runtime_error("GIF frame outside the screen");
        const unsigned lflags = byte();
        const unsigned char (*pal)[4] = gpal;
        if (lflags & 0x80) {
            read_palette(lpal, 2 << (lflags & 7), (eflags & 1) ? transparent : -1);
            pal = lpal;
        } else if (!(flags & 0x80)) {
            throw std::runtime_error("GIF without colour table");
        }
        std::vector<unsigned char> out(size_t(w) * h * 4, 0);
        std::vector<unsigned char> reached(size_t(w) * h, 0);
        // raster order, with the 4 passes of an interlaced frame
        const bool interlaced = lflags & 0x40;
        int pass = 0, cx = 0, cy = 0, step = interlaced ? 8 : 1;
        auto put = [&](unsigned idx) {
            if (cy >= fh) return;
            const size_t pi = size_t(y0 + cy) * w + (x0 + cx);
            reached[pi] = 1;
            if (pal[idx][3] > 128)
                for (int c = 0; c < 4; c++) out[4 * pi + c] = pal[idx][c];
            if (++cx >= fw) {
                cx = 0;
                cy += step;
                while (interlaced && cy >= fh && pass < 3) {
                    static const int start[4] = {0, 4, 2, 1}, steps[4] = {8, 8, 4, 2};
                    pass++;
                    cy = start[pass];
                    step = steps[pass];
                }
            }
        };
        if (fw == 0) cy = fh;
        // LZW over the data sub-blocks
        const unsigned min_size = byte();
        if (min_size > 12) throw std::runtime_error("corrupt GIF");
        const int clear = 1 << min_size;
        std::vector<int> prefix(4096, -1);
        std::vector<unsigned char> first(4096), suffix(4096), stack(4097);
        for (int c = 0; c < clear; c++) first[c] = suffix[c] = (unsigned char)c;
        int size = int(min_size) + 1, avail = clear + 2, old = -1;
        bool started = false;
        uint32_t bits = 0;
        int nbits = 0;
        size_t block = 0;  // bytes left in the current sub-block
        for (;;) {
            if (nbits < size) {
                if (block == 0) {
                    block = byte();
                    if (block == 0) break;  // data ended without an end code
                }
                block--;
                bits |= uint32_t(byte()) << nbits;
                nbits += 8;
                continue;
            }
            const int code = int(bits & ((1u << size) - 1));
            bits >>= size;
            nbits -= size;
            if (code == clear) {
                size = int(min_size) + 1;
                avail = clear + 2;
                old = -1;
                started = true;
                continue;
            }
            if (code == clear + 1) {  // end code: skip what is left of the data
                pos += block;
                for (unsigned len; (len = byte()) != 0;) pos += len;
                break;
            }
            if (code > avail) throw std::runtime_error("corrupt GIF raster");
            if (!started) throw std::runtime_error("GIF raster without a clear code");
            if (old >= 0 && avail < 4096) {  // a full table stays as it is until the next clear code
                prefix[avail] = old;
                first[avail] = first[old];
                suffix[avail] = code == avail ? first[old] : first[code];
                avail++;
            } else if (old < 0 && code == avail) {
                throw std::runtime_error("corrupt GIF raster");
            }
            int n = 0;
            for (int c = code; c >= 0; c = prefix[c]) stack[n++] = suffix[c];
            while (n) put(stack[--n]);
            if ((avail & ((1 << size) - 1)) == 0 && avail <= 0x0FFF) size++;
            old = code;
        }
        if (bgindex > 0)
            for (size_t pi = 0; pi < size_t(w) * h; pi++)
                if (!reached[pi]) {
                    out[4 * pi + 0] = gpal[bgindex][2];
                    out[4 * pi + 1] = gpal[bgindex][1];
                    out[4 * pi + 2] = gpal[bgindex][0];
                    out[4 * pi + 3] = 255;
                }
        InputImage img;
        img.width = w;
        img.height = h;
        img.data = std::move(out);
        return img;
    }
}

// Radiance HDR converted to 8 bits as stbi_load does: each colour channel is m * 2^(e - 136) (0 when
// e = 0), then (uint8) clamp(float(pow(v, 1 / 2.2f)) * 255 + 0.5f, 0, 255) with pow in double;
// alpha is 255.  Header: "#?RADIANCE" or "#?RGBE", a FORMAT=32-bit_rle_rgbe line, a blank line,
// then "-Y h +X w".  Scanlines of 8 to 32767 pixels may be run-length coded (2, 2, width, then
// each component's runs); a scanline that does not start that way switches the loader to flat
// RGBE quadruples from the first pixel on, the quadruple just read being pixel 0.
InputImage decode_hdr(const std::vector<unsigned char> &f) {
    size_t pos = 0;
    auto line = [&]() {
        std::string t;
        while (pos < f.size() && f[pos] != '\n' && t.size() < 1023) t += char(f[pos++]);
        while (pos < f.size() && f[pos] != '\n') pos++;  // an over-long line is cut, as the loader does
        if (pos < f.size()) pos++;
        return t;
    };
    const std::string magic = line();
    if (magic != "#?RADIANCE" && magic != "#?RGBE") throw std::runtime_error("not an HDR file");
    bool valid = false;
    for (std::string t; !(t = line()).empty();)
        if (t == "FORMAT=32-bit_rle_rgbe") valid = true;
    if (!valid) throw std::runtime_error("unsupported HDR format");
    const std::string res = line();
    if (res.compare(0, 3, "-Y ") != 0) throw std::runtime_error("unsupported HDR data layout");
    char *end = nullptr;
    const long h = std::strtol(res.c_str() + 3, &end, 10);
    while (*end == ' ') end++;
    if (std::strncmp(end, "+X ", 3) != 0) throw std::runtime_error("unsupported HDR data layout");
    const long w = std::strtol(end + 3, nullptr, 10);
    check_size(w, h);
    const size_t n = size_t(w) * h;
    std::vector<unsigned char> rgbe(n * 4);
    auto byte = [&]() -> unsigned {
        if (pos >= f.size()) throw std::runtime_error("truncated");
        return f[pos++];
    };
    auto flat_from = [&](size_t first) {
        for (size_t i = first; i < n; i++)
            for (int c = 0; c < 4; c++) rgbe[4 * i + c] = (unsigned char)byte();
    };
    if (w < 8 || w >= 32768) {
        flat_from(0);
    } else {
        std::vector<unsigned char> sl(size_t(w) * 4);
        for (long y = 0; y < h; y++) {
            const unsigned c1 = byte(), c2 = byte(), len = byte();
            if (c1 != 2 || c2 != 2 || (len & 0x80)) {
                rgbe[0] = (unsigned char)c1, rgbe[1] = (unsigned char)c2, rgbe[2] = (unsigned char)len;
                rgbe[3] = (unsigned char)byte();
                flat_from(1);
                break;
            }
            if (long((len << 8) | byte()) != w) throw std::runtime_error("corrupt HDR scanline");
            for (int k = 0; k < 4; k++)
                for (long i = 0; i < w;) {
                    unsigned count = byte();
                    if (count > 128) {
                        const unsigned char v = (unsigned char)byte();
                        count -= 128;
                        if (long(count) > w - i) throw std::runtime_error("corrupt HDR run");
                        while (count--) sl[4 * i++ + k] = v;
                    } else {
                        if (count == 0 || long(count) > w - i) throw std::runtime_error("corrupt HDR run");
                        while (count--) sl[4 * i++ + k] = (unsigned char)byte();
                    }
                }
            std::memcpy(&rgbe[size_t(y) * w * 4], sl.data(), sl.size());
        }
    }
    InputImage img;
    img.width = int(w);
    img.height = int(h);
    img.data.resize(n * 4);
    const float gamma = 1.0f / 2.2f;
    for (size_t i = 0; i < n; i++) {
        const unsigned char *q = &rgbe[4 * i];
        const float scale = q[3] ? std::ldexp(1.0f, int(q[3]) - 136) : 0.f;
        for (int c = 0; c < 3; c++) {
            const float v = q[3] ? float(q[c]) * scale : 0.f;
            float z = float(std::pow(double(v), double(gamma))) * 255 + 0.5f;
            z = z < 0 ? 0 : (z > 255 ? 255 : z);
            img.data[4 * i + c] = (unsigned char)int(z);
        }
        img.data[4 * i + 3] = 255;
    }
    return img;
}

// RGB Photoshop files as stbi_load reads them: the composite image after the header sections, 8-bit
// samples or the high byte of 16-bit ones; with PackBits compression every channel is one run of
// w * h bytes (the loader does this whatever the depth); missing channels are 0 (alpha 255); with 4
// or more channels, colours are un-premultiplied from the white matte in float, v * (1 / a) +
// 255 (1 - 1 / a) with a = alpha / 255, truncated to an integer and kept modulo 256 as the loader's
// float-to-byte conversion does on x86-64.
InputImage decode_psd(const std::vector<unsigned char> &f) {
    if (f.size() < 26 || be32(f, 0) != 0x38425053u) throw std::runtime_error("not a PSD file");
    if (be16(f, 4) != 1) throw std::runtime_error("unsupported PSD version");
    const int channels = int(be16(f, 12));
    if (channels > 16) throw std::runtime_error("unsupported PSD channel count");
    const int64_t h = be32(f, 14), w = be32(f, 18);
    const unsigned depth = be16(f, 22);
    if (depth != 8 && depth != 16) throw std::runtime_error("PSD bit depth is not 8 or 16");
    if (be16(f, 24) != 3) throw std::runtime_error("PSD is not in RGB colour mode");
    check_size(w, h);
    size_t pos = 26;
    for (int section = 0; section < 3; section++) pos += 4 + size_t(be32(f, pos));  // mode data, resources, layers
    const unsigned compression = be16(f, pos);
    pos += 2;
    if (compression > 1) throw std::runtime_error("unknown PSD compression");
    const size_t n = size_t(w) * size_t(h);
    auto byte = [&]() -> unsigned {
        if (pos >= f.size()) throw std::runtime_error("truncated");
        return f[pos++];
    };
    InputImage img;
    img.width = int(w);
    img.height = int(h);
    img.data.assign(n * 4, 0);
    unsigned char *out = img.data.data();
    if (compression) pos += size_t(h) * channels * 2;  // per-row byte counts, not needed
    for (int c = 0; c < 4; c++) {
        unsigned char *p = out + c;
        if (c >= channels) {
            for (size_t i = 0; i < n; i++, p += 4) *p = c == 3 ? 255 : 0;
        } else if (compression) {
            for (size_t i = 0; i < n;) {
                const unsigned len = byte();
                if (len == 128) continue;
                if (len < 128) {
                    if (len + 1 > n - i) throw std::runtime_error("corrupt PSD run");
                    for (unsigned k = 0; k <= len; k++, i++, p += 4) *p = (unsigned char)byte();
                } else {
                    const unsigned cnt = 257 - len;
                    if (cnt > n - i) throw std::runtime_error("corrupt PSD run");
                    const unsigned char v = (unsigned char)byte();
                    for (unsigned k = 0; k < cnt; k++, i++, p += 4) *p = v;
                }
            }
        } else if (depth == 16) {
            for (size_t i = 0; i < n; i++, p += 4) {
                const unsigned hi = byte();
                byte();
                *p = (unsigned char)hi;
            }
        } else {
            for (size_t i = 0; i < n; i++, p += 4) *p = (unsigned char)byte();
        }
    }
    if (channels >= 4)
        for (size_t i = 0; i < n; i++) {
            unsigned char *px = out + 4 * i;
            if (px[3] != 0 && px[3] != 255) {
                const float a = px[3] / 255.0f, ra = 1.0f / a, inv_a = 255.0f * (1 - ra);
                for (int c = 0; c < 3; c++) px[c] = (unsigned char)int(px[c] * ra + inv_a);
            }
        }
    return img;
}

// Softimage PIC (as stbi_load reads it): a 104-byte header (magic 0x5380F634, "PICT" at byte 88,
// big-endian width and height at 92 and 94), then a chain of channel packets (chained flag, bits
// per channel -- 8 only --, coding 0 raw / 1 pure run-length / 2 mixed run-length, and a channel
// mask R 0x80, G 0x40, B 0x20, A 0x10).  Every row holds each packet's data for that row in chain
// order; channels no packet carries stay 255.
InputImage decode_pic(const std::vector<unsigned char> &f) {
    if (f.size() < 104 || be32(f, 0) != 0x5380F634u || std::memcmp(&f[88], "PICT", 4) != 0)
        throw std::runtime_error("not a PIC file");
    const int w = int(be16(f, 92)), h = int(be16(f, 94));
    check_size(w, h);
    size_t pos = 104;
    auto byte = [&]() -> unsigned {
        if (pos >= f.size()) throw std::runtime_error("truncated");
        return f[pos++];
    };
    struct Packet {
        unsigned type, mask;
    };
    std::vector<Packet> packets;
    for (bool chained = true; chained;) {
        if (packets.size() == 10) throw std::runtime_error("too many PIC packets");
        chained = byte() != 0;
        const unsigned size = byte(), type = byte(), mask = byte();
        if (size != 8) throw std::runtime_error("PIC packet is not 8 bits per channel");
        if (type > 2) throw std::runtime_error("unknown PIC packet coding");
        packets.push_back({type, mask});
    }
    InputImage img;
    img.width = w;
    img.height = h;
    img.data.assign(size_t(w) * h * 4, 255);
    auto read_value = [&](unsigned mask, unsigned char *dst) {
        for (int c = 0; c < 4; c++)
            if (mask & (0x80u >> c)) dst[c] = (unsigned char)byte();
    };
    auto copy_value = [](unsigned mask, unsigned char *dst, const unsigned char *src) {
        for (int c = 0; c < 4; c++)
            if (mask & (0x80u >> c)) dst[c] = src[c];
    };
    for (int y = 0; y < h; y++)
        for (const Packet &pk : packets) {
            unsigned char *dst = &img.data[size_t(y) * w * 4];
            int left = w;
            if (pk.type == 0) {
                for (int x = 0; x < w; x++, dst += 4) read_value(pk.mask, dst);
                continue;
            }
            while (left > 0) {
                unsigned char v[4] = {};
                int count = int(byte());
                if (pk.type == 1) {  // a count and one value per run; a run past the row is cut
                    count = std::min(count, left);
                    read_value(pk.mask, v);
                    for (int i = 0; i < count; i++, dst += 4) copy_value(pk.mask, dst, v);
                } else if (count >= 128) {  // mixed: a repeated run (128: a 16-bit count follows)
                    if (count == 128) {
                        count = int(be16(f, pos));
                        pos += 2;
                    } else {
                        count -= 127;
                    }
                    if (count > left) throw std::runtime_error("PIC run past the row");
                    read_value(pk.mask, v);
                    for (int i = 0; i < count; i++, dst += 4) copy_value(pk.mask, dst, v);
                } else {  // mixed: count + 1 literal values
                    if (++count > left) throw std::runtime_error("PIC run past the row");
                    for (int i = 0; i < count; i++, dst += 4) read_value(pk.mask, dst);
                }
                left -= count;
            }
        }
    return img;
}

}  // namespace IQM
