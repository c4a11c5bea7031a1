// BMP, TGA, GIF, Radiance HDR, Photoshop PSD and Softimage PIC input for the command line, written
// from the formats' specifications (Microsoft's BITMAPINFOHEADER family; Truevision TGA 2.0;
// GIF89a; the Radiance RGBE picture format; Adobe's PSD file format; Softimage's PIC format).  Output is RGBA8 like the reference's
// stbi_load(..., 4) (src/main.cpp:37-57), including that loader's conversions where a format
// needs one (see each decoder).  Grey expands to R = G = B, a missing alpha becomes 255.
// Covered: BMP with 8-bit palettes, 24-bit and 32-bit pixels (BI_RGB, or BI_BITFIELDS with
// byte-aligned 8-bit masks), bottom-up or top-down rows; TGA types 1, 2, 3 and their run-length
// forms 9, 10, 11 with 8-, 24- or 32-bit pixels and 24- or 32-bit colour maps, either origin; the
// first frame of a GIF; HDR with run-length or flat RGBE scanlines; RGB PSD, 8 or 16 bits, raw or
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
