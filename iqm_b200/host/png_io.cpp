// PNG decoding per the PNG specification (ISO/IEC 15948): chunk stream, zlib-compressed IDAT,
// per-scanline filters (None, Sub, Up, Average, Paeth), Adam7 interlacing, bit depths 1-16.
#include "png_io.h"

#include <zlib.h>

#include <cstdint>
#include <cstring>
#include <fstream>
#include <iterator>
#include <stdexcept>

namespace {

uint32_t be32(const unsigned char *p) { return (uint32_t(p[0]) << 24) | (uint32_t(p[1]) << 16) | (uint32_t(p[2]) << 8) | p[3]; }

void put32(std::vector<unsigned char> &o, uint32_t v) {
    o.push_back((v >> 24) & 255);
    o.push_back((v >> 16) & 255);
    o.push_back((v >> 8) & 255);
    o.push_back(v & 255);
}

int paeth(int a, int b, int c) {
    const int p = a + b - c, pa = std::abs(p - a), pb = std::abs(p - b), pc = std::abs(p - c);
    if (pa <= pb && pa <= pc) return a;
    return pb <= pc ? b : c;
}

// Reverses the scanline filters of one (sub)image in place: `rows` x (1 + rowbytes) bytes.
void unfilter(unsigned char *data, int rows, size_t rowbytes, int bpp) {
    unsigned char *prev = nullptr;
    for (int y = 0; y < rows; y++) {
        unsigned char *line = data + size_t(y) * (rowbytes + 1);
        const int f = line[0];
        unsigned char *cur = line + 1;
        for (size_t i = 0; i < rowbytes; i++) {
            const int a = i >= size_t(bpp) ? cur[i - bpp] : 0;
            const int b = prev ? prev[i] : 0;
            const int c = (prev && i >= size_t(bpp)) ? prev[i - bpp] : 0;
            int v = cur[i];
            switch (f) {
                case 0: break;
                case 1: v += a; break;
                case 2: v += b; break;
                case 3: v += (a + b) / 2; break;
                case 4: v += paeth(a, b, c); break;
                default: throw std::runtime_error("bad PNG filter type");
            }
            cur[i] = (unsigned char)v;
        }
        prev = cur;
    }
}

}  // namespace

namespace IQM {

InputImage decode_png(const std::vector<unsigned char> &f) {
    static const unsigned char sig[8] = {137, 80, 78, 71, 13, 10, 26, 10};
    if (f.size() < 8 || std::memcmp(f.data(), sig, 8) != 0) throw std::runtime_error("not a PNG file");
    uint32_t w = 0, h = 0;
    int depth = 0, ctype = -1, interlace = 0;
    std::vector<unsigned char> idat, palette, trns;
    size_t pos = 8;
    bool end = false;
    while (!end) {
        if (pos + 8 > f.size()) throw std::runtime_error("truncated PNG");
        const uint32_t len = be32(&f[pos]);
        const char *type = reinterpret_cast<const char *>(&f[pos + 4]);
        if (pos + 12 + size_t(len) > f.size()) throw std::runtime_error("truncated PNG chunk");
        const unsigned char *d = &f[pos + 8];
        if (std::memcmp(type, "IHDR", 4) == 0) {
            if (len < 13) throw std::runtime_error("bad IHDR");
            w = be32(d);
            h = be32(d + 4);
            depth = d[8];
            ctype = d[9];
            interlace = d[12];
            if (d[10] != 0 || d[11] != 0) throw std::runtime_error("unsupported PNG compression/filter method");
        } else if (std::memcmp(type, "PLTE", 4) == 0) {
            palette.assign(d, d + len);
        } else if (std::memcmp(type, "tRNS", 4) == 0) {
            trns.assign(d, d + len);
        } else if (std::memcmp(type, "IDAT", 4) == 0) {
            idat.insert(idat.end(), d, d + len);
        } else if (std::memcmp(type, "IEND", 4) == 0) {
            end = true;
        }
        pos += 12 + size_t(len);
    }
    if (w == 0 || h == 0 || w > (1u << 16) || h > (1u << 16)) throw std::runtime_error("bad PNG dimensions");
    int channels;
    switch (ctype) {
        case 0: channels = 1; break;
        case 2: channels = 3; break;
        case 3: channels = 1; break;
        case 4: channels = 2; break;
        case 6: channels = 4; break;
        default: throw std::runtime_error("bad PNG colour type");
    }
    if (depth != 1 && depth != 2 && depth != 4 && depth != 8 && depth != 16) throw std::runtime_error("bad PNG bit depth");
    const int bits = channels * depth;
    const int bpp = std::max(1, bits / 8);
    // pass geometry (Adam7 or a single pass)
    struct Pass {
        int x0, y0, dx, dy;
    };
    const Pass adam7[7] = {{0, 0, 8, 8}, {4, 0, 8, 8}, {0, 4, 4, 8}, {2, 0, 4, 4}, {0, 2, 2, 4}, {1, 0, 2, 2}, {0, 1, 1, 2}};
    const Pass single[1] = {{0, 0, 1, 1}};
    const Pass *passes = interlace ? adam7 : single;
    const int npass = interlace ? 7 : 1;
    size_t raw_size = 0;
    for (int p = 0; p < npass; p++) {
        const size_t pw = (w + passes[p].dx - 1 - passes[p].x0) / passes[p].dx;
        const size_t ph = (h + passes[p].dy - 1 - passes[p].y0) / passes[p].dy;
        if (pw && ph) raw_size += ph * (1 + (pw * bits + 7) / 8);
    }
    std::vector<unsigned char> raw(raw_size);
    uLongf out_len = uLongf(raw_size);
    if (uncompress(raw.data(), &out_len, idat.data(), uLong(idat.size())) != Z_OK || out_len != raw_size)
        throw std::runtime_error("corrupt PNG image data");
    InputImage img{int(w), int(h), std::vector<unsigned char>(size_t(w) * h * 4)};
    size_t off = 0;
    for (int p = 0; p < npass; p++) {
        const Pass &P = passes[p];
        const size_t pw = (w + P.dx - 1 - P.x0) / P.dx;
        const size_t ph = (h + P.dy - 1 - P.y0) / P.dy;
        if (!pw || !ph) continue;
        const size_t rowbytes = (pw * bits + 7) / 8;
        unfilter(raw.data() + off, int(ph), rowbytes, bpp);
        for (size_t y = 0; y < ph; y++) {
            const unsigned char *line = raw.data() + off + y * (rowbytes + 1) + 1;
            for (size_t x = 0; x < pw; x++) {
                unsigned v[4] = {0, 0, 0, 255};
                auto sample = [&](int ch) -> unsigned {  // channel value scaled to 8 bits
                    if (depth == 8) return line[x * channels + ch];
                    if (depth == 16) return line[(x * channels + ch) * 2];
                    const size_t bit = (x * channels + ch) * depth;
                    const unsigned raw_v = (line[bit / 8] >> (8 - depth - bit % 8)) & ((1u << depth) - 1);
                    return ctype == 3 ? raw_v : raw_v * 255 / ((1u << depth) - 1);
                };
                if (ctype == 3) {
                    const unsigned idx = sample(0);
                    if (3 * idx + 2 >= palette.size()) throw std::runtime_error("PNG palette index out of range");
                    v[0] = palette[3 * idx];
                    v[1] = palette[3 * idx + 1];
                    v[2] = palette[3 * idx + 2];
                    v[3] = idx < trns.size() ? trns[idx] : 255;
                } else if (channels <= 2) {
                    v[0] = v[1] = v[2] = sample(0);
                    if (channels == 2) v[3] = sample(1);
                } else {
                    v[0] = sample(0);
                    v[1] = sample(1);
                    v[2] = sample(2);
                    if (channels == 4) v[3] = sample(3);
                }
                const size_t X = P.x0 + x * P.dx, Y = P.y0 + y * P.dy;
                unsigned char *dst = &img.data[(Y * w + X) * 4];
                for (int c = 0; c < 4; c++) dst[c] = (unsigned char)v[c];
            }
        }
        off += ph * (rowbytes + 1);
    }
    return img;
}

InputImage decode_pnm(const std::vector<unsigned char> &f) {
    // binary P5 (grey) / P6 (RGB) as stb_image reads them: samples taken as they are (no rescaling
    // by maxval); for maxval > 255 two bytes a sample, of which the loader keeps the second (it reads
    // the big-endian samples into host-order 16-bit words and keeps their high byte); comments run
    // to the end of the line (LF or CR)
    size_t pos = 0;
    auto token = [&]() -> std::string {
        std::string t;
        while (pos < f.size()) {
            const char c = char(f[pos]);
            if (c == '#') {
                while (pos < f.size() && f[pos] != '\n' && f[pos] != '\r') pos++;
            } else if (std::isspace((unsigned char)c)) {
                if (!t.empty()) break;
                pos++;
            } else {
                t.push_back(c);
                pos++;
            }
        }
        return t;
    };
    const std::string magic = token();
    if (magic != "P5" && magic != "P6") throw std::runtime_error("unsupported PNM type");
    const int w = std::stoi(token()), h = std::stoi(token()), maxv = std::stoi(token());
    pos++;  // the single whitespace after maxval
    if (w <= 0 || h <= 0 || maxv < 0 || maxv > 65535) throw std::runtime_error("unsupported PNM header");
    if (int64_t(w) * h >= (int64_t(1) << 31)) throw std::runtime_error("image size out of range");
    const int ch = magic == "P5" ? 1 : 3, bytes = maxv > 255 ? 2 : 1;
    if (f.size() < pos + size_t(w) * h * ch * bytes) throw std::runtime_error("truncated PNM");
    InputImage img{w, h, std::vector<unsigned char>(size_t(w) * h * 4)};
    for (size_t i = 0; i < size_t(w) * h; i++) {
        for (int c = 0; c < 3; c++) img.data[i * 4 + c] = f[pos + (i * ch + (ch == 3 ? c : 0)) * bytes + bytes - 1];
        img.data[i * 4 + 3] = 255;
    }
    return img;
}

InputImage load_image(const std::string &path) {
    std::ifstream in(path, std::ios::binary);
    try {
        if (!in) throw std::runtime_error("can't fopen");
        std::vector<unsigned char> f((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
        if (f.size() >= 8 && f[0] == 137 && f[1] == 'P' && f[2] == 'N' && f[3] == 'G') return decode_png(f);
        if (f.size() >= 2 && f[0] == 'P' && (f[1] == '5' || f[1] == '6')) return decode_pnm(f);
        if (f.size() >= 2 && f[0] == 'B' && f[1] == 'M') return decode_bmp(f);
        if (f.size() >= 3 && f[0] == 0xFF && f[1] == 0xD8 && f[2] == 0xFF) return decode_jpeg(f);
        auto starts = [&](const char *sig) {
            const size_t k = std::strlen(sig);
            return f.size() >= k && std::memcmp(f.data(), sig, k) == 0;
        };
        if (starts("GIF87a") || starts("GIF89a")) return decode_gif(f);
        if (starts("8BPS")) return decode_psd(f);
        if (starts("#?RADIANCE\n") || starts("#?RGBE\n")) return decode_hdr(f);
        if (f.size() >= 92 && starts("\x53\x80\xF6\x34") && std::memcmp(&f[88], "PICT", 4) == 0) return decode_pic(f);
        // TGA has no signature: like the reference's loader, try it when nothing else matched
        try {
            return decode_tga(f);
        } catch (const std::exception &) {
            throw std::runtime_error("unknown image type");
        }
    } catch (const std::exception &e) {
        throw std::runtime_error("Failed to load image '" + path + "', reason: " + e.what());
    }
}

std::vector<unsigned char> encode_png(int width, int height, int channels, const std::vector<unsigned char> &pixels) {
    if (channels != 1 && channels != 3 && channels != 4) throw std::runtime_error("PNG: 1, 3 or 4 channels");
    const size_t row = size_t(width) * channels;
    if (pixels.size() < row * size_t(height)) throw std::runtime_error("PNG: pixel buffer too small");
    std::vector<unsigned char> raw;
    raw.reserve(size_t(height) * (row + 1));
    for (int y = 0; y < height; y++) {
        raw.push_back(0);
        raw.insert(raw.end(), pixels.begin() + size_t(y) * row, pixels.begin() + size_t(y + 1) * row);
    }
    uLongf zlen = compressBound(uLong(raw.size()));
    std::vector<unsigned char> z(zlen);
    if (compress2(z.data(), &zlen, raw.data(), uLong(raw.size()), 6) != Z_OK) throw std::runtime_error("zlib failed");
    z.resize(zlen);
    std::vector<unsigned char> o = {137, 80, 78, 71, 13, 10, 26, 10};
    auto chunk = [&](const char *type, const std::vector<unsigned char> &data) {
        put32(o, uint32_t(data.size()));
        const size_t start = o.size();
        o.insert(o.end(), type, type + 4);
        o.insert(o.end(), data.begin(), data.end());
        put32(o, uint32_t(crc32(0, &o[start], uInt(o.size() - start))));
    };
    std::vector<unsigned char> ihdr;
    put32(ihdr, uint32_t(width));
    put32(ihdr, uint32_t(height));
    const unsigned char color_type = channels == 1 ? 0 : channels == 3 ? 2 : 6;
    ihdr.insert(ihdr.end(), {8, color_type, 0, 0, 0});
    chunk("IHDR", ihdr);
    chunk("IDAT", z);
    chunk("IEND", {});
    return o;
}

std::vector<unsigned char> encode_grey_png(int width, int height, const std::vector<unsigned char> &pixels) {
    return encode_png(width, height, 1, pixels);
}

bool write_png(const std::string &path, int width, int height, int channels, const std::vector<unsigned char> &pixels) {
    try {
        const auto bytes = encode_png(width, height, channels, pixels);
        std::ofstream out(path, std::ios::binary);
        out.write(reinterpret_cast<const char *>(bytes.data()), std::streamsize(bytes.size()));
        return bool(out);
    } catch (...) {
        return false;
    }
}

bool write_grey_png(const std::string &path, int width, int height, const std::vector<unsigned char> &pixels) {
    return write_png(path, width, height, 1, pixels);
}

}  // namespace IQM
