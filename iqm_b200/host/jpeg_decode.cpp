// Baseline JPEG input for the command line, written from the JPEG specification (ITU-T T.81,
// sequential DCT with Huffman coding, 8-bit samples; JFIF colour).  Output is RGBA8 like the
// reference's stbi_load(..., 4) (src/main.cpp:37-57).  A lossy format decodes to slightly different
// bytes in different decoders (IDCT arithmetic, chroma upsampling, colour rounding): this one uses a
// separable floating-point IDCT, the reference loader's integer triangle filters for 2x chroma
// upsampling (including its edge rule; the nearest sample for other factors) and the JFIF
// YCbCr->RGB equations, which keeps it within a few levels of the reference's loader.  Progressive files (T.81 Annex G: spectral selection
// and successive approximation, Huffman coded) keep every block's coefficients across their scans
// and are transformed after the last one.  Arithmetic-coded and lossless files, 12-bit samples and
// 4-component (CMYK) images are refused with a reason.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "png_io.h"

namespace IQM {
namespace {

// natural (row-major) position of the k-th coefficient in zig-zag order
const int kZigzag[64] = {0,  1,  8,  16, 9,  2,  3,  10, 17, 24, 32, 25, 18, 11, 4,  5,  12, 19, 26, 33, 40, 48,
                         41, 34, 27, 20, 13, 6,  7,  14, 21, 28, 35, 42, 49, 56, 57, 50, 43, 36, 29, 22, 15, 23,
                         30, 37, 44, 51, 58, 59, 52, 45, 38, 31, 39, 46, 53, 60, 61, 54, 47, 55, 62, 63};

struct Huffman {  // T.81 Annex C / F.2.2.3 decoding tables
    int mincode[17], maxcode[18], valptr[17];
    std::vector<unsigned char> vals;
    bool present = false;
    void build(const unsigned char *bits, const unsigned char *v, int nvals) {
        vals.assign(v, v + nvals);
        int code = 0, k = 0;
        for (int l = 1; l <= 16; l++) {
            valptr[l] = k;
            mincode[l] = code;
            code += bits[l - 1];
            k += bits[l - 1];
            maxcode[l] = bits[l - 1] ? code - 1 : -1;
            code <<= 1;
        }
        maxcode[17] = 0x7fffffff;
        present = true;
    }
};

struct Component {
    int id, h, v, tq, td = 0, ta = 0;
    int bw, bh;  // blocks per line / column (covering whole MCUs)
    std::vector<unsigned char> plane;  // bw*8 x bh*8 samples
    std::vector<int> coef;             // progressive: bw*bh blocks of 64 coefficients, zig-zag order
    int pred = 0;
};

class BitReader {
public:
    BitReader(const std::vector<unsigned char> &f, size_t pos) : f_(f), pos_(pos) {}
    int bit() {
        if (n_ == 0) fill();
        n_--;
        return (acc_ >> n_) & 1;
    }
    int bits(int s) {
        int v = 0;
        for (int i = 0; i < s; i++) v = (v << 1) | bit();
        return v;
    }
    // expects and consumes the restart marker RSTm, dropping buffered bits
    void restart() {
        n_ = 0;
        marker_ = false;
        while (pos_ + 1 < f_.size() && !(f_[pos_] == 0xFF && f_[pos_ + 1] >= 0xD0 && f_[pos_ + 1] <= 0xD7)) pos_++;
        if (pos_ + 1 >= f_.size()) throw std::runtime_error("JPEG restart marker missing");
        pos_ += 2;
    }
    size_t pos() const { return pos_; }

private:
    void fill() {
        unsigned b = 0;
        if (!marker_ && pos_ < f_.size()) {
            b = f_[pos_];
            if (b == 0xFF) {
                const unsigned nx = pos_ + 1 < f_.size() ? f_[pos_ + 1] : 0xD9;
                if (nx == 0x00) {
                    pos_ += 2;
                } else {
                    marker_ = true;  // a marker ends the segment: feed zero bits
                    b = 0;
                }
            } else {
                pos_++;
            }
        }
        acc_ = (acc_ << 8) | b;
        n_ = 8;
    }
    const std::vector<unsigned char> &f_;
    size_t pos_;
    uint32_t acc_ = 0;
    int n_ = 0;
    bool marker_ = false;
};

int decode_symbol(BitReader &br, const Huffman &h) {
    if (!h.present) throw std::runtime_error("JPEG Huffman table missing");
    int code = br.bit();
    for (int l = 1; l <= 16; l++) {
        if (code <= h.maxcode[l]) return h.vals.at(size_t(h.valptr[l] + code - h.mincode[l]));
        code = (code << 1) | br.bit();
    }
    throw std::runtime_error("corrupt JPEG Huffman code");
}

int receive_extend(BitReader &br, int s) {
    if (s == 0) return 0;
    if (s > 16) throw std::runtime_error("corrupt JPEG coefficient");
    const int v = br.bits(s);
    return v < (1 << (s - 1)) ? v - (1 << s) + 1 : v;
}

// 8x8 inverse DCT (T.81 A.3.3), level shift and clamp into `out` (stride `stride`).
void idct8x8(const float *coef, unsigned char *out, int stride) {
    static float c[8][8];
    static bool init = false;
    if (!init) {
        for (int x = 0; x < 8; x++)
            for (int u = 0; u < 8; u++)
                c[x][u] = float((u == 0 ? std::sqrt(0.5) : 1.0) * std::cos((2 * x + 1) * u * M_PI / 16.0) / 2.0);
        init = true;
    }
    float tmp[64];
    for (int v = 0; v < 8; v++)  // rows of coefficients along u
        for (int x = 0; x < 8; x++) {
            float s = 0.f;
            for (int u = 0; u < 8; u++) s += c[x][u] * coef[v * 8 + u];
            tmp[v * 8 + x] = s;
        }
    for (int y = 0; y < 8; y++)
        for (int x = 0; x < 8; x++) {
            float s = 0.f;
            for (int v = 0; v < 8; v++) s += c[y][v] * tmp[v * 8 + x];
            out[y * stride + x] = (unsigned char)std::clamp(int(std::lround(s + 128.0f)), 0, 255);
        }
}

}  // namespace

// One progressive scan (T.81 G.1.2): spectral band ss..se, successive approximation ah -> al.  DC
// scans may interleave components (MCU order); AC scans hold one component and walk its blocks.
void progressive_scan(BitReader &br, const std::vector<Component *> &sc, const Huffman *dc, const Huffman *ac, int ss,
                      int se, int ah, int al, int restart, int width, int height, int hmax, int vmax) {
    if (ss > se || se > 63 || (ss == 0 && se != 0) || (ss > 0 && sc.size() != 1) || al > 13)
        throw std::runtime_error("corrupt JPEG progressive scan");
    int eobrun = 0;
    const int p1 = 1 << al, m1 = -(1 << al);
    auto refine = [&](int &z) {  // one correction bit of an already non-zero coefficient
        if (br.bit() && (z & p1) == 0) z += z >= 0 ? p1 : m1;
    };
    auto block = [&](Component &c, int bx, int by) {
        int *z = &c.coef[(size_t(by) * c.bw + bx) * 64];
        if (ss == 0) {  // DC
            if (ah == 0) {
                c.pred += receive_extend(br, decode_symbol(br, dc[c.td]));
                z[0] = c.pred * (1 << al);
            } else if (br.bit()) {
                z[0] |= p1;
            }
            return;
        }
        if (ah == 0) {  // AC, first pass of the band
            if (eobrun > 0) {
                eobrun--;
                return;
            }
            for (int k = ss; k <= se; k++) {
                const int rs = decode_symbol(br, ac[c.ta]), r = rs >> 4, s = rs & 15;
                if (s == 0) {
                    if (r < 15) {
                        eobrun = (1 << r) - 1 + (r ? br.bits(r) : 0);
                        break;
                    }
                    k += 15;
                    continue;
                }
                k += r;
                if (k > se) throw std::runtime_error("corrupt JPEG block");
                z[k] = receive_extend(br, s) * (1 << al);
            }
            return;
        }
        int k = ss;  // AC refinement
        if (eobrun == 0) {
            for (; k <= se; k++) {
                const int rs = decode_symbol(br, ac[c.ta]);
                int r = rs >> 4, value = 0;
                const int s = rs & 15;
                if (s) {
                    if (s != 1) throw std::runtime_error("corrupt JPEG refinement");
                    value = br.bit() ? p1 : m1;
                } else if (r != 15) {
                    eobrun = (1 << r) + (r ? br.bits(r) : 0);
                    break;
                }
                for (; k <= se; k++) {  // pass r zero-history coefficients, refining the others
                    if (z[k] != 0) {
                        refine(z[k]);
                    } else {
                        if (r == 0) {
                            if (value) z[k] = value;
                            break;
                        }
                        r--;
                    }
                }
            }
        }
        if (eobrun > 0) {
            for (; k <= se; k++)
                if (z[k] != 0) refine(z[k]);
            eobrun--;
        }
    };
    int mcux, mcus;
    if (sc.size() == 1) {  // non-interleaved: blocks of the component's own (unpadded) extent
        const Component &c = *sc[0];
        const int cw = (width * c.h + hmax - 1) / hmax, ch = (height * c.v + vmax - 1) / vmax;
        mcux = (cw + 7) / 8;
        mcus = mcux * ((ch + 7) / 8);
    } else {
        mcux = (width + 8 * hmax - 1) / (8 * hmax);
        mcus = mcux * ((height + 8 * vmax - 1) / (8 * vmax));
    }
    for (auto *c : sc) c->pred = 0;
    for (int n = 0; n < mcus; n++) {
        if (restart && n && n % restart == 0) {
            br.restart();
            for (auto *c : sc) c->pred = 0;
            eobrun = 0;
        }
        const int mx = n % mcux, my = n / mcux;
        if (sc.size() == 1) {
            block(*sc[0], mx, my);
        } else {
            for (auto *c : sc)
                for (int v = 0; v < c->v; v++)
                    for (int h = 0; h < c->h; h++) block(*c, mx * c->h + h, my * c->v + v);
        }
    }
}

InputImage decode_jpeg(const std::vector<unsigned char> &f) {
    if (f.size() < 4 || f[0] != 0xFF || f[1] != 0xD8) throw std::runtime_error("not a JPEG file");
    uint16_t qt[4][64] = {};
    Huffman dc[4], ac[4];
    std::vector<Component> comps;
    int width = 0, height = 0, restart = 0, hmax = 1, vmax = 1;
    bool have_frame = false, done = false, progressive = false;
    size_t pos = 2;
    auto seg_len = [&](size_t p) -> size_t {
        if (p + 2 > f.size()) throw std::runtime_error("truncated JPEG");
        const size_t len = size_t(f[p]) << 8 | f[p + 1];
        if (len < 2 || p + len > f.size()) throw std::runtime_error("truncated JPEG");
        return len;
    };
    while (!done) {
        while (pos < f.size() && f[pos] != 0xFF) pos++;  // resynchronise on the next marker
        while (pos < f.size() && f[pos] == 0xFF) pos++;
        if (pos >= f.size()) throw std::runtime_error("truncated JPEG");
        const unsigned m = f[pos++];
        if (m == 0xD9) break;
        if (m == 0xD8 || (m >= 0xD0 && m <= 0xD7)) continue;
        const size_t len = seg_len(pos), p0 = pos + 2, end = pos + len;
        if (m == 0xDB) {  // quantisation tables, zig-zag order
            for (size_t p = p0; p < end;) {
                const int pq = f[p] >> 4, tq = f[p] & 15;
                p++;
                if (tq > 3) throw std::runtime_error("corrupt JPEG");
                for (int k = 0; k < 64; k++) {
                    if (p + (pq ? 2 : 1) > end) throw std::runtime_error("truncated JPEG");
                    qt[tq][k] = pq ? uint16_t(f[p] << 8 | f[p + 1]) : f[p];
                    p += pq ? 2 : 1;
                }
            }
        } else if (m == 0xC4) {  // Huffman tables
            for (size_t p = p0; p < end;) {
                const int tc = f[p] >> 4, th = f[p] & 15;
                if (th > 3 || tc > 1 || p + 17 > end) throw std::runtime_error("corrupt JPEG");
                int n = 0;
                for (int i = 0; i < 16; i++) n += f[p + 1 + i];
                if (p + 17 + size_t(n) > end) throw std::runtime_error("truncated JPEG");
                (tc ? ac : dc)[th].build(&f[p + 1], &f[p + 17], n);
                p += 17 + n;
            }
        } else if (m == 0xC0 || m == 0xC1 || m == 0xC2) {  // baseline / extended sequential / progressive, Huffman
            progressive = m == 0xC2;
            if (len < 8 || f[p0] != 8) throw std::runtime_error("only 8-bit JPEG samples are supported");
            height = f[p0 + 1] << 8 | f[p0 + 2];
            width = f[p0 + 3] << 8 | f[p0 + 4];
            const int nf = f[p0 + 5];
            if (nf != 1 && nf != 3) throw std::runtime_error("JPEG with " + std::to_string(nf) + " components is not supported");
            if (len < size_t(8 + 3 * nf)) throw std::runtime_error("truncated JPEG");
            if (width <= 0 || height <= 0 || width > 65535 || height > 65535) throw std::runtime_error("JPEG size out of range");
            for (int i = 0; i < nf; i++) {
                Component c{};
                c.id = f[p0 + 6 + 3 * i];
                c.h = f[p0 + 7 + 3 * i] >> 4;
                c.v = f[p0 + 7 + 3 * i] & 15;
                c.tq = f[p0 + 8 + 3 * i] & 3;
                if (c.h < 1 || c.h > 4 || c.v < 1 || c.v > 4) throw std::runtime_error("corrupt JPEG sampling factors");
                comps.push_back(c);
            }
            for (auto &c : comps) hmax = std::max(hmax, c.h), vmax = std::max(vmax, c.v);
            const int mcux = (width + 8 * hmax - 1) / (8 * hmax), mcuy = (height + 8 * vmax - 1) / (8 * vmax);
            for (auto &c : comps) {
                c.bw = mcux * c.h;
                c.bh = mcuy * c.v;
                c.plane.assign(size_t(c.bw) * 8 * c.bh * 8, 0);
                if (progressive) c.coef.assign(size_t(c.bw) * c.bh * 64, 0);
            }
            have_frame = true;
        } else if (m >= 0xC3 && m <= 0xCF && m != 0xC4 && m != 0xC8 && m != 0xCC) {
            throw std::runtime_error("lossless or arithmetic-coded JPEG is not supported");
        } else if (m == 0xDD) {
            restart = f[p0] << 8 | f[p0 + 1];
        } else if (m == 0xDA) {  // start of scan: entropy-coded data follows the header
            if (!have_frame) throw std::runtime_error("JPEG scan before frame header");
            const int ns = f[p0];
            std::vector<Component *> sc;
            for (int i = 0; i < ns; i++) {
                const int id = f[p0 + 1 + 2 * i];
                Component *c = nullptr;
                for (auto &cc : comps)
                    if (cc.id == id) c = &cc;
                if (!c) throw std::runtime_error("corrupt JPEG scan");
                c->td = f[p0 + 2 + 2 * i] >> 4 & 3;
                c->ta = f[p0 + 2 + 2 * i] & 3;
                c->pred = 0;
                sc.push_back(c);
            }
            BitReader br(f, end);
            if (progressive) {
                const size_t q = p0 + 1 + 2 * size_t(ns);
                if (q + 3 > end) throw std::runtime_error("truncated JPEG");
                progressive_scan(br, sc, dc, ac, f[q], f[q + 1], f[q + 2] >> 4, f[q + 2] & 15, restart, width,
                                 height, hmax, vmax);
                pos = br.pos();
                continue;
            }
            float coef[64];
            auto block = [&](Component &c, int bx, int by) {
                std::fill(coef, coef + 64, 0.f);
                const int t = decode_symbol(br, dc[c.td]);
                c.pred += receive_extend(br, t);
                coef[0] = float(c.pred * qt[c.tq][0]);
                for (int k = 1; k < 64;) {
                    const int rs = decode_symbol(br, ac[c.ta]), r = rs >> 4, s = rs & 15;
                    if (s == 0) {
                        if (r != 15) break;  // end of block
                        k += 16;
                        continue;
                    }
                    k += r;
                    if (k > 63) throw std::runtime_error("corrupt JPEG block");
                    coef[kZigzag[k]] = float(receive_extend(br, s) * qt[c.tq][k]);
                    k++;
                }
                const int stride = c.bw * 8;
                idct8x8(coef, &c.plane[size_t(by) * 8 * stride + size_t(bx) * 8], stride);
            };
            int mcus, mcux = 0;
            if (ns == 1) {  // non-interleaved: blocks of the component's own (unpadded) extent
                Component &c = *sc[0];
                const int cw = (width * c.h + hmax - 1) / hmax, ch = (height * c.v + vmax - 1) / vmax;
                mcux = (cw + 7) / 8;
                mcus = mcux * ((ch + 7) / 8);
            } else {
                mcux = (width + 8 * hmax - 1) / (8 * hmax);
                mcus = mcux * ((height + 8 * vmax - 1) / (8 * vmax));
            }
            for (int n = 0; n < mcus; n++) {
                if (restart && n && n % restart == 0) {
                    br.restart();
                    for (auto *c : sc) c->pred = 0;
                }
                const int mx = n % mcux, my = n / mcux;
                if (ns == 1) {
                    block(*sc[0], mx, my);
                } else {
                    for (auto *c : sc)
                        for (int v = 0; v < c->v; v++)
                            for (int h = 0; h < c->h; h++) block(*c, mx * c->h + h, my * c->v + v);
                }
            }
            pos = br.pos();
            if (comps.size() == 1 || ns == int(comps.size())) done = true;  // baseline: the frame's last scan
            continue;
        }
        pos = end;
    }
    if (!have_frame) throw std::runtime_error("JPEG has no frame");
    if (progressive)  // dequantise with the tables in force at the end, transform every block
        for (auto &c : comps) {
            float coef[64];
            const int stride = c.bw * 8;
            for (int by = 0; by < c.bh; by++)
                for (int bx = 0; bx < c.bw; bx++) {
                    const int *z = &c.coef[(size_t(by) * c.bw + bx) * 64];
                    for (int k = 0; k < 64; k++) coef[kZigzag[k]] = float(z[k] * qt[c.tq][k]);
                    idct8x8(coef, &c.plane[size_t(by) * 8 * stride + size_t(bx) * 8], stride);
                }
        }
    InputImage img;
    img.width = width;
    img.height = height;
    img.data.resize(size_t(width) * height * 4);
    // Component sample at full resolution, as the reference's loader upsamples chroma (integer
    // triangle filters, each output rounded to a byte):
    //   2x across:       (3 a + b + 2) >> 2 with b the neighbour on the output's side; the row's
    //                    first output is a[0], its last a[w-1], and the output before the last
    //                    weighs the second-to-last sample by 3 -- the loader's own edge rule;
    //   2x down:         (3 near + far + 2) >> 2 with the neighbouring row (clamped) as far;
    //   2x both ways:    t = 3 near + far per column, then (3 t + t' + 8) >> 4 with the neighbouring
    //                    column's t', and (t + 2) >> 2 at the row's first and last output;
    //   other factors:   the nearest sample.
    auto sample = [&](const Component &c, int x, int y) -> float {
        const int fx = hmax / c.h, fy = vmax / c.v, stride = c.bw * 8;
        const int pw = (width * c.h + hmax - 1) / hmax, ph = (height * c.v + vmax - 1) / vmax;  // real extent
        auto at = [&](int xx, int yy) {
            return int(c.plane[size_t(std::clamp(yy, 0, ph - 1)) * stride + std::clamp(xx, 0, pw - 1)]);
        };
        const int cx = x / fx, cy = y / fy;
        if (fy == 2 && fx <= 2) {
            const int far_row = (y & 1) ? cy + 1 : cy - 1;  // clamped by at()
            auto t = [&](int xx) { return 3 * at(xx, cy) + at(xx, far_row); };
            if (fx == 1) return float((t(cx) + 2) >> 2);
            if (pw == 1 || x == 0 || x == 2 * pw - 1) return float((t(cx) + 2) >> 2);
            return float((x & 1) ? (3 * t(cx) + t(cx + 1) + 8) >> 4 : (3 * t(cx) + t(cx - 1) + 8) >> 4);
        }
        if (fx == 2 && fy == 1) {
            if (pw == 1 || x == 0) return float(at(cx, cy));
            if (x & 1) return float(cx == pw - 1 ? at(cx, cy) : (3 * at(cx, cy) + at(cx + 1, cy) + 2) >> 2);
            if (cx == pw - 1) return float((3 * at(cx - 1, cy) + at(cx, cy) + 2) >> 2);
            return float((3 * at(cx, cy) + at(cx - 1, cy) + 2) >> 2);
        }
        return float(at(cx, cy));
    };
    for (int y = 0; y < height; y++)
        for (int x = 0; x < width; x++) {
            unsigned char *o = &img.data[(size_t(y) * width + x) * 4];
            const float Y = sample(comps[0], x, y);
            if (comps.size() == 1) {
                o[0] = o[1] = o[2] = (unsigned char)Y;
            } else {  // JFIF YCbCr -> RGB
                const float cb = sample(comps[1], x, y) - 128.f, cr = sample(comps[2], x, y) - 128.f;
                auto px = [](float v) { return (unsigned char)std::clamp(int(std::lround(v)), 0, 255); };
                o[0] = px(Y + 1.402f * cr);
                o[1] = px(Y - 0.344136f * cb - 0.714136f * cr);
                o[2] = px(Y + 1.772f * cb);
            }
            o[3] = 255;
        }
    return img;
}

}  // namespace IQM
