// JPEG decoding for diffuse textures (ITU-T T.81 with the JFIF colour
// convention), to 8-bit RGBA with rows top-down, as the reference's texture
// loader receives every texture format through stbi_load with 4 requested
// channels (Texture::Load, Src/Core/texture.cu:207-240).
//
// Supported: baseline and extended sequential (SOF0, SOF1) and progressive
// (SOF2) Huffman-coded 8-bit images with 1 (grey) or 3 (YCbCr, or RGB when
// an Adobe APP14 marker says so) components, any sampling factors 1-4,
// restart intervals, 8- and 16-bit quantisation tables. Arithmetic coding,
// lossless, hierarchical and 12-bit processes and 4-component (CMYK) images
// are refused with a message.
//
// Pipeline: entropy-decode every scan into per-component coefficient planes
// (progressive scans refine them in place: DC first/refine, AC first/refine
// with end-of-band runs, per T.81 G.1.2), then dequantise and inverse-DCT
// each 8x8 block in double precision, upsample chroma (2:1 planes with the
// triangle filter that weights the nearer sample 3/4, other ratios by
// replication) and convert YCbCr to RGB. Results agree with the reference's
// decoder to within a few levels: the inverse DCT, the upsampling filter's
// rounding and the colour conversion are computed independently.
#include "scene_data.h"
#include "common.cuh"
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

namespace crt {
namespace {

[[noreturn]] void bad(const char *msg) { throw Error(CRT_ERR_PARSE, std::string("JPEG: ") + msg); }

// Natural (row-major) index of the k-th coefficient in zig-zag order.
const uint8_t kZigzag[64] = {0,  1,  8,  16, 9,  2,  3,  10, 17, 24, 32, 25, 18, 11, 4,  5,
                             12, 19, 26, 33, 40, 48, 41, 34, 27, 20, 13, 6,  7,  14, 21, 28,
                             35, 42, 49, 56, 57, 50, 43, 36, 29, 22, 15, 23, 30, 37, 44, 51,
                             58, 59, 52, 45, 38, 31, 39, 46, 53, 60, 61, 54, 47, 55, 62, 63};

struct HuffTable {
    bool present = false;
    // canonical code ranges per length (T.81 F.2.2.3): codes of length l are
    // mincode[l] .. maxcode[l], their symbols start at valptr[l]
    int mincode[17], maxcode[18], valptr[17];
    std::vector<uint8_t> vals;
    // 9-bit lookahead: (length << 8 | symbol), 0 = longer code
    uint16_t fast[512];
    void build(const uint8_t counts[16], const uint8_t *symbols, int nsym) {
        vals.assign(symbols, symbols + nsym);
        int code = 0, k = 0;
        std::memset(fast, 0, sizeof(fast));
        for (int l = 1; l <= 16; ++l) {
            const int c = counts[l - 1];
            valptr[l] = k;
            mincode[l] = code;
            maxcode[l] = c ? code + c - 1 : -1;
            for (int i = 0; i < c; ++i, ++code, ++k) {
                if (l <= 9) {
                    const int shift = 9 - l;
                    for (int f = code << shift; f < ((code + 1) << shift); ++f)
                        fast[f] = (uint16_t)((l << 8) | vals[k]);
                }
            }
            if (code > (1 << l)) bad("over-subscribed Huffman table");
            code <<= 1;
        }
        maxcode[17] = INT32_MAX;
        present = true;
    }
};

// Bits of an entropy-coded segment: 0xFF 0x00 stands for 0xFF; a marker ends
// the segment, after which zero bits are supplied.
struct Bits {
    const uint8_t *p;
    size_t n, pos;
    uint32_t acc = 0;
    int cnt = 0;
    int marker = -1;  // marker met inside the entropy data (RSTn or the next segment)
    void fill() {
        while (cnt <= 24) {
            uint32_t b = 0;
            if (marker < 0 && pos < n) {
                b = p[pos];
                if (b == 0xFF) {
                    const uint8_t nx = pos + 1 < n ? p[pos + 1] : 0xD9;
                    if (nx == 0x00) {
                        pos += 2;
                    } else {
                        marker = nx;
                        b = 0;
                    }
                } else {
                    ++pos;
                }
            }
            acc |= b << (24 - cnt);
            cnt += 8;
        }
    }
    int peek9() {
        fill();
        return (int)(acc >> 23);
    }
    void skip(int k) {
        acc <<= k;
        cnt -= k;
    }
    int bit() {
        fill();
        const int b = (int)(acc >> 31);
        skip(1);
        return b;
    }
    int get(int k) {
        if (k == 0) return 0;
        fill();
        const int v = (int)(acc >> (32 - k));
        skip(k);
        return v;
    }
    void reset() {
        acc = 0;
        cnt = 0;
    }
};

int huff_decode(Bits &b, const HuffTable &h) {
    if (!h.present) bad("scan uses an undefined Huffman table");
    const uint16_t f = h.fast[b.peek9()];
    if (f) {
        b.skip(f >> 8);
        return f & 0xFF;
    }
    int code = 0;
    for (int l = 1; l <= 16; ++l) {
        code = (code << 1) | b.bit();
        if (h.maxcode[l] >= 0 && code <= h.maxcode[l] && code >= h.mincode[l]) return h.vals[h.valptr[l] + code - h.mincode[l]];
    }
    bad("bad Huffman code");
}

// EXTEND (T.81 F.2.2.1): the s-bit magnitude category value v as a signed
// coefficient.
inline int extend(int v, int s) { return s == 0 ? 0 : (v < (1 << (s - 1)) ? v - (1 << s) + 1 : v); }

struct Component {
    int id, h, v, tq;
    int bw, bh;                 // blocks per row / column of the coefficient plane (MCU-padded)
    int cw, ch;                 // component size in samples
    std::vector<int16_t> coef;  // bw * bh * 64, natural order
    int dc_pred = 0;
    int td = 0, ta = 0;
};

struct Decoder {
    const std::vector<uint8_t> &f;
    size_t pos = 0;
    uint16_t qt[4][64];  // natural order
    bool qt_present[4] = {false, false, false, false};
    HuffTable dc[4], ac[4];
    std::vector<Component> comps;
    int width = 0, height = 0, hmax = 1, vmax = 1, mcux = 0, mcuy = 0;
    bool progressive = false, frame = false, adobe = false;
    int adobe_transform = -1;
    int restart = 0;
    int eobrun = 0;

    explicit Decoder(const std::vector<uint8_t> &data) : f(data) {}

    int u8() {
        if (pos >= f.size()) bad("truncated file");
        return f[pos++];
    }
    int u16() {
        const int a = u8();
        return (a << 8) | u8();
    }

    void read_dqt(size_t end) {
        while (pos < end) {
            const int pq = u8();
            const int t = pq & 15, prec = pq >> 4;
            if (t > 3 || prec > 1) bad("bad quantisation table");
            for (int k = 0; k < 64; ++k) qt[t][kZigzag[k]] = (uint16_t)(prec ? u16() : u8());
            qt_present[t] = true;
        }
    }
    void read_dht(size_t end) {
        while (pos < end) {
            const int tc = u8();
            const int cls = tc >> 4, id = tc & 15;
            if (cls > 1 || id > 3) bad("bad Huffman table id");
            uint8_t counts[16];
            int total = 0;
            for (int i = 0; i < 16; ++i) total += counts[i] = (uint8_t)u8();
            if (total > 256 || pos + total > end) bad("bad Huffman table");
            (cls ? ac : dc)[id].build(counts, f.data() + pos, total);
            pos += total;
        }
    }
    void read_sof(int marker) {
        if (frame) bad("more than one frame");
        frame = true;
        progressive = marker == 0xC2;
        if (u8() != 8) bad("only 8-bit samples are decoded");
        height = u16();
        width = u16();
        const int nf = u8();
        if (width <= 0 || height <= 0) bad("image without a height (DNL) or width");
        if (width > (1 << 15) || height > (1 << 15)) bad("image larger than 32768 pixels");
        if (nf != 1 && nf != 3) bad("only grey and 3-component images are decoded");
        comps.resize(nf);
        for (auto &c : comps) {
            c.id = u8();
            const int hv = u8();
            c.h = hv >> 4;
            c.v = hv & 15;
            c.tq = u8();
            if (c.h < 1 || c.h > 4 || c.v < 1 || c.v > 4 || c.tq > 3) bad("bad component parameters");
            hmax = std::max(hmax, c.h);
            vmax = std::max(vmax, c.v);
        }
        mcux = (width + 8 * hmax - 1) / (8 * hmax);
        mcuy = (height + 8 * vmax - 1) / (8 * vmax);
        for (auto &c : comps) {
            if (hmax % c.h || vmax % c.v) bad("sampling factors that are not integer ratios");
            c.bw = mcux * c.h;
            c.bh = mcuy * c.v;
            c.cw = (width * c.h + hmax - 1) / hmax;
            c.ch = (height * c.v + vmax - 1) / vmax;
            c.coef.assign((size_t)c.bw * c.bh * 64, 0);
        }
    }

    // One scan's entropy-coded data, up to the next non-RST marker.
    void read_scan(size_t header_end) {
        if (!frame) bad("scan before the frame header");
        const int ns = u8();
        if (ns < 1 || ns > 4) bad("bad scan header");
        std::vector<Component *> sc;
        for (int i = 0; i < ns; ++i) {
            const int cid = u8(), t = u8();
            Component *c = nullptr;
            for (auto &cc : comps)
                if (cc.id == cid) c = &cc;
            if (!c) bad("scan names an unknown component");
            c->td = t >> 4;
            c->ta = t & 15;
            if (c->td > 3 || c->ta > 3) bad("bad table selector");
            sc.push_back(c);
        }
        const int ss = u8(), se = u8(), a = u8();
        const int ah = a >> 4, al = a & 15;
        if (pos != header_end) bad("bad scan header length");
        if (!progressive) {
            if (ss != 0 || se != 63 || a != 0) bad("bad sequential scan parameters");
        } else {
            if (ss > se || se > 63 || (ss == 0 && se != 0) || (ss > 0 && ns != 1) || al > 13) bad("bad progressive scan");
        }
        for (auto *c : sc) c->dc_pred = 0;
        eobrun = 0;
        Bits b{f.data(), f.size(), pos};
        // blocks of the scan, in MCU order
        const bool single = ns == 1;
        const int units_x = single ? (sc[0]->cw + 7) / 8 : mcux;
        const int units_y = single ? (sc[0]->ch + 7) / 8 : mcuy;
        int todo = restart;
        for (int my = 0; my < units_y; ++my)
            for (int mx = 0; mx < units_x; ++mx) {
                if (restart && todo == 0) {
                    // expect RSTn, then restart the predictors and the bit reader
                    if (b.marker >= 0xD0 && b.marker <= 0xD7) {
                        b.pos += 2;
                        b.marker = -1;
                    } else if (b.marker < 0) {
                        // not yet reached: skip to it
                        while (b.pos + 1 < b.n && !(b.p[b.pos] == 0xFF && b.p[b.pos + 1] >= 0xD0 &&
                                                     b.p[b.pos + 1] <= 0xD7))
                            ++b.pos;
                        if (b.pos + 1 < b.n) b.pos += 2;
                    }
                    b.reset();
                    for (auto *c : sc) c->dc_pred = 0;
                    eobrun = 0;
                    todo = restart;
                }
                if (single) {
                    Component *c = sc[0];
                    decode_block(b, *c, &c->coef[((size_t)my * c->bw + mx) * 64], ss, se, ah, al);
                } else {
                    for (auto *c : sc)
                        for (int by = 0; by < c->v; ++by)
                            for (int bx = 0; bx < c->h; ++bx) {
                                const size_t bi = (size_t)(my * c->v + by) * c->bw + (mx * c->h + bx);
                                decode_block(b, *c, &c->coef[bi * 64], ss, se, ah, al);
                            }
                }
                if (restart) --todo;
            }
        // continue after the entropy data: find the next marker that is not RSTn
        size_t p = b.marker >= 0 ? b.pos : b.pos;
        while (p + 1 < f.size() && !(f[p] == 0xFF && f[p + 1] != 0x00 && !(f[p + 1] >= 0xD0 && f[p + 1] <= 0xD7)))
            ++p;
        pos = p;
    }

    void decode_block(Bits &b, Component &c, int16_t *blk, int ss, int se, int ah, int al) {
        if (!progressive) {
            const int t = huff_decode(b, dc[c.td]);
            if (t > 11) bad("bad DC magnitude");
            c.dc_pred += extend(b.get(t), t);
            blk[0] = (int16_t)c.dc_pred;
            for (int k = 1; k < 64;) {
                const int rs = huff_decode(b, ac[c.ta]);
                const int r = rs >> 4, s = rs & 15;
                if (s == 0) {
                    if (r != 15) break;
                    k += 16;
                    continue;
                }
                k += r;
                if (k > 63) bad("AC coefficient index beyond 63");
                blk[kZigzag[k]] = (int16_t)extend(b.get(s), s);
                ++k;
            }
            return;
        }
        if (ss == 0) {  // DC scans
            if (ah == 0) {
                const int t = huff_decode(b, dc[c.td]);
                if (t > 11) bad("bad DC magnitude");
                c.dc_pred += extend(b.get(t), t);
                blk[0] = (int16_t)(c.dc_pred * (1 << al));
            } else if (b.bit()) {
                blk[0] = (int16_t)(blk[0] | (1 << al));
            }
            return;
        }
        if (ah == 0) {  // AC first pass
            if (eobrun > 0) {
                --eobrun;
                return;
            }
            for (int k = ss; k <= se;) {
                const int rs = huff_decode(b, ac[c.ta]);
                const int r = rs >> 4, s = rs & 15;
                if (s == 0) {
                    if (r < 15) {
                        eobrun = (1 << r) - 1;
                        if (r) eobrun += b.get(r);
                        break;
                    }
                    k += 16;
                    continue;
                }
                k += r;
                if (k > 63) bad("AC coefficient index beyond 63");
                blk[kZigzag[k]] = (int16_t)(extend(b.get(s), s) * (1 << al));
                ++k;
            }
            return;
        }
        // AC refinement: one more bit of every coefficient already non-zero
        // in the band, and new coefficients of magnitude 1 << al placed after
        // runs of still-zero ones
        const int p1 = 1 << al, m1 = -(1 << al);
        auto refine = [&](int16_t &v) {
            if (b.bit() && (v & p1) == 0) v = (int16_t)(v + (v >= 0 ? p1 : m1));
        };
        int k = ss;
        if (eobrun == 0) {
            for (; k <= se; ++k) {
                const int rs = huff_decode(b, ac[c.ta]);
                int r = rs >> 4;
                const int s = rs & 15;
                int val = 0;
                if (s) {
                    if (s != 1) bad("bad refinement magnitude");
                    val = b.bit() ? p1 : m1;
                } else if (r != 15) {
                    eobrun = 1 << r;
                    if (r) eobrun += b.get(r);
                    break;
                }
                while (k <= se) {
                    int16_t &v = blk[kZigzag[k]];
                    if (v != 0) {
                        refine(v);
                    } else {
                        if (r == 0) {
                            if (val) v = (int16_t)val;
                            break;
                        }
                        --r;
                    }
                    ++k;
                }
            }
        }
        if (eobrun > 0) {
            for (; k <= se; ++k) {
                int16_t &v = blk[kZigzag[k]];
                if (v != 0) refine(v);
            }
            --eobrun;
        }
    }

    void parse() {
        if (u16() != 0xFFD8) bad("missing start-of-image marker");
        bool scans = false;
        while (true) {
            int m = u8();
            if (m != 0xFF) bad("expected a marker");
            while ((m = u8()) == 0xFF) {
            }
            if (m == 0xD9) break;                          // EOI
            if (m >= 0xD0 && m <= 0xD7) continue;          // stray RST
            const size_t start = pos;
            const int len = u16();
            if (len < 2 || start + len > f.size()) bad("bad segment length");
            const size_t end = start + len;
            switch (m) {
                case 0xDB: read_dqt(end); break;
                case 0xC4: read_dht(end); break;
                case 0xC0:
                case 0xC1:
                case 0xC2: read_sof(m); break;
                case 0xDD:
                    restart = u16();
                    break;
                case 0xDA:
                    read_scan(end);
                    scans = true;
                    continue;  // pos already after the entropy data
                case 0xEE:
                    if (len >= 14 && std::memcmp(&f[start + 2], "Adobe", 5) == 0) {
                        adobe = true;
                        adobe_transform = f[start + 13];
                    }
                    break;
                default:
                    if ((m >= 0xC3 && m <= 0xCF) && m != 0xC4 && m != 0xC8 && m != 0xCC)
                        bad("unsupported coding process (lossless, hierarchical or arithmetic)");
                    break;  // APPn, COM and others: skipped
            }
            pos = end;
            if (pos >= f.size()) break;
        }
        if (!frame || !scans) bad("no image data");
    }

    void finish(HostTexture &t) {
        // dequantise + inverse DCT into per-component planes
        // cosk[x][u] = C(u) cos((2x + 1) u pi / 16) / 2, C(0) = 1/sqrt(2)
        double cosk[8][8];
        for (int x = 0; x < 8; ++x)
            for (int u = 0; u < 8; ++u)
                cosk[x][u] = (u == 0 ? std::sqrt(0.5) : 1.0) * std::cos((2 * x + 1) * u * M_PI / 16.0) / 2.0;
        std::vector<std::vector<uint8_t>> planes(comps.size());
        for (size_t ci = 0; ci < comps.size(); ++ci) {
            Component &c = comps[ci];
            if (!qt_present[c.tq]) bad("component uses an undefined quantisation table");
            const int pw = c.bw * 8, ph = c.bh * 8;
            planes[ci].assign((size_t)pw * ph, 0);
            double in[64], tmp[64];
            for (int by = 0; by < c.bh; ++by)
                for (int bx = 0; bx < c.bw; ++bx) {
                    const int16_t *blk = &c.coef[((size_t)by * c.bw + bx) * 64];
                    for (int i = 0; i < 64; ++i) in[i] = (double)blk[i] * qt[c.tq][i];
                    for (int y = 0; y < 8; ++y)  // rows: inverse over u for each v row
                        for (int x = 0; x < 8; ++x) {
                            double s = 0.0;
                            for (int u = 0; u < 8; ++u) s += cosk[x][u] * in[y * 8 + u];
                            tmp[y * 8 + x] = s;
                        }
                    for (int x = 0; x < 8; ++x)
                        for (int y = 0; y < 8; ++y) {
                            double s = 0.0;
                            for (int v = 0; v < 8; ++v) s += cosk[y][v] * tmp[v * 8 + x];
                            const long q = std::lround(s + 128.0);
                            planes[ci][(size_t)(by * 8 + y) * pw + bx * 8 + x] = (uint8_t)std::min(255L, std::max(0L, q));
                        }
                }
        }
        // upsample every component to the full image
        std::vector<std::vector<uint8_t>> full(comps.size());
        for (size_t ci = 0; ci < comps.size(); ++ci) {
            const Component &c = comps[ci];
            const int pw = c.bw * 8;
            const int sx = hmax / c.h, sy = vmax / c.v;
            const std::vector<uint8_t> &p = planes[ci];
            std::vector<uint8_t> &o = full[ci];
            o.assign((size_t)width * height, 0);
            auto at = [&](int x, int y) -> int {
                x = std::min(std::max(x, 0), c.cw - 1);
                y = std::min(std::max(y, 0), c.ch - 1);
                return p[(size_t)y * pw + x];
            };
            for (int y = 0; y < height; ++y)
                for (int x = 0; x < width; ++x) {
                    int val;
                    if (sx == 1 && sy == 1) {
                        val = at(x, y);
                    } else if (sx == 2 && sy == 1) {
                        const int n = x >> 1, far = (x & 1) ? n + 1 : n - 1;
                        val = (3 * at(n, y) + at(far, y) + 2) >> 2;
                    } else if (sx == 1 && sy == 2) {
                        const int n = y >> 1, far = (y & 1) ? n + 1 : n - 1;
                        val = (3 * at(x, n) + at(x, far) + 2) >> 2;
                    } else if (sx == 2 && sy == 2) {
                        const int nx = x >> 1, fx = (x & 1) ? nx + 1 : nx - 1;
                        const int ny = y >> 1, fy = (y & 1) ? ny + 1 : ny - 1;
                        const int near_col = 3 * at(nx, ny) + at(nx, fy);
                        const int far_col = 3 * at(fx, ny) + at(fx, fy);
                        val = (3 * near_col + far_col + 8) >> 4;
                    } else {
                        val = at(x / sx, y / sy);
                    }
                    o[(size_t)y * width + x] = (uint8_t)val;
                }
        }
        t.width = width;
        t.height = height;
        t.rgba.assign((size_t)width * height * 4, 255);
        const bool rgb = comps.size() == 3 &&
                         ((adobe && adobe_transform == 0) ||
                          (comps[0].id == 'R' && comps[1].id == 'G' && comps[2].id == 'B'));
        for (size_t i = 0; i < (size_t)width * height; ++i) {
            uint8_t *px = &t.rgba[i * 4];
            if (comps.size() == 1) {
                px[0] = px[1] = px[2] = full[0][i];
            } else if (rgb) {
                px[0] = full[0][i];
                px[1] = full[1][i];
                px[2] = full[2][i];
            } else {
                const double y = full[0][i], cb = full[1][i] - 128.0, cr = full[2][i] - 128.0;
                const double rgbv[3] = {y + 1.402 * cr, y - 0.344136 * cb - 0.714136 * cr, y + 1.772 * cb};
                for (int k = 0; k < 3; ++k)
                    px[k] = (uint8_t)std::min(255L, std::max(0L, std::lround(rgbv[k])));
            }
        }
    }
};

}  // namespace

void decode_jpeg(const std::vector<uint8_t> &f, HostTexture &t) {
    Decoder d(f);
    d.parse();
    d.finish(t);
}

}  // namespace crt
