// Image decoding for diffuse textures: PNG (zlib/deflate per RFC 1950/1951,
// the PNG row filters and colour types) and binary PPM, to 8-bit RGBA with
// rows top-down. This is what the reference's texture loader hands to its
// uchar4 CUDA array (Texture::Load, Src/Core/texture.cu:207-240, through
// stbi_load with 4 requested channels): 16-bit samples keep their high byte,
// low-bit-depth grey is scaled to 0..255, palette entries expand with their
// tRNS alpha, absent alpha is 255. JPEG is decoded in jpeg.cpp. Interlaced
// PNGs and other formats are refused with a message (the scene loader then
// keeps the basecolor).
#include "scene_data.h"
#include "common.cuh"
#include <algorithm>
#include <cctype>
#include <cstring>
#include <fstream>
#include <iterator>

namespace crt {
namespace {

// ---------------------------------------------------------------------------
// inflate
// ---------------------------------------------------------------------------

struct BitReader {
    const uint8_t *p;
    size_t n, pos = 0;
    uint32_t bitbuf = 0;
    int bitcnt = 0;
    BitReader(const uint8_t *d, size_t len) : p(d), n(len) {}
    int bit() {
        if (bitcnt == 0) {
            if (pos >= n) throw Error(CRT_ERR_PARSE, "PNG: truncated deflate stream");
            bitbuf = p[pos++];
            bitcnt = 8;
        }
        int b = bitbuf & 1;
        bitbuf >>= 1;
        --bitcnt;
        return b;
    }
    uint32_t bits(int k) {  // LSB first
        uint32_t v = 0;
        for (int i = 0; i < k; ++i) v |= (uint32_t)bit() << i;
        return v;
    }
    void align() { bitcnt = 0; }
};

// Canonical Huffman code: counts per length and symbols in code order.
struct Huffman {
    uint16_t count[16] = {};
    std::vector<uint16_t> symbol;
    void build(const uint8_t *lengths, int n) {
        std::memset(count, 0, sizeof(count));
        for (int i = 0; i < n; ++i) count[lengths[i]]++;
        count[0] = 0;
        uint16_t offs[16];
        offs[1] = 0;
        for (int len = 1; len < 15; ++len) offs[len + 1] = offs[len] + count[len];
        symbol.assign(n, 0);
        for (int i = 0; i < n; ++i)
            if (lengths[i]) symbol[offs[lengths[i]]++] = (uint16_t)i;
    }
    int decode(BitReader &br) const {
        int code = 0, first = 0, index = 0;
        for (int len = 1; len <= 15; ++len) {
            code |= br.bit();
            const int c = count[len];
            if (code - first < c) return symbol[index + (code - first)];
            index += c;
            first = (first + c) << 1;
            code <<= 1;
        }
        throw Error(CRT_ERR_PARSE, "PNG: bad Huffman code");
    }
};

const uint16_t kLenBase[29] = {3,  4,  5,  6,  7,  8,  9,  10, 11,  13,  15,  17,  19,  23, 27,
                               31, 35, 43, 51, 59, 67, 83, 99, 115, 131, 163, 195, 227, 258};
const uint8_t kLenExtra[29] = {0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 2, 2, 2, 2, 3, 3, 3, 3, 4, 4, 4, 4, 5, 5, 5, 5, 0};
const uint16_t kDistBase[30] = {1,   2,   3,   4,   5,   7,    9,    13,   17,   25,   33,   49,   65,    97,    129,
                                193, 257, 385, 513, 769, 1025, 1537, 2049, 3073, 4097, 6145, 8193, 12289, 16385, 24577};
const uint8_t kDistExtra[30] = {0, 0, 0, 0, 1, 1, 2, 2, 3, 3, 4, 4, 5, 5, 6, 6, 7, 7, 8, 8, 9, 9, 10, 10, 11, 11, 12, 12, 13, 13};

void inflate_codes(BitReader &br, const Huffman &lit, const Huffman &dist, std::vector<uint8_t> &out) {
    for (;;) {
        int sym = lit.decode(br);
        if (sym < 256) {
            out.push_back((uint8_t)sym);
        } else if (sym == 256) {
            return;
        } else {
            sym -= 257;
            if (sym >= 29) throw Error(CRT_ERR_PARSE, "PNG: bad length symbol");
            const size_t len = kLenBase[sym] + br.bits(kLenExtra[sym]);
            const int ds = dist.decode(br);
            if (ds >= 30) throw Error(CRT_ERR_PARSE, "PNG: bad distance symbol");
            const size_t d = kDistBase[ds] + br.bits(kDistExtra[ds]);
            if (d > out.size()) throw Error(CRT_ERR_PARSE, "PNG: distance before the start of the data");
            const size_t from = out.size() - d;
            for (size_t k = 0; k < len; ++k) out.push_back(out[from + k]);
        }
    }
}

std::vector<uint8_t> zlib_inflate(const std::vector<uint8_t> &z, size_t expected) {
    if (z.size() < 2 || (z[0] & 0x0F) != 8 || ((z[0] << 8) | z[1]) % 31 != 0)
        throw Error(CRT_ERR_PARSE, "PNG: bad zlib header");
    if (z[1] & 0x20) throw Error(CRT_ERR_PARSE, "PNG: zlib preset dictionary");
    BitReader br(z.data() + 2, z.size() - 2);
    std::vector<uint8_t> out;
    out.reserve(expected);
    int final = 0;
    while (!final) {
        final = br.bit();
        const int type = (int)br.bits(2);
        if (type == 0) {
            br.align();
            if (br.pos + 4 > br.n) throw Error(CRT_ERR_PARSE, "PNG: truncated stored block");
            const uint32_t len = br.p[br.pos] | (br.p[br.pos + 1] << 8);
            const uint32_t nlen = br.p[br.pos + 2] | (br.p[br.pos + 3] << 8);
            br.pos += 4;
            if ((len ^ 0xFFFFu) != nlen || br.pos + len > br.n) throw Error(CRT_ERR_PARSE, "PNG: bad stored block");
            out.insert(out.end(), br.p + br.pos, br.p + br.pos + len);
            br.pos += len;
        } else if (type == 1) {
            uint8_t l[288], d[30];
            for (int i = 0; i < 288; ++i) l[i] = i < 144 ? 8 : (i < 256 ? 9 : (i < 280 ? 7 : 8));
            for (int i = 0; i < 30; ++i) d[i] = 5;
            Huffman lit, dist;
            lit.build(l, 288);
            dist.build(d, 30);
            inflate_codes(br, lit, dist, out);
        } else if (type == 2) {
            const int hlit = (int)br.bits(5) + 257, hdist = (int)br.bits(5) + 1, hclen = (int)br.bits(4) + 4;
            static const uint8_t order[19] = {16, 17, 18, 0, 8, 7, 9, 6, 10, 5, 11, 4, 12, 3, 13, 2, 14, 1, 15};
            uint8_t cl[19] = {};
            for (int i = 0; i < hclen; ++i) cl[order[i]] = (uint8_t)br.bits(3);
            Huffman clh;
            clh.build(cl, 19);
            uint8_t lens[320] = {};
            int k = 0;
            while (k < hlit + hdist) {
                const int sym = clh.decode(br);
                if (sym < 16) {
                    lens[k++] = (uint8_t)sym;
                } else {
                    int rep = 0;
                    uint8_t val = 0;
                    if (sym == 16) {
                        if (k == 0) throw Error(CRT_ERR_PARSE, "PNG: repeat with no previous length");
                        val = lens[k - 1];
                        rep = 3 + (int)br.bits(2);
                    } else if (sym == 17) {
                        rep = 3 + (int)br.bits(3);
                    } else {
                        rep = 11 + (int)br.bits(7);
                    }
                    if (k + rep > hlit + hdist) throw Error(CRT_ERR_PARSE, "PNG: code lengths overflow");
                    for (int r = 0; r < rep; ++r) lens[k++] = val;
                }
            }
            Huffman lit, dist;
            lit.build(lens, hlit);
            dist.build(lens + hlit, hdist);
            inflate_codes(br, lit, dist, out);
        } else {
            throw Error(CRT_ERR_PARSE, "PNG: reserved deflate block type");
        }
    }
    return out;
}

uint32_t be32(const uint8_t *p) { return ((uint32_t)p[0] << 24) | ((uint32_t)p[1] << 16) | ((uint32_t)p[2] << 8) | p[3]; }

int paeth(int a, int b, int c) {
    const int p = a + b - c, pa = p > a ? p - a : a - p, pb = p > b ? p - b : b - p, pc = p > c ? p - c : c - p;
    if (pa <= pb && pa <= pc) return a;
    return pb <= pc ? b : c;
}

void decode_png(const std::vector<uint8_t> &f, HostTexture &t) {
    static const uint8_t sig[8] = {137, 80, 78, 71, 13, 10, 26, 10};
    if (f.size() < 8 || std::memcmp(f.data(), sig, 8) != 0) throw Error(CRT_ERR_PARSE, "not a PNG file");
    size_t pos = 8;
    int w = 0, h = 0, depth = 0, ctype = -1, interlace = 0;
    std::vector<uint8_t> idat, plte, trns;
    bool have_hdr = false;
    while (pos + 8 <= f.size()) {
        const uint32_t len = be32(&f[pos]);
        const char *type = (const char *)&f[pos + 4];
        if (pos + 12 + (size_t)len > f.size()) throw Error(CRT_ERR_PARSE, "PNG: truncated chunk");
        const uint8_t *d = &f[pos + 8];
        if (!std::memcmp(type, "IHDR", 4)) {
            if (len < 13) throw Error(CRT_ERR_PARSE, "PNG: short IHDR");
            w = (int)be32(d);
            h = (int)be32(d + 4);
            depth = d[8];
            ctype = d[9];
            interlace = d[12];
            have_hdr = true;
        } else if (!std::memcmp(type, "PLTE", 4)) {
            plte.assign(d, d + len);
        } else if (!std::memcmp(type, "tRNS", 4)) {
            trns.assign(d, d + len);
        } else if (!std::memcmp(type, "IDAT", 4)) {
            idat.insert(idat.end(), d, d + len);
        } else if (!std::memcmp(type, "IEND", 4)) {
            break;
        }
        pos += 12 + len;
    }
    if (!have_hdr || w <= 0 || h <= 0 || w > (1 << 15) || h > (1 << 15)) throw Error(CRT_ERR_PARSE, "PNG: bad IHDR");
    if (interlace) throw Error(CRT_ERR_PARSE, "PNG: interlaced images are not supported");
    int channels;
    switch (ctype) {
        case 0: channels = 1; break;
        case 2: channels = 3; break;
        case 3: channels = 1; break;
        case 4: channels = 2; break;
        case 6: channels = 4; break;
        default: throw Error(CRT_ERR_PARSE, "PNG: bad colour type");
    }
    const bool ok_depth = depth == 8 || depth == 16 || ((ctype == 0 || ctype == 3) && (depth == 1 || depth == 2 || depth == 4));
    if (!ok_depth || (ctype == 3 && depth == 16)) throw Error(CRT_ERR_PARSE, "PNG: unsupported bit depth");
    const size_t bits_pp = (size_t)channels * depth;
    const size_t row_bytes = ((size_t)w * bits_pp + 7) / 8;
    const size_t bpp = std::max<size_t>(1, bits_pp / 8);  // filter byte distance
    std::vector<uint8_t> raw = zlib_inflate(idat, (row_bytes + 1) * h);
    if (raw.size() < (row_bytes + 1) * (size_t)h) throw Error(CRT_ERR_PARSE, "PNG: image data too short");
    std::vector<uint8_t> img((size_t)h * row_bytes);
    for (int y = 0; y < h; ++y) {
        const uint8_t ft = raw[(size_t)y * (row_bytes + 1)];
        const uint8_t *src = &raw[(size_t)y * (row_bytes + 1) + 1];
        uint8_t *cur = &img[(size_t)y * row_bytes];
        const uint8_t *prev = y > 0 ? &img[(size_t)(y - 1) * row_bytes] : nullptr;
        for (size_t x = 0; x < row_bytes; ++x) {
            const int a = x >= bpp ? cur[x - bpp] : 0, b = prev ? prev[x] : 0, c = (prev && x >= bpp) ? prev[x - bpp] : 0;
            int v = src[x];
            switch (ft) {
                case 0: break;
                case 1: v += a; break;
                case 2: v += b; break;
                case 3: v += (a + b) >> 1; break;
                case 4: v += paeth(a, b, c); break;
                default: throw Error(CRT_ERR_PARSE, "PNG: bad row filter");
            }
            cur[x] = (uint8_t)v;
        }
    }
    t.width = w;
    t.height = h;
    t.rgba.assign((size_t)w * h * 4, 255);
    auto sample = [&](const uint8_t *row, int x, int ch) -> int {  // channel value, 8-bit or high byte
        if (depth == 16) return row[(size_t)(x * channels + ch) * 2];
        if (depth == 8) return row[(size_t)x * channels + ch];
        const int per = 8 / depth, byte = row[x / per], shift = (per - 1 - x % per) * depth;
        return (byte >> shift) & ((1 << depth) - 1);
    };
    static const int scale_low[9] = {0, 0xff, 0x55, 0, 0x11, 0, 0, 0, 0x01};
    for (int y = 0; y < h; ++y) {
        const uint8_t *row = &img[(size_t)y * row_bytes];
        for (int x = 0; x < w; ++x) {
            uint8_t *o = &t.rgba[((size_t)y * w + x) * 4];
            if (ctype == 3) {
                const int i = sample(row, x, 0);
                if ((size_t)i * 3 + 2 >= plte.size()) throw Error(CRT_ERR_PARSE, "PNG: palette index out of range");
                o[0] = plte[i * 3];
                o[1] = plte[i * 3 + 1];
                o[2] = plte[i * 3 + 2];
                o[3] = (size_t)i < trns.size() ? trns[i] : 255;
            } else if (ctype == 0 || ctype == 4) {
                int g = sample(row, x, 0);
                if (depth < 8) g *= scale_low[depth];
                o[0] = o[1] = o[2] = (uint8_t)g;
                if (ctype == 4) o[3] = (uint8_t)sample(row, x, 1);
            } else {
                for (int k = 0; k < 3; ++k) o[k] = (uint8_t)sample(row, x, k);
                if (ctype == 6) o[3] = (uint8_t)sample(row, x, 3);
            }
        }
    }
}

// Binary PPM (P6, maxval <= 255).
void decode_ppm(const std::vector<uint8_t> &f, HostTexture &t) {
    size_t pos = 2;
    auto next_int = [&]() {
        for (;;) {
            while (pos < f.size() && isspace(f[pos])) ++pos;
            if (pos < f.size() && f[pos] == '#') {
                while (pos < f.size() && f[pos] != '\n') ++pos;
                continue;
            }
            break;
        }
        int v = 0;
        bool any = false;
        while (pos < f.size() && isdigit(f[pos])) {
            v = v * 10 + (f[pos++] - '0');
            any = true;
            if (v > (1 << 20)) break;
        }
        if (!any) throw Error(CRT_ERR_PARSE, "PPM: bad header");
        return v;
    };
    const int w = next_int(), h = next_int(), maxv = next_int();
    ++pos;  // single whitespace before the raster
    if (w <= 0 || h <= 0 || w > (1 << 15) || h > (1 << 15) || maxv <= 0 || maxv > 255)
        throw Error(CRT_ERR_PARSE, "PPM: unsupported header");
    if (pos + (size_t)w * h * 3 > f.size()) throw Error(CRT_ERR_PARSE, "PPM: truncated raster");
    t.width = w;
    t.height = h;
    t.rgba.assign((size_t)w * h * 4, 255);
    for (size_t i = 0; i < (size_t)w * h; ++i)
        for (int k = 0; k < 3; ++k) t.rgba[i * 4 + k] = (uint8_t)(f[pos + i * 3 + k] * 255 / maxv);
}

}  // namespace

void decode_jpeg(const std::vector<uint8_t> &f, HostTexture &t);  // jpeg.cpp

void load_texture_image(const std::string &path, HostTexture &t) {
    std::ifstream in(path, std::ios::binary);
    if (!in) throw Error(CRT_ERR_IO, "cannot open texture " + path);
    std::vector<uint8_t> f((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
    if (f.size() >= 8 && f[0] == 137 && f[1] == 'P' && f[2] == 'N' && f[3] == 'G')
        decode_png(f, t);
    else if (f.size() >= 2 && f[0] == 'P' && f[1] == '6')
        decode_ppm(f, t);
    else if (f.size() >= 3 && f[0] == 0xFF && f[1] == 0xD8 && f[2] == 0xFF)
        decode_jpeg(f, t);
    else
        throw Error(CRT_ERR_PARSE, "unsupported texture format (PNG, JPEG and binary PPM are decoded): " + path);
}

}  // namespace crt

extern "C" crt_status crt_image_decode(const char *path, int32_t *w, int32_t *h, uint8_t *rgba) {
    try {
        CRT_CHECK(path && w && h, CRT_ERR_INVALID, "crt_image_decode: null argument");
        crt::HostTexture t;
        crt::load_texture_image(path, t);
        *w = t.width;
        *h = t.height;
        if (rgba) std::memcpy(rgba, t.rgba.data(), t.rgba.size());
        crt::set_last_error("");
        return CRT_OK;
    } catch (const crt::Error &e) {
        crt::set_last_error(e.what());
        return e.status;
    } catch (const std::exception &e) {
        crt::set_last_error(e.what());
        return CRT_ERR_INVALID;
    }
}
