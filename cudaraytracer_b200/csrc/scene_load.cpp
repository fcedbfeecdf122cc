// Scene loader: the reference's scene JSON schema and semantics, its OBJ
// import rules and Radiance HDR environment maps, parsed with a small JSON
// reader, an OBJ reader and an RGBE decoder written for this library.
//
// Reference behaviour reproduced (Src/Core/scene.cpp, Src/Utils/objloader.cpp):
//  * camera block: type must be "pinhole"; resolution, fov (vertical,
//    degrees), max_bounces (default 5), rr (0.8), spp (16), direction
//    (0,0,-1), denoise (false)                               scene.cpp:187-252
//  * materials: diffuse | light | pbr | subsurface | dielectric | glass with
//    the per-type defaults; unknown types are skipped          scene.cpp:254-396
//  * objects: transform = T * R * S, rotations pre-multiplied in list order;
//    one mesh per (OBJ shape, OBJ material); material resolution order
//    "material" -> "material_overrides" -> OBJ material name ->
//    "default_material"; meshes without a valid material are skipped;
//    mesh names "<object>" or "<object>::<shape>[::<mtl>]"    scene.cpp:12-48, 398-537
//  * OBJ: positions T*p, normals (T^-1)^T*n normalised; a face lacking any
//    vn gets the face normal on all three vertices            objloader.cpp:10-50, 185-198
//  * lights: "area" (lightMeshName, emission from the named material's ke
//    or "ke") and "env" (path to an HDR image)                 scene.cpp:539-616
#include "scene_data.h"
#include "common.cuh"
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <memory>
#include <sstream>
#include <array>
#include <unordered_map>

namespace crt {
namespace {

// ---------------------------------------------------------------------------
// JSON
// ---------------------------------------------------------------------------
struct Json {
    enum Kind { NUL, BOOL, NUM, STR, ARR, OBJ } kind = NUL;
    bool b = false;
    double num = 0;
    std::string str;
    std::vector<Json> arr;
    std::vector<std::pair<std::string, Json>> obj;

    bool has(const std::string &k) const {
        if (kind != OBJ) return false;
        for (auto &kv : obj)
            if (kv.first == k) return true;
        return false;
    }
    const Json &operator[](const std::string &k) const {
        static const Json null;
        if (kind == OBJ)
            for (auto &kv : obj)
                if (kv.first == k) return kv.second;
        return null;
    }
    double number(const char *what) const {
        if (kind == NUM) return num;
        if (kind == BOOL) return b ? 1.0 : 0.0;
        throw Error(CRT_ERR_PARSE, std::string("expected a number for ") + what);
    }
    const std::string &string(const char *what) const {
        if (kind != STR) throw Error(CRT_ERR_PARSE, std::string("expected a string for ") + what);
        return str;
    }
};

class JsonParser {
   public:
    explicit JsonParser(const std::string &s) : s_(s) {}
    Json parse() {
        Json v = value();
        ws();
        if (i_ != s_.size()) fail("trailing characters");
        return v;
    }

   private:
    const std::string &s_;
    size_t i_ = 0;
    [[noreturn]] void fail(const char *m) {
        throw Error(CRT_ERR_PARSE, std::string("JSON: ") + m + " at offset " + std::to_string(i_));
    }
    void ws() {
        while (i_ < s_.size() && std::isspace((unsigned char)s_[i_])) ++i_;
    }
    bool lit(const char *w) {
        size_t n = std::strlen(w);
        if (s_.compare(i_, n, w) == 0) {
            i_ += n;
            return true;
        }
        return false;
    }
    Json value() {
        ws();
        if (i_ >= s_.size()) fail("unexpected end");
        char c = s_[i_];
        Json v;
        if (c == '{') {
            v.kind = Json::OBJ;
            ++i_;
            ws();
            if (i_ < s_.size() && s_[i_] == '}') {
                ++i_;
                return v;
            }
            for (;;) {
                ws();
                if (i_ >= s_.size() || s_[i_] != '"') fail("expected key");
                std::string k = str();
                ws();
                if (i_ >= s_.size() || s_[i_] != ':') fail("expected ':'");
                ++i_;
                v.obj.emplace_back(k, value());
                ws();
                if (i_ < s_.size() && s_[i_] == ',') {
                    ++i_;
                    continue;
                }
                if (i_ < s_.size() && s_[i_] == '}') {
                    ++i_;
                    return v;
                }
                fail("expected ',' or '}'");
            }
        }
        if (c == '[') {
            v.kind = Json::ARR;
            ++i_;
            ws();
            if (i_ < s_.size() && s_[i_] == ']') {
                ++i_;
                return v;
            }
            for (;;) {
                v.arr.push_back(value());
                ws();
                if (i_ < s_.size() && s_[i_] == ',') {
                    ++i_;
                    continue;
                }
                if (i_ < s_.size() && s_[i_] == ']') {
                    ++i_;
                    return v;
                }
                fail("expected ',' or ']'");
            }
        }
        if (c == '"') {
            v.kind = Json::STR;
            v.str = str();
            return v;
        }
        if (lit("true")) {
            v.kind = Json::BOOL;
            v.b = true;
            return v;
        }
        if (lit("false")) {
            v.kind = Json::BOOL;
            return v;
        }
        if (lit("null")) return v;
        const char *start = s_.c_str() + i_;
        char *end = nullptr;
        v.num = std::strtod(start, &end);
        if (end == start) fail("bad value");
        v.kind = Json::NUM;
        i_ += end - start;
        return v;
    }
    std::string str() {
        ++i_;  // opening quote
        std::string out;
        while (i_ < s_.size() && s_[i_] != '"') {
            char c = s_[i_++];
            if (c == '\\') {
                if (i_ >= s_.size()) fail("bad escape");
                char e = s_[i_++];
                switch (e) {
                    case 'n': out += '\n'; break;
                    case 't': out += '\t'; break;
                    case 'r': out += '\r'; break;
                    case 'b': out += '\b'; break;
                    case 'f': out += '\f'; break;
                    case 'u': {
                        if (i_ + 4 > s_.size()) fail("bad \\u escape");
                        unsigned cp = std::strtoul(s_.substr(i_, 4).c_str(), nullptr, 16);
                        i_ += 4;
                        if (cp < 0x80) {
                            out += (char)cp;
                        } else if (cp < 0x800) {
                            out += (char)(0xC0 | (cp >> 6));
                            out += (char)(0x80 | (cp & 0x3F));
                        } else {
                            out += (char)(0xE0 | (cp >> 12));
                            out += (char)(0x80 | ((cp >> 6) & 0x3F));
                            out += (char)(0x80 | (cp & 0x3F));
                        }
                        break;
                    }
                    default: out += e;
                }
            } else {
                out += c;
            }
        }
        if (i_ >= s_.size()) fail("unterminated string");
        ++i_;
        return out;
    }
};

std::string read_file(const std::string &path) {
    std::ifstream f(path, std::ios::binary);
    if (!f) throw Error(CRT_ERR_IO, "cannot open " + path);
    std::ostringstream ss;
    ss << f.rdbuf();
    return ss.str();
}

// ---------------------------------------------------------------------------
// 4x4 transforms (row-major), evaluated in double and rounded to float.
// ---------------------------------------------------------------------------
struct M4 {
    double m[4][4];
    static M4 identity() {
        M4 r{};
        for (int i = 0; i < 4; ++i) r.m[i][i] = 1;
        return r;
    }
    M4 operator*(const M4 &b) const {
        M4 r{};
        for (int i = 0; i < 4; ++i)
            for (int j = 0; j < 4; ++j)
                for (int k = 0; k < 4; ++k) r.m[i][j] += m[i][k] * b.m[k][j];
        return r;
    }
};

// Angle conversion as AngleToRadian (Src/Utils/mathutil.cu:4-7), PI = 3.1415926.
double deg2rad(float a) { return (float)(a / 180.0f * 3.1415926); }

M4 rot(int axis, float deg) {
    double r = deg2rad(deg), c = (float)std::cos((float)r), s = (float)std::sin((float)r);
    M4 m = M4::identity();
    int a = (axis + 1) % 3, b = (axis + 2) % 3;
    if (axis == 1) {  // RotateY: (0,0)=c (0,2)=s (2,0)=-s (2,2)=c
        m.m[0][0] = c; m.m[0][2] = s; m.m[2][0] = -s; m.m[2][2] = c;
    } else {
        m.m[a][a] = c; m.m[a][b] = -s; m.m[b][a] = s; m.m[b][b] = c;
    }
    return m;
}

bool invert(const M4 &a, M4 &inv) {
    double m[4][8];
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 8; ++j) m[i][j] = j < 4 ? a.m[i][j] : (j - 4 == i ? 1 : 0);
    for (int c = 0; c < 4; ++c) {
        int p = c;
        for (int r = c + 1; r < 4; ++r)
            if (std::fabs(m[r][c]) > std::fabs(m[p][c])) p = r;
        if (std::fabs(m[p][c]) < 1e-300) return false;
        for (int j = 0; j < 8; ++j) std::swap(m[c][j], m[p][j]);
        double d = m[c][c];
        for (int j = 0; j < 8; ++j) m[c][j] /= d;
        for (int r = 0; r < 4; ++r)
            if (r != c) {
                double f = m[r][c];
                for (int j = 0; j < 8; ++j) m[r][j] -= f * m[c][j];
            }
    }
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) inv.m[i][j] = m[i][j + 4];
    return true;
}

bool is_identity(const M4 &m) {
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j)
            if (m.m[i][j] != (i == j ? 1.0 : 0.0)) return false;
    return true;
}

// float vector helpers with single rounding per operation (same order as
// the reference's Eigen expressions).
inline void fcross(const float *a, const float *b, float *o) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}
inline float fdot(const float *a, const float *b) { return a[0] * b[0] + (a[1] * b[1] + a[2] * b[2]); }
inline void fnormalize(float *v) {
    float z = fdot(v, v);
    if (z > 0.f) {
        float s = std::sqrt(z);
        v[0] /= s;
        v[1] /= s;
        v[2] /= s;
    }
}

// ---------------------------------------------------------------------------
// OBJ
// ---------------------------------------------------------------------------
struct ObjMesh {
    std::string name, material;
    std::vector<float> verts, normals, uvs;
};

std::string dir_of(const std::string &p) {
    size_t k = p.find_last_of('/');
    return k == std::string::npos ? "" : p.substr(0, k + 1);
}
std::string stem_of(const std::string &p) {
    size_t k = p.find_last_of('/');
    std::string f = k == std::string::npos ? p : p.substr(k + 1);
    size_t d = f.find_last_of('.');
    return (d != std::string::npos && d > 0) ? f.substr(0, d) : f;
}

void load_mtl_names(const std::string &path, std::vector<std::string> &names) {
    std::ifstream f(path);
    if (!f) return;
    std::string line;
    while (std::getline(f, line)) {
        std::istringstream ls(line);
        std::string tag;
        ls >> tag;
        if (tag == "newmtl") {
            std::string n;
            std::getline(ls >> std::ws, n);
            while (!n.empty() && (n.back() == '\r' || n.back() == ' ')) n.pop_back();
            names.push_back(n);
        }
    }
}

std::vector<ObjMesh> load_obj(const std::string &path, const M4 &T, const M4 &Tinv, bool identity) {
    std::ifstream f(path);
    if (!f) throw Error(CRT_ERR_IO, "cannot open OBJ " + path);
    std::vector<float> P, N, UV;
    std::vector<std::string> mtl_names;
    struct Face {
        int v[3], t[3], n[3];
    };
    struct Shape {
        std::string name;
        std::vector<Face> faces;
        std::vector<int> mat;
    };
    std::vector<Shape> shapes(1);
    int cur_mat = -1;
    std::string line;
    auto resolve = [](long i, size_t n) -> int {
        if (i > 0) return (int)(i - 1);
        if (i < 0) return (int)((long)n + i);
        return -1;
    };
    while (std::getline(f, line)) {
        if (!line.empty() && line.back() == '\r') line.pop_back();
        const char *s = line.c_str();
        while (*s == ' ' || *s == '\t') ++s;
        if (s[0] == 'v' && (s[1] == ' ' || s[1] == '\t')) {
            float x = 0, y = 0, z = 0;
            std::sscanf(s + 2, "%f %f %f", &x, &y, &z);
            P.push_back(x); P.push_back(y); P.push_back(z);
        } else if (s[0] == 'v' && s[1] == 'n') {
            float x = 0, y = 0, z = 0;
            std::sscanf(s + 3, "%f %f %f", &x, &y, &z);
            N.push_back(x); N.push_back(y); N.push_back(z);
        } else if (s[0] == 'v' && s[1] == 't') {
            float x = 0, y = 0;
            std::sscanf(s + 3, "%f %f", &x, &y);
            UV.push_back(x); UV.push_back(y);
        } else if (s[0] == 'f' && (s[1] == ' ' || s[1] == '\t')) {
            std::vector<std::array<int, 3>> corners;
            std::istringstream ls(s + 2);
            std::string tok;
            while (ls >> tok) {
                long vi = 0, ti = 0, ni = 0;
                const char *t = tok.c_str();
                char *e;
                vi = std::strtol(t, &e, 10);
                if (*e == '/') {
                    ++e;
                    if (*e != '/') ti = std::strtol(e, &e, 10);
                    if (*e == '/') ni = std::strtol(e + 1, &e, 10);
                }
                corners.push_back({resolve(vi, P.size() / 3), resolve(ti, UV.size() / 2), resolve(ni, N.size() / 3)});
            }
            for (size_t k = 1; k + 1 < corners.size(); ++k) {  // fan triangulation
                Face fc;
                const std::array<int, 3> *cs[3] = {&corners[0], &corners[k], &corners[k + 1]};
                for (int c = 0; c < 3; ++c) {
                    fc.v[c] = (*cs[c])[0];
                    fc.t[c] = (*cs[c])[1];
                    fc.n[c] = (*cs[c])[2];
                }
                shapes.back().faces.push_back(fc);
                shapes.back().mat.push_back(cur_mat);
            }
        } else if ((s[0] == 'o' || s[0] == 'g') && (s[1] == ' ' || s[1] == '\t' || s[1] == 0)) {
            std::string n = s[1] ? std::string(s + 2) : std::string();
            if (shapes.back().faces.empty())
                shapes.back().name = n;
            else {
                shapes.emplace_back();
                shapes.back().name = n;
            }
        } else if (std::strncmp(s, "usemtl", 6) == 0) {
            std::string n = s + 6;
            n.erase(0, n.find_first_not_of(" \t"));
            cur_mat = -1;
            for (size_t k = 0; k < mtl_names.size(); ++k)
                if (mtl_names[k] == n) cur_mat = (int)k;
        } else if (std::strncmp(s, "mtllib", 6) == 0) {
            std::string n = s + 6;
            n.erase(0, n.find_first_not_of(" \t"));
            load_mtl_names(dir_of(path) + n, mtl_names);
        }
    }
    // One mesh per (shape, material) in first-face order (objloader.cpp:151-178).
    std::vector<ObjMesh> meshes;
    std::unordered_map<std::string, size_t> lookup;
    for (size_t si = 0; si < shapes.size(); ++si) {
        const Shape &sh = shapes[si];
        for (size_t fi = 0; fi < sh.faces.size(); ++fi) {
            int mi = sh.mat[fi];
            std::string mname = (mi >= 0 && mi < (int)mtl_names.size()) ? mtl_names[mi] : "";
            std::string key = std::to_string(si) + ":" + std::to_string(mi);
            auto it = lookup.find(key);
            size_t idx;
            if (it == lookup.end()) {
                ObjMesh m;
                std::string shape_name = sh.name.empty() ? stem_of(path) + "_shape_" + std::to_string(si) : sh.name;
                m.name = mname.empty() ? shape_name : shape_name + "::" + mname;
                m.material = mname;
                idx = meshes.size();
                lookup[key] = idx;
                meshes.push_back(m);
            } else {
                idx = it->second;
            }
            const Face &fc = sh.faces[fi];
            float pv[3][3], nv[3][3], tv[3][2];
            bool has_n = true;
            for (int c = 0; c < 3; ++c) {
                int v = fc.v[c];
                if (v < 0 || 3 * v + 2 >= (int)P.size()) throw Error(CRT_ERR_PARSE, "OBJ face index out of range in " + path);
                double p[3] = {P[3 * v], P[3 * v + 1], P[3 * v + 2]};
                for (int k = 0; k < 3; ++k)
                    pv[c][k] = identity ? (float)p[k]
                                        : (float)(T.m[k][0] * p[0] + T.m[k][1] * p[1] + T.m[k][2] * p[2] + T.m[k][3]);
                int n = fc.n[c];
                if (n >= 0 && 3 * n + 2 < (int)N.size()) {
                    double q[3] = {N[3 * n], N[3 * n + 1], N[3 * n + 2]};
                    for (int k = 0; k < 3; ++k)  // (T^-1)^T row k = column k of T^-1
                        nv[c][k] = (float)(Tinv.m[0][k] * q[0] + Tinv.m[1][k] * q[1] + Tinv.m[2][k] * q[2] + Tinv.m[3][k]);
                    fnormalize(nv[c]);
                } else {
                    has_n = false;
                }
                int t = fc.t[c];
                tv[c][0] = (t >= 0 && 2 * t + 1 < (int)UV.size()) ? UV[2 * t] : 0.f;
                tv[c][1] = (t >= 0 && 2 * t + 1 < (int)UV.size()) ? UV[2 * t + 1] : 0.f;
            }
            if (!has_n) {
                float e1[3], e2[3], fn[3];
                for (int k = 0; k < 3; ++k) {
                    e1[k] = pv[1][k] - pv[0][k];
                    e2[k] = pv[2][k] - pv[0][k];
                }
                fcross(e1, e2, fn);
                fnormalize(fn);
                for (int c = 0; c < 3; ++c)
                    for (int k = 0; k < 3; ++k) nv[c][k] = fn[k];
            }
            ObjMesh &m = meshes[idx];
            for (int c = 0; c < 3; ++c) {
                for (int k = 0; k < 3; ++k) m.verts.push_back(pv[c][k]);
                for (int k = 0; k < 3; ++k) m.normals.push_back(nv[c][k]);
                m.uvs.push_back(tv[c][0]);
                m.uvs.push_back(tv[c][1]);
            }
        }
    }
    return meshes;
}

// ---------------------------------------------------------------------------
// Radiance HDR (RGBE; flat or new-style run-length scanlines). Values are
// byte * 2^(e - 136), alpha 1: the convention of the loader the reference
// uses (stbi_loadf with 4 components).
// ---------------------------------------------------------------------------
void load_hdr(const std::string &path, int &w, int &h, std::vector<float> &rgba) {
    std::string data = read_file(path);
    size_t p = 0;
    auto getline = [&](std::string &l) {
        l.clear();
        while (p < data.size() && data[p] != '\n') l += data[p++];
        if (p < data.size()) ++p;
    };
    std::string l;
    getline(l);
    if (l.rfind("#?RADIANCE", 0) != 0 && l.rfind("#?RGBE", 0) != 0)
        throw Error(CRT_ERR_PARSE, "not a Radiance HDR file: " + path);
    for (;;) {
        if (p >= data.size()) throw Error(CRT_ERR_PARSE, "truncated HDR header: " + path);
        getline(l);
        if (l.empty()) break;
        if (l.rfind("FORMAT=", 0) == 0 && l != "FORMAT=32-bit_rle_rgbe")
            throw Error(CRT_ERR_PARSE, "unsupported HDR format " + l);
    }
    getline(l);
    char ys[3] = {0}, xs[3] = {0};
    if (std::sscanf(l.c_str(), "%2s %d %2s %d", ys, &h, xs, &w) != 4 || std::strcmp(ys, "-Y") || std::strcmp(xs, "+X"))
        throw Error(CRT_ERR_PARSE, "unsupported HDR orientation: " + l);
    CRT_CHECK(w > 0 && h > 0 && (size_t)w * h < (1u << 30), CRT_ERR_PARSE, "bad HDR size");
    rgba.assign((size_t)w * h * 4, 0.f);
    std::vector<unsigned char> scan((size_t)w * 4);
    auto byte = [&]() -> unsigned char {
        if (p >= data.size()) throw Error(CRT_ERR_PARSE, "truncated HDR data: " + path);
        return (unsigned char)data[p++];
    };
    for (int y = 0; y < h; ++y) {
        bool rle = false;
        if (w >= 8 && w < 32768 && p + 4 <= data.size()) {
            unsigned char c0 = data[p], c1 = data[p + 1], c2 = data[p + 2];
            rle = c0 == 2 && c1 == 2 && !(c2 & 0x80);
        }
        if (rle) {
            p += 4;
            for (int c = 0; c < 4; ++c) {
                int x = 0;
                while (x < w) {
                    unsigned char n = byte();
                    if (n > 128) {
                        n -= 128;
                        unsigned char v = byte();
                        CRT_CHECK(x + n <= w, CRT_ERR_PARSE, "HDR run overflows scanline");
                        for (int k = 0; k < n; ++k) scan[(size_t)(x++) * 4 + c] = v;
                    } else {
                        CRT_CHECK(n > 0 && x + n <= w, CRT_ERR_PARSE, "HDR dump overflows scanline");
                        for (int k = 0; k < n; ++k) scan[(size_t)(x++) * 4 + c] = byte();
                    }
                }
            }
        } else {
            for (int x = 0; x < w; ++x)
                for (int c = 0; c < 4; ++c) scan[(size_t)x * 4 + c] = byte();
        }
        for (int x = 0; x < w; ++x) {
            const unsigned char *e = &scan[(size_t)x * 4];
            float *o = &rgba[((size_t)y * w + x) * 4];
            if (e[3]) {
                float f = std::ldexp(1.0f, (int)e[3] - 136);
                o[0] = e[0] * f;
                o[1] = e[1] * f;
                o[2] = e[2] * f;
            }
            o[3] = 1.f;
        }
    }
}

// ---------------------------------------------------------------------------
// scene JSON
// ---------------------------------------------------------------------------
void vec3(const Json &j, float *out, const char *what) {
    if (j.kind != Json::ARR || j.arr.size() < 3) throw Error(CRT_ERR_PARSE, std::string("expected [x,y,z] for ") + what);
    for (int k = 0; k < 3; ++k) out[k] = (float)j.arr[k].number(what);
}

void parse_camera(const Json &c, HostScene &s) {
    CRT_CHECK(c.has("type"), CRT_ERR_PARSE, "camera missing 'type'");
    CRT_CHECK(c["type"].string("camera.type") == "pinhole", CRT_ERR_PARSE,
              "unsupported camera type " + c["type"].str);
    if (c.has("resolution")) {
        s.width = (int)c["resolution"].arr.at(0).number("resolution");
        s.height = (int)c["resolution"].arr.at(1).number("resolution");
    }
    if (c.has("fov")) s.fovy = (float)c["fov"].number("fov");
    if (c.has("max_bounces")) s.max_bounces = (int)c["max_bounces"].number("max_bounces");
    if (c.has("rr")) s.rr = (float)c["rr"].number("rr");
    if (c.has("spp")) s.spp = (int)c["spp"].number("spp");
    if (c.has("direction")) vec3(c["direction"], s.direction, "direction");
    if (c.has("denoise")) s.denoise = c["denoise"].kind == Json::BOOL ? c["denoise"].b : c["denoise"].num != 0;
    CRT_CHECK(s.width > 0 && s.height > 0, CRT_ERR_PARSE, "camera resolution missing or invalid");
}

DMaterial default_material() {
    DMaterial m;
    std::memset(&m, 0, sizeof(m));
    m.type = MAT_DIFFUSE;
    m.roughness = 0.5f;
    m.metallic = 0.f;
    m.transmission = 1.f;
    m.ior = 1.f;
    m.tex = -1;
    return m;
}

void parse_materials(const Json &arr, HostScene &s, std::unordered_map<std::string, int> &map) {
    CRT_CHECK(arr.kind == Json::ARR, CRT_ERR_PARSE, "'materials' should be an array");
    s.materials.assign(arr.arr.size(), default_material());
    s.material_names.assign(arr.arr.size(), "");
    for (size_t i = 0; i < arr.arr.size(); ++i) {
        const Json &j = arr.arr[i];
        if (!j.has("name") || !j.has("type")) {
            s.warnings.push_back("material missing 'name' or 'type'");
            continue;
        }
        DMaterial m = default_material();
        std::string type = j["type"].string("material.type");
        if (type == "diffuse") m.type = MAT_DIFFUSE;
        else if (type == "light") m.type = MAT_LIGHT;
        else if (type == "pbr") m.type = MAT_PBR;
        else if (type == "subsurface") m.type = MAT_SUBSURFACE;
        else if (type == "dielectric" || type == "glass") m.type = MAT_DIELECTRIC;
        else {
            s.warnings.push_back("unsupported material type " + type);
            continue;
        }
        if (m.type == MAT_DIFFUSE || m.type == MAT_PBR || m.type == MAT_SUBSURFACE) {
            if (j.has("basecolor")) vec3(j["basecolor"], m.base, "basecolor");
        }
        if (m.type == MAT_LIGHT && j.has("emission")) vec3(j["emission"], m.ke, "emission");
        if (m.type == MAT_PBR) {
            m.metallic = j.has("metallic") ? (float)j["metallic"].number("metallic") : 0.f;
            m.roughness = j.has("roughness") ? (float)j["roughness"].number("roughness") : 0.5f;
        }
        if (m.type == MAT_SUBSURFACE) {
            if (j.has("scatter_distance"))
                vec3(j["scatter_distance"], m.scatter, "scatter_distance");
            else
                m.scatter[0] = m.scatter[1] = m.scatter[2] = 1.f;
            if (j.has("ior")) m.ior = (float)j["ior"].number("ior");
            if (j.has("roughness")) m.roughness = (float)j["roughness"].number("roughness");
            m.metallic = 0.f;
        }
        if (m.type == MAT_DIELECTRIC) {
            if (j.has("basecolor"))
                vec3(j["basecolor"], m.base, "basecolor");
            else
                m.base[0] = m.base[1] = m.base[2] = 1.f;
            m.ior = j.has("ior") ? (float)j["ior"].number("ior") : 1.5f;
            m.transmission = j.has("transmission") ? (float)j["transmission"].number("transmission") : 1.f;
            m.roughness = j.has("roughness") ? (float)j["roughness"].number("roughness") : 0.f;
            m.metallic = 0.f;
        }
        if (j.has("diffuse_texture")) {  // Src/Core/scene.cpp:380-386
            const std::string tn = j["diffuse_texture"].string("diffuse_texture");
            int found = -1;
            for (size_t t = 0; t < s.textures.size(); ++t)
                if (s.textures[t].name == tn) found = (int)t;
            if (found >= 0)
                m.tex = found;
            else
                s.warnings.push_back("texture '" + tn + "' not found for material '" + j["name"].str + "'");
        }
        std::string name = j["name"].string("material.name");
        s.materials[i] = m;
        s.material_names[i] = name;
        map[name] = (int)i;
    }
}

std::string resolve_material(const Json &obj, const ObjMesh &m, const std::unordered_map<std::string, int> &map) {
    if (obj.has("material")) return obj["material"].string("object.material");
    if (obj.has("material_overrides") && obj["material_overrides"].kind == Json::OBJ) {
        const Json &ov = obj["material_overrides"];
        if (!m.material.empty() && ov.has(m.material)) return ov[m.material].string("material_overrides");
    }
    if (!m.material.empty() && map.count(m.material)) return m.material;
    if (obj.has("default_material")) return obj["default_material"].string("default_material");
    return "";
}

void parse_objects(const Json &arr, HostScene &s, const std::unordered_map<std::string, int> &mat_map,
                   std::unordered_map<std::string, int> &mesh_map) {
    CRT_CHECK(arr.kind == Json::ARR, CRT_ERR_PARSE, "'objects' should be an array");
    for (const Json &o : arr.arr) {
        if (!o.has("name") || !o.has("path")) {
            s.warnings.push_back("object missing 'name' or 'path'");
            continue;
        }
        M4 T = M4::identity(), R = M4::identity(), S = M4::identity();
        if (o.has("translate")) {
            float t[3];
            vec3(o["translate"], t, "translate");
            for (int k = 0; k < 3; ++k) T.m[k][3] = t[k];
        }
        if (o.has("rotate") && o["rotate"].kind == Json::ARR)
            for (const Json &r : o["rotate"].arr) {
                if (r.has("rotateX")) R = rot(0, (float)r["rotateX"].number("rotateX")) * R;
                else if (r.has("rotateY")) R = rot(1, (float)r["rotateY"].number("rotateY")) * R;
                else if (r.has("rotateZ")) R = rot(2, (float)r["rotateZ"].number("rotateZ")) * R;
            }
        if (o.has("scale")) {
            float sc[3];
            vec3(o["scale"], sc, "scale");
            for (int k = 0; k < 3; ++k) S.m[k][k] = sc[k];
        }
        M4 X = T * R * S, Xinv;
        CRT_CHECK(invert(X, Xinv), CRT_ERR_PARSE, "singular object transform");
        std::string oname = o["name"].string("object.name");
        std::vector<ObjMesh> meshes = load_obj(o["path"].string("object.path"), X, Xinv, is_identity(X));
        if (meshes.empty()) {
            s.warnings.push_back("object '" + oname + "' produced no meshes");
            continue;
        }
        bool expanded = meshes.size() > 1;
        for (const ObjMesh &m : meshes) {
            if (m.verts.empty()) continue;
            std::string mname = resolve_material(o, m, mat_map);
            auto it = mat_map.find(mname);
            if (mname.empty() || it == mat_map.end()) {
                s.warnings.push_back("no valid material binding for mesh '" + m.name + "' of object '" + oname + "'");
                continue;
            }
            DMesh dm;
            std::memset(&dm, 0, sizeof(dm));
            dm.material = it->second;
            dm.light = -1;
            dm.start = (int)s.prim_mesh.size();
            dm.count = (int)(m.verts.size() / 9);
            float area = 0.f;
            int mesh_id = (int)s.meshes.size();
            for (int t = 0; t < dm.count; ++t) {
                area += triangle_area(&m.verts[9 * (size_t)t]);
                s.prim_mesh.push_back(mesh_id);
            }
            dm.area = area;
            s.verts.insert(s.verts.end(), m.verts.begin(), m.verts.end());
            s.normals.insert(s.normals.end(), m.normals.begin(), m.normals.end());
            s.uvs.insert(s.uvs.end(), m.uvs.begin(), m.uvs.end());
            std::string name = expanded ? oname + "::" + m.name : oname;
            mesh_map[name] = mesh_id;
            s.meshes.push_back(dm);
            s.mesh_names.push_back(name);
        }
    }
}

void parse_lights(const Json &arr, HostScene &s, const std::unordered_map<std::string, int> &mat_map,
                  const std::unordered_map<std::string, int> &mesh_map) {
    CRT_CHECK(arr.kind == Json::ARR, CRT_ERR_PARSE, "'lights' should be an array");
    for (const Json &l : arr.arr) {
        if (!l.has("type")) {
            s.warnings.push_back("light missing 'type'");
            continue;
        }
        DLight dl;
        std::memset(&dl, 0, sizeof(dl));
        dl.mesh = -1;
        std::string type = l["type"].string("light.type");
        if (type == "area") {
            dl.type = LIGHT_AREA;
            if (l.has("ke")) vec3(l["ke"], dl.emission, "ke");
            if (l.has("material")) {
                auto it = mat_map.find(l["material"].string("light.material"));
                if (it != mat_map.end())
                    for (int k = 0; k < 3; ++k) dl.emission[k] = s.materials[it->second].ke[k];
                else
                    s.warnings.push_back("light material not found");
            }
            auto mit = mesh_map.find(l["lightMeshName"].kind == Json::STR ? l["lightMeshName"].str : "");
            if (mit == mesh_map.end()) {
                s.warnings.push_back("light mesh '" + l["lightMeshName"].str + "' not found; light skipped");
                continue;
            }
            dl.mesh = mit->second;
            s.meshes[dl.mesh].light = (int)s.lights.size();
        } else if (type == "env") {
            dl.type = LIGHT_ENV;
            CRT_CHECK(l.has("path"), CRT_ERR_PARSE, "env light missing 'path'");
            load_hdr(l["path"].string("light.path"), s.env_w, s.env_h, s.env);
            s.env_light = (int)s.lights.size();
        } else {
            s.warnings.push_back("unsupported light type " + type);
            continue;
        }
        s.lights.push_back(dl);
    }
}

}  // namespace

float triangle_area(const float *v) {
    float e1[3], e2[3], n[3];
    for (int k = 0; k < 3; ++k) {
        e1[k] = v[3 + k] - v[k];
        e2[k] = v[6 + k] - v[k];
    }
    fcross(e1, e2, n);
    return 0.5f * std::sqrt(fdot(n, n));
}

void face_normal(const float *v, float *n) {
    float e1[3], e2[3];
    for (int k = 0; k < 3; ++k) {
        e1[k] = v[3 + k] - v[k];
        e2[k] = v[6 + k] - v[k];
    }
    fcross(e1, e2, n);
    fnormalize(n);
}

DMaterial default_material_record() { return default_material(); }

void load_scene_json(const std::string &path, HostScene &s) {
    std::string text = read_file(path);
    Json root = JsonParser(text).parse();
    CRT_CHECK(root.kind == Json::OBJ, CRT_ERR_PARSE, "scene file is not a JSON object");
    parse_camera(root["camera"], s);
    std::unordered_map<std::string, int> mat_map, mesh_map;
    CRT_CHECK(root["textures"].kind == Json::ARR, CRT_ERR_PARSE, "'textures' should be an array");
    // ParseTextures (Src/Core/scene.cpp:618-644); an image that does not
    // decode leaves its materials on their basecolor
    for (const Json &tj : root["textures"].arr) {
        if (!tj.has("path") || !tj.has("name")) {
            s.warnings.push_back("texture missing 'path' or 'name'");
            continue;
        }
        HostTexture t;
        t.name = tj["name"].string("texture.name");
        try {
            load_texture_image(tj["path"].string("texture.path"), t);
        } catch (const Error &e) {
            s.warnings.push_back(std::string("texture '") + t.name + "' not loaded: " + e.what());
            continue;
        }
        s.textures.push_back(std::move(t));
    }
    parse_materials(root["materials"], s, mat_map);
    parse_objects(root["objects"], s, mat_map, mesh_map);
    parse_lights(root["lights"], s, mat_map, mesh_map);
    CRT_CHECK(!s.prim_mesh.empty(), CRT_ERR_PARSE, "scene has no triangles");
}

}  // namespace crt
