// SVGF denoiser and its primary-hit G-buffer.
//
// G-buffer: the reference rasterises one with OpenGL (RenderGBuffer,
// Src/Core/renderer.cuh:1446-1503; Shader/gbuffer.vs, gbuffer.fs). Here a
// primary ray through each pixel centre finds the nearest surface (no face
// culling, as the raster pass culls none) and writes the same four planes
// with the same encodings:
//   pos_tri      float4  world position, triangle index within its mesh
//   normal_mat   ushort4 uint((n * 0.5 + 0.5) * 65535) of the interpolated
//                        vertex normal, material id
//   bary_mesh    ushort4 uint(barycentrics * 65535), mesh id + 1
//   motion_depth float4  NDC(current) - NDC(previous camera), linear view
//                        depth, fwidth(depth) from 2x2 quad differences
// Background pixels are all zero (the raster pass's clear values).
//
// SVGF: TemporalDenoising (renderer.cuh:524-677), ComputeVarianceKernel
// (:689-805) and AtrousKernel (:807-954) restated pixel for pixel, driven in
// the order of RenderLoop's denoise block (:1208-1258): temporal reprojection
// (which also writes the history the reference copies afterwards), 7x7
// variance estimate, then atrous_iterations a-trous passes at steps 1, 2,
// 4, ... (skipped on the first frame), the last of them writing the
// caller's output. The temporal pass also stores, per pixel, the decoded
// normal, depth, material/mesh ids and history length that every later tap
// compares against (one 16 B and one 8 B load per tap instead of four
// G-buffer loads and a normal decode).
#include "svgf.h"
#include "shade.cuh"
#include <cstring>
#include <cstdlib>

namespace crt {

// ---------------------------------------------------------------------------
// G-buffer
// ---------------------------------------------------------------------------
struct Mat4 {
    float m[16];  // row-major
};

// Perspective (Src/Utils/mathutil.cu:163-172).
static Mat4 perspective(float fovy, float aspect, float n, float f) {
    Mat4 r;
    std::memset(&r, 0, sizeof(r));
    float ff = 1.0f / std::tan((float)((double)(fovy / 180) * kPiD) / 2.0f);
    r.m[0] = ff / aspect;
    r.m[5] = ff;
    r.m[10] = (f + n) / (n - f);
    r.m[11] = (2 * f * n) / (n - f);
    r.m[14] = -1.0f;
    return r;
}

// LookAt (Src/Utils/mathutil.cu:175-193).
static Mat4 look_at(const float *eye, const float *center, const float *up) {
    auto nrm = [](float *v) {
        float z = v[0] * v[0] + (v[1] * v[1] + v[2] * v[2]);
        if (z > 0) {
            float s = std::sqrt(z);
            v[0] /= s; v[1] /= s; v[2] /= s;
        }
    };
    auto crs = [](const float *a, const float *b, float *o) {
        o[0] = a[1] * b[2] - a[2] * b[1];
        o[1] = a[2] * b[0] - a[0] * b[2];
        o[2] = a[0] * b[1] - a[1] * b[0];
    };
    auto dt = [](const float *a, const float *b) { return a[0] * b[0] + (a[1] * b[1] + a[2] * b[2]); };
    float f[3] = {center[0] - eye[0], center[1] - eye[1], center[2] - eye[2]}, s[3], u[3];
    nrm(f);
    crs(f, up, s);
    nrm(s);
    crs(s, f, u);
    Mat4 r;
    std::memset(&r, 0, sizeof(r));
    r.m[0] = s[0]; r.m[1] = s[1]; r.m[2] = s[2]; r.m[3] = -dt(s, eye);
    r.m[4] = u[0]; r.m[5] = u[1]; r.m[6] = u[2]; r.m[7] = -dt(u, eye);
    r.m[8] = -f[0]; r.m[9] = -f[1]; r.m[10] = -f[2]; r.m[11] = dt(f, eye);
    r.m[15] = 1.f;
    return r;
}

static Mat4 mul(const Mat4 &a, const Mat4 &b) {
    Mat4 r;
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) {
            float s = 0.f;
            for (int k = 0; k < 4; ++k) s += a.m[4 * i + k] * b.m[4 * k + j];
            r.m[4 * i + j] = s;
        }
    return r;
}

struct GbufCam {
    float pos[3], ld[3], du[3], dv[3];
    float view[16];
    float vp[16], prev_vp[16];
};

__device__ __forceinline__ float4 xform(const float *M, V3 p) {
    return make_float4(M[0] * p.x + M[1] * p.y + M[2] * p.z + M[3], M[4] * p.x + M[5] * p.y + M[6] * p.z + M[7],
                       M[8] * p.x + M[9] * p.y + M[10] * p.z + M[11], M[12] * p.x + M[13] * p.y + M[14] * p.z + M[15]);
}

__global__ void k_gbuffer(SceneView s, GbufCam cam, int W, int H, float4 *pos_tri, ushort4 *normal_mat,
                          ushort4 *bary_mesh, float4 *motion_depth) {
    int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= W || j >= H) return;
    int pix = j * W + i;
    V3 ld = ld3(cam.ld), du = ld3(cam.du), dv = ld3(cam.dv), pos = ld3(cam.pos);
    V3 pp = (ld + (i + 0.5f) * du) + (j + 0.5f) * dv;
    V3 d = normalized(pp - pos);
    Hit h = closest_hit<false, false>(s.bvh, pos, d, 0.f, kTriTMax);
    if (h.slot < 0) {
        pos_tri[pix] = make_float4(0.f, 0.f, 0.f, 0.f);
        normal_mat[pix] = make_ushort4(0, 0, 0, 0);
        bary_mesh[pix] = make_ushort4(0, 0, 0, 0);
        motion_depth[pix] = make_float4(0.f, 0.f, 0.f, 0.f);
        return;
    }
    int prim = tri_prim(s.bvh, h.slot);
    V3 p = hit_point(s.bvh, h);
    const float4 *ap = s.attr + 4 * (size_t)prim;
    float4 A0 = __ldg(ap), A1 = __ldg(ap + 1), A2 = __ldg(ap + 2), A3 = __ldg(ap + 3);
    float b0 = 1.f - h.b1 - h.b2;
    V3 n = normalized((b0 * V3{A0.x, A0.y, A0.z} + h.b1 * V3{A1.x, A1.y, A1.z}) + h.b2 * V3{A2.x, A2.y, A2.z});
    int mesh = __float_as_int(A3.w);
    const DMesh &M = s.meshes[mesh];
    auto enc = [](float x) -> unsigned short {
        float v = x * 65535.0f;
        return (unsigned short)(v <= 0.f ? 0.f : (v >= 65535.f ? 65535.f : v));
    };
    pos_tri[pix] = make_float4(p.x, p.y, p.z, (float)(prim - M.start));
    normal_mat[pix] = make_ushort4(enc(n.x * 0.5f + 0.5f), enc(n.y * 0.5f + 0.5f), enc(n.z * 0.5f + 0.5f),
                                   (unsigned short)M.material);
    bary_mesh[pix] = make_ushort4(enc(b0), enc(h.b1), enc(h.b2), (unsigned short)(mesh + 1));
    float4 c = xform(cam.vp, p), q = xform(cam.prev_vp, p);
    float4 e = xform(cam.view, p);
    motion_depth[pix] = make_float4(c.x / c.w - q.x / q.w, c.y / c.w - q.y / q.w, -e.z, 0.f);
}

// fwidth(depth) = |dFdx| + |dFdy| with the derivative taken within each 2x2
// pixel quad, as a fragment shader computes it.
__global__ void k_gbuffer_dz(int W, int H, const float4 *pos_tri_unused, float4 *motion_depth) {
    int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= W || j >= H) return;
    int pix = j * W + i;
    float4 md = motion_depth[pix];
    if (md.z == 0.f) return;
    int ix = i ^ 1, jy = j ^ 1;
    float dx = 0.f, dy = 0.f;
    if (ix < W) {
        float z = motion_depth[j * W + ix].z;
        if (z != 0.f) dx = (i & 1) ? md.z - z : z - md.z;
    }
    if (jy < H) {
        float z = motion_depth[jy * W + i].z;
        if (z != 0.f) dy = (j & 1) ? md.z - z : z - md.z;
    }
    motion_depth[pix].w = fabsf(dx) + fabsf(dy);
}

void gbuffer_from_primary(const SceneView &view, const CameraState &cur, const CameraState &prev, const float bmin[3],
                          const float bmax[3], const GBufferPlanes &g, cudaStream_t stream) {
    GbufCam gc;
    for (int k = 0; k < 3; ++k) {
        gc.pos[k] = cur.position[k];
        gc.ld[k] = cur.left_down[k];
        gc.du[k] = cur.du[k];
        gc.dv[k] = cur.dv[k];
    }
    // Near 0.1, far = diagonal + |camera - centre| (renderer.cuh:1469-1471).
    float c[3], e[3], dc[3];
    for (int k = 0; k < 3; ++k) {
        c[k] = (bmin[k] + bmax[k]) * 0.5f;
        e[k] = bmax[k] - bmin[k];
        dc[k] = cur.position[k] - c[k];
    }
    float far = std::sqrt(e[0] * e[0] + (e[1] * e[1] + e[2] * e[2])) +
                std::sqrt(dc[0] * dc[0] + (dc[1] * dc[1] + dc[2] * dc[2]));
    Mat4 P = perspective(cur.fovy, cur.ratio, 0.1f, far);
    Mat4 V = look_at(cur.position, cur.lookat, cur.up);
    Mat4 Vp = look_at(prev.position, prev.lookat, prev.up);
    Mat4 VP = mul(P, V), PVP = mul(perspective(prev.fovy, prev.ratio, 0.1f, far), Vp);
    std::memcpy(gc.view, V.m, sizeof(gc.view));
    std::memcpy(gc.vp, VP.m, sizeof(gc.vp));
    std::memcpy(gc.prev_vp, PVP.m, sizeof(gc.prev_vp));
    dim3 b(16, 16), gr((cur.width + 15) / 16, (cur.height + 15) / 16);
    k_gbuffer<<<gr, b, 0, stream>>>(view, gc, cur.width, cur.height, g.pos_tri, g.normal_mat, g.bary_mesh,
                                    g.motion_depth);
    k_gbuffer_dz<<<gr, b, 0, stream>>>(cur.width, cur.height, g.pos_tri, g.motion_depth);
    CRT_CUDA(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// SVGF
// ---------------------------------------------------------------------------
struct GB {
    const float4 *pos_tri;
    const ushort4 *normal_mat;
    const ushort4 *bary_mesh;
    const float4 *motion_depth;
};

__device__ __forceinline__ V3 decode_normal(ushort4 n) {
    return normalized(V3{n.x / 65535.0f * 2.f - 1.f, n.y / 65535.0f * 2.f - 1.f, n.z / 65535.0f * 2.f - 1.f});
}
__device__ __forceinline__ V3 rgb(const float4 *b, int i) {
    float4 v = b[i];
    return V3{v.x, v.y, v.z};
}

// IsValidTemporalReprojectionTap (renderer.cuh:460-497).
__device__ __forceinline__ bool valid_tap(int tx, int ty, int W, int H, int mesh, int mat, int tri, V3 n, float depth,
                                          float dz, float pixdist, const GB &last, float reproj) {
    if (tx < 0 || tx >= W || ty < 0 || ty >= H) return false;
    int k = ty * W + tx;
    float4 lp = last.pos_tri[k];
    ushort4 lb = last.bary_mesh[k], ln = last.normal_mat[k];
    float4 lm = last.motion_depth[k];
    float dotn = dot(n, decode_normal(ln));
    float dd = fabsf(depth - lm.z);
    float thr = fmaxf(dz, lm.w) * (pixdist + 1.f) + reproj * fmaxf(depth, lm.z);
    return mesh == (int)lb.w && mat == (int)ln.w && tri == (int)lp.w && dotn >= 0.9f && dd <= thr;
}

// Per-pixel edge-stopping record written by the temporal pass and read by
// the variance and a-trous taps: the decoded G-buffer normal and linear
// depth (edge), and the material | mesh << 16 id with the history length
// (tag). decode_normal runs once per pixel instead of once per tap; the
// values are the same.
struct EdgeOut {
    float4 *edge;
    int2 *tag;
};

struct TemporalArgs {
    int W, H, max_hist;
    float reproj;
    const float4 *noisy_d, *noisy_i;      // current noisy frame
    float4 *cur_d, *cur_i;                // blended result
    float4 *hist_out_d, *hist_out_i;      // the same, kept as next frame's history
    const float4 *hist_d, *hist_i;        // last frame's temporal history
    float2 *mom_d, *mom_i;                // moments written this frame
    const float2 *lmom_d, *lmom_i;        // last frame's moments
    int *hlen;                            // history length written
    const int *lhlen;
    bool first;
};

// TemporalDenoising (renderer.cuh:524-677). Reads the noisy frame, writes
// the blended result both as the frame's working buffer and as the next
// frame's history, and the pixel's edge-stopping record.
__global__ void k_svgf_temporal(TemporalArgs a, GB cur, GB last, EdgeOut eo) {
    int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= a.W || y >= a.H) return;
    int idx = y * a.W + x;
    const float4 nd4 = a.noisy_d[idx], ni4 = a.noisy_i[idx];
    V3 cd{nd4.x, nd4.y, nd4.z}, ci{ni4.x, ni4.y, ni4.z};
    float4 pt = cur.pos_tri[idx];
    ushort4 bm = cur.bary_mesh[idx], nm = cur.normal_mat[idx];
    float4 md = cur.motion_depth[idx];
    int mat = nm.w, mesh = bm.w, tri = (int)pt.w;
    V3 n = decode_normal(nm);
    float depth = md.z, dz = md.w;
    eo.edge[idx] = make_float4(n.x, n.y, n.z, depth);
    if (a.first) {
        float dl = luminance(cd), il = luminance(ci);
        a.mom_d[idx] = make_float2(dl, dl * dl);
        a.mom_i[idx] = make_float2(il, il * il);
        const float4 od = make_float4(nd4.x, nd4.y, nd4.z, 1.f), oi = make_float4(ni4.x, ni4.y, ni4.z, 1.f);
        a.cur_d[idx] = od;
        a.cur_i[idx] = oi;
        a.hist_out_d[idx] = od;
        a.hist_out_i[idx] = oi;
        a.hlen[idx] = 1;
        eo.tag[idx] = make_int2(mat | (mesh << 16), 1);
        return;
    }
    float mvx = md.x * a.W * 0.5f, mvy = md.y * a.H * 0.5f;
    float pixdist = sqrtf(mvx * mvx + mvy * mvy);
    // GetLastFramePos (renderer.cuh:446-455)
    float px = ((float)x + 0.5f) - mvx, py = ((float)y + 0.5f) - mvy;
    bool inside = px >= 0.5f && px < a.W - 0.5f && py >= 0.5f && py < a.H - 0.5f;
    bool valid = false;
    V3 rd{0.f, 0.f, 0.f}, ri{0.f, 0.f, 0.f};
    float2 rmd = make_float2(0.f, 0.f), rmi = make_float2(0.f, 0.f);
    float rh = 0.f;
    auto tap = [&](float w, int k) {
        rd = rd + rgb(a.hist_d, k) * w;
        ri = ri + rgb(a.hist_i, k) * w;
        rmd.x += a.lmom_d[k].x * w;
        rmd.y += a.lmom_d[k].y * w;
        rmi.x += a.lmom_i[k].x * w;
        rmi.y += a.lmom_i[k].y * w;
        rh += (float)a.lhlen[k] * w;
    };
    if (inside) {
        float fx = px - 0.5f, fy = py - 0.5f;
        int bx = (int)floorf(fx), by = (int)floorf(fy);
        float frx = fx - (float)bx, fry = fy - (float)by;
        float tw = 0.f;
        bool all = true;
        for (int oy = 0; oy <= 1; oy++)
            for (int ox = 0; ox <= 1; ox++) {
                int tx = bx + ox, ty = by + oy;
                if (!valid_tap(tx, ty, a.W, a.H, mesh, mat, tri, n, depth, dz, pixdist, last, a.reproj)) {
                    all = false;
                    continue;
                }
                float w = (ox == 0 ? (1.f - frx) : frx) * (oy == 0 ? (1.f - fry) : fry);
                tap(w, ty * a.W + tx);
                tw += w;
            }
        if (all && tw > 1e-6f) {
            float inv = 1.f / tw;
            rd = rd * inv;
            ri = ri * inv;
            rmd.x *= inv; rmd.y *= inv;
            rmi.x *= inv; rmi.y *= inv;
            rh *= inv;
            valid = true;
        } else {
            rd = ri = V3{0.f, 0.f, 0.f};
            rmd = rmi = make_float2(0.f, 0.f);
            rh = 0.f;
            tw = 0.f;
            const float kw[2] = {0.5f, 0.25f};
            int cx = max(0, min(a.W - 1, (int)floorf(px))), cy = max(0, min(a.H - 1, (int)floorf(py)));
            for (int oy = -1; oy <= 1; oy++)
                for (int ox = -1; ox <= 1; ox++) {
                    int tx = cx + ox, ty = cy + oy;
                    if (!valid_tap(tx, ty, a.W, a.H, mesh, mat, tri, n, depth, dz, pixdist, last, a.reproj)) continue;
                    float w = kw[abs(ox)] * kw[abs(oy)];
                    tap(w, ty * a.W + tx);
                    tw += w;
                }
            if (tw > 1e-6f) {
                float inv = 1.f / tw;
                rd = rd * inv;
                ri = ri * inv;
                rmd.x *= inv; rmd.y *= inv;
                rmi.x *= inv; rmi.y *= inv;
                rh *= inv;
                valid = true;
            }
        }
    }
    int hl = 1;
    if (valid) hl = min(max(1, (int)floorf(rh + 0.5f)) + 1, a.max_hist);
    float alpha = valid ? 1.f / hl : 1.0f;
    float dl = luminance(cd), il = luminance(ci);
    float4 od, oi;
    od.x = alpha * cd.x + (1 - alpha) * rd.x;
    od.y = alpha * cd.y + (1 - alpha) * rd.y;
    od.z = alpha * cd.z + (1 - alpha) * rd.z;
    oi.x = alpha * ci.x + (1 - alpha) * ri.x;
    oi.y = alpha * ci.y + (1 - alpha) * ri.y;
    oi.z = alpha * ci.z + (1 - alpha) * ri.z;
    float2 lmd = valid ? rmd : make_float2(0.f, 0.f), lmi = valid ? rmi : make_float2(0.f, 0.f);
    float2 mdd, mii;
    mdd.x = alpha * dl + (1 - alpha) * lmd.x;
    mdd.y = alpha * dl * dl + (1 - alpha) * lmd.y;
    mii.x = alpha * il + (1 - alpha) * lmi.x;
    mii.y = alpha * il * il + (1 - alpha) * lmi.y;
    a.mom_d[idx] = mdd;
    a.mom_i[idx] = mii;
    if (valid) {
        od.w = mdd.y - mdd.x * mdd.x;
        oi.w = mii.y - mii.x * mii.x;
    } else {
        od.w = 1.f;
        oi.w = 1.f;
        hl = 1;
    }
    a.hlen[idx] = hl;
    eo.tag[idx] = make_int2(mat | (mesh << 16), hl);
    a.cur_d[idx] = od;
    a.cur_i[idx] = oi;
    a.hist_out_d[idx] = od;
    a.hist_out_i[idx] = oi;
}

struct VarianceArgs {
    int W, H, half;
    float sigma_depth, sigma_normal, sigma_light;
    const float4 *in_d, *in_i;
    float4 *out_d, *out_i;
    const float2 *mom_d, *mom_i;
    const float4 *edge;
    const int2 *tag;
};

// Tap sources for the variance body (global memory or a shared tile).
struct VarGlobalTaps {
    const VarianceArgs &a;
    __device__ __forceinline__ float4 d(int x, int y) const { return a.in_d[y * a.W + x]; }
    __device__ __forceinline__ float4 i(int x, int y) const { return a.in_i[y * a.W + x]; }
    __device__ __forceinline__ float4 e(int x, int y) const { return a.edge[y * a.W + x]; }
    __device__ __forceinline__ int t(int x, int y) const { return a.tag[y * a.W + x].x; }
    __device__ __forceinline__ float4 m(int x, int y) const {
        const float2 md = a.mom_d[y * a.W + x], mi = a.mom_i[y * a.W + x];
        return make_float4(md.x, md.y, mi.x, mi.y);
    }
};

struct VarTileTaps {
    const float4 *sd, *si, *se, *sm;
    const int *st;
    int x0, y0, rw;
    __device__ __forceinline__ int at(int x, int y) const { return (y - y0) * rw + (x - x0); }
    __device__ __forceinline__ float4 d(int x, int y) const { return sd[at(x, y)]; }
    __device__ __forceinline__ float4 i(int x, int y) const { return si[at(x, y)]; }
    __device__ __forceinline__ float4 e(int x, int y) const { return se[at(x, y)]; }
    __device__ __forceinline__ int t(int x, int y) const { return st[at(x, y)]; }
    __device__ __forceinline__ float4 m(int x, int y) const { return sm[at(x, y)]; }
};

// Edge-stopping weights in the log domain. The reference's tap weight
// powf(c, s) * expf(w) (c the clamped normal dot, w the summed depth and
// luminance terms) equals exp2(s * log2(c) + w * log2(e)); it is evaluated
// with one lg2 and one ex2 of the special-function unit (relative error
// about 1e-6, against the filters' 1e-3 parity bound) instead of powf, expf
// and their range reductions. c = 0 gives log2 = -inf and a weight of 0, as
// powf(0, s) does for s > 0.
constexpr float kLog2e = 1.44269504088896341f;
__device__ __forceinline__ float log_weight(float c, float s) { return s * __log2f(c); }
__device__ __forceinline__ float sqrt_fast(float x) { return x * rsqrtf(x); }  // x > 0

// sqrt(ki^2 + kj^2) for |ki|, |kj| <= 3, at [|kj| * 4 + |ki|] (correctly
// rounded values; the tap loops index it with warp-uniform offsets).
__constant__ float c_tap_dist[16] = {0.f,         1.f,         2.f,         3.f,
                                     1.f,         1.41421356f, 2.23606798f, 3.16227766f,
                                     2.f,         2.23606798f, 2.82842712f, 3.60555128f,
                                     3.f,         3.16227766f, 3.60555128f, 4.24264069f};

// ComputeVarianceKernel (renderer.cuh:689-805) for pixel (x, y) with a
// history shorter than 4 frames: 7x7 edge-stopped filter of colour and
// moments, variance from the filtered moments.
template <class Taps>
__device__ __forceinline__ void variance_pixel(const VarianceArgs &a, const GB &g, const Taps &src, int x, int y, int h,
                                               int ctag) {
    int idx = y * a.W + x;
    const float4 cd4 = src.d(x, y), ci4 = src.i(x, y);
    V3 cd{cd4.x, cd4.y, cd4.z}, ci{ci4.x, ci4.y, ci4.z};
    float cdl = luminance(cd), cil = luminance(ci);
    const float4 ce = src.e(x, y);
    float cdepth = ce.w, dz = fmaxf(g.motion_depth[idx].w, 1e-4f);
    V3 cn{ce.x, ce.y, ce.z};
    V3 fd{0.f, 0.f, 0.f}, fi{0.f, 0.f, 0.f};
    float fmd0 = 0.f, fmd1 = 0.f, fmi0 = 0.f, fmi1 = 0.f, twd = 0.f, twi = 0.f;
    float sd = a.sigma_depth * fmaxf(dz, 1e-4f);
    // quotients as products with per-pixel reciprocals (see atrous_pixel)
    const float inv_sl = 1.f / a.sigma_light;
    const float il_scale = sqrtf(cil) * inv_sl;
    for (int kj = -a.half; kj <= a.half; kj++)
        for (int ki = -a.half; ki <= a.half; ki++) {
            int ni = x + ki, nj = y + kj;
            if (!(ni >= 0 && ni < a.W && nj >= 0 && nj < a.H)) continue;
            if (src.t(ni, nj) != ctag) continue;
            const float4 nd4 = src.d(ni, nj), ni4 = src.i(ni, nj);
            V3 nd{nd4.x, nd4.y, nd4.z}, nid{ni4.x, ni4.y, ni4.z};
            const float4 ne = src.e(ni, nj);
            float nz = ne.w;
            V3 nn{ne.x, ne.y, ne.z};
            float ndl = luminance(nd), nil = luminance(nid);
            const float4 mm = src.m(ni, nj);
            const float dist = c_tap_dist[abs(kj) * 4 + abs(ki)];
            float wz = -__fdividef(fabsf(cdepth - nz), sd * dist + 1e-4f);
            const float ln = log_weight(fmaxf(0.f, dot(cn, nn)), a.sigma_normal);
            float dref = fmaxf(fmaxf(cdl, ndl), 1e-4f);
            float wdl = -fabsf(cdl - ndl) * sqrt_fast(dref) * inv_sl;
            float wil = -fabsf(cil - nil) * il_scale;
            float dw = exp2f(fmaf(wz + wdl, kLog2e, ln)), iw = exp2f(fmaf(wz + wil, kLog2e, ln));
            fd = fd + nd * dw;
            fi = fi + nid * iw;
            fmd0 += mm.x * dw;
            fmd1 += mm.y * dw;
            fmi0 += mm.z * iw;
            fmi1 += mm.w * iw;
            twd += dw;
            twi += iw;
        }
    twd = fmaxf(twd, 1e-6f);
    twi = fmaxf(twi, 1e-6f);
    fmd0 /= twd; fmd1 /= twd;
    fmi0 /= twi; fmi1 /= twi;
    fd = fd / twd;
    fi = fi / twi;
    float vd = fmaxf(0.f, fmd1 - fmd0 * fmd0), vi = fmaxf(0.f, fmi1 - fmi0 * fmi0);
    vd *= 4.f / h;
    vi *= 4.f / h;
    a.out_d[idx] = make_float4(fd.x, fd.y, fd.z, vd);
    a.out_i[idx] = make_float4(fi.x, fi.y, fi.z, vi);
}

// One thread per pixel, taps from global memory.
__global__ void k_svgf_variance(VarianceArgs a, GB g) {
    int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= a.W || y >= a.H) return;
    int idx = y * a.W + x;
    const int2 ctag = a.tag[idx];
    if (ctag.y >= 4) {
        a.out_d[idx] = a.in_d[idx];
        a.out_i[idx] = a.in_i[idx];
        return;
    }
    variance_pixel(a, g, VarGlobalTaps{a}, x, y, ctag.y, ctag.x);
}

// Tiled: a block whose pixels all have 4 frames of history only copies
// (the steady state); otherwise its 32 x 8 pixels and a 3-pixel halo
// (colour, edge record, tag, moments: 68 B per pixel) are staged in shared
// memory for the 7x7 taps.
constexpr int kVarTileX = 32, kVarTileY = 8, kVarHalf = 3;

__global__ void __launch_bounds__(kVarTileX * kVarTileY) k_svgf_variance_tiled(VarianceArgs a, GB g) {
    constexpr int R = kVarHalf, RW = kVarTileX + 2 * R, RH = kVarTileY + 2 * R, N = RW * RH;
    __shared__ float4 sd[N], si[N], se[N], sm[N];
    __shared__ int stg[N];
    const int bx = blockIdx.x * kVarTileX, by = blockIdx.y * kVarTileY;
    const int x = bx + threadIdx.x, y = by + threadIdx.y;
    const bool inside = x < a.W && y < a.H;
    int2 ctag = make_int2(0, 4);
    if (inside) ctag = a.tag[y * a.W + x];
    const bool filter = inside && ctag.y < 4;
    if (!__syncthreads_or(filter)) {
        if (inside) {
            a.out_d[y * a.W + x] = a.in_d[y * a.W + x];
            a.out_i[y * a.W + x] = a.in_i[y * a.W + x];
        }
        return;
    }
    const int tid = threadIdx.y * kVarTileX + threadIdx.x;
    for (int k = tid; k < N; k += kVarTileX * kVarTileY) {
        const int gx = bx - R + k % RW, gy = by - R + k / RW;
        if (gx < 0 || gx >= a.W || gy < 0 || gy >= a.H) continue;  // never read: taps check the image bounds
        const int gi = gy * a.W + gx;
        sd[k] = a.in_d[gi];
        si[k] = a.in_i[gi];
        se[k] = a.edge[gi];
        stg[k] = a.tag[gi].x;
        const float2 md = a.mom_d[gi], mi = a.mom_i[gi];
        sm[k] = make_float4(md.x, md.y, mi.x, mi.y);
    }
    __syncthreads();
    if (!inside) return;
    if (!filter) {
        const VarTileTaps t{sd, si, se, sm, stg, bx - R, by - R, RW};
        a.out_d[y * a.W + x] = t.d(x, y);
        a.out_i[y * a.W + x] = t.i(x, y);
        return;
    }
    variance_pixel(a, g, VarTileTaps{sd, si, se, sm, stg, bx - R, by - R, RW}, x, y, ctag.y, ctag.x);
}

struct AtrousArgs {
    int W, H, step;
    float sigma_depth, sigma_normal, sigma_light;
    const float4 *in_d, *in_i;
    float4 *out_d, *out_i;
    const float4 *edge;
    const int2 *tag;
};

// Tap sources for the a-trous body: straight from global memory, or from a
// shared-memory tile that covers the block and its halo.
struct GlobalTaps {
    const AtrousArgs &a;
    __device__ __forceinline__ float4 d(int x, int y) const { return a.in_d[y * a.W + x]; }
    __device__ __forceinline__ float4 i(int x, int y) const { return a.in_i[y * a.W + x]; }
    __device__ __forceinline__ float4 e(int x, int y) const { return a.edge[y * a.W + x]; }
    __device__ __forceinline__ int2 t(int x, int y) const { return a.tag[y * a.W + x]; }
};

struct TileTaps {
    const float4 *sd, *si, *se;
    const int2 *st;
    int x0, y0, rw;  // tile origin (image coordinates of its first element) and row width
    __device__ __forceinline__ int at(int x, int y) const { return (y - y0) * rw + (x - x0); }
    __device__ __forceinline__ float4 d(int x, int y) const { return sd[at(x, y)]; }
    __device__ __forceinline__ float4 i(int x, int y) const { return si[at(x, y)]; }
    __device__ __forceinline__ float4 e(int x, int y) const { return se[at(x, y)]; }
    __device__ __forceinline__ int2 t(int x, int y) const { return st[at(x, y)]; }
};

// AtrousKernel (renderer.cuh:807-954) for pixel (x, y): 3x3 pre-blur of
// the variance, then the 5x5 edge-stopped filter at a.step.
template <class Taps>
__device__ __forceinline__ void atrous_pixel(const AtrousArgs &a, const GB &g, const Taps &src, int x, int y) {
    int idx = y * a.W + x;
    const int2 ctag = src.t(x, y);
    int ch = max(ctag.y, 1);
    const float4 cd4 = src.d(x, y), ci4 = src.i(x, y);
    V3 cd{cd4.x, cd4.y, cd4.z}, ci{ci4.x, ci4.y, ci4.z};
    float cdl = luminance(cd), cil = luminance(ci);
    const float4 ce = src.e(x, y);
    float cdepth = ce.w, dz = fmaxf(g.motion_depth[idx].w, 1e-4f);
    V3 cn{ce.x, ce.y, ce.z};
    const float vk[2] = {0.5f, 0.25f};
    float fvd = 0.f, fvi = 0.f, fvw = 0.f;
    for (int vj = -1; vj <= 1; vj++)
        for (int vi = -1; vi <= 1; vi++) {
            int sx = x + vi, sy = y + vj;
            if (sx < 0 || sx >= a.W || sy < 0 || sy >= a.H) continue;
            float w = vk[abs(vi)] * vk[abs(vj)];
            fvd += w * fmaxf(0.0f, src.d(sx, sy).w);
            fvi += w * fmaxf(0.0f, src.i(sx, sy).w);
            fvw += w;
        }
    fvw = fmaxf(fvw, 1e-6f);
    fvd /= fvw;
    fvi /= fvw;
    float sdd = sqrtf(fvd) + 1e-3f, sdi = sqrtf(fvi) + 1e-3f;
    V3 fd{0.f, 0.f, 0.f}, fi{0.f, 0.f, 0.f};
    float twd = 0.f, twi = 0.f, vard = 0.f, vari = 0.f;
    float boot = fminf(1.f, fmaxf(0.f, (4.f - (float)ch) / 3.f));
    float sdep = fmaxf(a.sigma_depth, 1e-3f) * fmaxf(dz, 1e-4f) * (1.f + 2.5f * boot);
    float sld = a.sigma_light * (1.f + 2.0f * boot);
    float sli = a.sigma_light * (1.f + 1.5f * boot);
    float sn = fmaxf(8.f, a.sigma_normal * (1.f - 0.85f * boot));
    const float kw[3] = {3.f / 8.f, 1.f / 4.f, 1.f / 16.f};
    // The per-tap quotients of the reference's weights become products with
    // per-pixel reciprocals (same formula; the roundings differ by an ulp):
    // wz = -|dz| / (sdep * dist + 1e-6) over the six tap distances of the
    // 5x5 stencil, wdl = -|dl| * sqrt(dref) / (sld * sdd), and the indirect
    // term's sqrt(iref) / (sli * sdi), constant over the taps.
    const float inv_ld = 1.f / (sld * sdd);
    const float il_scale = sqrtf(fmaxf(cil, 1e-4f)) / (sli * sdi);
    float inv_z[6];
    {
        const int d2[6] = {0, 1, 2, 4, 5, 8};  // ki^2 + kj^2 of the stencil
#pragma unroll
        for (int k = 0; k < 6; ++k) inv_z[k] = 1.f / (sdep * (sqrtf(float(d2[k])) * a.step) + 1e-6f);
    }
    for (int kj = -2; kj <= 2; kj++)
        for (int ki = -2; ki <= 2; ki++) {
            int ni = x + ki * a.step, nj = y + kj * a.step;
            if (!(ni >= 0 && ni < a.W && nj >= 0 && nj < a.H)) continue;
            const int2 ntag = src.t(ni, nj);
            if (ntag.x != ctag.x) continue;
            int nh = max(ntag.y, 1);
            const float4 ne = src.e(ni, nj);
            float nz = ne.w;
            V3 nn{ne.x, ne.y, ne.z};
            float4 nd4 = src.d(ni, nj), ni4 = src.i(ni, nj);
            V3 nd{nd4.x, nd4.y, nd4.z}, nic{ni4.x, ni4.y, ni4.z};
            float nvd = fmaxf(0.0f, nd4.w), nvi = fmaxf(0.0f, ni4.w);
            const int r2 = ki * ki + kj * kj;
            const int zi = r2 == 0 ? 0 : (r2 == 1 ? 1 : (r2 == 2 ? 2 : (r2 == 4 ? 3 : (r2 == 5 ? 4 : 5))));
            float wz = -fabsf(cdepth - nz) * inv_z[zi];
            const float ln = log_weight(fmaxf(0.f, dot(cn, nn)), sn);
            float ndl = luminance(nd), nil = luminance(nic);
            float dref = fmaxf(fmaxf(cdl, ndl), 1e-4f);
            float wdl = -fabsf(cdl - ndl) * sqrt_fast(dref) * inv_ld;
            float wil = -fabsf(cil - nil) * il_scale;
            float hc = boot > 0.f ? (0.5f + 0.5f * fminf((float)nh / 4.f, 1.f)) : 1.f;
            float kwt = kw[abs(ki)] * kw[abs(kj)] * hc;
            float dw = exp2f(fmaf(wz + wdl, kLog2e, ln)) * kwt, iw = exp2f(fmaf(wz + wil, kLog2e, ln)) * kwt;
            fd = fd + dw * nd;
            fi = fi + iw * nic;
            twd += dw;
            twi += iw;
            vard += dw * dw * nvd;
            vari += iw * iw * nvi;
        }
    if (twd > 1e-6f)
        a.out_d[idx] = make_float4(fd.x / twd, fd.y / twd, fd.z / twd, vard / (twd * twd));
    else
        a.out_d[idx] = make_float4(cd.x, cd.y, cd.z, 1.f);
    if (twi > 1e-6f)
        a.out_i[idx] = make_float4(fi.x / twi, fi.y / twi, fi.z / twi, vari / (twi * twi));
    else
        a.out_i[idx] = make_float4(ci.x, ci.y, ci.z, 1.f);
}

// One thread per pixel, taps from global memory (large steps).
__global__ void k_svgf_atrous(AtrousArgs a, GB g) {
    int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= a.W || y >= a.H) return;
    atrous_pixel(a, g, GlobalTaps{a}, x, y);
}

// Small steps (1 and 2): the block's kTileX x kTileY pixels and their halo
// of 2 * kStep (the 5x5 taps; it also covers the 3x3 pre-blur) are staged
// once in shared memory (colour, variance, edge record and tag: 56 B per
// pixel), so each loaded pixel serves up to 25 taps of the block instead
// of being fetched per tap.
constexpr int kTileX = 32, kTileY = 8;

template <int kStep>
__global__ void __launch_bounds__(kTileX * kTileY) k_svgf_atrous_tiled(AtrousArgs a, GB g) {
    constexpr int R = 2 * kStep, RW = kTileX + 2 * R, RH = kTileY + 2 * R, N = RW * RH;
    __shared__ float4 sd[N], si[N], se[N];
    __shared__ int2 stg[N];
    const int bx = blockIdx.x * kTileX, by = blockIdx.y * kTileY;
    const int tid = threadIdx.y * kTileX + threadIdx.x;
    for (int k = tid; k < N; k += kTileX * kTileY) {
        const int gx = bx - R + k % RW, gy = by - R + k / RW;
        if (gx < 0 || gx >= a.W || gy < 0 || gy >= a.H) continue;  // never read: taps check the image bounds
        const int gi = gy * a.W + gx;
        sd[k] = a.in_d[gi];
        si[k] = a.in_i[gi];
        se[k] = a.edge[gi];
        stg[k] = a.tag[gi];
    }
    __syncthreads();
    const int x = bx + threadIdx.x, y = by + threadIdx.y;
    if (x >= a.W || y >= a.H) return;
    atrous_pixel(a, g, TileTaps{sd, si, se, stg, bx - R, by - R, RW}, x, y);
}

// ---------------------------------------------------------------------------
// host: state and frame
// ---------------------------------------------------------------------------
void SvgfState::allocate(int w, int h) {
    release();
    W = w;
    H = h;
    size_t n = (size_t)w * h;
    for (int k = 0; k < 2; ++k) {
        CRT_CUDA(cudaMalloc(&buf_d[k], n * sizeof(float4)));
        CRT_CUDA(cudaMalloc(&buf_i[k], n * sizeof(float4)));
        CRT_CUDA(cudaMalloc(&hist_d[k], n * sizeof(float4)));
        CRT_CUDA(cudaMalloc(&hist_i[k], n * sizeof(float4)));
        CRT_CUDA(cudaMalloc(&mom_d[k], n * sizeof(float2)));
        CRT_CUDA(cudaMalloc(&mom_i[k], n * sizeof(float2)));
        CRT_CUDA(cudaMalloc(&hlen[k], n * sizeof(int)));
    }
    CRT_CUDA(cudaMalloc(&edge, n * sizeof(float4)));
    CRT_CUDA(cudaMalloc(&tag, n * sizeof(int2)));
    reset_sync();
}

void SvgfState::reset_sync() {
    size_t n = (size_t)W * H;
    for (int k = 0; k < 2; ++k) {
        CRT_CUDA(cudaMemset(hist_d[k], 0, n * sizeof(float4)));
        CRT_CUDA(cudaMemset(hist_i[k], 0, n * sizeof(float4)));
        CRT_CUDA(cudaMemset(mom_d[k], 0, n * sizeof(float2)));
        CRT_CUDA(cudaMemset(mom_i[k], 0, n * sizeof(float2)));
        CRT_CUDA(cudaMemset(hlen[k], 0, n * sizeof(int)));
    }
    t = 0;
    first = true;
}

void SvgfState::release() {
    if (edge) cudaFree(edge), edge = nullptr;
    if (tag) cudaFree(tag), tag = nullptr;
    for (int k = 0; k < 2; ++k) {
        for (void **p : {(void **)&buf_d[k], (void **)&buf_i[k], (void **)&hist_d[k], (void **)&hist_i[k],
                         (void **)&mom_d[k], (void **)&mom_i[k], (void **)&hlen[k]})
            if (*p) {
                cudaFree(*p);
                *p = nullptr;
            }
    }
}

int svgf_frame(SvgfState &st, const DenoiseParams &p, const GBufferPlanes &cur, const GBufferPlanes &last,
               const float4 *noisy_d, const float4 *noisy_i, float4 *out_d, float4 *out_i, cudaStream_t s) {
    const int W = st.W, H = st.H;
    dim3 b(16, 16), g((W + 15) / 16, (H + 15) / 16);
    dim3 bt(kTileX, kTileY), gt((W + kTileX - 1) / kTileX, (H + kTileY - 1) / kTileY);
    // CRT_SVGF_TILED=0 runs every a-trous pass from global memory
    const char *tv = getenv("CRT_SVGF_TILED");
    const bool tiled = !(tv && tv[0] == '0');
    GB gc{cur.pos_tri, cur.normal_mat, cur.bary_mesh, cur.motion_depth};
    GB gl{last.pos_tri, last.normal_mat, last.bary_mesh, last.motion_depth};
    const int t = st.t;
    const int passes = st.first ? 0 : (p.atrous_iterations < 1 ? 1 : (p.atrous_iterations > 8 ? 8 : p.atrous_iterations));
    // The passes ping-pong between buf[0] and buf[1]; the last one writes
    // the caller's output directly.
    int c = 0;  // buffer holding the current result
    TemporalArgs ta;
    ta.W = W;
    ta.H = H;
    ta.max_hist = p.max_history_length;
    ta.reproj = p.reprojection_depth_factor;
    ta.noisy_d = noisy_d;
    ta.noisy_i = noisy_i;
    ta.cur_d = st.buf_d[c];
    ta.cur_i = st.buf_i[c];
    ta.hist_out_d = st.hist_d[t];
    ta.hist_out_i = st.hist_i[t];
    ta.hist_d = st.hist_d[1 - t];
    ta.hist_i = st.hist_i[1 - t];
    ta.mom_d = st.mom_d[t];
    ta.mom_i = st.mom_i[t];
    ta.lmom_d = st.mom_d[1 - t];
    ta.lmom_i = st.mom_i[1 - t];
    ta.hlen = st.hlen[t];
    ta.lhlen = st.hlen[1 - t];
    ta.first = st.first;
    k_svgf_temporal<<<g, b, 0, s>>>(ta, gc, gl, EdgeOut{st.edge, st.tag});
    int launches = 1;
    VarianceArgs va;
    va.W = W;
    va.H = H;
    va.half = 7 / 2;
    va.sigma_depth = p.sigma_depth;
    va.sigma_normal = p.sigma_normal;
    va.sigma_light = p.sigma_light;
    va.in_d = st.buf_d[c];
    va.in_i = st.buf_i[c];
    va.out_d = passes ? st.buf_d[1 - c] : out_d;
    va.out_i = passes ? st.buf_i[1 - c] : out_i;
    va.mom_d = st.mom_d[t];
    va.mom_i = st.mom_i[t];
    va.edge = st.edge;
    va.tag = st.tag;
    if (tiled && va.half == kVarHalf)
        k_svgf_variance_tiled<<<dim3((W + kVarTileX - 1) / kVarTileX, (H + kVarTileY - 1) / kVarTileY),
                                dim3(kVarTileX, kVarTileY), 0, s>>>(va, gc);
    else
        k_svgf_variance<<<g, b, 0, s>>>(va, gc);
    ++launches;
    c = 1 - c;
    for (int i = 0; i < passes; ++i) {
        AtrousArgs aa;
        aa.W = W;
        aa.H = H;
        aa.step = 1 << i;
        aa.sigma_depth = p.sigma_depth;
        aa.sigma_normal = p.sigma_normal;
        aa.sigma_light = p.sigma_light;
        aa.in_d = st.buf_d[c];
        aa.in_i = st.buf_i[c];
        const bool last_pass = i == passes - 1;
        aa.out_d = last_pass ? out_d : st.buf_d[1 - c];
        aa.out_i = last_pass ? out_i : st.buf_i[1 - c];
        aa.edge = st.edge;
        aa.tag = st.tag;
        if (aa.step == 1 && tiled)
            k_svgf_atrous_tiled<1><<<gt, bt, 0, s>>>(aa, gc);
        else if (aa.step == 2 && tiled)
            k_svgf_atrous_tiled<2><<<gt, bt, 0, s>>>(aa, gc);
        else
            k_svgf_atrous<<<g, b, 0, s>>>(aa, gc);
        ++launches;
        c = 1 - c;
    }
    CRT_CUDA(cudaGetLastError());
    st.t = 1 - t;
    st.first = false;
    return launches;
}

}  // namespace crt
