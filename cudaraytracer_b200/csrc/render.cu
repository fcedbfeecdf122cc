// Wavefront path tracer: raygen -> (extend -> shade -> shadow) x max_bounces.
//
// Replaces Renderer::RenderLoop's frame body (Src/Core/renderer.cuh:1144-1193):
// GenerateRayKernel (:96-115), IntersectionKernel (:132-163), ShadingKernel /
// PathTracing (:170-440) and the thrust StreamCompaction with two host syncs
// per call (:1032-1049). Here:
//  * path state is SoA (5 x float4 = 80 B per path) in two ping-pong queues;
//  * extend writes a 16 B hit record per path; shade runs the reference's
//    per-hit logic, defers the next-event-estimation visibility test to a
//    record (64 B) for the shadow kernel, and pushes surviving paths to the
//    other queue with warp-aggregated atomics (no scan, no host round trip);
//  * queue lengths live on the device, kernels are launched with a fixed
//    persistent grid that reads them, so a bounce needs no host
//    synchronisation and the whole pass can be captured in a CUDA graph;
//  * a path's radiance is added to the pixel (float4 atomics) only when the
//    path terminates, so paths still alive after max_bounces are dropped,
//    exactly as the reference drops them (renderer.cuh:1166-1193).
// Rows are bottom-up (pixel j = 0 is the bottom row), as the reference's
// accumulation buffers.
#include "path.cuh"
#include "traverse.cuh"
#include <algorithm>
#include <cmath>
#include <cstring>

namespace crt {

// ---------------------------------------------------------------------------
// host: scene upload
// ---------------------------------------------------------------------------
RenderData::~RenderData() {
    if (attr) cudaFree(attr);
    if (slot_class) cudaFree(slot_class);
    if (meshes) cudaFree(meshes);
    if (materials) cudaFree(materials);
    if (lights) cudaFree(lights);
    if (env_tex) cudaDestroyTextureObject(env_tex);
    if (env_array) cudaFreeArray(env_array);
    if (env_ucdf) cudaFree(env_ucdf);
    if (env_vcdf) cudaFree(env_vcdf);
    if (env_row_alias) cudaFree(env_row_alias);
    if (env_col_alias) cudaFree(env_col_alias);
    for (cudaTextureObject_t t : tex_objects) cudaDestroyTextureObject(t);
    for (cudaArray_t a : tex_arrays) cudaFreeArray(a);
    if (d_textures) cudaFree(d_textures);
}

template <class T>
static T *upload(const std::vector<T> &v) {
    T *d = nullptr;
    if (v.empty()) return nullptr;
    CRT_CUDA(cudaMalloc(&d, v.size() * sizeof(T)));
    CRT_CUDA(cudaMemcpy(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
    return d;
}

// Vose's alias method (deterministic worklist order) over weights w; the
// sampled index has probability w[i] / sum(w).
static void build_alias(const std::vector<double> &w, float2 *out) {
    const int n = (int)w.size();
    double sum = 0;
    for (double x : w) sum += x;
    std::vector<double> p(n);
    for (int i = 0; i < n; ++i) p[i] = sum > 0 ? w[i] * n / sum : 1.0;
    std::vector<int> small, large;
    for (int i = 0; i < n; ++i) (p[i] < 1.0 ? small : large).push_back(i);
    std::vector<float> prob(n, 1.f);
    std::vector<int> alias(n);
    for (int i = 0; i < n; ++i) alias[i] = i;
    while (!small.empty() && !large.empty()) {
        int s = small.back();
        small.pop_back();
        int l = large.back();
        prob[s] = (float)p[s];
        alias[s] = l;
        p[l] = (p[l] + p[s]) - 1.0;
        if (p[l] < 1.0) {
            large.pop_back();
            small.push_back(l);
        }
    }
    for (int i : large) prob[i] = 1.f;
    for (int i : small) prob[i] = 1.f;
    for (int i = 0; i < n; ++i) {
        int a = alias[i];
        float fa;
        std::memcpy(&fa, &a, 4);
        out[i] = make_float2(prob[i], fa);
    }
}

void upload_render_data(const HostScene &hs, RenderData &rd) {
    const size_t n = hs.prim_mesh.size();
    std::vector<float4> attr(n * 4);
    for (size_t p = 0; p < n; ++p) {
        const float *nn = &hs.normals[9 * p];
        const float *uv = &hs.uvs[6 * p];
        int m = hs.prim_mesh[p];
        float mf;
        std::memcpy(&mf, &m, 4);
        attr[4 * p + 0] = make_float4(nn[0], nn[1], nn[2], uv[0]);
        attr[4 * p + 1] = make_float4(nn[3], nn[4], nn[5], uv[1]);
        attr[4 * p + 2] = make_float4(nn[6], nn[7], nn[8], uv[2]);
        attr[4 * p + 3] = make_float4(uv[3], uv[4], uv[5], mf);
    }
    rd.attr = upload(attr);
    rd.meshes = upload(hs.meshes);
    rd.materials = upload(hs.materials);
    rd.lights = upload(hs.lights);
    rd.num_meshes = (int)hs.meshes.size();
    rd.num_materials = (int)hs.materials.size();
    rd.num_lights = (int)hs.lights.size();
    rd.env_light = hs.env_light;
    // Texture::Load (Src/Core/texture.cu:207-240): uchar4 array, wrap u,
    // clamp v, linear filtering, normalised coordinates, [0, 255] -> [0, 1]
    for (const HostTexture &t : hs.textures) {
        cudaChannelFormatDesc cd = cudaCreateChannelDesc<uchar4>();
        cudaArray_t arr = nullptr;
        CRT_CUDA(cudaMallocArray(&arr, &cd, t.width, t.height));
        rd.tex_arrays.push_back(arr);
        CRT_CUDA(cudaMemcpy2DToArray(arr, 0, 0, t.rgba.data(), (size_t)t.width * 4, (size_t)t.width * 4, t.height,
                                     cudaMemcpyHostToDevice));
        cudaResourceDesc res;
        std::memset(&res, 0, sizeof(res));
        res.resType = cudaResourceTypeArray;
        res.res.array.array = arr;
        cudaTextureDesc td;
        std::memset(&td, 0, sizeof(td));
        td.addressMode[0] = cudaAddressModeWrap;
        td.addressMode[1] = cudaAddressModeClamp;
        td.filterMode = cudaFilterModeLinear;
        td.readMode = cudaReadModeNormalizedFloat;
        td.normalizedCoords = 1;
        cudaTextureObject_t obj = 0;
        CRT_CUDA(cudaCreateTextureObject(&obj, &res, &td, nullptr));
        rd.tex_objects.push_back(obj);
    }
    rd.d_textures = upload(rd.tex_objects);
    if (hs.env_light >= 0) {
        const int W = hs.env_w, H = hs.env_h;
        rd.env_w = W;
        rd.env_h = H;
        cudaChannelFormatDesc cd = cudaCreateChannelDesc<float4>();
        CRT_CUDA(cudaMallocArray(&rd.env_array, &cd, W, H));
        CRT_CUDA(cudaMemcpy2DToArray(rd.env_array, 0, 0, hs.env.data(), (size_t)W * 16, (size_t)W * 16, H,
                                     cudaMemcpyHostToDevice));
        cudaResourceDesc res;
        std::memset(&res, 0, sizeof(res));
        res.resType = cudaResourceTypeArray;
        res.res.array.array = rd.env_array;
        cudaTextureDesc td;
        std::memset(&td, 0, sizeof(td));
        td.addressMode[0] = cudaAddressModeWrap;   // as HDRTexture::Load (texture.cu:95-100)
        td.addressMode[1] = cudaAddressModeClamp;
        td.filterMode = cudaFilterModeLinear;
        td.readMode = cudaReadModeElementType;
        td.normalizedCoords = 1;
        CRT_CUDA(cudaCreateTextureObject(&rd.env_tex, &res, &td, nullptr));
        // Importance-sampling CDFs of HDRTexture::Load (texture.cu:40-83), in
        // the same float arithmetic and order.
        std::vector<float> u((size_t)W * H), v(H);
        for (int y = 0; y < H; ++y) {
            float vsum = 0.0f;
            for (int x = 0; x < W; ++x) {
                size_t i = (size_t)y * W + x;
                float r = hs.env[4 * i], g = hs.env[4 * i + 1], b = hs.env[4 * i + 2];
                float lum = 0.2126f * r + 0.7152f * g + 0.0722f * b;
                float theta = (float)((double)(((float)y + 0.5f) / (float)H) * kPiD);
                lum *= sinf(theta);
                vsum += lum;
                u[i] = vsum;
            }
            v[y] = vsum;
        }
        for (int y = 0; y < H; ++y) {
            float rs = v[y];
            for (int x = 0; x < W; ++x) {
                size_t i = (size_t)y * W + x;
                u[i] = rs > 0.0f ? u[i] / rs : 0.0f;
            }
        }
        for (int i = 1; i < H; ++i) v[i] += v[i - 1];
        float tot = v[H - 1];
        for (int i = 0; i < H; ++i) v[i] = tot > 0.0f ? v[i] / tot : 0.0f;
        // Alias tables carrying the CDFs' discrete distribution.
        std::vector<float2> ra(H), ca((size_t)W * H);
        std::vector<double> w(H);
        for (int y = 0; y < H; ++y) w[y] = y == 0 ? v[0] : (double)(v[y] - v[y - 1]);
        build_alias(w, ra.data());
        std::vector<double> wc(W);
        for (int y = 0; y < H; ++y) {
            const float *row = &u[(size_t)y * W];
            for (int x = 0; x < W; ++x) wc[x] = x == 0 ? row[0] : (double)(row[x] - row[x - 1]);
            build_alias(wc, &ca[(size_t)y * W]);
        }
        rd.env_ucdf = upload(u);
        rd.env_vcdf = upload(v);
        rd.env_row_alias = upload(ra);
        rd.env_col_alias = upload(ca);
    }
}

namespace {
__global__ void k_slot_class(const float4 *tris, const float4 *attr, const DMesh *meshes, const DMaterial *mats, int n,
                             uint8_t *cls) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        const int prim = __float_as_int(tris[3 * (size_t)s].w);
        const int mesh = __float_as_int(attr[4 * (size_t)prim + 3].w);
        cls[s] = mats[meshes[mesh].material].type == MAT_SUBSURFACE ? 1 : 0;
    }
}
}  // namespace

void build_slot_class(const BvhBuffers &bvh, const HostScene &hs, RenderData &rd, cudaStream_t stream) {
    if (rd.slot_class) cudaFree(rd.slot_class), rd.slot_class = nullptr;
    const int n = (int)bvh.num_tris;
    bool any_sss = false;
    for (const DMaterial &m : hs.materials) any_sss = any_sss || m.type == MAT_SUBSURFACE;
    if (n <= 0 || !any_sss) return;  // no class array: every hit goes to the first region
    CRT_CUDA(cudaMalloc(&rd.slot_class, (size_t)n));
    k_slot_class<<<std::min((n + 255) / 256, 148 * 8), 256, 0, stream>>>(bvh.tris, rd.attr, rd.meshes, rd.materials,
                                                                          n, rd.slot_class);
    CRT_CUDA(cudaGetLastError());
}

SceneView make_view(const BvhBuffers &bvh, const RenderData &rd) {
    SceneView s;
    std::memset(&s, 0, sizeof(s));
    s.bvh = bvh.view();
    s.slot_of_prim = bvh.slot_of_prim;
    s.attr = rd.attr;
    s.slot_class = rd.slot_class;
    s.meshes = rd.meshes;
    s.materials = rd.materials;
    s.lights = rd.lights;
    s.num_lights = rd.num_lights;
    s.env_light = rd.env_light;
    s.env.tex = rd.env_tex;
    s.env.w = rd.env_w;
    s.env.h = rd.env_h;
    s.env.ucdf = rd.env_ucdf;
    s.env.vcdf = rd.env_vcdf;
    s.env.row_alias = rd.env_row_alias;
    s.env.col_alias = rd.env_col_alias;
    s.textures = rd.d_textures;
    // Bounds3D::Center / DiagonalLength of the scene bounds (Src/Core/bounds.h:110-118).
    float e[3];
    for (int k = 0; k < 3; ++k) {
        s.center[k] = (bvh.bounds_min[k] + bvh.bounds_max[k]) * 0.5f;
        e[k] = bvh.bounds_max[k] - bvh.bounds_min[k];
    }
    s.diag = std::sqrt(e[0] * e[0] + (e[1] * e[1] + e[2] * e[2]));
    return s;
}

// ---------------------------------------------------------------------------
// host: camera
// ---------------------------------------------------------------------------
static float deg2rad(float a) { return (float)((double)(a / 180) * kPiD); }
static float rad2deg(float r) { return (float)((double)r * 180 / kPiD); }

void compute_camera(CameraState &c) {
    float th = deg2rad(c.theta), ph = deg2rad(c.phi);
    float x = c.distance * std::sin(th) * std::sin(ph);
    float y = c.distance * std::cos(th);
    float z = c.distance * std::sin(th) * std::cos(ph);
    float off[3] = {x, y, z};
    for (int k = 0; k < 3; ++k) {
        c.position[k] = c.target[k] + off[k];
        c.lookat[k] = c.target[k];
    }
    c.up[0] = 0.f; c.up[1] = 1.f; c.up[2] = 0.f;
    auto nrm = [](float *v) {
        float z = v[0] * v[0] + (v[1] * v[1] + v[2] * v[2]);
        if (z > 0.f) {
            float s = std::sqrt(z);
            v[0] /= s; v[1] /= s; v[2] /= s;
        }
    };
    auto crs = [](const float *a, const float *b, float *o) {
        o[0] = a[1] * b[2] - a[2] * b[1];
        o[1] = a[2] * b[0] - a[0] * b[2];
        o[2] = a[0] * b[1] - a[1] * b[0];
    };
    float lp[3];
    for (int k = 0; k < 3; ++k) lp[k] = c.lookat[k] - c.position[k];
    float wv[3] = {lp[0], lp[1], lp[2]};
    nrm(wv);
    for (int k = 0; k < 3; ++k) c.w[k] = -wv[k];
    float upn[3] = {c.up[0], c.up[1], c.up[2]};
    nrm(upn);
    crs(upn, c.w, c.u);
    nrm(c.u);
    crs(c.w, c.u, c.v);
    nrm(c.v);
    c.focal = std::sqrt(lp[0] * lp[0] + (lp[1] * lp[1] + lp[2] * lp[2]));
    c.ratio = 1.f * c.width / c.height;
    float hh = 2 * c.focal * std::tan(deg2rad(c.fovy / 2));
    float ww = hh * c.ratio;
    for (int k = 0; k < 3; ++k) {
        c.du[k] = ww * c.u[k] / c.width;
        c.dv[k] = hh * c.v[k] / c.height;
        c.left_down[k] = c.lookat[k] - c.width / 2 * c.du[k] - c.height / 2 * c.dv[k];
    }
}

void init_camera(CameraState &c, const float bmin[3], const float bmax[3], const float dir[3], float fovy, int w,
                 int h) {
    float e[3];
    for (int k = 0; k < 3; ++k) {
        c.target[k] = (bmin[k] + bmax[k]) * 0.5f;
        e[k] = bmax[k] - bmin[k];
    }
    float diag = std::sqrt(e[0] * e[0] + (e[1] * e[1] + e[2] * e[2]));
    c.fovy = fovy;
    c.width = w;
    c.height = h;
    c.distance = diag * 0.5f / std::sin(deg2rad(fovy) / 2.f) * 0.6f;
    float d[3] = {dir[0], dir[1], dir[2]};
    float z = d[0] * d[0] + (d[1] * d[1] + d[2] * d[2]);
    if (z > 0.f) {
        float s = std::sqrt(z);
        for (int k = 0; k < 3; ++k) d[k] /= s;
    }
    float dn = std::sqrt(d[0] * d[0] + (d[1] * d[1] + d[2] * d[2]));
    c.theta = rad2deg(std::acos(d[1] / dn));
    c.phi = rad2deg(std::atan2(d[0], d[2]));
    compute_camera(c);
}

// ---------------------------------------------------------------------------
// wavefront buffers
// ---------------------------------------------------------------------------
void Wavefront::reserve(size_t paths) {
    if (!counters) {
        // kept across growth: [0..3] queue counts, [8..11] two 64-bit ray counters
        CRT_CUDA(cudaMalloc(&counters, kWavefrontCounters * sizeof(int)));
        CRT_CUDA(cudaMemset(counters, 0, kWavefrontCounters * sizeof(int)));
    }
    if (paths <= cap) return;
    release_paths();
    for (int q = 0; q < 2; ++q)
        for (int k = 0; k < 5; ++k) CRT_CUDA(cudaMalloc(&this->q[q][k], paths * sizeof(float4)));
    CRT_CUDA(cudaMalloc(&hits, paths * sizeof(float4)));
    for (int k = 0; k < 4; ++k) CRT_CUDA(cudaMalloc(&shadow[k], paths * sizeof(float4)));
    for (int k = 0; k < 2; ++k) CRT_CUDA(cudaMalloc(&term[k], paths * sizeof(float4)));
    CRT_CUDA(cudaMalloc(&order, 2 * paths * sizeof(int)));
    cap = paths;
}

void Wavefront::release() {
    release_paths();
    if (counters) cudaFree(counters), counters = nullptr;
}

void Wavefront::release_paths() {
    for (int q = 0; q < 2; ++q)
        for (int k = 0; k < 5; ++k)
            if (this->q[q][k]) cudaFree(this->q[q][k]), this->q[q][k] = nullptr;
    if (hits) cudaFree(hits), hits = nullptr;
    for (int k = 0; k < 4; ++k)
        if (shadow[k]) cudaFree(shadow[k]), shadow[k] = nullptr;
    for (int k = 0; k < 2; ++k)
        if (term[k]) cudaFree(term[k]), term[k] = nullptr;
    if (order) cudaFree(order), order = nullptr;
    cap = 0;
}

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------

// GenerateRayKernel + PinholeGeneratingRay (renderer.cuh:96-115,
// camera.cu:27-35): jitter (u, v), pixel (i + u, j + v) from the bottom-left.
__global__ void k_raygen(CamView cam, StepParams sp, int n, QueueView q, int *counters) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) {
        counters[0] = n;
        counters[kHitCounter] = 0;
        counters[kMissCounter] = 0;
        counters[kSssCounter] = 0;
    }
    if (i >= n) return;
    uint32_t pixel = (uint32_t)(i % sp.pixels);
    uint32_t sample = (uint32_t)(sp.first_sample + i / sp.pixels);
    int px = (int)pixel % cam.w, py = (int)pixel / cam.w;
    PathState s;
    s.rng = pcg32_seed(sp.seed, pixel, sample);
    float u0 = pcg32_uniform(s.rng), u1 = pcg32_uniform(s.rng);
    V3 ld = ld3(cam.ld), du = ld3(cam.du), dv = ld3(cam.dv), pos = ld3(cam.pos);
    V3 pp = (ld + (px + u0) * du) + (py + u1) * dv;
    s.o = pos;
    s.d = normalized(pp - pos);
    s.w = V3{1.f, 1.f, 1.f};
    s.dc = s.ic = V3{0.f, 0.f, 0.f};
    s.pdf = 0.f;
    s.pixel = pixel;
    s.first = true;
    s.spec = false;
    store_path(q, i, s);
}

// Extend: closest hit of every live path (TraceRay, renderer.cuh:124-130:
// tMin 0, closest starts at 1e8), and the path's place in the shade order.
// Also clears the next bounce's queue counters.
__global__ void __launch_bounds__(256) k_extend(BvhView bvh, QueueView q, const int *n_in, float4 *hits, int *counters,
                                                int out_idx, int mode, ShadeOrder ord) {
    __shared__ unsigned s_stack[kStageShort * kStageMaxBlock];
    ShortStack<kStageShort> st;
    st.col = s_stack + threadIdx.x;
    st.stride = blockDim.x;
    const int n = *n_in;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        counters[out_idx] = 0;
        counters[2] = 0;
        counters[3] = 0;
        atomicAdd(reinterpret_cast<unsigned long long *>(counters + kExtendRaysCounter), (unsigned long long)n);
    }
    if (mode == kStageWarp) {
        // whole warps over 32 consecutive paths; the warp's (link, mask)
        // stack takes 2 x kStackSize words of s_stack
        static_assert(kStageShort * kStageMaxBlock >= (kStageMaxBlock / 32) * 2 * kStackSize, "warp stacks");
        int *ws_link = reinterpret_cast<int *>(s_stack) + (threadIdx.x >> 5) * 2 * kStackSize;
        unsigned *ws_mask = reinterpret_cast<unsigned *>(ws_link + kStackSize);
        for (int i0 = blockIdx.x * blockDim.x + (threadIdx.x & ~31); i0 < n; i0 += gridDim.x * blockDim.x) {
            const int i = i0 + (threadIdx.x & 31);
            const bool active = i < n;
            V3 o{0.f, 0.f, 0.f}, d{0.f, 0.f, 1.f};
            if (active) {
                const float4 a = q.p[0][i], b = q.p[1][i];
                o = V3{a.x, a.y, a.z};
                d = V3{b.x, b.y, b.z};
            }
            const Hit h = closest_hit_warp(bvh, ws_link, ws_mask, active, o, d, 0.f, kTriTMax);
            if (active) {
                hits[i] = make_float4(h.t, __int_as_float(h.slot), h.b1, h.b2);
                shade_order_put(ord, counters, h.slot, i);
            }
        }
        return;
    }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float4 a = q.p[0][i], b = q.p[1][i];
        const V3 o{a.x, a.y, a.z}, d{b.x, b.y, b.z};
        Hit h = stage_closest<false>(bvh, st, mode, o, d, 0.f, kTriTMax);
        hits[i] = make_float4(h.t, __int_as_float(h.slot), h.b1, h.b2);
        shade_order_put(ord, counters, h.slot, i);
    }
}

// One shade launch over the hits (the full material code) or over the
// misses (the environment only) of a bounce's shade order: the two sets in
// separate kernels keep the misses' warps out of the hit kernel's large
// instruction footprint.
enum ShadeSet { kShadeHits = 1, kShadeMisses = 2 };

template <int kSet>
__device__ __forceinline__ void shade_body(const SceneView &s, const StepParams &sp, const QueueView &qin,
                                           const float4 *hits, const int *n_in, const QueueView &qout, int *counters,
                                           int out_idx, const ShadowView &sh, float4 *term0, float4 *term1,
                                           const AccumView &acc, const ShadeOrder &ord) {
    (void)n_in;
    const int nhit = counters[kHitCounter];
    const int t_end = kSet == kShadeHits ? nhit + counters[kSssCounter] : counters[kMissCounter];
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < t_end; t += gridDim.x * blockDim.x) {
        const int i = kSet == kShadeHits ? shade_hit_index(ord, t, nhit) : shade_miss_index(ord, t);
        PathState ps = load_path(qin, i);
        float4 hr = hits[i];
        Hit h;
        h.t = hr.x;
        h.slot = __float_as_int(hr.y);
        h.b1 = hr.z;
        h.b2 = hr.w;
        NeeRecord nee;
        nee.valid = false;
        StepResult res;
        if (kSet == kShadeMisses) {
            // miss (IntersectionKernel, renderer.cuh:139-157): environment
            // radiance weighted into direct (first bounce) or indirect.
            if (s.env_light >= 0) {
                V3 bg = env_emission(s.env, ps.d);
                if (ps.first)
                    ps.dc = ps.dc + mul(ps.w, bg);
                else
                    ps.ic = ps.ic + mul(ps.w, bg);
            }
            res = kTerminate;
        } else {
            res = path_step(s, sp, ps, h, nee);
        }
        bool cont = res == kContinue;
        int slot = warp_alloc(&counters[out_idx], cont);
        if (cont) store_path(qout, slot, ps);
        bool need_term = !cont && nee.valid;
        int tslot = warp_alloc(&counters[3], need_term);
        if (need_term) {
            term0[tslot] = make_float4(ps.dc.x, ps.dc.y, ps.dc.z, __uint_as_float(ps.pixel));
            term1[tslot] = make_float4(ps.ic.x, ps.ic.y, ps.ic.z, 0.f);
        } else if (!cont) {
            accumulate(acc, ps.pixel, ps.dc, ps.ic);
        }
        int sslot = warp_alloc(&counters[2], nee.valid);
        if (nee.valid) {
            uint32_t target = cont ? (uint32_t)slot : (kTermBit | (uint32_t)tslot);
            if (nee.direct) target |= kDirectBit;
            sh.r[0][sslot] = make_float4(nee.hp.x, nee.hp.y, nee.hp.z, nee.hn.x);
            sh.r[1][sslot] = make_float4(nee.hn.y, nee.hn.z, nee.lp.x, nee.lp.y);
            sh.r[2][sslot] = make_float4(nee.lp.z, nee.ln.x, nee.ln.y, nee.ln.z);
            sh.r[3][sslot] = make_float4(nee.C.x, nee.C.y, nee.C.z, __uint_as_float(target));
        }
    }
}

// Registers capped at 64 (4 blocks of 256 or 8 of 128 threads per SM): the
// shade body is bound by instruction fetch, and twice the resident warps of
// its natural 112 registers cover more of it than the spills cost (measured
// 5% faster per 1080p frame).
__global__ void __launch_bounds__(256, 4) k_shade(SceneView s, StepParams sp, QueueView qin, const float4 *hits,
                                                  const int *n_in, QueueView qout, int *counters, int out_idx,
                                                  ShadowView sh, float4 *term0, float4 *term1, AccumView acc,
                                                  ShadeOrder ord) {
    shade_body<kShadeHits>(s, sp, qin, hits, n_in, qout, counters, out_idx, sh, term0, term1, acc, ord);
}

// The same compiled for kMinBlocks resident 128-thread blocks per SM (4: no
// cap, 112 registers; 6: 80; 10: 48), to measure the trade against the
// default; selected by CRT_SHADE_MIN_BLOCKS for blocks of at most 128 threads.
template <int kMinBlocks>
__global__ void __launch_bounds__(128, kMinBlocks) k_shade_mb(SceneView s, StepParams sp, QueueView qin,
                                                               const float4 *hits, const int *n_in, QueueView qout,
                                                               int *counters, int out_idx, ShadowView sh,
                                                               float4 *term0, float4 *term1, AccumView acc,
                                                               ShadeOrder ord) {
    shade_body<kShadeHits>(s, sp, qin, hits, n_in, qout, counters, out_idx, sh, term0, term1, acc, ord);
}

// The misses of the shade order: a small kernel (environment lookup and
// accumulation), at full occupancy.
__global__ void __launch_bounds__(256) k_shade_miss(SceneView s, StepParams sp, QueueView qin, const float4 *hits,
                                                    const int *n_in, QueueView qout, int *counters, int out_idx,
                                                    ShadowView sh, float4 *term0, float4 *term1, AccumView acc,
                                                    ShadeOrder ord) {
    shade_body<kShadeMisses>(s, sp, qin, hits, n_in, qout, counters, out_idx, sh, term0, term1, acc, ord);
}

static int shade_min_blocks(int block) {
    const char *e = getenv("CRT_SHADE_MIN_BLOCKS");
    const int v = e ? atoi(e) : 0;
    return (block <= 128 && (v == 4 || v == 6 || v == 10)) ? v : 0;
}

// The effect of deferred NEE sample i once its visibility is known: a
// visible sample's contribution joins its path's direct or indirect
// radiance; a path that already terminated is then added to its pixel.
__device__ __forceinline__ void shadow_apply(const ShadowView &sh, int i, bool vis, const QueueView &qout,
                                             float4 *term0, float4 *term1, const AccumView &acc) {
    const float4 d = sh.r[3][i];
    uint32_t target = __float_as_uint(d.w);
    uint32_t idx = target & kIndexMask;
    bool direct = (target & kDirectBit) != 0;
    V3 C{d.x, d.y, d.z};
    if (target & kTermBit) {
        float4 t0 = term0[idx], t1 = term1[idx];
        V3 dc{t0.x, t0.y, t0.z}, ic{t1.x, t1.y, t1.z};
        if (vis) {
            if (direct)
                dc = dc + C;
            else
                ic = ic + C;
        }
        accumulate(acc, __float_as_uint(t0.w), dc, ic);
    } else if (vis) {
        if (direct) {
            float4 p2 = qout.p[2][idx], p3 = qout.p[3][idx];
            p2.w += C.x;
            p3.x += C.y;
            p3.y += C.z;
            qout.p[2][idx] = p2;
            qout.p[3][idx] = p3;
        } else {
            float4 p3 = qout.p[3][idx], p4 = qout.p[4][idx];
            p3.z += C.x;
            p3.w += C.y;
            p4.x += C.z;
            qout.p[3][idx] = p3;
            qout.p[4][idx] = p4;
        }
    }
}

// Shadow: Light::Visible for each deferred NEE sample; a visible sample's
// contribution joins its path's direct or indirect radiance; a path that
// already terminated is then added to its pixel.
__global__ void __launch_bounds__(256) k_shadow(BvhView bvh, ShadowView sh, int *counters, QueueView qout,
                                                float4 *term0, float4 *term1, AccumView acc, int mode) {
    __shared__ unsigned s_stack[kStageShort * kStageMaxBlock];
    ShortStack<kStageShort> st;
    st.col = s_stack + threadIdx.x;
    st.stride = blockDim.x;
    const int n = counters[2];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        atomicAdd(reinterpret_cast<unsigned long long *>(counters + kShadowRaysCounter), (unsigned long long)n);
        // the shade order of the next bounce starts empty (shade has read it)
        counters[kHitCounter] = 0;
        counters[kMissCounter] = 0;
        counters[kSssCounter] = 0;
    }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float4 a = sh.r[0][i], b = sh.r[1][i], c = sh.r[2][i];
        const V3 hp{a.x, a.y, a.z}, hn{a.w, b.x, b.y}, lp{b.z, b.w, c.x}, ln{c.y, c.z, c.w};
        const bool vis = stage_visible(bvh, st, mode, hp, hn, lp, ln);
        shadow_apply(sh, i, vis, qout, term0, term1, acc);
    }
}

// Extend and shadow with per-lane ray refill (trace_dynamic, traverse.cuh):
// each warp keeps 32 rays in flight over its share of the queue and a lane
// whose ray finished takes the next one. For the incoherent rays after the
// first bounce and for shadow rays (kStageRefill); same traversal and the
// same results as the one-path-per-thread kernels.
struct StageExtendJob {
    BvhView bvh;
    QueueView q;
    float4 *hits;
    int *counters;
    ShadeOrder ord;
    __device__ void setup(int i, BvhView &b, V3 &o, V3 &d, float &tmin, float &tmax, float &t_exit) {
        b = bvh;
        const float4 a = q.p[0][i], bb = q.p[1][i];
        o = V3{a.x, a.y, a.z};
        d = V3{bb.x, bb.y, bb.z};
        tmin = 0.f;
        tmax = kTriTMax;
        t_exit = 0.f;
    }
    __device__ void finish(int i, const BvhView &, const Hit &h) {
        hits[i] = make_float4(h.t, __int_as_float(h.slot), h.b1, h.b2);
        shade_order_put(ord, counters, h.slot, i);
    }
};

struct StageShadowJob {
    BvhView bvh;
    ShadowView sh;
    QueueView qout;
    float4 *term0, *term1;
    AccumView acc;
    ShadowRay r;
    __device__ void setup(int i, BvhView &b, V3 &o, V3 &d, float &tmin, float &tmax, float &t_exit) {
        b = bvh;
        const float4 a = sh.r[0][i], bb = sh.r[1][i], c = sh.r[2][i];
        shadow_ray_init(r, V3{a.x, a.y, a.z}, V3{a.w, bb.x, bb.y}, V3{bb.z, bb.w, c.x}, V3{c.y, c.z, c.w});
        o = r.o;
        d = r.dir;
        tmin = 1e-6f;
        tmax = 1e8f;
        t_exit = r.t_exit;
    }
    __device__ void finish(int i, const BvhView &b, const Hit &h) {
        shadow_apply(sh, i, shadow_ray_visible(r, b, h), qout, term0, term1, acc);
    }
};

__global__ void __launch_bounds__(256) k_extend_refill(BvhView bvh, QueueView q, const int *n_in, float4 *hits,
                                                       int *counters, int out_idx, ShadeOrder ord) {
    const int n = *n_in;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        counters[out_idx] = 0;
        counters[2] = 0;
        counters[3] = 0;
        atomicAdd(reinterpret_cast<unsigned long long *>(counters + kExtendRaysCounter), (unsigned long long)n);
    }
    StageExtendJob job{bvh, q, hits, counters, ord};
    trace_dynamic<true>(job, n);
}

__global__ void __launch_bounds__(256) k_shadow_refill(BvhView bvh, ShadowView sh, int *counters, QueueView qout,
                                                       float4 *term0, float4 *term1, AccumView acc) {
    const int n = counters[2];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        atomicAdd(reinterpret_cast<unsigned long long *>(counters + kShadowRaysCounter), (unsigned long long)n);
        counters[kHitCounter] = 0;  // the shade order of the next bounce starts empty
        counters[kMissCounter] = 0;
        counters[kSssCounter] = 0;
    }
    StageShadowJob job{bvh, sh, qout, term0, term1, acc, {}};
    trace_dynamic<true>(job, n);
}

void launch_extend_stage(const BvhView &bvh, const QueueView &q, const int *n_in, float4 *hits, int *counters,
                         int out_idx, int mode, int bounce, const ShadeOrder &ord, int block, cudaStream_t s) {
    if (mode == kStageRefill && bounce > 0) {
        k_extend_refill<<<persistent_grid((const void *)k_extend_refill, block), block, 0, s>>>(bvh, q, n_in, hits,
                                                                                             counters, out_idx, ord);
    } else {
        k_extend<<<persistent_grid((const void *)k_extend, block), block, 0, s>>>(bvh, q, n_in, hits, counters,
                                                                                   out_idx, extend_mode(mode, bounce),
                                                                                   ord);
    }
}

void launch_shadow_stage(const BvhView &bvh, const ShadowView &sh, int *counters, const QueueView &qout,
                         float4 *term0, float4 *term1, const AccumView &acc, int mode, int block, cudaStream_t s) {
    if (mode == kStageRefill)
        k_shadow_refill<<<persistent_grid((const void *)k_shadow_refill, block), block, 0, s>>>(bvh, sh, counters,
                                                                                             qout, term0, term1, acc);
    else
        k_shadow<<<persistent_grid((const void *)k_shadow, block), block, 0, s>>>(bvh, sh, counters, qout, term0,
                                                                                   term1, acc, mode);
}

// The mode named by CRT_STAGE_TRAVERSAL, or -1.
static int env_traversal() {
    const char *e = getenv("CRT_STAGE_TRAVERSAL");
    if (!e) return -1;
    const std::string v(e);
    if (v == "local") return kStageLocal;
    if (v == "shared") return kStageShared;
    if (v == "local-quant") return kStageLocalQuant;
    if (v == "shared-quant") return kStageSharedQuant;
    if (v == "warp") return kStageWarp;
    if (v == "refill") return kStageRefill;
    return -1;
}

int stage_traversal_env() {
    const int e = env_traversal();
    return e >= 0 ? e : kStageTraversalDefault;
}

int RenderParams::traversal(int64_t num_tris) const {
    // CRT_STAGE_LOCAL..CRT_STAGE_REFILL are the StageTraversal modes + 1
    if (stage_traversal > 0) return stage_traversal - 1;
    const int e = env_traversal();
    if (e >= 0) return e;
    // Per-lane refill pays for its bookkeeping once traversals are long:
    // measured 8% faster per 1080p frame on the 1.31M-triangle icosphere
    // field and 26% slower on the 36-triangle Cornell box.
    return num_tris >= kRefillMinTriangles ? kStageRefill : kStageLocal;
}

int persistent_grid(const void *kernel, int block) {
    static int sms = 0;
    if (!sms) {
        int dev;
        CRT_CUDA(cudaGetDevice(&dev));
        CRT_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    }
    int per = 0;
    CRT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, block, 0));
    return sms * std::max(1, per);
}

int render_samples(const SceneView &view, const CameraState &cam, const RenderParams &rp, int first_sample, int spp,
                   Wavefront &wf, Accum &acc, cudaStream_t stream) {
    const int pixels = cam.width * cam.height;
    CRT_CHECK(pixels > 0 && pixels <= (int)kPixelMask, CRT_ERR_INVALID, "bad resolution");
    int per_pass = rp.spp_per_pass > 0 ? rp.spp_per_pass : std::max(1, (int)((8u << 20) / (unsigned)pixels));
    per_pass = std::min(per_pass, spp);
    size_t need = (size_t)pixels * per_pass;
    CRT_CHECK(need <= kIndexMask, CRT_ERR_CAPACITY, "wavefront larger than 2^30 paths");
    wf.reserve(need);
    CamView cv;
    for (int k = 0; k < 3; ++k) {
        cv.pos[k] = cam.position[k];
        cv.ld[k] = cam.left_down[k];
        cv.du[k] = cam.du[k];
        cv.dv[k] = cam.dv[k];
    }
    cv.w = cam.width;
    cv.h = cam.height;
    AccumView av{acc.direct, acc.indirect, acc.sumsq};
    QueueView q[2];
    for (int j = 0; j < 2; ++j)
        for (int k = 0; k < 5; ++k) q[j].p[k] = wf.q[j][k];
    ShadowView sh{{wf.shadow[0], wf.shadow[1], wf.shadow[2], wf.shadow[3]}};
    const ShadeOrder ord{wf.order, (int)wf.cap, view.slot_class};
    const int blk = rp.block();
    const int smem = rp.traversal(view.bvh.num_tris);
    const int mb = shade_min_blocks(blk);
    const void *shade_fn = mb == 4    ? (const void *)k_shade_mb<4>
                           : mb == 6  ? (const void *)k_shade_mb<6>
                           : mb == 10 ? (const void *)k_shade_mb<10>
                                      : (const void *)k_shade;
    const int g_sh = persistent_grid(shade_fn, blk);
    const int g_sm = persistent_grid((const void *)k_shade_miss, blk);
    int launches = 0;
    for (int done = 0; done < spp; done += per_pass) {
        int s_here = std::min(per_pass, spp - done);
        int n = pixels * s_here;
        StepParams sp;
        sp.bounce = 0;
        sp.rr = rp.rr;
        sp.rr_start = rp.rr_start_bounce;
        sp.seed = rp.seed;
        sp.first_sample = first_sample + done;
        sp.pixels = pixels;
        k_raygen<<<(n + 255) / 256, 256, 0, stream>>>(cv, sp, n, q[0], wf.counters);
        ++launches;
        for (int b = 0; b < rp.max_bounces; ++b) {
            int in = b & 1, out = 1 - in;
            sp.bounce = b;
            launch_extend_stage(view.bvh, q[in], wf.counters + in, wf.hits, wf.counters, out, smem, b, ord, blk,
                                stream);
            if (mb == 4)
                k_shade_mb<4><<<g_sh, blk, 0, stream>>>(view, sp, q[in], wf.hits, wf.counters + in, q[out],
                                                        wf.counters, out, sh, wf.term[0], wf.term[1], av, ord);
            else if (mb == 6)
                k_shade_mb<6><<<g_sh, blk, 0, stream>>>(view, sp, q[in], wf.hits, wf.counters + in, q[out],
                                                        wf.counters, out, sh, wf.term[0], wf.term[1], av, ord);
            else if (mb == 10)
                k_shade_mb<10><<<g_sh, blk, 0, stream>>>(view, sp, q[in], wf.hits, wf.counters + in, q[out],
                                                         wf.counters, out, sh, wf.term[0], wf.term[1], av, ord);
            else
                k_shade<<<g_sh, blk, 0, stream>>>(view, sp, q[in], wf.hits, wf.counters + in, q[out], wf.counters,
                                                  out, sh, wf.term[0], wf.term[1], av, ord);
            k_shade_miss<<<g_sm, blk, 0, stream>>>(view, sp, q[in], wf.hits, wf.counters + in, q[out], wf.counters,
                                                   out, sh, wf.term[0], wf.term[1], av, ord);
            launch_shadow_stage(view.bvh, sh, wf.counters, q[out], wf.term[0], wf.term[1], av, smem, blk, stream);
            launches += 4;
        }
        CRT_CUDA(cudaGetLastError());
    }
    return launches;
}

}  // namespace crt
