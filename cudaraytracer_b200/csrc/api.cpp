// C ABI of libcrt.so (declared in include/crt.h): contexts, scenes and ray
// queries. Every entry point converts exceptions into a crt_status and keeps
// the message in a thread-local slot (crt_last_error).
#include "api_internal.h"
#include <cstring>
#include <new>

namespace crt {

static thread_local std::string g_last_error;
void set_last_error(const std::string &msg) { g_last_error = msg; }

void DeviceScratch::reserve(size_t bytes) {
    if (bytes <= cap) return;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    CRT_CUDA(cudaMalloc(&p, bytes));
    cap = bytes;
}
DeviceScratch::~DeviceScratch() {
    if (p) cudaFree(p);
}

Scene::~Scene() {
    free_bvh(bvh);
    if (d_verts) cudaFree(d_verts);
}

}  // namespace crt

using namespace crt;

// Ray batches larger than this are streamed through the device in chunks on
// two streams so host<->device copies overlap the kernels.
static const int64_t kChunkRays = 2 << 20;

extern "C" {

const char *crt_last_error(void) { return g_last_error.c_str(); }
const char *crt_version(void) { return "crt 0.1 (sm_100a)"; }

crt_status crt_create(int device, crt_ctx **out) {
    return guard([&] {
        CRT_CHECK(out != nullptr, CRT_ERR_INVALID, "crt_create: out is null");
        int n = 0;
        CRT_CUDA(cudaGetDeviceCount(&n));
        CRT_CHECK(device >= 0 && device < n, CRT_ERR_INVALID, "crt_create: no such CUDA device");
        CRT_CUDA(cudaSetDevice(device));
        auto *c = new crt_ctx();
        c->device = device;
        for (int i = 0; i < 2; ++i) CRT_CUDA(cudaStreamCreateWithFlags(&c->streams[i], cudaStreamNonBlocking));
        c->stream = c->streams[0];
        *out = c;
    });
}

void crt_destroy(crt_ctx *ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    for (int i = 0; i < 2; ++i)
        if (ctx->streams[i]) cudaStreamDestroy(ctx->streams[i]);
    delete ctx;
}

crt_status crt_scene_from_triangles(crt_ctx *ctx, const float *tri_verts, int64_t n_tris, crt_scene **out) {
    return guard([&] {
        CRT_CHECK(ctx && tri_verts && out, CRT_ERR_INVALID, "crt_scene_from_triangles: null argument");
        CRT_CHECK(n_tris > 0, CRT_ERR_INVALID, "crt_scene_from_triangles: n_tris must be > 0");
        CRT_CUDA(cudaSetDevice(ctx->device));
        auto *s = new crt_scene();
        s->ctx = ctx;
        try {
            size_t bytes = (size_t)n_tris * 9 * sizeof(float);
            CRT_CUDA(cudaMalloc(&s->d_verts, bytes));
            CRT_CUDA(cudaMemcpyAsync(s->d_verts, tri_verts, bytes, cudaMemcpyHostToDevice, ctx->stream));
            build_bvh(s->d_verts, (int)n_tris, ctx->stream, s->bvh);
        } catch (...) {
            delete s;
            throw;
        }
        *out = s;
    });
}

void crt_scene_free(crt_scene *scene) {
    if (!scene) return;
    cudaSetDevice(scene->ctx->device);
    cudaStreamSynchronize(scene->ctx->stream);
    delete scene;
}

crt_status crt_scene_info(const crt_scene *scene, crt_scene_info_t *info) {
    return guard([&] {
        CRT_CHECK(scene && info, CRT_ERR_INVALID, "crt_scene_info: null argument");
        std::memset(info, 0, sizeof(*info));
        info->num_triangles = scene->bvh.num_tris;
        info->num_bvh_nodes = scene->bvh.num_nodes;
        info->bvh_depth = scene->bvh.depth;
        for (int k = 0; k < 3; ++k) {
            info->bounds_min[k] = scene->bvh.bounds_min[k];
            info->bounds_max[k] = scene->bvh.bounds_max[k];
        }
        info->build_ms = scene->bvh.build_ms;
        scene->fill_info(*info);
    });
}

crt_status crt_trace_closest_device(crt_scene *scene, const crt_ray *d_rays, int64_t n, crt_hit *d_hits,
                                    void *stream) {
    return guard([&] {
        CRT_CHECK(scene && (n == 0 || (d_rays && d_hits)), CRT_ERR_INVALID, "crt_trace_closest_device: null");
        CRT_CHECK(n >= 0, CRT_ERR_INVALID, "crt_trace_closest_device: negative n");
        CRT_CHECK(((uintptr_t)d_rays & 15) == 0 && ((uintptr_t)d_hits & 15) == 0, CRT_ERR_INVALID,
                  "crt_trace_closest_device: buffers must be 16-byte aligned");
        cudaStream_t s = stream ? (cudaStream_t)stream : scene->ctx->stream;
        launch_trace_closest(scene->bvh.view(), reinterpret_cast<const float4 *>(d_rays), n,
                             reinterpret_cast<float4 *>(d_hits), s);
    });
}

crt_status crt_trace_closest(crt_scene *scene, const crt_ray *rays, int64_t n, crt_hit *hits) {
    return guard([&] {
        CRT_CHECK(scene && (n == 0 || (rays && hits)), CRT_ERR_INVALID, "crt_trace_closest: null argument");
        CRT_CHECK(n >= 0, CRT_ERR_INVALID, "crt_trace_closest: negative n");
        if (n == 0) return;
        crt_ctx *ctx = scene->ctx;
        CRT_CUDA(cudaSetDevice(ctx->device));
        int64_t chunk = n < kChunkRays ? n : kChunkRays;
        size_t in_b = (size_t)chunk * sizeof(crt_ray), out_b = (size_t)chunk * sizeof(crt_hit);
        for (int k = 0; k < 2; ++k) ctx->stage[k].reserve(in_b + out_b);
        for (int64_t off = 0, c = 0; off < n; off += chunk, ++c) {
            int64_t m = (n - off) < chunk ? (n - off) : chunk;
            int k = (int)(c & 1);
            cudaStream_t s = ctx->streams[k];
            char *base = (char *)ctx->stage[k].p;
            CRT_CUDA(cudaMemcpyAsync(base, rays + off, m * sizeof(crt_ray), cudaMemcpyHostToDevice, s));
            launch_trace_closest(scene->bvh.view(), (const float4 *)base, m, (float4 *)(base + in_b), s);
            CRT_CUDA(cudaMemcpyAsync(hits + off, base + in_b, m * sizeof(crt_hit), cudaMemcpyDeviceToHost, s));
        }
        for (int k = 0; k < 2; ++k) CRT_CUDA(cudaStreamSynchronize(ctx->streams[k]));
    });
}

crt_status crt_trace_shadow_device(crt_scene *scene, const crt_shadow_query *d_q, int64_t n, uint8_t *d_occ,
                                   void *stream) {
    return guard([&] {
        CRT_CHECK(scene && (n == 0 || (d_q && d_occ)), CRT_ERR_INVALID, "crt_trace_shadow_device: null");
        CRT_CHECK(n >= 0, CRT_ERR_INVALID, "crt_trace_shadow_device: negative n");
        CRT_CHECK(((uintptr_t)d_q & 15) == 0, CRT_ERR_INVALID,
                  "crt_trace_shadow_device: queries must be 16-byte aligned");
        cudaStream_t s = stream ? (cudaStream_t)stream : scene->ctx->stream;
        launch_trace_shadow(scene->bvh.view(), reinterpret_cast<const float *>(d_q), n, d_occ, s);
    });
}

crt_status crt_trace_shadow(crt_scene *scene, const crt_shadow_query *q, int64_t n, uint8_t *occluded) {
    return guard([&] {
        CRT_CHECK(scene && (n == 0 || (q && occluded)), CRT_ERR_INVALID, "crt_trace_shadow: null argument");
        CRT_CHECK(n >= 0, CRT_ERR_INVALID, "crt_trace_shadow: negative n");
        if (n == 0) return;
        crt_ctx *ctx = scene->ctx;
        CRT_CUDA(cudaSetDevice(ctx->device));
        int64_t chunk = n < kChunkRays ? n : kChunkRays;
        size_t in_b = (size_t)chunk * sizeof(crt_shadow_query), out_b = ((size_t)chunk + 15) & ~(size_t)15;
        for (int k = 0; k < 2; ++k) ctx->stage[k].reserve(in_b + out_b);
        for (int64_t off = 0, c = 0; off < n; off += chunk, ++c) {
            int64_t m = (n - off) < chunk ? (n - off) : chunk;
            int k = (int)(c & 1);
            cudaStream_t s = ctx->streams[k];
            char *base = (char *)ctx->stage[k].p;
            CRT_CUDA(cudaMemcpyAsync(base, q + off, m * sizeof(crt_shadow_query), cudaMemcpyHostToDevice, s));
            launch_trace_shadow(scene->bvh.view(), (const float *)base, m, (uint8_t *)(base + in_b), s);
            CRT_CUDA(cudaMemcpyAsync(occluded + off, base + in_b, m, cudaMemcpyDeviceToHost, s));
        }
        for (int k = 0; k < 2; ++k) CRT_CUDA(cudaStreamSynchronize(ctx->streams[k]));
    });
}

}  // extern "C"
