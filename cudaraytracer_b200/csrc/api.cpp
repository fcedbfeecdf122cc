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
    if (scratch_done) {
        cudaEventSynchronize(scratch_done);
        cudaEventDestroy(scratch_done);
    }
    free_bvh(bvh);
    if (d_verts) cudaFree(d_verts);
}

void Scene::acquire_scratch(cudaStream_t s) {
    if (scratch_done) CRT_CUDA(cudaStreamWaitEvent(s, scratch_done, 0));
}

void Scene::release_scratch(cudaStream_t s) {
    if (!scratch_done) CRT_CUDA(cudaEventCreateWithFlags(&scratch_done, cudaEventDisableTiming));
    CRT_CUDA(cudaEventRecord(scratch_done, s));
}

void Scene::fill_info(crt_scene_info_t &info) const {
    info.num_meshes = (int32_t)host.meshes.size();
    info.num_materials = (int32_t)host.materials.size();
    info.num_lights = (int32_t)host.lights.size();
    info.width = rp.width;
    info.height = rp.height;
    info.spp = rp.spp;
    info.max_bounces = rp.max_bounces;
    info.rr = rp.rr;
    info.fovy = cam.fovy;
    info.denoise = host.denoise ? 1 : 0;
    info.has_env = host.env_light >= 0 ? 1 : 0;
}

}  // namespace crt

using namespace crt;

// Ray batches larger than this are streamed through the device in chunks on
// two streams so host<->device copies overlap the kernels. 1M rays (32-48 MB
// per chunk) keeps the unoverlapped first copy and last kernel of a call
// short; measured on B200 over PCIe at 16M rays: 26.0 ms per extend+shadow
// step against 27.1 ms with 2M-ray chunks and 30.9 ms with 256K.
static const int64_t kChunkRays = 1 << 20;

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
        CRT_CUDA(cudaMalloc(&c->d_err, sizeof(int)));
        CRT_CUDA(cudaMemset(c->d_err, 0, sizeof(int)));
        *out = c;
    });
}

void crt_destroy(crt_ctx *ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    for (int i = 0; i < 2; ++i)
        if (ctx->streams[i]) cudaStreamDestroy(ctx->streams[i]);
    if (ctx->d_err) cudaFree(ctx->d_err);
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
            s->bvh.err = ctx->d_err;
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
        info->num_wide_nodes = scene->bvh.num_wide_nodes;
        info->wide_depth = scene->bvh.wide_depth;
        info->wide_build_ms = scene->bvh.wide_build_ms;
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

crt_status crt_scene_ray_counts(crt_scene *scene, void *stream, int64_t *extend_rays, int64_t *shadow_rays) {
    return guard([&] {
        CRT_CHECK(scene && extend_rays && shadow_rays, CRT_ERR_INVALID, "crt_scene_ray_counts: null argument");
        CRT_CUDA(cudaSetDevice(scene->ctx->device));
        *extend_rays = *shadow_rays = 0;
        if (!scene->wf.counters) return;
        if (stream) CRT_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
        CRT_CUDA(cudaStreamSynchronize(scene->ctx->stream));
        unsigned long long c[2];
        CRT_CUDA(cudaMemcpy(&c[0], scene->wf.counters + kExtendRaysCounter, 8, cudaMemcpyDeviceToHost));
        CRT_CUDA(cudaMemcpy(&c[1], scene->wf.counters + kShadowRaysCounter, 8, cudaMemcpyDeviceToHost));
        *extend_rays = (int64_t)c[0];
        *shadow_rays = (int64_t)c[1];
    });
}

crt_status crt_bvh8_collapse(const float *bin_nodes, int64_t num_bin_nodes, float *wide_nodes, int32_t *wide_links,
                             int64_t *num_wide, int32_t *wide_depth) {
    return guard([&] {
        CRT_CHECK(bin_nodes && num_bin_nodes > 0 && num_wide, CRT_ERR_INVALID, "crt_bvh8_collapse: bad argument");
        std::vector<float4> nodes;
        std::vector<int> links;
        const int depth = collapse_bvh8(reinterpret_cast<const float4 *>(bin_nodes), num_bin_nodes, nodes, links);
        const int64_t count = (int64_t)(nodes.size() / 4);
        if (wide_nodes && wide_links) {
            CRT_CHECK(*num_wide >= count, CRT_ERR_CAPACITY, "crt_bvh8_collapse: output arrays too small");
            std::memcpy(wide_nodes, nodes.data(), nodes.size() * sizeof(float4));
            std::memcpy(wide_links, links.data(), links.size() * sizeof(int));
        }
        *num_wide = count;
        if (wide_depth) *wide_depth = depth;
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

extern "C" {

namespace {

// Host scene -> device: BVH build over the vertices, render data upload,
// render parameters and the orbit camera from the camera block
// (Scene::Scene, Src/Core/scene.cpp:50-57 with BuildBVH :115 and
// InitCameraParam :646).
void finish_scene(crt_scene *s) {
    HostScene &h = s->host;
    size_t n = h.prim_mesh.size();
    CRT_CHECK(n < (size_t)(1 << 27) - 1, CRT_ERR_CAPACITY, "too many triangles");
    CRT_CUDA(cudaMalloc(&s->d_verts, h.verts.size() * sizeof(float)));
    CRT_CUDA(cudaMemcpy(s->d_verts, h.verts.data(), h.verts.size() * sizeof(float), cudaMemcpyHostToDevice));
    s->bvh.err = s->ctx->d_err;
    build_bvh(s->d_verts, (int)n, s->ctx->stream, s->bvh);
    upload_render_data(h, s->rd);
    build_slot_class(s->bvh, h, s->rd, s->ctx->stream);
    CRT_CUDA(cudaStreamSynchronize(s->ctx->stream));
    s->rp.width = h.width;
    s->rp.height = h.height;
    s->rp.spp = h.spp;
    s->rp.max_bounces = h.max_bounces;
    s->rp.rr = h.rr;
    init_camera(s->cam, s->bvh.bounds_min, s->bvh.bounds_max, h.direction, h.fovy, h.width, h.height);
    s->renderable = true;
}

void host_scene_from_desc(const crt_scene_desc &d, HostScene &h) {
    CRT_CHECK(d.n_tris > 0 && d.verts, CRT_ERR_INVALID, "crt_scene_from_arrays: no triangles");
    CRT_CHECK(d.n_tris < (1 << 27) - 1, CRT_ERR_CAPACITY, "crt_scene_from_arrays: too many triangles");
    CRT_CHECK(d.n_meshes > 0 && d.meshes && d.n_materials > 0 && d.materials, CRT_ERR_INVALID,
              "crt_scene_from_arrays: meshes and materials required");
    CRT_CHECK(d.n_lights >= 0 && (d.n_lights == 0 || d.lights), CRT_ERR_INVALID, "crt_scene_from_arrays: lights");
    CRT_CHECK(d.width > 0 && d.height > 0 && d.spp >= 0 && d.max_bounces >= 0, CRT_ERR_INVALID,
              "crt_scene_from_arrays: bad camera block");
    const size_t n = (size_t)d.n_tris;
    h.width = d.width;
    h.height = d.height;
    h.spp = d.spp;
    h.max_bounces = d.max_bounces;
    h.rr = d.rr;
    h.fovy = d.fovy;
    for (int k = 0; k < 3; ++k) h.direction[k] = d.direction[k];
    CRT_CHECK(d.n_textures >= 0 && (d.n_textures == 0 || d.textures), CRT_ERR_INVALID,
              "crt_scene_from_arrays: textures");
    for (int i = 0; i < d.n_textures; ++i) {
        const crt_texture_desc &td = d.textures[i];
        CRT_CHECK(td.width > 0 && td.height > 0 && td.width <= (1 << 15) && td.height <= (1 << 15) && td.rgba,
                  CRT_ERR_INVALID, "crt_scene_from_arrays: bad texture");
        HostTexture t;
        t.name = "texture" + std::to_string(i);
        t.width = td.width;
        t.height = td.height;
        t.rgba.assign(td.rgba, td.rgba + (size_t)4 * td.width * td.height);
        h.textures.push_back(std::move(t));
    }
    h.materials.resize(d.n_materials);
    h.material_names.resize(d.n_materials);
    for (int i = 0; i < d.n_materials; ++i) {
        const crt_material_desc &md = d.materials[i];
        CRT_CHECK(md.type >= MAT_LIGHT && md.type <= MAT_SUBSURFACE, CRT_ERR_INVALID,
                  "crt_scene_from_arrays: bad material type");
        DMaterial m = default_material_record();
        m.type = md.type;
        for (int k = 0; k < 3; ++k) {
            m.base[k] = md.basecolor[k];
            m.ke[k] = md.emission[k];
            m.scatter[k] = md.scatter_distance[k];
        }
        m.roughness = md.roughness;
        m.metallic = md.metallic;
        m.transmission = md.transmission;
        m.ior = md.ior;
        CRT_CHECK(md.texture >= -1 && md.texture < d.n_textures, CRT_ERR_INVALID,
                  "crt_scene_from_arrays: bad material texture");
        m.tex = md.texture;
        h.materials[i] = m;
        h.material_names[i] = "material" + std::to_string(i);
    }
    h.verts.assign(d.verts, d.verts + 9 * n);
    if (d.normals) {
        h.normals.assign(d.normals, d.normals + 9 * n);
    } else {
        h.normals.resize(9 * n);
        for (size_t t = 0; t < n; ++t) {
            float fn[3];
            face_normal(&h.verts[9 * t], fn);
            for (int c = 0; c < 3; ++c)
                for (int k = 0; k < 3; ++k) h.normals[9 * t + 3 * c + k] = fn[k];
        }
    }
    if (d.uvs)
        h.uvs.assign(d.uvs, d.uvs + 6 * n);
    else
        h.uvs.assign(6 * n, 0.f);
    h.prim_mesh.resize(n);
    int64_t next = 0;
    for (int i = 0; i < d.n_meshes; ++i) {
        const crt_mesh_desc &md = d.meshes[i];
        CRT_CHECK(md.first == next && md.count > 0 && md.first + (int64_t)md.count <= d.n_tris, CRT_ERR_INVALID,
                  "crt_scene_from_arrays: meshes must tile the triangles in order");
        CRT_CHECK(md.material >= 0 && md.material < d.n_materials, CRT_ERR_INVALID,
                  "crt_scene_from_arrays: bad mesh material");
        DMesh dm;
        std::memset(&dm, 0, sizeof(dm));
        dm.material = md.material;
        dm.light = -1;
        dm.start = md.first;
        dm.count = md.count;
        float area = 0.f;
        for (int t = 0; t < md.count; ++t) {
            area += triangle_area(&h.verts[9 * (size_t)(md.first + t)]);
            h.prim_mesh[md.first + t] = i;
        }
        dm.area = area;
        h.meshes.push_back(dm);
        h.mesh_names.push_back("mesh" + std::to_string(i));
        next += md.count;
    }
    CRT_CHECK(next == d.n_tris, CRT_ERR_INVALID, "crt_scene_from_arrays: meshes must cover every triangle");
    for (int i = 0; i < d.n_lights; ++i) {
        const crt_light_desc &ld = d.lights[i];
        DLight dl;
        std::memset(&dl, 0, sizeof(dl));
        dl.mesh = -1;
        if (ld.type == LIGHT_AREA) {
            CRT_CHECK(ld.mesh >= 0 && ld.mesh < d.n_meshes, CRT_ERR_INVALID, "crt_scene_from_arrays: bad light mesh");
            dl.type = LIGHT_AREA;
            dl.mesh = ld.mesh;
            for (int k = 0; k < 3; ++k) dl.emission[k] = ld.emission[k];
            h.meshes[ld.mesh].light = (int)h.lights.size();
        } else if (ld.type == LIGHT_ENV) {
            CRT_CHECK(d.env_rgba && d.env_width > 0 && d.env_height > 0, CRT_ERR_INVALID,
                      "crt_scene_from_arrays: environment light without an image");
            dl.type = LIGHT_ENV;
            h.env_w = d.env_width;
            h.env_h = d.env_height;
            h.env.assign(d.env_rgba, d.env_rgba + (size_t)4 * d.env_width * d.env_height);
            h.env_light = (int)h.lights.size();
        } else {
            throw Error(CRT_ERR_INVALID, "crt_scene_from_arrays: unsupported light type");
        }
        h.lights.push_back(dl);
    }
}

}  // namespace

crt_status crt_scene_load_json(crt_ctx *ctx, const char *path, crt_scene **out) {
    return guard([&] {
        CRT_CHECK(ctx && path && out, CRT_ERR_INVALID, "crt_scene_load_json: null argument");
        CRT_CUDA(cudaSetDevice(ctx->device));
        auto *s = new crt_scene();
        s->ctx = ctx;
        try {
            load_scene_json(path, s->host);
            finish_scene(s);
        } catch (...) {
            delete s;
            throw;
        }
        *out = s;
    });
}

crt_status crt_scene_from_arrays(crt_ctx *ctx, const crt_scene_desc *desc, crt_scene **out) {
    return guard([&] {
        CRT_CHECK(ctx && desc && out, CRT_ERR_INVALID, "crt_scene_from_arrays: null argument");
        CRT_CUDA(cudaSetDevice(ctx->device));
        auto *s = new crt_scene();
        s->ctx = ctx;
        try {
            host_scene_from_desc(*desc, s->host);
            finish_scene(s);
        } catch (...) {
            delete s;
            throw;
        }
        *out = s;
    });
}

crt_status crt_scene_export_geometry(const crt_scene *scene, float *verts, float *normals, float *uvs,
                                     int32_t *prim_mesh) {
    return guard([&] {
        CRT_CHECK(scene && scene->renderable, CRT_ERR_INVALID, "crt_scene_export_geometry: not a loaded scene");
        const HostScene &h = scene->host;
        if (verts) std::memcpy(verts, h.verts.data(), h.verts.size() * sizeof(float));
        if (normals) std::memcpy(normals, h.normals.data(), h.normals.size() * sizeof(float));
        if (uvs) std::memcpy(uvs, h.uvs.data(), h.uvs.size() * sizeof(float));
        if (prim_mesh) std::memcpy(prim_mesh, h.prim_mesh.data(), h.prim_mesh.size() * sizeof(int32_t));
    });
}

crt_status crt_scene_export_tables(const crt_scene *scene, float *materials, float *meshes, float *lights) {
    return guard([&] {
        CRT_CHECK(scene && scene->renderable, CRT_ERR_INVALID, "crt_scene_export_tables: not a loaded scene");
        const HostScene &h = scene->host;
        if (materials)
            for (size_t i = 0; i < h.materials.size(); ++i) {
                const DMaterial &m = h.materials[i];
                float *o = materials + 16 * i;
                float v[16] = {(float)m.type, m.base[0], m.base[1], m.base[2], m.ke[0], m.ke[1], m.ke[2], m.roughness,
                               m.metallic, m.transmission, m.scatter[0], m.scatter[1], m.scatter[2], m.ior,
                               (float)m.tex, 0.f};
                std::memcpy(o, v, sizeof(v));
            }
        if (meshes)
            for (size_t i = 0; i < h.meshes.size(); ++i) {
                const DMesh &m = h.meshes[i];
                float v[8] = {(float)m.material, (float)m.light, (float)m.start, (float)m.count, m.area, 0, 0, 0};
                std::memcpy(meshes + 8 * i, v, sizeof(v));
            }
        if (lights)
            for (size_t i = 0; i < h.lights.size(); ++i) {
                const DLight &l = h.lights[i];
                float v[8] = {(float)l.type, (float)l.mesh, l.emission[0], l.emission[1], l.emission[2], 0, 0, 0};
                std::memcpy(lights + 8 * i, v, sizeof(v));
            }
    });
}

crt_status crt_get_render_params(const crt_scene *scene, crt_render_params *p) {
    return guard([&] {
        CRT_CHECK(scene && p, CRT_ERR_INVALID, "crt_get_render_params: null argument");
        std::memset(p, 0, sizeof(*p));
        p->width = scene->rp.width;
        p->height = scene->rp.height;
        p->spp = scene->rp.spp;
        p->max_bounces = scene->rp.max_bounces;
        p->rr = scene->rp.rr;
        p->rr_start_bounce = scene->rp.rr_start_bounce;
        p->seed = scene->rp.seed;
        p->spp_per_pass = scene->rp.spp_per_pass;
        p->paths_per_pass = scene->rp.paths_per_pass;
        p->stage_block = scene->rp.stage_block;
        p->stage_traversal = scene->rp.stage_traversal;
    });
}

crt_status crt_set_render_params(crt_scene *scene, const crt_render_params *p) {
    return guard([&] {
        CRT_CHECK(scene && p && scene->renderable, CRT_ERR_INVALID, "crt_set_render_params: not a loaded scene");
        CRT_CHECK(p->width > 0 && p->height > 0 && (int64_t)p->width * p->height < (1 << 30), CRT_ERR_INVALID,
                  "crt_set_render_params: bad resolution");
        CRT_CHECK(p->spp >= 0 && p->max_bounces >= 0 && p->spp_per_pass >= 0 && p->paths_per_pass >= 0,
                  CRT_ERR_INVALID, "crt_set_render_params: negative count");
        CRT_CHECK(p->stage_block == 0 || p->stage_block == 64 || p->stage_block == 128 || p->stage_block == 256,
                  CRT_ERR_INVALID, "crt_set_render_params: stage_block must be 0, 64, 128 or 256");
        CRT_CHECK(p->stage_traversal >= CRT_STAGE_DEFAULT && p->stage_traversal <= CRT_STAGE_REFILL,
                  CRT_ERR_INVALID, "crt_set_render_params: stage_traversal must be 0-6");
        bool resized = p->width != scene->rp.width || p->height != scene->rp.height;
        scene->rp.width = p->width;
        scene->rp.height = p->height;
        scene->rp.spp = p->spp;
        scene->rp.max_bounces = p->max_bounces;
        scene->rp.rr = p->rr;
        scene->rp.rr_start_bounce = p->rr_start_bounce;
        scene->rp.seed = p->seed;
        scene->rp.spp_per_pass = p->spp_per_pass;
        scene->rp.paths_per_pass = p->paths_per_pass;
        scene->rp.stage_block = p->stage_block;
        scene->rp.stage_traversal = p->stage_traversal;
        if (resized) {
            scene->cam.width = p->width;
            scene->cam.height = p->height;
            compute_camera(scene->cam);
        }
    });
}

crt_status crt_get_camera(const crt_scene *scene, crt_camera *c) {
    return guard([&] {
        CRT_CHECK(scene && c && scene->renderable, CRT_ERR_INVALID, "crt_get_camera: not a loaded scene");
        const CameraState &s = scene->cam;
        for (int k = 0; k < 3; ++k) {
            c->target[k] = s.target[k];
            c->position[k] = s.position[k];
            c->u[k] = s.u[k];
            c->v[k] = s.v[k];
            c->w[k] = s.w[k];
            c->du[k] = s.du[k];
            c->dv[k] = s.dv[k];
            c->left_down[k] = s.left_down[k];
        }
        c->distance = s.distance;
        c->theta_deg = s.theta;
        c->phi_deg = s.phi;
        c->fovy_deg = s.fovy;
    });
}

crt_status crt_set_camera_orbit(crt_scene *scene, const crt_camera *c) {
    return guard([&] {
        CRT_CHECK(scene && c && scene->renderable, CRT_ERR_INVALID, "crt_set_camera_orbit: not a loaded scene");
        CameraState &s = scene->cam;
        for (int k = 0; k < 3; ++k) s.target[k] = c->target[k];
        s.distance = c->distance;
        s.theta = c->theta_deg;
        s.phi = c->phi_deg;
        s.fovy = c->fovy_deg;
        compute_camera(s);
    });
}

crt_status crt_render_device(crt_scene *scene, int32_t first_sample, int32_t spp, float *d_direct, float *d_indirect,
                             float *d_sumsq, void *stream) {
    return guard([&] {
        CRT_CHECK(scene && scene->renderable, CRT_ERR_INVALID, "crt_render_device: not a loaded scene");
        CRT_CHECK(d_direct && d_indirect && spp >= 0 && first_sample >= 0, CRT_ERR_INVALID,
                  "crt_render_device: bad argument");
        CRT_CUDA(cudaSetDevice(scene->ctx->device));
        cudaStream_t s = stream ? (cudaStream_t)stream : scene->ctx->stream;
        Accum acc;
        acc.direct = (float4 *)d_direct;
        acc.indirect = (float4 *)d_indirect;
        acc.sumsq = (float4 *)d_sumsq;
        acc.pixels = (size_t)scene->rp.width * scene->rp.height;
        scene->acquire_scratch(s);
        if (spp > 0)
            render_samples(make_view(scene->bvh, scene->rd), scene->cam, scene->rp, first_sample, spp, scene->wf, acc, s);
        scene->release_scratch(s);
    });
}

crt_status crt_render(crt_scene *scene, int32_t spp, float *direct, float *indirect, float *sumsq) {
    return guard([&] {
        CRT_CHECK(scene && scene->renderable, CRT_ERR_INVALID, "crt_render: not a loaded scene");
        CRT_CHECK(spp >= 0, CRT_ERR_INVALID, "crt_render: negative spp");
        CRT_CUDA(cudaSetDevice(scene->ctx->device));
        cudaStream_t s = scene->ctx->stream;
        size_t px = (size_t)scene->rp.width * scene->rp.height;
        size_t bytes = px * sizeof(float4);
        scene->acquire_scratch(s);
        CRT_CUDA(cudaStreamSynchronize(s));  // the accumulators may be reallocated below
        scene->accum.reserve(3 * bytes);
        char *base = (char *)scene->accum.p;
        CRT_CUDA(cudaMemsetAsync(base, 0, 3 * bytes, s));
        Accum acc;
        acc.direct = (float4 *)base;
        acc.indirect = (float4 *)(base + bytes);
        acc.sumsq = sumsq ? (float4 *)(base + 2 * bytes) : nullptr;
        acc.pixels = px;
        if (spp > 0)
            render_samples(make_view(scene->bvh, scene->rd), scene->cam, scene->rp, 0, spp, scene->wf, acc, s);
        if (direct) CRT_CUDA(cudaMemcpyAsync(direct, acc.direct, bytes, cudaMemcpyDeviceToHost, s));
        if (indirect) CRT_CUDA(cudaMemcpyAsync(indirect, acc.indirect, bytes, cudaMemcpyDeviceToHost, s));
        if (sumsq) CRT_CUDA(cudaMemcpyAsync(sumsq, acc.sumsq, bytes, cudaMemcpyDeviceToHost, s));
        scene->release_scratch(s);
        CRT_CUDA(cudaStreamSynchronize(s));
    });
}

}  // extern "C"

crt_svgf::~crt_svgf() {
    for (int k = 0; k < 2; ++k)
        for (void *p : {(void *)gb[k].pos_tri, (void *)gb[k].normal_mat, (void *)gb[k].bary_mesh,
                        (void *)gb[k].motion_depth})
            if (p) cudaFree(p);
    if (noisy_d) cudaFree(noisy_d);
    if (noisy_i) cudaFree(noisy_i);
}

static crt::DenoiseParams to_params(const crt_denoise_params *p) {
    crt::DenoiseParams d;
    if (p) {
        d.max_history_length = p->max_history_length;
        d.sigma_light = p->sigma_light;
        d.sigma_normal = p->sigma_normal;
        d.sigma_depth = p->sigma_depth;
        d.reprojection_depth_factor = p->reprojection_depth_factor;
        d.atrous_iterations = p->atrous_iterations;
    }
    return d;
}

static crt::GBufferPlanes to_planes(const crt_gbuffer *g) {
    crt::GBufferPlanes o;
    o.pos_tri = (float4 *)g->pos_tri;
    o.normal_mat = (ushort4 *)g->normal_mat;
    o.bary_mesh = (ushort4 *)g->bary_mesh;
    o.motion_depth = (float4 *)g->motion_depth;
    return o;
}

static crt::CameraState camera_from(const crt::CameraState &base, const crt_camera *c) {
    crt::CameraState s = base;
    for (int k = 0; k < 3; ++k) s.target[k] = c->target[k];
    s.distance = c->distance;
    s.theta = c->theta_deg;
    s.phi = c->phi_deg;
    s.fovy = c->fovy_deg;
    crt::compute_camera(s);
    return s;
}

extern "C" {

crt_status crt_denoise_params_default(crt_denoise_params *p) {
    return guard([&] {
        CRT_CHECK(p, CRT_ERR_INVALID, "crt_denoise_params_default: null");
        crt::DenoiseParams d;
        p->max_history_length = d.max_history_length;
        p->sigma_light = d.sigma_light;
        p->sigma_normal = d.sigma_normal;
        p->sigma_depth = d.sigma_depth;
        p->reprojection_depth_factor = d.reprojection_depth_factor;
        p->atrous_iterations = d.atrous_iterations;
    });
}

crt_status crt_gbuffer_from_primary(crt_scene *scene, const crt_camera *prev, const crt_gbuffer *out, void *stream) {
    return guard([&] {
        CRT_CHECK(scene && scene->renderable && out && out->pos_tri && out->normal_mat && out->bary_mesh &&
                      out->motion_depth,
                  CRT_ERR_INVALID, "crt_gbuffer_from_primary: bad argument");
        CRT_CUDA(cudaSetDevice(scene->ctx->device));
        cudaStream_t s = stream ? (cudaStream_t)stream : scene->ctx->stream;
        crt::CameraState pc = prev ? camera_from(scene->cam, prev) : scene->cam;
        gbuffer_from_primary(make_view(scene->bvh, scene->rd), scene->cam, pc, scene->bvh.bounds_min,
                             scene->bvh.bounds_max, to_planes(out), s);
    });
}

crt_status crt_svgf_create(crt_ctx *ctx, int32_t width, int32_t height, crt_svgf **out) {
    return guard([&] {
        CRT_CHECK(ctx && out && width > 0 && height > 0, CRT_ERR_INVALID, "crt_svgf_create: bad argument");
        CRT_CUDA(cudaSetDevice(ctx->device));
        auto *v = new crt_svgf();
        v->ctx = ctx;
        try {
            v->st.allocate(width, height);
        } catch (...) {
            delete v;
            throw;
        }
        *out = v;
    });
}

void crt_svgf_free(crt_svgf *s) {
    if (!s) return;
    cudaSetDevice(s->ctx->device);
    cudaStreamSynchronize(s->ctx->stream);
    delete s;
}

crt_status crt_svgf_reset(crt_svgf *s) {
    return guard([&] {
        CRT_CHECK(s, CRT_ERR_INVALID, "crt_svgf_reset: null");
        CRT_CUDA(cudaSetDevice(s->ctx->device));
        CRT_CUDA(cudaDeviceSynchronize());
        s->st.reset_sync();
        s->have_prev_cam = false;
    });
}

crt_status crt_svgf_frame(crt_svgf *s, const crt_denoise_params *p, const crt_gbuffer *cur, const crt_gbuffer *prev,
                          const float *noisy_direct, const float *noisy_indirect, float *out_direct,
                          float *out_indirect, void *stream) {
    return guard([&] {
        CRT_CHECK(s && cur && prev && noisy_direct && noisy_indirect && out_direct && out_indirect, CRT_ERR_INVALID,
                  "crt_svgf_frame: null argument");
        CRT_CUDA(cudaSetDevice(s->ctx->device));
        cudaStream_t st = stream ? (cudaStream_t)stream : s->ctx->stream;
        svgf_frame(s->st, to_params(p), to_planes(cur), to_planes(prev), (const float4 *)noisy_direct,
                   (const float4 *)noisy_indirect, (float4 *)out_direct, (float4 *)out_indirect, st);
    });
}

crt_status crt_render_svgf_frame(crt_scene *scene, crt_svgf *s, const crt_denoise_params *p, int32_t frame_index,
                                 float *out_direct, float *out_indirect, void *stream) {
    return guard([&] {
        CRT_CHECK(scene && scene->renderable && s && out_direct && out_indirect && frame_index >= 0, CRT_ERR_INVALID,
                  "crt_render_svgf_frame: bad argument");
        CRT_CHECK(s->st.W == scene->rp.width && s->st.H == scene->rp.height, CRT_ERR_INVALID,
                  "crt_render_svgf_frame: SVGF state size differs from the render resolution");
        CRT_CUDA(cudaSetDevice(scene->ctx->device));
        cudaStream_t st = stream ? (cudaStream_t)stream : scene->ctx->stream;
        size_t n = (size_t)s->st.W * s->st.H;
        if (!s->noisy_d) {
            CRT_CUDA(cudaMalloc(&s->noisy_d, n * sizeof(float4)));
            CRT_CUDA(cudaMalloc(&s->noisy_i, n * sizeof(float4)));
            for (int k = 0; k < 2; ++k) {
                CRT_CUDA(cudaMalloc(&s->gb[k].pos_tri, n * sizeof(float4)));
                CRT_CUDA(cudaMalloc(&s->gb[k].normal_mat, n * sizeof(ushort4)));
                CRT_CUDA(cudaMalloc(&s->gb[k].bary_mesh, n * sizeof(ushort4)));
                CRT_CUDA(cudaMalloc(&s->gb[k].motion_depth, n * sizeof(float4)));
                CRT_CUDA(cudaMemsetAsync(s->gb[k].pos_tri, 0, n * sizeof(float4), st));
                CRT_CUDA(cudaMemsetAsync(s->gb[k].normal_mat, 0, n * sizeof(ushort4), st));
                CRT_CUDA(cudaMemsetAsync(s->gb[k].bary_mesh, 0, n * sizeof(ushort4), st));
                CRT_CUDA(cudaMemsetAsync(s->gb[k].motion_depth, 0, n * sizeof(float4), st));
            }
        }
        scene->acquire_scratch(st);
        // framebufferReset: each denoised frame starts from cleared buffers
        CRT_CUDA(cudaMemsetAsync(s->noisy_d, 0, n * sizeof(float4), st));
        CRT_CUDA(cudaMemsetAsync(s->noisy_i, 0, n * sizeof(float4), st));
        Accum acc;
        acc.direct = s->noisy_d;
        acc.indirect = s->noisy_i;
        acc.pixels = n;
        render_samples(make_view(scene->bvh, scene->rd), scene->cam, scene->rp, frame_index, 1, scene->wf, acc, st);
        const crt::CameraState &pc = s->have_prev_cam ? s->prev_cam : scene->cam;
        gbuffer_from_primary(make_view(scene->bvh, scene->rd), scene->cam, pc, scene->bvh.bounds_min,
                             scene->bvh.bounds_max, s->gb[s->gi], st);
        svgf_frame(s->st, to_params(p), s->gb[s->gi], s->gb[1 - s->gi], s->noisy_d, s->noisy_i, (float4 *)out_direct,
                   (float4 *)out_indirect, st);
        scene->release_scratch(st);
        s->gi = 1 - s->gi;
        s->prev_cam = scene->cam;
        s->have_prev_cam = true;
    });
}

}  // extern "C"
