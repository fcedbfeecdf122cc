/*
 * crt.h — C ABI of the B200 wavefront path tracer (libcrt.so).
 *
 * Plain C types only: opaque handles, POD structs, pointers and sizes.
 * Every entry point returns a crt_status; no C++ exception crosses the ABI.
 * Host-buffer entry points copy inputs host->device and results back inside
 * the call; "_device" variants take device pointers and a CUDA stream
 * (a cudaStream_t passed as void*; NULL selects the context's own stream,
 * cudaStreamLegacy = (void*)1 the legacy default stream) and do not
 * synchronise.
 *
 * Reference interfaces these replace (DarrenChen-CN/CudaRayTracer):
 *   Scene(const std::string&)          Src/Core/scene.cpp:50
 *   BVH::BVH / CreateBVH               Src/Core/bvh.cu:9, :308
 *   BVH::IsIntersect (closest hit)     Src/Core/bvh.cu:253
 *   Light::Visible (shadow predicate)  Src/Core/light.cu:5
 *   Renderer::RenderLoop (frame loop)  Src/Core/renderer.cuh:1106
 * The reference exposes these as in-process C++ classes and global
 * singletons (renderParam, Src/Core/scene.h:46; cameraParam,
 * Src/Core/camera.h:48); it has no FFI of its own.
 */
#ifndef CRT_H
#define CRT_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum crt_status {
    CRT_OK = 0,
    CRT_ERR_INVALID = 1,   /* bad argument (null pointer, negative size, ...) */
    CRT_ERR_IO = 2,        /* file could not be opened or read               */
    CRT_ERR_PARSE = 3,     /* malformed JSON / OBJ / HDR                     */
    CRT_ERR_CUDA = 4,      /* a CUDA runtime call failed                     */
    CRT_ERR_OOM = 5,       /* device allocation failed                       */
    CRT_ERR_CAPACITY = 6,  /* request exceeds a fixed capacity               */
    CRT_ERR_TIMEOUT = 7    /* a bounded device-side wait gave up             */
} crt_status;

typedef struct crt_ctx crt_ctx;
typedef struct crt_scene crt_scene;

/* One ray: origin + tmin, direction + tmax (32 B, two float4).
 * tmin only prunes BVH boxes and tmax is the initial closest distance, as in
 * BVH::IsIntersect(ray, info, tMin, tMax) (Src/Core/bvh.cu:253,263,283-284);
 * triangles accept 0 <= t <= 1e8 (Src/Core/bvh.cu:271 default arguments,
 * Src/Core/triangle.cu:125). */
typedef struct crt_ray {
    float ox, oy, oz, tmin;
    float dx, dy, dz, tmax;
} crt_ray;

/* Closest-hit record (16 B): distance, original primitive index (-1 = miss)
 * and the barycentrics (b1, b2) of Src/Core/triangle.cu:116-118. */
typedef struct crt_hit {
    float t;
    int32_t prim;
    float u, v;
} crt_hit;

/* Inputs of Light::Visible (Src/Core/light.cu:5-27): the shading point and its
 * geometric normal, the light sample point and its normal (48 B). */
typedef struct crt_shadow_query {
    float px, py, pz;
    float nx, ny, nz;
    float lx, ly, lz;
    float lnx, lny, lnz;
} crt_shadow_query;

/* Scene summary returned by crt_scene_info. */
typedef struct crt_scene_info_t {
    int64_t num_triangles;
    int64_t num_bvh_nodes;
    int32_t bvh_depth;
    int32_t num_meshes;
    int32_t num_materials;
    int32_t num_lights;
    float bounds_min[3];
    float bounds_max[3];
    float build_ms;        /* device BVH build time (CUDA events) */
    int32_t width, height, spp, max_bounces;
    float rr, fovy;
    int32_t denoise;
    int32_t has_env;
    int64_t num_wide_nodes;  /* nodes of the 8-wide quantised tree the traversal kernels use */
    int32_t wide_depth;
    float wide_build_ms;     /* collapse of the binary tree into it (host clock) */
} crt_scene_info_t;

/* ---- context ---------------------------------------------------------- */

/* Creates a context bound to CUDA device `device` with its own stream.
 * Replaces the implicit device/global state of the reference
 * (Src/Utils/ui.cpp:164 cudaSetDevice(0); Src/Core/scene.h:46). */
crt_status crt_create(int device, crt_ctx **out);
void crt_destroy(crt_ctx *ctx);
/* Message of the last failing call on this thread ("" if none). */
const char *crt_last_error(void);
/* Library version string. */
const char *crt_version(void);

/* ---- scenes ----------------------------------------------------------- */

/* Geometry-only scene from a triangle soup (n_tris x 9 floats: v0,v1,v2),
 * primitive index = position in the array. Builds the BVH on the device.
 * Replaces BVH::BVH(Triangle*, int, 4, SAH) + CreateBVH
 * (Src/Core/bvh.cu:9-32, :308-314; called from Src/Core/scene.cpp:115-127). */
crt_status crt_scene_from_triangles(crt_ctx *ctx, const float *tri_verts,
                                    int64_t n_tris, crt_scene **out);
void crt_scene_free(crt_scene *scene);
crt_status crt_scene_info(const crt_scene *scene, crt_scene_info_t *info);

/* Loads a scene JSON with the reference's schema and semantics (camera,
 * materials, objects as OBJ files, area and environment lights) and builds
 * its BVH on the device. Replaces Scene::Scene(path) (Src/Core/scene.cpp:50)
 * with ParseSceneFile (:129), BuildBVH (:115), InitCameraParam (:646). */
crt_status crt_scene_load_json(crt_ctx *ctx, const char *path, crt_scene **out);

/* A renderable scene from in-memory arrays, for generators: the same scene
 * crt_scene_load_json builds from the equivalent JSON/OBJ/HDR files, with
 * the JSON references already resolved (material per mesh, light mesh and
 * emission per light). Material types follow Src/Core/material.h:6-12. */
typedef struct crt_material_desc {
    int32_t type;                /* 0 light, 1 diffuse, 2 pbr, 3 dielectric, 4 subsurface */
    float basecolor[3];
    float emission[3];           /* ke (light materials) */
    float roughness, metallic, transmission;
    float scatter_distance[3];
    float ior;
    int32_t texture;             /* diffuse texture index, -1 = none */
} crt_material_desc;

typedef struct crt_texture_desc {
    int32_t width, height;
    const uint8_t *rgba;         /* width x height RGBA bytes, top row first (as decoded from the image file) */
} crt_texture_desc;

typedef struct crt_mesh_desc {
    int32_t material;            /* index into materials */
    int32_t first, count;        /* triangle range; meshes tile [0, n_tris) in order */
} crt_mesh_desc;

typedef struct crt_light_desc {
    int32_t type;                /* 0 area (over `mesh`), 2 environment (env_rgba) */
    int32_t mesh;
    float emission[3];           /* area lights */
} crt_light_desc;

typedef struct crt_scene_desc {
    int64_t n_tris;
    const float *verts;          /* n_tris x 9 (v0, v1, v2) */
    const float *normals;        /* n_tris x 9 per-vertex normals, or NULL for face normals */
    const float *uvs;            /* n_tris x 6, or NULL for zeros */
    int32_t n_meshes, n_materials, n_lights;
    const crt_mesh_desc *meshes;
    const crt_material_desc *materials;
    const crt_light_desc *lights;
    int32_t env_width, env_height;
    const float *env_rgba;       /* env_width x env_height RGBA floats, top row first */
    int32_t n_textures;
    const crt_texture_desc *textures;
    int32_t width, height, spp, max_bounces;  /* camera block (Src/Core/scene.cpp:187-252) */
    float rr, fovy;
    float direction[3];
} crt_scene_desc;

crt_status crt_scene_from_arrays(crt_ctx *ctx, const crt_scene_desc *desc, crt_scene **out);

/* Decodes a texture image as the scene loader does (PNG: all colour types,
 * 1-16 bit, non-interlaced; binary PPM) to 8-bit RGBA, top row first - the
 * pixels the reference's Texture::Load gets from stbi_load with 4 channels
 * (Src/Core/texture.cu:207-211). Host only. Call with rgba = NULL for the
 * size, then again with a w*h*4-byte buffer. */
crt_status crt_image_decode(const char *path, int32_t *w, int32_t *h, uint8_t *rgba);

/* Loaded geometry in scene order (arrays sized by crt_scene_info):
 * verts n x 9, normals n x 9 (per vertex), uvs n x 6, prim_mesh n. Any
 * pointer may be NULL. Mirrors Scene's host triangle arrays
 * (Src/Core/scene.cpp:508-536). */
crt_status crt_scene_export_geometry(const crt_scene *scene, float *verts, float *normals, float *uvs,
                                     int32_t *prim_mesh);
/* Material / mesh / light tables: materials n x 16 floats (type, base[3],
 * ke[3], roughness, metallic, transmission, scatter[3], ior, tex, 0),
 * meshes n x 8 (material, light, start, count, area, 0, 0, 0), lights
 * n x 8 (type, mesh, emission[3], 0, 0, 0); integers stored as float values. */
crt_status crt_scene_export_tables(const crt_scene *scene, float *materials, float *meshes, float *lights);

/* ---- rendering -------------------------------------------------------- */

/* Render parameters; defaults come from the scene JSON camera block
 * (Src/Core/scene.cpp:187-252) and CameraParam (Src/Core/camera.h:40-44). */
typedef struct crt_render_params {
    int32_t width, height;    /* resolution */
    int32_t spp;              /* samples per pixel of one crt_render call */
    int32_t max_bounces;      /* extend/shade iterations (renderer.cuh:1166) */
    float rr;                 /* Russian-roulette continuation probability */
    int32_t rr_start_bounce;  /* extension: first bounce that applies RR; 0 = reference */
    uint64_t seed;            /* PCG32 seed of the per-path streams */
    int32_t spp_per_pass;     /* samples per wavefront of crt_render*; 0 = automatic */
    int32_t paths_per_pass;   /* paths per wavefront of crt_render_views; 0 = 8M */
    int32_t stage_block;      /* threads per block of the extend/shade/shadow wavefront stages
                                 (64, 128 or 256); 0 = 128 */
    int32_t stage_traversal;  /* BVH traversal of the extend and shadow stages: 0 = library
                                 default, else one of CRT_STAGE_* below */
} crt_render_params;

/* crt_render_params.stage_traversal: where each path's traversal stack lives
 * and which node layout it reads. */
#define CRT_STAGE_DEFAULT 0       /* CRT_STAGE_TRAVERSAL from the environment, else LOCAL */
#define CRT_STAGE_LOCAL 1         /* 64-entry stack in local memory, 64 B float nodes */
#define CRT_STAGE_SHARED 2        /* top 8 entries in shared memory, 64 B float nodes */
#define CRT_STAGE_LOCAL_QUANT 3   /* local stack, 32 B nodes with 16-bit quantised boxes */
#define CRT_STAGE_SHARED_QUANT 4  /* shared short stack, 32 B quantised nodes */
#define CRT_STAGE_WARP 5          /* primary rays as warp-coherent packets, one stack per warp in shared
                                     memory; later bounces and shadow rays as LOCAL */
#define CRT_STAGE_REFILL 6        /* primary rays as LOCAL; later bounces and shadow rays with per-lane
                                     ray refill (each warp keeps 32 rays in flight), local stack */

crt_status crt_get_render_params(const crt_scene *scene, crt_render_params *p);
crt_status crt_set_render_params(crt_scene *scene, const crt_render_params *p);

/* Orbit camera (CameraParam, Src/Core/camera.h:11-46). Setting recomputes
 * the pinhole basis as Camera::ComputeCameraParam (camera.h:58-84). */
typedef struct crt_camera {
    float target[3];
    float distance, theta_deg, phi_deg, fovy_deg;
    float position[3], u[3], v[3], w[3];  /* derived, ignored on set */
    float du[3], dv[3], left_down[3];     /* derived: pixel steps, corner */
} crt_camera;

crt_status crt_get_camera(const crt_scene *scene, crt_camera *cam);
crt_status crt_set_camera_orbit(crt_scene *scene, const crt_camera *cam);

/* Renders spp samples per pixel from a cleared frame and copies the float
 * accumulators to host buffers of width*height*4 floats: sums over samples
 * of the direct and indirect radiance (rgb + 0) and, optionally, the sum of
 * squares of each sample's total radiance (rgb + sample count). Rows are
 * bottom-up, as the reference's direct/indirect lighting buffers
 * (Src/Core/renderer.cuh:56-59, 117-122); divide by spp for the image.
 * Replaces the non-denoised progressive loop of Renderer::RenderLoop
 * (Src/Core/renderer.cuh:1144-1193). Any output pointer may be NULL. */
crt_status crt_render(crt_scene *scene, int32_t spp, float *direct, float *indirect, float *sumsq);
/* Adds samples [first_sample, first_sample + spp) into device accumulators
 * (float4 per pixel; sumsq may be NULL) on `stream`, asynchronously. */
crt_status crt_render_device(crt_scene *scene, int32_t first_sample, int32_t spp, float *d_direct,
                             float *d_indirect, float *d_sumsq, void *stream);

/* Running totals of the rays the scene's wavefront renders have traced
 * since it was created (crt_render, crt_render_device, crt_render_views):
 * closest-hit extend rays (path vertices) and shadow rays (Light::Visible
 * tests). Subsurface probe rays, traced inside the shade stage, are not
 * counted. Waits for the scene's work on the context stream and `stream`.
 * No counterpart in the reference. */
crt_status crt_scene_ray_counts(crt_scene *scene, void *stream, int64_t *extend_rays, int64_t *shadow_rays);

/* Same as crt_render_device but allocates no device memory: the path queues
 * live in a fixed scratch area inside the library's device image (18.4 MB
 * per GPU that loads the library, held until exit), for hosts that own the
 * GPU memory pool and forbid foreign cudaMalloc/cudaFree during a frame
 * (engines, viewport plugins, real-time services). At most 65,536 paths per
 * wavefront: images with more than 65,536 pixels return CRT_ERR_CAPACITY;
 * smaller images run ceil(spp / per_pass) wavefronts of per_pass samples,
 * per_pass = min(65,536 / pixels, spp_per_pass when set). The stage block
 * size follows stage_block as in crt_render_device. The first call on a device looks up the scratch address and must come
 * before any stream capture on that device. All calls share the scratch,
 * so calls whose GPU work overlaps race; the caller must order them.
 * No counterpart in the reference (its renderer allocates its buffers in
 * Renderer::CudaInit). */
crt_status crt_render_device_noalloc(crt_scene *scene, int32_t first_sample, int32_t spp, float *d_direct,
                                     float *d_indirect, float *d_sumsq, void *stream);

/* Batched multi-view rendering (no reference counterpart: the reference
 * renders one view, one sample per pixel per frame). Renders samples
 * [first_sample, first_sample + spp) of n_views orbit cameras (same
 * resolution as the scene's render params) into view-major device
 * accumulators of n_views*width*height float4 each. All views' paths share
 * wavefronts of paths_per_pass paths; with use_graph != 0 one pass (raygen,
 * max_bounces x (extend, shade, shadow), pass advance) is captured once as a
 * CUDA graph and replayed. Asynchronous on `stream`. */
crt_status crt_render_views(crt_scene *scene, int32_t n_views, const crt_camera *cams, int32_t first_sample,
                            int32_t spp, float *d_direct, float *d_indirect, float *d_sumsq, int32_t use_graph,
                            void *stream);

/* ---- multi-scene render server ----------------------------------------- */

/* Continuous batching of render requests over resident scenes (no reference
 * counterpart: the reference renders one scene, one request at a time, behind
 * the renderParam singleton, Src/Core/scene.h:20-46, and
 * Renderer::RenderLoop, Src/Core/renderer.cuh:1106-1307). Scenes added to a
 * server stay resident and owned by the caller, who keeps them alive until
 * crt_server_free. Requests (scene, resolution, spp, camera, seed) queue and
 * are admitted, oldest first, while a request slot is free and the HBM
 * budget holds the scenes, the shared wavefront and every admitted request's
 * accumulators. Each wavefront pass packs up to paths_per_pass paths of the
 * admitted requests in admission order; up to passes_in_flight passes are
 * queued on the GPU ahead of the host. A request's image equals that of
 * crt_render_device with the same camera, render parameters and seed, up to
 * the order of float additions into its pixels. */
typedef struct crt_server crt_server;

typedef struct crt_server_config {
    int64_t hbm_budget_bytes; /* scenes + wavefront + request accumulators; 0 = 150 GiB */
    int32_t paths_per_pass;   /* shared wavefront size; 0 = 8M paths */
    int32_t max_requests;     /* admitted (unreleased) request slots; 0 = 4096; at most 2^20 */
    int32_t passes_in_flight; /* passes queued on the GPU; 0 = 2; at most 64 */
    int32_t schedule;         /* how a pass is filled from the admitted requests:
                                 CRT_SCHED_SHORTEST_FIRST (0, default) or CRT_SCHED_ADMISSION_ORDER */
} crt_server_config;

/* Pass filling. Shortest first: the oldest admitted request takes up to half
 * of each pass (so no request starves), the rest of the pass goes to the
 * requests with the fewest paths left, which keeps small requests' latency
 * low behind large ones. Admission order: requests in the order they were
 * admitted (first come, first served). */
#define CRT_SCHED_SHORTEST_FIRST 0
#define CRT_SCHED_ADMISSION_ORDER 1

typedef struct crt_request {
    int32_t scene;            /* id from crt_server_add_scene */
    int32_t width, height;    /* resolution */
    int32_t spp;              /* samples per pixel */
    int32_t max_bounces;      /* extend/shade iterations */
    float rr;                 /* Russian-roulette continuation probability */
    int32_t rr_start_bounce;  /* first bounce that applies RR; 0 = reference */
    uint64_t seed;            /* PCG32 seed of the request's path streams */
    crt_camera camera;        /* orbit parameters (target, distance, theta, phi, fovy); derived fields ignored */
} crt_request;

typedef enum crt_request_state { CRT_REQ_QUEUED = 0, CRT_REQ_RUNNING = 1, CRT_REQ_DONE = 2 } crt_request_state;

typedef struct crt_server_stats {
    int64_t queued, running, done; /* requests by state (done = finished, not yet released) */
    int64_t passes, paths;         /* wavefront passes and paths enqueued so far */
    int64_t bytes_budget, bytes_scenes, bytes_wavefront, bytes_requests, bytes_pool;
    int32_t num_scenes, passes_in_flight;
} crt_server_stats;

crt_status crt_server_create(crt_ctx *ctx, const crt_server_config *cfg, crt_server **out);
void crt_server_free(crt_server *srv);
/* Makes a loaded scene resident in the server; CRT_ERR_CAPACITY when its
 * device bytes do not fit the budget. */
crt_status crt_server_add_scene(crt_server *srv, crt_scene *scene, int32_t *scene_id);
/* Queues a request; CRT_ERR_CAPACITY when it could never fit the budget. */
crt_status crt_server_submit(crt_server *srv, const crt_request *req, int64_t *request_id);
/* Retires finished passes, admits queued requests and enqueues passes up to
 * passes_in_flight. Non-blocking unless `wait` != 0, which blocks until at
 * least one request finishes when work is in flight. *n_done (may be NULL)
 * = requests that finished during this call. */
crt_status crt_server_step(crt_server *srv, int32_t wait, int32_t *n_done);
/* *state = a crt_request_state. */
crt_status crt_server_poll(crt_server *srv, int64_t request_id, int32_t *state);
/* Copies a finished request's accumulators (width*height float4 each, sums
 * over spp, rows bottom-up) to host memory. */
crt_status crt_server_result(crt_server *srv, int64_t request_id, float *direct, float *indirect);
/* Device pointers to a finished request's accumulators, valid until release. */
crt_status crt_server_result_device(crt_server *srv, int64_t request_id, const float **d_direct,
                                    const float **d_indirect);
/* Frees a finished or still-queued request's slot and buffers. */
crt_status crt_server_release(crt_server *srv, int64_t request_id);
crt_status crt_server_get_stats(crt_server *srv, crt_server_stats *st);

/* ---- SVGF denoising ---------------------------------------------------- */

/* G-buffer planes in device memory, width*height entries each, rows
 * bottom-up, with the encodings of the reference's raster G-buffer
 * (Shader/gbuffer.fs:16-38; Src/Core/renderer.cuh:32-54):
 *   pos_tri      4 floats  world position, triangle index within its mesh
 *   normal_mat   4 uint16  uint((n*0.5+0.5)*65535) of the interpolated normal, material id
 *   bary_mesh    4 uint16  uint(barycentrics*65535), mesh id + 1
 *   motion_depth 4 floats  NDC motion (current - previous camera), linear depth, fwidth(depth)
 * Background pixels are all zero. */
typedef struct crt_gbuffer {
    float *pos_tri;
    uint16_t *normal_mat;
    uint16_t *bary_mesh;
    float *motion_depth;
} crt_gbuffer;

/* DenoiseParam (Src/Utils/ui.h:14-25). */
typedef struct crt_denoise_params {
    int32_t max_history_length; /* 24 */
    float sigma_light;          /* 8 */
    float sigma_normal;         /* 256 */
    float sigma_depth;          /* 1 */
    float reprojection_depth_factor; /* 0.1 */
    int32_t atrous_iterations;  /* 5 */
} crt_denoise_params;

typedef struct crt_svgf crt_svgf;

crt_status crt_denoise_params_default(crt_denoise_params *p);

/* G-buffer of the scene's current camera from primary rays through pixel
 * centres (nearest surface of either facing, as the reference's raster pass
 * without culling); motion vectors against `prev` (NULL = the current
 * camera, i.e. no motion). Replaces RenderGBuffer (renderer.cuh:1446-1503). */
crt_status crt_gbuffer_from_primary(crt_scene *scene, const crt_camera *prev, const crt_gbuffer *out,
                                    void *stream);

/* Display resolve and debug views (GatherKernel, Src/Core/renderer.cuh:956-1030)
 * into width*height uchar4 device pixels (the scene's render resolution), in
 * the reference's display-buffer layout: mode 0 colour ((direct + indirect)
 * / spp, or the sum as is when `denoised`; gamma 1/2.2; vertically flipped
 * rows), 1 linear depth, 2 shading normal, 3 mesh id colours, 4 position in
 * the scene bounds (modes 1-4 from the G-buffer `gb`, which may be NULL for
 * mode 0). Asynchronous on `stream`. */
crt_status crt_gather(crt_scene *scene, int32_t mode, int32_t spp, int32_t denoised, const float *d_direct,
                      const float *d_indirect, const crt_gbuffer *gb, void *d_pixels, void *stream);

/* SVGF state (temporal history, moments, history lengths) for a w x h image. */
crt_status crt_svgf_create(crt_ctx *ctx, int32_t width, int32_t height, crt_svgf **out);
void crt_svgf_free(crt_svgf *s);
/* Clears the history; the next frame is a first frame. */
crt_status crt_svgf_reset(crt_svgf *s);

/* One SVGF frame over device buffers (float4 per pixel, rgb used): temporal
 * reprojection against the history (TemporalDenoising, renderer.cuh:524),
 * 7x7 variance estimate while history < 4 (ComputeVarianceKernel, :689) and
 * atrous_iterations a-trous passes at steps 1, 2, 4, ... (AtrousKernel, :807;
 * none on the first frame), in the order of RenderLoop's denoise block
 * (:1208-1258). Outputs are float4 (rgb, variance). */
crt_status crt_svgf_frame(crt_svgf *s, const crt_denoise_params *p, const crt_gbuffer *cur, const crt_gbuffer *prev,
                          const float *noisy_direct, const float *noisy_indirect, float *out_direct,
                          float *out_indirect, void *stream);

/* The reference's denoised frame (renderParam.denoise, renderer.cuh:1144-1304):
 * renders 1 sample per pixel (sample index = frame_index), builds the
 * G-buffer against the camera of the previous frame of this state, runs
 * SVGF and writes the denoised direct/indirect float4 planes (device). */
crt_status crt_render_svgf_frame(crt_scene *scene, crt_svgf *s, const crt_denoise_params *p, int32_t frame_index,
                                 float *out_direct, float *out_indirect, void *stream);

/* ---- ray queries ------------------------------------------------------ */

/* Closest hit for n rays in host memory (BVH::IsIntersect, Src/Core/bvh.cu:253
 * with Triangle::IsIntersect, Src/Core/triangle.cu:15). */
crt_status crt_trace_closest(crt_scene *scene, const crt_ray *rays, int64_t n,
                             crt_hit *hits);
/* Same on device buffers, asynchronous on `stream` (cudaStream_t or NULL). */
crt_status crt_trace_closest_device(crt_scene *scene, const crt_ray *d_rays,
                                    int64_t n, crt_hit *d_hits, void *stream);

/* Light::Visible predicate (Src/Core/light.cu:5-27) for n queries; writes
 * occluded[i] = 1 when the reference would return false (not visible). */
crt_status crt_trace_shadow(crt_scene *scene, const crt_shadow_query *q,
                            int64_t n, uint8_t *occluded);
crt_status crt_trace_shadow_device(crt_scene *scene, const crt_shadow_query *d_q,
                                   int64_t n, uint8_t *d_occluded, void *stream);

/* Host-side collapse of a binary node array (this library's 64 B two-child
 * layout, 16 floats per node, root at 0, as built on the device for every
 * scene) into the 8-wide quantised layout the trace kernels read: 16 floats
 * (64 B) per wide node and 8 child links per wide node. With wide_nodes or
 * wide_links NULL only the counts are returned; otherwise both arrays must
 * hold *num_wide (in: capacity, out: count) nodes. No counterpart in the
 * reference, whose traversal reads the binary tree it builds
 * (BVH::FlattenBVHTree, Src/Core/bvh.cu:186-206). */
crt_status crt_bvh8_collapse(const float *bin_nodes, int64_t num_bin_nodes, float *wide_nodes,
                             int32_t *wide_links, int64_t *num_wide, int32_t *wide_depth);

/* ---- tensor-core 3x3 convolutions (learned denoiser) ------------------- */

/* No reference counterpart: the dense contractions of the kernel-predicting
 * denoiser, as BF16 x BF16 -> FP32 implicit GEMMs on the sm_100a tensor cores
 * (tcgen05). Activations are NHWC BF16 (bit patterns as uint16), n images of
 * h x w pixels; channel counts are multiples of 16 (input channels up to
 * 512, output channels in [16, 256]; the data gradient's output is the
 * forward's input, so it takes cin <= 256); stride 1, zero padding 1; tap
 * t = 3 * (dy + 1) + (dx + 1). Activation, weight, mask and BF16 output
 * buffers are 16-byte aligned (the kernels read them with TMA and store
 * 16 B vectors); FP32 outputs 4-byte aligned; other alignments are refused
 * with CRT_ERR_INVALID. All asynchronous on `stream` (NULL = the context
 * stream). */
/* out[p, o] = bias[o] + sum_{t, c} in[p + off(t), c] * w[t][o][c], ReLU if
 * relu != 0; written as BF16 (d_out_bf16) and/or FP32 (d_out_f32). */
crt_status crt_conv3x3_forward(crt_ctx *ctx, const void *d_in, int32_t n, int32_t h, int32_t w, int32_t cin,
                               const void *d_weights, const float *d_bias, int32_t cout, int32_t relu,
                               void *d_out_bf16, float *d_out_f32, void *stream);
/* grad_in[p, c] = sum_{t, o} grad_out[p - off(t), o] * wt[t][c][o] with
 * wt[t] = w[t] transposed; multiplied by (mask[p, c] > 0) when d_mask (the
 * layer input, a ReLU output) is given. */
crt_status crt_conv3x3_backward_data(crt_ctx *ctx, const void *d_grad_out, int32_t n, int32_t h, int32_t w,
                                     int32_t cout, const void *d_weights_t, int32_t cin, const void *d_mask,
                                     void *d_grad_in, void *stream);
/* grad_w[t][o][c] += sum_p in[p + off(t), c] * grad_out[p, o] (FP32). */
crt_status crt_conv3x3_backward_weights(crt_ctx *ctx, const void *d_in, const void *d_grad_out, int32_t n,
                                        int32_t h, int32_t w, int32_t cin, int32_t cout, float *d_grad_w,
                                        void *stream);
/* ---- learned kernel-predicting denoiser (KPCN) ------------------------ */

/* A 3-level U-Net (32/64/96 channels) on the tensor-core convolutions above
 * that predicts a 5x5 filter per pixel, applied to the noisy radiance; no
 * reference counterpart (the reference filters with SVGF only). Images are
 * n x h x w with h, w multiples of 4. Features: 16 BF16 channels per pixel
 * (crt_kpcn_features); radiance: float4 per pixel (rgb, unused). */
typedef struct crt_kpcn crt_kpcn;
crt_status crt_kpcn_create(crt_ctx *ctx, uint64_t seed, crt_kpcn **out);
void crt_kpcn_free(crt_kpcn *k);
/* Parameters as one FP32 vector: per layer (e0a e0b e1a e1b e2a e2b d1a d1b
 * d0a d0b out) the weights [9][cout][cin] then the bias [cout]. */
crt_status crt_kpcn_num_params(const crt_kpcn *k, int64_t *n);
crt_status crt_kpcn_get_params(crt_kpcn *k, float *host);
crt_status crt_kpcn_set_params(crt_kpcn *k, const float *host);
crt_status crt_kpcn_get_grads(crt_kpcn *k, float *host);
/* Network input from a render: noisy = (direct + indirect) / spp per pixel
 * (float4) and the 16 feature channels: log(1 + noisy rgb), albedo of the
 * primary-hit material, decoded shading normal, linear depth / depth_scale,
 * motion (from a crt_gbuffer of the same view), 1 / sqrt(spp), 3 zeros. */
crt_status crt_kpcn_features(crt_scene *scene, const crt_gbuffer *gb, const float *d_direct, const float *d_indirect,
                             int32_t spp, int64_t pixels, float depth_scale, void *d_features, float *d_noisy,
                             void *stream);
/* d_out (float4 per pixel) = the filtered radiance. */
crt_status crt_kpcn_forward(crt_kpcn *k, int32_t n, int32_t h, int32_t w, const void *d_features,
                            const float *d_noisy, float *d_out, void *stream);
/* Forward, relMSE loss against d_target (mean over pixels and RGB of
 * (out - ref)^2 / (ref^2 + 0.01)), backward; then an Adam step when lr > 0.
 * *loss (may be NULL) receives the batch loss (synchronises). */
crt_status crt_kpcn_train_step(crt_kpcn *k, int32_t n, int32_t h, int32_t w, const void *d_features,
                               const float *d_noisy, const float *d_target, float lr, float *loss, void *stream);
/* Internal tensors of the last forward (tests): 0..9 layer outputs (BF16),
 * 10 filter logits (FP32, 32 per pixel), 11 pool0, 12 pool1, 13 cat1,
 * 14 cat0; `bytes` must equal the tensor's size. */
crt_status crt_kpcn_debug_tensor(crt_kpcn *k, int32_t which, void *host, int64_t bytes);

/* Synchronises the device and reports (clearing the flag) a device-side
 * error recorded by this context's kernels: CRT_ERR_TIMEOUT when a
 * tensor-core kernel gave up a bounded wait, CRT_ERR_CUDA when a BVH
 * traversal met a node, leaf or stack depth outside the tree and stopped
 * that ray instead of reading out of bounds. */
crt_status crt_check_device_errors(crt_ctx *ctx);

#ifdef __cplusplus
}
#endif
#endif /* CRT_H */
