// Wavefront renderer interface (render.cu).
#pragma once
#include "shade.cuh"
#include "bvh_build.h"
#include <vector>

namespace crt {

constexpr int64_t kRefillMinTriangles = 65536;

struct RenderParams {
    int width = 0, height = 0;
    int spp = 16;
    int max_bounces = 5;
    float rr = 0.8f;
    int rr_start_bounce = 0;  // extension; 0 = reference (RR at every shading event)
    uint64_t seed = 1;
    int spp_per_pass = 0;     // samples per wavefront; 0 = automatic
    int paths_per_pass = 0;   // paths per wavefront of multi-view batches; 0 = 8M
    int stage_block = 0;      // threads per block of the wavefront stage kernels; 0 = 128
    int stage_traversal = 0;  // CRT_STAGE_*: 0 = stage_traversal_env() (environment or default)
    int block() const { return stage_block ? stage_block : 128; }
    // The StageTraversal mode (render_kernels.cuh) of the extend/shadow
    // stages for a scene of num_tris triangles: stage_traversal if set, else
    // CRT_STAGE_TRAVERSAL, else per-lane refill from kRefillMinTriangles up
    // and the local stack below.
    int traversal(int64_t num_tris) const;
};

// Device-resident render data of a scene (everything but the BVH).
struct RenderData {
    float4 *attr = nullptr;
    uint8_t *slot_class = nullptr;  // per leaf-ordered triangle slot: 1 = subsurface material (build_slot_class)
    DMesh *meshes = nullptr;
    DMaterial *materials = nullptr;
    DLight *lights = nullptr;
    int num_meshes = 0, num_materials = 0, num_lights = 0, env_light = -1;
    cudaArray_t env_array = nullptr;
    cudaTextureObject_t env_tex = 0;
    float *env_ucdf = nullptr, *env_vcdf = nullptr;
    float2 *env_row_alias = nullptr, *env_col_alias = nullptr;
    int env_w = 0, env_h = 0;
    // diffuse textures: uchar4 arrays behind normalised-float texture objects
    std::vector<cudaArray_t> tex_arrays;
    std::vector<cudaTextureObject_t> tex_objects;
    cudaTextureObject_t *d_textures = nullptr;
    ~RenderData();
};

// Path-state buffers of one wavefront, reused across renders.
// Words of a wavefront's counter block: queue counts in [0, 4), the counts
// of the bounce's hit (other than subsurface), miss and subsurface-hit
// paths in the shade order at kHitCounter, kMissCounter and kSssCounter,
// and two 64-bit running totals of the rays the stage kernels
// traced (extend rays at word 8, shadow rays at word 10; the subsurface
// probe rays that the shade stage traces inline are not counted).
constexpr int kWavefrontCounters = 16;
constexpr int kHitCounter = 4;
constexpr int kMissCounter = 5;
constexpr int kSssCounter = 6;
constexpr int kExtendRaysCounter = 8;
constexpr int kShadowRaysCounter = 10;

struct Wavefront {
    size_t cap = 0;
    float4 *q[2][5] = {};      // two path queues, 5 x float4 per path
    float4 *hits = nullptr;    // (t, slot, b1, b2)
    float4 *shadow[4] = {};    // shadow-test records
    float4 *term[2] = {};      // terminated paths waiting for their shadow test
    int *order = nullptr;      // shade order, 2 x cap (render_kernels.cuh)
    int *counters = nullptr;   // [in0, in1, shadow, term] per bounce parity, hit/miss counts; ray counters
    void reserve(size_t paths);
    void release();
    void release_paths();
    ~Wavefront() { release(); }
};

// Accumulators (float4 per pixel, rows bottom-up as the reference's).
struct Accum {
    float4 *direct = nullptr, *indirect = nullptr, *sumsq = nullptr;
    size_t pixels = 0;
};

void upload_render_data(const HostScene &hs, RenderData &rd);
// rd.slot_class from the BVH's leaf-ordered triangles and the uploaded
// meshes and materials (after upload_render_data); left null when no
// material is subsurface.
void build_slot_class(const BvhBuffers &bvh, const HostScene &hs, RenderData &rd, cudaStream_t stream);
SceneView make_view(const BvhBuffers &bvh, const RenderData &rd);
// ComputeCameraParam (Src/Core/camera.h:58-84) from the orbit parameters.
void compute_camera(CameraState &c);
// InitCameraParam (Src/Core/scene.cpp:646-667): orbit from scene bounds.
void init_camera(CameraState &c, const float bmin[3], const float bmax[3], const float dir[3], float fovy, int w,
                 int h);
// Renders `spp` samples into acc (added to its contents) on `stream`.
// Returns the number of kernel launches issued.
int render_samples(const SceneView &view, const CameraState &cam, const RenderParams &rp, int first_sample, int spp,
                   Wavefront &wf, Accum &acc, cudaStream_t stream);

}  // namespace crt
