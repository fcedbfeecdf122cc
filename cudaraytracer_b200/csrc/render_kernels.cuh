// Kernel-level interface of the wavefront renderer: path-state encoding,
// kernel parameter blocks and the stage kernels (defined in render.cu).
#pragma once
#include "render.h"
#include "trace.cuh"

namespace crt {

// Path metadata word: pixel index in bits 0-29, flags in 30-31.
constexpr uint32_t kFirst = 1u << 31, kSpec = 1u << 30, kPixelMask = (1u << 30) - 1;
constexpr uint32_t kTermBit = 1u << 31, kDirectBit = 1u << 30, kIndexMask = (1u << 30) - 1;

// Path queue: five float4 planes per path (SoA).
struct QueueView {
    float4 *p[5];
};

// Pixel accumulators (float4 per pixel).
struct AccumView {
    float4 *direct, *indirect, *sumsq;
};

// Pinhole camera vectors used by raygen.
struct CamView {
    float pos[3], ld[3], du[3], dv[3];
    int w, h;
};

// Per-launch constants of a bounce.
struct StepParams {
    int bounce;
    float rr;
    int rr_start;
    uint64_t seed;
    int first_sample;
    int pixels;
};

// Deferred next-event-estimation visibility records (four float4 planes).
struct ShadowView {
    float4 *r[4];
};

// The order in which the shade stage visits a bounce's paths, written by
// the extend stage into idx (2 x cap entries): the queue indices of paths
// that hit a triangle of any material but subsurface in idx[0 .. hits), of
// paths that missed in idx[cap - misses .. cap), and of subsurface hits in
// idx[cap .. cap + sss); the counts at kHitCounter, kMissCounter and
// kSssCounter of the counter block (reset by raygen and by the shadow stage
// for the next bounce). cls is the scene's slot class (1 = subsurface) or
// null. Misses only add the environment, so most warps of a sparse scene's
// first bounce are miss-only; subsurface hits trace probe rays inside the
// shade stage, so they run in warps of their own.
struct ShadeOrder {
    int *idx;
    int cap;
    const uint8_t *cls;
};

__global__ void k_raygen(CamView cam, StepParams sp, int n, QueueView q, int *counters);
__global__ void k_extend(BvhView bvh, QueueView q, const int *n_in, float4 *hits, int *counters, int out_idx,
                         int mode, ShadeOrder ord);
// Shade runs as two launches per bounce: k_shade over the shade order's
// hits, then k_shade_miss over its misses.
__global__ void k_shade(SceneView s, StepParams sp, QueueView qin, const float4 *hits, const int *n_in, QueueView qout,
                        int *counters, int out_idx, ShadowView sh, float4 *term0, float4 *term1, AccumView acc,
                        ShadeOrder ord);
__global__ void k_shade_miss(SceneView s, StepParams sp, QueueView qin, const float4 *hits, const int *n_in,
                             QueueView qout, int *counters, int out_idx, ShadowView sh, float4 *term0, float4 *term1,
                             AccumView acc, ShadeOrder ord);
__global__ void k_shadow(BvhView bvh, ShadowView sh, int *counters, QueueView qout, float4 *term0, float4 *term1,
                         AccumView acc, int mode);
// The extend stage of bounce `bounce` and the shadow stage in traversal
// mode `mode` (StageTraversal below): picks the kernel (one path per thread
// or per-lane refill) and its persistent grid for `block` threads.
void launch_extend_stage(const BvhView &bvh, const QueueView &q, const int *n_in, float4 *hits, int *counters,
                         int out_idx, int mode, int bounce, const ShadeOrder &ord, int block, cudaStream_t s);
void launch_shadow_stage(const BvhView &bvh, const ShadowView &sh, int *counters, const QueueView &qout,
                         float4 *term0, float4 *term1, const AccumView &acc, int mode, int block, cudaStream_t s);

// Blocks per grid for a persistent launch of `kernel` (all SMs at full
// occupancy).
int persistent_grid(const void *kernel, int block);

// Traversal stack entries per thread kept in shared memory by the extend
// and shadow stages (deeper entries spill to local memory), and the
// largest block those stages are launched with.
constexpr int kStageShort = 8;
constexpr int kStageMaxBlock = 256;
// How the extend and shadow stages traverse: the top of each lane's stack
// in shared memory (ShortStack) or the whole stack in local memory
// (LocalStack), over the float nodes or their 16-bit quantised copy; or
// (kStageWarp) the primary rays of bounce 0 as warp-coherent packets with
// one stack per warp in shared memory (closest_hit_warp, bvh.cuh), every
// later bounce and every shadow ray with the local stack; or (kStageRefill)
// bounce 0 one path per thread and every later extend and every shadow ray
// with per-lane ray refill (trace_dynamic, traverse.cuh), local stack.
enum StageTraversal : int {
    kStageLocal = 0,
    kStageShared = 1,
    kStageLocalQuant = 2,
    kStageSharedQuant = 3,
    kStageWarp = 4,
    kStageRefill = 5,
};
constexpr int kStageTraversalDefault = kStageLocal;

// The extend stage's mode at bounce `bounce` (kStageWarp covers bounce 0).
inline int extend_mode(int mode, int bounce) {
    return ((mode == kStageWarp && bounce > 0) || mode == kStageRefill) ? kStageLocal : mode;
}

// The server's mode: kStageTraversalDefault, or the one named by
// CRT_STAGE_TRAVERSAL (local, shared, local-quant, shared-quant, warp,
// refill; the server's stages treat warp and refill as local). The
// renderers resolve theirs with RenderParams::traversal (render.h).
int stage_traversal_env();

#ifdef __CUDACC__
// Closest hit and Light::Visible in the given mode (`sst` is the lane's
// shared-memory stack column).
template <bool kEarlyExit>
__device__ __forceinline__ Hit stage_closest(const BvhView &bvh, ShortStack<kStageShort> &sst, int mode, V3 o, V3 d,
                                             float tmin, float tmax, float t_exit = 0.f) {
    if (mode == kStageShared) return closest_hit_st<kEarlyExit, true, false>(bvh, sst, o, d, tmin, tmax, t_exit);
    if (mode == kStageSharedQuant) return closest_hit_st<kEarlyExit, true, true>(bvh, sst, o, d, tmin, tmax, t_exit);
    LocalStack lst;
    if (mode == kStageLocalQuant) return closest_hit_st<kEarlyExit, true, true>(bvh, lst, o, d, tmin, tmax, t_exit);
    return closest_hit_st<kEarlyExit, true, false>(bvh, lst, o, d, tmin, tmax, t_exit);
}

__device__ __forceinline__ bool stage_visible(const BvhView &bvh, ShortStack<kStageShort> &sst, int mode, V3 hp, V3 hn,
                                              V3 lp, V3 ln) {
    ShadowRay r;
    shadow_ray_init(r, hp, hn, lp, ln);
    const Hit hit = stage_closest<true>(bvh, sst, mode, r.o, r.dir, 1e-6f, 1e8f, r.t_exit);
    return shadow_ray_visible(r, bvh, hit);
}
#endif

}  // namespace crt
