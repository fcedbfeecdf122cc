// Standalone extend (closest-hit) and shadow (Light::Visible) kernels over
// ray batches in HBM.
//
// Extend replaces IntersectionKernel's traversal (Src/Core/renderer.cuh:132
// -> TraceRay :124 -> BVH::IsIntersect Src/Core/bvh.cu:253): 32 B in per ray
// (two float4 loads), 16 B out (one float4 store), node boxes and triangles
// through the read-only path, persistent warps with lane refill.
#include "trace.cuh"
#include "traverse.cuh"
#include "render_kernels.cuh"  // persistent_grid
#include <algorithm>
#include <cstdlib>

namespace crt {

constexpr int kTraceBlock = 128;

namespace {

struct ClosestJob {
    BvhView bvh;
    const float4 *rays;
    float4 *hits;
    __device__ void setup(int i, BvhView &b, V3 &o, V3 &d, float &tmin, float &tmax, float &t_exit) {
        b = bvh;
        float4 r0 = __ldg(rays + 2 * (size_t)i), r1 = __ldg(rays + 2 * (size_t)i + 1);
        o = v3(r0.x, r0.y, r0.z);
        d = v3(r1.x, r1.y, r1.z);
        tmin = r0.w;
        tmax = r1.w;
        t_exit = 0.f;
    }
    __device__ void finish(int i, const BvhView &b, const Hit &h) {
        int prim = h.slot >= 0 ? tri_prim(b, h.slot) : -1;
        hits[i] = make_float4(h.t, __int_as_float(prim), h.b1, h.b2);
    }
};

struct ShadowJob {
    BvhView bvh;
    const float4 *q;
    uint8_t *occ;
    ShadowRay r;
    __device__ void setup(int i, BvhView &b, V3 &o, V3 &d, float &tmin, float &tmax, float &t_exit) {
        b = bvh;
        float4 a = __ldg(q + 3 * (size_t)i), bb = __ldg(q + 3 * (size_t)i + 1), c = __ldg(q + 3 * (size_t)i + 2);
        shadow_ray_init(r, v3(a.x, a.y, a.z), v3(a.w, bb.x, bb.y), v3(bb.z, bb.w, c.x), v3(c.y, c.z, c.w));
        o = r.o;
        d = r.dir;
        tmin = 1e-6f;
        tmax = 1e8f;
        t_exit = r.t_exit;
    }
    __device__ void finish(int i, const BvhView &b, const Hit &h) { occ[i] = shadow_ray_visible(r, b, h) ? 0 : 1; }
};

// Light::Visible in two passes, with the same answer. Pass 1 looks for the
// closest hit on [0, sd + 0.2] only (sd = distance from the light point to
// the shading point), which prunes every box beyond the shading point from
// the start; a hit found there is the closest hit of the whole ray, and the
// predicate is evaluated on it as before. With no hit there, the closest
// hit of the whole ray is absent (visible) or at t >= sd + 0.2, more than
// 0.1 from the shading point and from the sample distance (occluded), so
// pass 2 only asks whether any triangle is hit on [sd + 0.2, 1e8] and stops
// at the first.
struct ShadowJob2 {
    BvhView bvh;
    const float4 *q;
    uint8_t *occ;
    ShadowRay r;
    bool second;
    __device__ void setup(int i, BvhView &b, V3 &o, V3 &d, float &tmin, float &tmax, float &t_exit) {
        b = bvh;
        float4 a = __ldg(q + 3 * (size_t)i), bb = __ldg(q + 3 * (size_t)i + 1), c = __ldg(q + 3 * (size_t)i + 2);
        shadow_ray_init(r, v3(a.x, a.y, a.z), v3(a.w, bb.x, bb.y), v3(bb.z, bb.w, c.x), v3(c.y, c.z, c.w));
        o = r.o;
        d = r.dir;
        tmin = 1e-6f;
        tmax = r.sd + 0.2f;
        t_exit = r.t_exit;
        second = false;
    }
    __device__ bool again(int, Hit &hit, float &tmin, float &t_exit) {
        if (second || hit.slot >= 0) return false;
        second = true;
        tmin = r.sd + 0.2f;
        hit.t = 1e8f;
        hit.slot = -1;
        t_exit = 1e8f;  // any accepted hit ends pass 2
        return true;
    }
    __device__ void finish(int i, const BvhView &b, const Hit &h) {
        occ[i] = second ? (h.slot >= 0 ? 1 : 0) : (shadow_ray_visible(r, b, h) ? 0 : 1);
    }
};

}  // namespace

// Each warp traces its contiguous share of the batch, refilling lanes as
// their rays finish (traverse.cuh).
__global__ void __launch_bounds__(kTraceBlock) k_trace_closest(BvhView bvh, const float4 *__restrict__ rays, int n,
                                                               float4 *__restrict__ hits) {
    ClosestJob job{bvh, rays, hits};
    trace_dynamic<true>(job, n);
}

__global__ void __launch_bounds__(kTraceBlock) k_trace_shadow(BvhView bvh, const float4 *__restrict__ q, int n,
                                                              uint8_t *__restrict__ occ) {
    ShadowJob job{bvh, q, occ, {}};
    trace_dynamic<true>(job, n);
}

// The binary traversal with its local stack, compiled for kMinBlocks
// resident 128-thread blocks per SM (a register cap of 65536 / (128 x
// kMinBlocks) per thread: more warps to hide load latency, against spills).
template <int kMinBlocks>
__global__ void __launch_bounds__(kTraceBlock, kMinBlocks) k_trace_closest_o(BvhView bvh, const float4 *__restrict__ rays,
                                                                            int n, float4 *__restrict__ hits) {
    ClosestJob job{bvh, rays, hits};
    trace_dynamic<true>(job, n);
}

template <int kMinBlocks>
__global__ void __launch_bounds__(kTraceBlock, kMinBlocks) k_trace_shadow_o(BvhView bvh, const float4 *__restrict__ q,
                                                                           int n, uint8_t *__restrict__ occ) {
    ShadowJob job{bvh, q, occ, {}};
    trace_dynamic<true>(job, n);
}

// The binary traversal over the 16-bit quantised nodes (bvh16.cuh), local
// stack.
__global__ void __launch_bounds__(kTraceBlock, 8) k_trace_closest_q(BvhView bvh, const float4 *__restrict__ rays, int n,
                                                                 float4 *__restrict__ hits) {
    ClosestJob job{bvh, rays, hits};
    LocalStack st;
    trace_dynamic_st<true, true>(job, n, st);
}

__global__ void __launch_bounds__(kTraceBlock, 8) k_trace_shadow_q(BvhView bvh, const float4 *__restrict__ q, int n,
                                                                uint8_t *__restrict__ occ) {
    ShadowJob job{bvh, q, occ, {}};
    LocalStack st;
    trace_dynamic_st<true, true>(job, n, st);
}

// One ray per thread, no refill (closest_hit / its early-exit form over the
// local stack): for small scenes, whose traversals are a few nodes long and
// do not repay the refill loop's bookkeeping.
__global__ void __launch_bounds__(kTraceBlock) k_trace_closest_1(BvhView bvh, const float4 *__restrict__ rays, int n,
                                                                 float4 *__restrict__ hits) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    ClosestJob job{bvh, rays, hits};
    BvhView b;
    V3 o, d;
    float tmin, tmax, t_exit;
    job.setup(i, b, o, d, tmin, tmax, t_exit);
    job.finish(i, b, closest_hit<false>(b, o, d, tmin, tmax));
}

__global__ void __launch_bounds__(kTraceBlock) k_trace_shadow_1(BvhView bvh, const float4 *__restrict__ q, int n,
                                                                uint8_t *__restrict__ occ) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    ShadowJob job{bvh, q, occ, {}};
    BvhView b;
    V3 o, d;
    float tmin, tmax, t_exit;
    job.setup(i, b, o, d, tmin, tmax, t_exit);
    job.finish(i, b, closest_hit<true>(b, o, d, tmin, tmax, t_exit));
}

// --- Scenes whose tree fits in shared memory ---
//
// Interior nodes (4 float4 each) and triangles (3 float4 each: v0 with the
// primitive index, e1 = v1 - v0, e2 = v2 - v0 rounded to nearest as the
// triangle test forms them) of a scene of at most kTinyBytes are copied
// into each block's shared memory once; the traversal then reads them there
// (closest_hit's order, tests and bounds checks, so the same hits). It is
// the default up to kTinyDefaultBytes. Over 1M random rays + 1M shadow
// queries (extend + shadow ms, against the refill traversal from global
// memory) it is faster on trees of 1.1 KB (0.169 vs 0.218), 2.1 KB (the
// Cornell box, 0.248 vs 0.286) and 8.9 KB (0.183 vs 0.203), and slower at
// 9.6 KB (0.280 vs 0.253), 19.3 KB (0.234 vs 0.214) and 29.1 KB (0.323 vs
// 0.256): each block's copy of the tree grows with it, and deeper trees
// gain more from the refill loop.
constexpr int kTinyBytes = 32 * 1024;
constexpr int kTinyDefaultBytes = 8 * 1024;

static int64_t tiny_bytes(const BvhView &bvh) {
    return ((int64_t)4 * bvh.num_nodes + (int64_t)3 * bvh.num_tris) * (int64_t)sizeof(float4);
}

template <bool kEarlyExit, class Stack>
__device__ __forceinline__ Hit closest_hit_tiny(const float4 *sn, const float4 *se, const BvhView &bvh, Stack &st,
                                                V3 o, V3 d, float tmin, float tmax, float t_exit) {
    Hit hit;
    hit.t = tmax;
    hit.slot = -1;
    hit.b1 = hit.b2 = 0.f;
    const V3 inv = v3(rrcp(d.x), rrcp(d.y), rrcp(d.z));
    unsigned lm[Stack::kLocal];
    st.reset();
    int link = 0;
    while (link != kSentinel) {
        while (link >= 0) {
            if (link >= bvh.num_nodes) {
                report_traversal_bounds(bvh);
                return hit;
            }
            const float4 *nd = sn + 4 * link;
            const float4 n0 = nd[0], n1 = nd[1], n2 = nd[2];
            const int4 n3 = reinterpret_cast<const int4 *>(nd)[3];
            float t0, t1;
            const bool h0 = slab(n0.x, n0.y, n0.z, n0.w, n2.x, n2.y, o, inv, tmin, hit.t, t0);
            const bool h1 = slab(n1.x, n1.y, n1.z, n1.w, n2.z, n2.w, o, inv, tmin, hit.t, t1);
            if (h0 && h1) {
                int near = n3.x, far = n3.y;
                if (t1 < t0) {
                    near = n3.y;
                    far = n3.x;
                }
                if (st.sp >= kStackSize) {
                    report_traversal_bounds(bvh);
                    return hit;
                }
                st.push((unsigned)far, lm);
                link = near;
            } else if (h0) {
                link = n3.x;
            } else if (h1) {
                link = n3.y;
            } else {
                link = st.empty() ? kSentinel : (int)st.pop(lm);
            }
        }
        if (link == kSentinel) break;
        const int code = ~link;
        const int first = code >> 4, count = code & 15;
        if (first + count > bvh.num_tris) {
            report_traversal_bounds(bvh);
            return hit;
        }
        for (int k = 0; k < count; ++k) {
            const int slot = first + k;
            const float4 *tp = se + 3 * slot;
            const float4 a = tp[0], b = tp[1], c = tp[2];
            const bool acc = intersect_triangle_e<true>(o, d, v3(a.x, a.y, a.z), v3(b.x, b.y, b.z), v3(c.x, c.y, c.z),
                                                        slot, hit);
            if (kEarlyExit && acc && hit.t < t_exit) return hit;
        }
        link = st.empty() ? kSentinel : (int)st.pop(lm);
    }
    return hit;
}

// Copies the interior nodes and the triangles as (v0, e1, e2) records into
// s_tree (the caller synchronises the block afterwards).
__device__ __forceinline__ void tiny_fill(float4 *s_tree, const BvhView &bvh) {
    const int nn = 4 * bvh.num_nodes;
    for (int k = threadIdx.x; k < nn; k += blockDim.x) s_tree[k] = __ldg(bvh.nodes + k);
    for (int k = threadIdx.x; k < bvh.num_tris; k += blockDim.x) {
        const float4 a = __ldg(bvh.tris + 3 * k), b = __ldg(bvh.tris + 3 * k + 1), c = __ldg(bvh.tris + 3 * k + 2);
        s_tree[nn + 3 * k] = a;
        s_tree[nn + 3 * k + 1] = make_float4(rsub(b.x, a.x), rsub(b.y, a.y), rsub(b.z, a.z), 0.f);
        s_tree[nn + 3 * k + 2] = make_float4(rsub(c.x, a.x), rsub(c.y, a.y), rsub(c.z, a.z), 0.f);
    }
}

// Grid-stride over the batch (one ray per thread when the grid covers it);
// kShort > 0 keeps the top kShort stack entries per lane in shared memory.
template <class Job, bool kEarlyExit, int kShort>
__global__ void __launch_bounds__(kTraceBlock) k_trace_tiny(Job job, int n) {
    extern __shared__ float4 s_tree[];
    __shared__ unsigned s_stack[kShort > 0 ? kShort * kTraceBlock : 1];
    const BvhView &bvh = job.bvh;
    const int nn = 4 * bvh.num_nodes;
    tiny_fill(s_tree, bvh);
    __syncthreads();
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += stride) {
        const int i = (int)r;
        BvhView b;
        V3 o, d;
        float tmin, tmax, t_exit;
        job.setup(i, b, o, d, tmin, tmax, t_exit);
        Hit h;
        if constexpr (kShort > 0) {
            ShortStack<kShort> st;
            st.col = s_stack + threadIdx.x;
            st.stride = blockDim.x;
            h = closest_hit_tiny<kEarlyExit>(s_tree, s_tree + nn, b, st, o, d, tmin, tmax, t_exit);
        } else {
            LocalStack st;
            h = closest_hit_tiny<kEarlyExit>(s_tree, s_tree + nn, b, st, o, d, tmin, tmax, t_exit);
        }
        job.finish(i, b, h);
    }
}

// Launches k_trace_tiny over n rays: one ray per thread (persistent false)
// or a grid of all SMs at full occupancy.
template <class Job, bool kEarlyExit, int kShort>
static void launch_tiny(const Job &job, int64_t n, bool persistent, cudaStream_t s) {
    const int smem = (int)tiny_bytes(job.bvh);
    const void *kernel = (const void *)k_trace_tiny<Job, kEarlyExit, kShort>;
    int64_t blocks = (n + kTraceBlock - 1) / kTraceBlock;
    if (persistent) {
        static int sms = 0;
        if (!sms) {
            int dev;
            CRT_CUDA(cudaGetDevice(&dev));
            CRT_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        }
        int per = 0;
        CRT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, kTraceBlock, smem));
        blocks = std::min<int64_t>(blocks, (int64_t)sms * std::max(1, per));
    }
    k_trace_tiny<Job, kEarlyExit, kShort><<<(int)blocks, kTraceBlock, smem, s>>>(job, (int)n);
}

// Light::Visible in two passes (ShadowJob2), local stack, for at least
// kMinBlocks resident blocks per SM (1: no register cap).
template <int kMinBlocks>
__global__ void __launch_bounds__(kTraceBlock, kMinBlocks) k_trace_shadow_2p(BvhView bvh,
                                                                            const float4 *__restrict__ q, int n,
                                                                            uint8_t *__restrict__ occ) {
    ShadowJob2 job{bvh, q, occ, {}, false};
    LocalStack st;
    trace_dynamic_st<true, false, ShadowJob2, LocalStack, false, true>(job, n, st);
}

// The binary traversal with the local stack and pipelined triangle loads,
// for at least kMinBlocks resident blocks per SM (1: no register cap).
template <int kMinBlocks>
__global__ void __launch_bounds__(kTraceBlock, kMinBlocks) k_trace_closest_pf(BvhView bvh,
                                                                             const float4 *__restrict__ rays, int n,
                                                                             float4 *__restrict__ hits) {
    ClosestJob job{bvh, rays, hits};
    LocalStack st;
    trace_dynamic_st<true, false, ClosestJob, LocalStack, true>(job, n, st);
}

template <int kMinBlocks>
__global__ void __launch_bounds__(kTraceBlock, kMinBlocks) k_trace_shadow_pf(BvhView bvh, const float4 *__restrict__ q,
                                                                            int n, uint8_t *__restrict__ occ) {
    ShadowJob job{bvh, q, occ, {}};
    LocalStack st;
    trace_dynamic_st<true, false, ShadowJob, LocalStack, true>(job, n, st);
}

// The binary traversal with postponed leaves (traverse.cuh), local stack.
__global__ void __launch_bounds__(kTraceBlock) k_trace_closest_p(BvhView bvh, const float4 *__restrict__ rays, int n,
                                                                 float4 *__restrict__ hits) {
    ClosestJob job{bvh, rays, hits};
    LocalStack st;
    trace_dynamic_spec<true>(job, n, st);
}

__global__ void __launch_bounds__(kTraceBlock) k_trace_shadow_p(BvhView bvh, const float4 *__restrict__ q, int n,
                                                                uint8_t *__restrict__ occ) {
    ShadowJob job{bvh, q, occ, {}};
    LocalStack st;
    trace_dynamic_spec<true>(job, n, st);
}

// The binary traversal with the per-lane short stack in shared memory
// (kShort entries per lane, kShort x 128 words per block).
template <int kShort, bool kQuant>
__global__ void __launch_bounds__(kTraceBlock) k_trace_closest_s(BvhView bvh, const float4 *__restrict__ rays, int n,
                                                                 float4 *__restrict__ hits) {
    __shared__ unsigned s_stack[kShort * kTraceBlock];
    ShortStack<kShort> st;
    st.col = s_stack + threadIdx.x;
    st.stride = blockDim.x;
    ClosestJob job{bvh, rays, hits};
    trace_dynamic_st<true, kQuant>(job, n, st);
}

template <int kShort, bool kQuant>
__global__ void __launch_bounds__(kTraceBlock) k_trace_shadow_s(BvhView bvh, const float4 *__restrict__ q, int n,
                                                                uint8_t *__restrict__ occ) {
    __shared__ unsigned s_stack[kShort * kTraceBlock];
    ShortStack<kShort> st;
    st.col = s_stack + threadIdx.x;
    st.stride = blockDim.x;
    ShadowJob job{bvh, q, occ, {}};
    trace_dynamic_st<true, kQuant>(job, n, st);
}

// The same over the 8-wide quantised tree with the shared-memory short
// stack (kShort entries per lane, kShort x 128 words per block).
template <int kShort>
__global__ void __launch_bounds__(kTraceBlock) k_trace_closest8(BvhView bvh, const float4 *__restrict__ rays, int n,
                                                                float4 *__restrict__ hits) {
    __shared__ unsigned s_stack[kShort * kTraceBlock];
    ClosestJob job{bvh, rays, hits};
    trace_dynamic8<true, kShort>(job, n, s_stack);
}

template <int kShort>
__global__ void __launch_bounds__(kTraceBlock) k_trace_shadow8(BvhView bvh, const float4 *__restrict__ q, int n,
                                                               uint8_t *__restrict__ occ) {
    __shared__ unsigned s_stack[kShort * kTraceBlock];
    ShadowJob job{bvh, q, occ, {}};
    trace_dynamic8<true, kShort>(job, n, s_stack);
}

template <int kShort>
__global__ void __launch_bounds__(kTraceBlock) k_trace_closest8r(BvhView bvh, const float4 *__restrict__ rays, int n,
                                                                 float4 *__restrict__ hits) {
    __shared__ unsigned s_stack[kShort * kTraceBlock];
    ClosestJob job{bvh, rays, hits};
    trace_dynamic8<true, kShort, ClosestJob, true>(job, n, s_stack);
}

template <int kShort>
__global__ void __launch_bounds__(kTraceBlock) k_trace_shadow8r(BvhView bvh, const float4 *__restrict__ q, int n,
                                                                uint8_t *__restrict__ occ) {
    __shared__ unsigned s_stack[kShort * kTraceBlock];
    ShadowJob job{bvh, q, occ, {}};
    trace_dynamic8<true, kShort, ShadowJob, true>(job, n, s_stack);
}

// Traversal variant of the trace kernels. The default is kTinyVariant for
// scenes of at most kTinyDefaultBytes and kTraceVariant otherwise;
// CRT_TRAVERSAL overrides it.
//   2        binary tree, stack in local memory, per-lane refill;
//   210/212  the same capped at 51 / 42 registers (10 / 12 blocks per SM);
//   1        one ray per thread without refill;
//   3        postponed leaves;
//   5/58     pipelined triangle loads (no register cap / 8 blocks per SM);
//   6/68     shadow queries in two passes (ShadowJob2; no cap / 8 blocks per
//            SM; extend as 2);
//   4/416    the 16-bit quantised nodes, stack in local / shared memory;
//   28/216   top 8 / 16 stack entries per lane in shared memory;
//   8/82     8-wide quantised tree (built only with CRT_BVH8=1), 16 / 8
//            shared-memory entries; 83 as 8 with the visited node's links
//            in registers;
//   11/12/13 the tree in shared memory (k_trace_tiny; scenes of at most
//            kTinyBytes, else 2): one ray per thread with the local stack /
//            a persistent grid / one ray per thread with 8 stack entries
//            per lane in shared memory.
// On the Cornell box (36 triangles, 1M random rays) 11 issues from 85% of
// the scheduler slots with 11-12 of 32 lanes active: divergence between the
// lanes' paths, not memory, bounds it. Capping it at 40 / 32 registers (12 /
// 16 blocks per SM), and binning each block's rays by direction and origin
// octant before tracing them, measured 8-20% and 2-10% slower.
constexpr int kTraceVariant = 2;
constexpr int kTinyVariant = 11;

static int traversal_variant(const BvhView &bvh) {
    const char *e = getenv("CRT_TRAVERSAL");
    const int64_t tb = tiny_bytes(bvh);
    const bool tiny = tb <= kTinyBytes;
    int v = e ? atoi(e) : (tb <= kTinyDefaultBytes ? kTinyVariant : kTraceVariant);
    if ((v == 8 || v == 82 || v == 83) && !bvh.wnodes) v = 2;
    if ((v == 4 || v == 416) && !bvh.cnodes) v = 2;
    if (v >= 11 && v <= 13 && !tiny) v = 2;
    return v;
}

// Persistent grid (all SMs at full occupancy), fewer blocks for small
// batches so every warp gets rays.
static int trace_grid(const void *kernel, int64_t n) {
    const int full = persistent_grid(kernel, kTraceBlock);
    const int64_t want = (n + kTraceBlock - 1) / kTraceBlock;
    return (int)(want < full ? (want > 0 ? want : 1) : full);
}

void launch_trace_closest(const BvhView &bvh, const float4 *d_rays, int64_t n, float4 *d_hits, cudaStream_t s) {
    if (n <= 0) return;
    CRT_CHECK(n < (int64_t)1 << 31, CRT_ERR_CAPACITY, "trace batch larger than 2^31 rays");
    const int v = traversal_variant(bvh);
    if (v >= 11 && v <= 13) {
        const ClosestJob job{bvh, d_rays, d_hits};
        if (v == 13)
            launch_tiny<ClosestJob, false, 8>(job, n, false, s);
        else
            launch_tiny<ClosestJob, false, 0>(job, n, v == 12, s);
    } else if (v == 4)
        k_trace_closest_q<<<trace_grid((const void *)k_trace_closest_q, n), kTraceBlock, 0, s>>>(bvh, d_rays, (int)n,
                                                                                                d_hits);
    else if (v == 416)
        k_trace_closest_s<16, true><<<trace_grid((const void *)k_trace_closest_s<16, true>, n), kTraceBlock, 0, s>>>(
            bvh, d_rays, (int)n, d_hits);
    else if (v == 3)
        k_trace_closest_p<<<trace_grid((const void *)k_trace_closest_p, n), kTraceBlock, 0, s>>>(bvh, d_rays, (int)n,
                                                                                                d_hits);
    else if (v == 1)
        k_trace_closest_1<<<(int)((n + kTraceBlock - 1) / kTraceBlock), kTraceBlock, 0, s>>>(bvh, d_rays, (int)n,
                                                                                           d_hits);
    else if (v == 5)
        k_trace_closest_pf<1><<<trace_grid((const void *)k_trace_closest_pf<1>, n), kTraceBlock, 0, s>>>(
            bvh, d_rays, (int)n, d_hits);
    else if (v == 58)
        k_trace_closest_pf<8><<<trace_grid((const void *)k_trace_closest_pf<8>, n), kTraceBlock, 0, s>>>(
            bvh, d_rays, (int)n, d_hits);
    else if (v == 210)
        k_trace_closest_o<10><<<trace_grid((const void *)k_trace_closest_o<10>, n), kTraceBlock, 0, s>>>(
            bvh, d_rays, (int)n, d_hits);
    else if (v == 212)
        k_trace_closest_o<12><<<trace_grid((const void *)k_trace_closest_o<12>, n), kTraceBlock, 0, s>>>(
            bvh, d_rays, (int)n, d_hits);
    else if (v == 28)
        k_trace_closest_s<8, false><<<trace_grid((const void *)k_trace_closest_s<8, false>, n), kTraceBlock, 0, s>>>(
            bvh, d_rays, (int)n, d_hits);
    else if (v == 216)
        k_trace_closest_s<16, false><<<trace_grid((const void *)k_trace_closest_s<16, false>, n), kTraceBlock, 0, s>>>(
            bvh, d_rays, (int)n, d_hits);
    else if (v == 8)
        k_trace_closest8<16><<<trace_grid((const void *)k_trace_closest8<16>, n), kTraceBlock, 0, s>>>(
            bvh, d_rays, (int)n, d_hits);
    else if (v == 82)
        k_trace_closest8<8><<<trace_grid((const void *)k_trace_closest8<8>, n), kTraceBlock, 0, s>>>(
            bvh, d_rays, (int)n, d_hits);
    else if (v == 83)
        k_trace_closest8r<16><<<trace_grid((const void *)k_trace_closest8r<16>, n), kTraceBlock, 0, s>>>(
            bvh, d_rays, (int)n, d_hits);
    else
        k_trace_closest<<<trace_grid((const void *)k_trace_closest, n), kTraceBlock, 0, s>>>(bvh, d_rays, (int)n,
                                                                                            d_hits);
    CRT_CUDA(cudaGetLastError());
}

void launch_trace_shadow(const BvhView &bvh, const float *d_q, int64_t n, uint8_t *d_occ, cudaStream_t s) {
    if (n <= 0) return;
    CRT_CHECK(n < (int64_t)1 << 31, CRT_ERR_CAPACITY, "trace batch larger than 2^31 queries");
    const float4 *q = reinterpret_cast<const float4 *>(d_q);
    const int v = traversal_variant(bvh);
    if (v >= 11 && v <= 13) {
        const ShadowJob job{bvh, q, d_occ, {}};
        if (v == 13)
            launch_tiny<ShadowJob, true, 8>(job, n, false, s);
        else
            launch_tiny<ShadowJob, true, 0>(job, n, v == 12, s);
    } else if (v == 4)
        k_trace_shadow_q<<<trace_grid((const void *)k_trace_shadow_q, n), kTraceBlock, 0, s>>>(bvh, q, (int)n, d_occ);
    else if (v == 416)
        k_trace_shadow_s<16, true><<<trace_grid((const void *)k_trace_shadow_s<16, true>, n), kTraceBlock, 0, s>>>(
            bvh, q, (int)n, d_occ);
    else if (v == 3)
        k_trace_shadow_p<<<trace_grid((const void *)k_trace_shadow_p, n), kTraceBlock, 0, s>>>(bvh, q, (int)n, d_occ);
    else if (v == 1)
        k_trace_shadow_1<<<(int)((n + kTraceBlock - 1) / kTraceBlock), kTraceBlock, 0, s>>>(bvh, q, (int)n, d_occ);
    else if (v == 5)
        k_trace_shadow_pf<1><<<trace_grid((const void *)k_trace_shadow_pf<1>, n), kTraceBlock, 0, s>>>(bvh, q,
                                                                                                      (int)n, d_occ);
    else if (v == 6)
        k_trace_shadow_2p<1><<<trace_grid((const void *)k_trace_shadow_2p<1>, n), kTraceBlock, 0, s>>>(bvh, q,
                                                                                                      (int)n, d_occ);
    else if (v == 68)
        k_trace_shadow_2p<8><<<trace_grid((const void *)k_trace_shadow_2p<8>, n), kTraceBlock, 0, s>>>(bvh, q,
                                                                                                      (int)n, d_occ);
    else if (v == 58)
        k_trace_shadow_pf<8><<<trace_grid((const void *)k_trace_shadow_pf<8>, n), kTraceBlock, 0, s>>>(bvh, q,
                                                                                                      (int)n, d_occ);
    else if (v == 210)
        k_trace_shadow_o<10><<<trace_grid((const void *)k_trace_shadow_o<10>, n), kTraceBlock, 0, s>>>(bvh, q, (int)n,
                                                                                                    d_occ);
    else if (v == 212)
        k_trace_shadow_o<12><<<trace_grid((const void *)k_trace_shadow_o<12>, n), kTraceBlock, 0, s>>>(bvh, q, (int)n,
                                                                                                    d_occ);
    else if (v == 28)
        k_trace_shadow_s<8, false><<<trace_grid((const void *)k_trace_shadow_s<8, false>, n), kTraceBlock, 0, s>>>(bvh, q, (int)n,
                                                                                                  d_occ);
    else if (v == 216)
        k_trace_shadow_s<16, false><<<trace_grid((const void *)k_trace_shadow_s<16, false>, n), kTraceBlock, 0, s>>>(bvh, q, (int)n,
                                                                                                    d_occ);
    else if (v == 8)
        k_trace_shadow8<16><<<trace_grid((const void *)k_trace_shadow8<16>, n), kTraceBlock, 0, s>>>(bvh, q, (int)n,
                                                                                                    d_occ);
    else if (v == 82)
        k_trace_shadow8<8><<<trace_grid((const void *)k_trace_shadow8<8>, n), kTraceBlock, 0, s>>>(bvh, q, (int)n,
                                                                                                  d_occ);
    else if (v == 83)
        k_trace_shadow8r<16><<<trace_grid((const void *)k_trace_shadow8r<16>, n), kTraceBlock, 0, s>>>(bvh, q, (int)n,
                                                                                                      d_occ);
    else
        k_trace_shadow<<<trace_grid((const void *)k_trace_shadow, n), kTraceBlock, 0, s>>>(bvh, q, (int)n, d_occ);
    CRT_CUDA(cudaGetLastError());
}

}  // namespace crt
