// Persistent-warp BVH traversal with dynamic ray refill.
//
// Random rays in one warp need very different numbers of traversal steps, so
// a warp that traces one ray per lane runs until its slowest ray finishes
// with most lanes idle. Here each warp keeps up to 32 rays in flight: one
// loop turn runs one while-while iteration per active lane (descend interior
// nodes to a leaf, test the leaf's triangles), and lanes whose ray finished
// take the next rays of the warp's contiguous share of [0, n) (no atomics:
// with incoherent rays the shares even out). Per ray, the node visit order
// and every
// arithmetic step are those of closest_hit (bvh.cuh), so results are
// bit-identical.
//
// Used by the standalone ray-batch kernels (trace.cu), whose rays are
// incoherent. The wavefront stages keep one path per thread: their primary
// rays are coherent within a warp, and refilling lanes would break that.
//
// A Job supplies, per ray index, the BVH and ray (setup) and consumes the
// hit (finish):
//   __device__ void setup(int i, BvhView &bvh, V3 &o, V3 &d, float &tmin,
//                         float &tmax, float &t_exit);
//   __device__ void finish(int i, const BvhView &bvh, const Hit &hit);
// An accepted hit with t < t_exit ends the traversal (closest_hit<true>'s
// early exit; t_exit = 0 never fires).
#pragma once
#include "bvh.cuh"
#include "bvh8.cuh"

namespace crt {

#ifdef __CUDACC__

template <bool kCull, bool kQuant, class Job, class Stack, bool kPipe = false, bool kMultiPass = false>
__device__ __forceinline__ void trace_dynamic_st(Job &job, int n, Stack &st);

// The stack in local memory, float nodes.
template <bool kCull, class Job>
__device__ __forceinline__ void trace_dynamic(Job &job, int n) {
    LocalStack st;
    trace_dynamic_st<kCull, false>(job, n, st);
}

// Over a given per-lane stack (LocalStack or ShortStack, bvh.cuh), and over
// the float nodes or (kQuant) their 16-bit quantised copy (bvh16.cuh). With
// kPipe the leaf loop loads triangle k + 1 before testing triangle k, so its
// 48 B are in flight during the test (same tests in the same order). With
// kMultiPass a finished ray is offered to
//   __device__ bool again(int i, Hit &hit, float &tmin, float &t_exit);
// which may set a new box interval start, closest bound (hit.t, with
// hit.slot = -1) and exit distance and return true to traverse again from
// the root before finish.
template <bool kCull, bool kQuant, class Job, class Stack, bool kPipe, bool kMultiPass>
__device__ __forceinline__ void trace_dynamic_st(Job &job, int n, Stack &st) {
    const unsigned lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    // warp-uniform: the rays [cbase, cbase + cleft) of this warp not yet started
    const int64_t warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int cbase = (int)(w * n / warps);
    int cleft = (int)((w + 1) * n / warps) - cbase;
    // per-lane ray state
    int idx = -1;
    BvhView bvh{nullptr, nullptr, 0, nullptr, nullptr, 0, nullptr, nullptr, {}};
    V3 o{0.f, 0.f, 0.f}, d{0.f, 0.f, 0.f}, inv{0.f, 0.f, 0.f};
    float tmin = 0.f, t_exit = 0.f;
    Hit hit;
    hit.t = 0.f;
    hit.slot = -1;
    hit.b1 = hit.b2 = 0.f;
    int link = kSentinel;
    unsigned lm[Stack::kLocal];
    st.reset();

    auto start = [&](int k) {
        idx = k;
        float tmax;
        job.setup(k, bvh, o, d, tmin, tmax, t_exit);
        inv = v3(rrcp(d.x), rrcp(d.y), rrcp(d.z));
        hit.t = tmax;
        hit.slot = -1;
        hit.b1 = hit.b2 = 0.f;
        st.reset();
        link = 0;
    };

    while (true) {
        const unsigned idle = __ballot_sync(0xffffffffu, idx < 0);
        if (idle && cleft > 0) {
            const int take = min(__popc(idle), cleft);
            const int rank = __popc(idle & lt);
            if (idx < 0 && rank < take) start(cbase + rank);
            cbase += take;
            cleft -= take;
        }
        if (__ballot_sync(0xffffffffu, idx >= 0) == 0) break;  // nothing in flight and nothing left
        if (idx < 0) continue;
        // one while-while iteration of closest_hit
        bool bad = false;
        while (link >= 0) {
            if (link >= bvh.num_nodes) {
                bad = true;
                break;
            }
            float4 n0, n1, n2;
            int4 n3;
            if (kQuant)
                load_node16(bvh.cnodes, link, bvh.grid, n0, n1, n2, n3);
            else
                load_node(bvh.nodes + 4 * (size_t)link, n0, n1, n2, n3);
            float t0, t1;
            bool h0 = slab(n0.x, n0.y, n0.z, n0.w, n2.x, n2.y, o, inv, tmin, hit.t, t0);
            bool h1 = slab(n1.x, n1.y, n1.z, n1.w, n2.z, n2.w, o, inv, tmin, hit.t, t1);
            if (h0 && h1) {
                int near = n3.x, far = n3.y;
                if (t1 < t0) {
                    near = n3.y;
                    far = n3.x;
                }
                if (st.sp >= kStackSize) {
                    bad = true;
                    break;
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
        bool finished = link == kSentinel;
        if (!finished && !bad) {
            const int code = ~link;
            const int first = code >> 4, count = code & 15;
            bad = first + count > bvh.num_tris;
        }
        if (bad) {
            // an index outside the tree: record it and end this ray
            report_traversal_bounds(bvh);
            finished = true;
        }
        if (!finished) {
            const int code = ~link;
            const int first = code >> 4, count = code & 15;
            if (kPipe && count > 0) {
                // [first, first + count) checked against num_tris above
                const float4 *tp = bvh.tris + 3 * (size_t)first;
                float4 a = __ldg(tp + 0), b = __ldg(tp + 1), c = __ldg(tp + 2);
                for (int k = 0; k < count; ++k) {
                    float4 na = a, nb = b, nc = c;
                    if (k + 1 < count) {
                        na = __ldg(tp + 3 * (k + 1));
                        nb = __ldg(tp + 3 * (k + 1) + 1);
                        nc = __ldg(tp + 3 * (k + 1) + 2);
                    }
                    const bool acc = intersect_triangle<kCull>(o, d, a, b, c, first + k, hit);
                    if (acc && hit.t < t_exit) {
                        finished = true;
                        break;
                    }
                    a = na;
                    b = nb;
                    c = nc;
                }
            } else if (!kPipe) {
                for (int k = 0; k < count; ++k) {
                    const int slot = first + k;
                    const float4 *tp = bvh.tris + 3 * (size_t)slot;
                    float4 a = __ldg(tp + 0), b = __ldg(tp + 1), c = __ldg(tp + 2);
                    const bool acc = intersect_triangle<kCull>(o, d, a, b, c, slot, hit);
                    if (acc && hit.t < t_exit) {
                        finished = true;
                        break;
                    }
                }
            }
            if (!finished) {
                link = st.empty() ? kSentinel : (int)st.pop(lm);
                finished = link == kSentinel;
            }
        }
        if (finished) {
            bool again = false;
            if constexpr (kMultiPass) again = !bad && job.again(idx, hit, tmin, t_exit);
            if (again) {
                st.reset();
                link = 0;
            } else {
                job.finish(idx, bvh, hit);
                idx = -1;
            }
        }
    }
}

// trace_dynamic with postponed leaves (the speculative while-while loop of
// Aila and Laine, "Understanding the Efficiency of Ray Traversal on GPUs",
// HPG 2009): a lane that reaches a leaf keeps it pending and goes on
// descending while other lanes of the warp are still looking for their
// first leaf, so the node loop runs with more lanes busy; a lane that
// meets a second leaf stops there and keeps it for the next turn. Leaves
// are tested in the order they are found; the extra node visits use the
// closest hit of the leaves tested so far, so results equal closest_hit's
// up to the order in which equal-t triangles are met.
template <bool kCull, class Job, class Stack>
__device__ __forceinline__ void trace_dynamic_spec(Job &job, int n, Stack &st) {
    const unsigned lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    const int64_t warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int cbase = (int)(w * n / warps);
    int cleft = (int)((w + 1) * n / warps) - cbase;
    int idx = -1;
    BvhView bvh{nullptr, nullptr, 0, nullptr, nullptr, 0, nullptr, nullptr, {}};
    V3 o{0.f, 0.f, 0.f}, d{0.f, 0.f, 0.f}, inv{0.f, 0.f, 0.f};
    float tmin = 0.f, t_exit = 0.f;
    Hit hit;
    hit.t = 0.f;
    hit.slot = -1;
    hit.b1 = hit.b2 = 0.f;
    int link = kSentinel;
    unsigned lm[Stack::kLocal];
    st.reset();

    while (true) {
        const unsigned idle = __ballot_sync(0xffffffffu, idx < 0);
        if (idle && cleft > 0) {
            const int take = min(__popc(idle), cleft);
            const int rank = __popc(idle & lt);
            if (idx < 0 && rank < take) {
                idx = cbase + rank;
                float tmax;
                job.setup(idx, bvh, o, d, tmin, tmax, t_exit);
                inv = v3(rrcp(d.x), rrcp(d.y), rrcp(d.z));
                hit.t = tmax;
                hit.slot = -1;
                hit.b1 = hit.b2 = 0.f;
                st.reset();
                link = 0;
            }
            cbase += take;
            cleft -= take;
        }
        if (__ballot_sync(0xffffffffu, idx >= 0) == 0) break;
        if (idx < 0) continue;
        int pending = 0;  // postponed leaf link (< 0), 0 = none
        bool bad = false;
        while (true) {
            if (link >= 0) {
                if (link >= bvh.num_nodes) {
                    bad = true;
                    break;
                }
                float4 n0, n1, n2;
                int4 n3;
                load_node(bvh.nodes + 4 * (size_t)link, n0, n1, n2, n3);
                float t0, t1;
                bool h0 = slab(n0.x, n0.y, n0.z, n0.w, n2.x, n2.y, o, inv, tmin, hit.t, t0);
                bool h1 = slab(n1.x, n1.y, n1.z, n1.w, n2.z, n2.w, o, inv, tmin, hit.t, t1);
                if (h0 && h1) {
                    int near = n3.x, far = n3.y;
                    if (t1 < t0) {
                        near = n3.y;
                        far = n3.x;
                    }
                    if (st.sp >= kStackSize) {
                        bad = true;
                        break;
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
            if (link < 0 && link != kSentinel && pending == 0) {
                pending = link;
                link = st.empty() ? kSentinel : (int)st.pop(lm);
            }
            // go on while some lane of the warp still has no leaf to test
            // (lanes holding a second leaf in `link`, or done, idle meanwhile)
            const bool searching = pending == 0 && link != kSentinel;
            if (!__any_sync(__activemask(), searching)) break;
        }
        bool finished = false;
        if (!bad && pending != 0) {
            const int code = ~pending;
            const int first = code >> 4, count = code & 15;
            if (first + count > bvh.num_tris) {
                bad = true;
            } else {
                for (int k = 0; k < count; ++k) {
                    const int slot = first + k;
                    const float4 *tp = bvh.tris + 3 * (size_t)slot;
                    float4 a = __ldg(tp + 0), b = __ldg(tp + 1), c = __ldg(tp + 2);
                    const bool acc = intersect_triangle<kCull>(o, d, a, b, c, slot, hit);
                    if (acc && hit.t < t_exit) {
                        finished = true;
                        break;
                    }
                }
            }
        }
        if (bad) {
            report_traversal_bounds(bvh);
            finished = true;
        }
        // nothing left: no leaf in hand and the stack exhausted (no push
        // follows a pop of the empty stack)
        if (!finished && link == kSentinel) finished = true;
        if (finished) {
            job.finish(idx, bvh, hit);
            idx = -1;
        }
    }
}

// trace_dynamic over the 8-wide quantised tree (bvh8.cuh) with the
// per-lane short stack in shared memory: `s_stack` is the block's
// kShort x blockDim.x word array. One loop turn finds the next leaf
// (visiting wide nodes on the way) and tests its triangles; lanes whose ray
// finished take new rays as above. Hit records equal closest_hit's (same
// triangle test, conservative boxes); only the order in which equal-t
// triangles are met may differ.
template <bool kCull, int kShort, class Job, bool kRegLinks = false>
__device__ __forceinline__ void trace_dynamic8(Job &job, int n, unsigned *s_stack) {
    const unsigned lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    const int64_t warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int cbase = (int)(w * n / warps);
    int cleft = (int)((w + 1) * n / warps) - cbase;
    int idx = -1;
    BvhView bvh{nullptr, nullptr, 0, nullptr, nullptr, 0, nullptr, nullptr, {}};
    V3 o{0.f, 0.f, 0.f}, d{0.f, 0.f, 0.f}, inv{0.f, 0.f, 0.f};
    float tmin = 0.f, t_exit = 0.f;
    unsigned oct = 0, cur = 0;
    Hit hit;
    hit.t = 0.f;
    hit.slot = -1;
    hit.b1 = hit.b2 = 0.f;
    ShortStack<kShort> st;
    st.col = s_stack + threadIdx.x;
    st.stride = blockDim.x;
    st.sp = 0;
    int lk[8];
    bool fresh = false;
    unsigned lm[ShortStack<kShort>::kLocal];

    while (true) {
        const unsigned idle = __ballot_sync(0xffffffffu, idx < 0);
        if (idle && cleft > 0) {
            const int take = min(__popc(idle), cleft);
            const int rank = __popc(idle & lt);
            if (idx < 0 && rank < take) {
                idx = cbase + rank;
                float tmax;
                job.setup(idx, bvh, o, d, tmin, tmax, t_exit);
                inv = v3(rrcp(d.x), rrcp(d.y), rrcp(d.z));
                oct = ray_octant(d);
                hit.t = tmax;
                hit.slot = -1;
                hit.b1 = hit.b2 = 0.f;
                st.reset();
                if (kRegLinks) load_links8(bvh.wlinks, 0, lk);
                fresh = kRegLinks;
                cur = visit8(bvh.wnodes, 0, o, inv, tmin, hit.t, oct);
            }
            cbase += take;
            cleft -= take;
        }
        if (__ballot_sync(0xffffffffu, idx >= 0) == 0) break;
        if (idx < 0) continue;
        const int leaf = next_leaf8<kShort, kRegLinks>(bvh, cur, st, lm, o, inv, tmin, hit.t, oct, lk, fresh);
        bool finished = leaf == 0;
        if (!finished) {
            const int code = ~leaf;
            const int first = code >> 4, count = code & 15;
            for (int k = 0; k < count; ++k) {
                const int slot = first + k;
                const float4 *tp = bvh.tris + 3 * (size_t)slot;
                const float4 a = __ldg(tp + 0), b = __ldg(tp + 1), c = __ldg(tp + 2);
                const bool acc = intersect_triangle<kCull>(o, d, a, b, c, slot, hit);
                if (acc && hit.t < t_exit) {
                    finished = true;
                    break;
                }
            }
            if (!finished && (cur & 0xffu) == 0 && st.empty()) finished = true;
        }
        if (finished) {
            job.finish(idx, bvh, hit);
            idx = -1;
        }
    }
}

#endif  // __CUDACC__

}  // namespace crt
