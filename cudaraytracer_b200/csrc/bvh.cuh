// BVH layout and traversal shared by the extend, shadow and shade kernels.
//
// Layout in HBM (all 16-byte aligned, read with 128-bit __ldg loads):
//   nodes: 64 B per interior node, the boxes of BOTH children in the parent so
//          one node fetch (4 x float4) decides the whole step:
//            [0] c0.lo.x c0.hi.x c0.lo.y c0.hi.y
//            [1] c1.lo.x c1.hi.x c1.lo.y c1.hi.y
//            [2] c0.lo.z c0.hi.z c1.lo.z c1.hi.z
//            [3] link0 link1 (int bits) , 0, 0
//          link >= 0 : interior node index
//          link <  0 : leaf, ~((first << 4) | count), count in [0, 15]
//   tris:  48 B per triangle in leaf order: v0 (w = original primitive index
//          as int bits), v1, v2. Edges are formed in-kernel exactly as the
//          reference does (e1 = v1 - v0, Src/Core/triangle.cu:102-103), so
//          the stored vertices give bit-identical arithmetic. (A second
//          leaf-order array of v0, e1, e2 saved the six subtractions but
//          measured 6-8% slower on a 1.3M-triangle scene, whose traversal
//          then keeps both arrays in L2; only the shared-memory copy of a
//          small tree holds edges, trace.cu.)
// The reference node is a 32 B {triIndex, count/right, Bounds3D} with the
// child boxes stored in the children (Src/Core/bvh.h:25-33) and a 176 B AoS
// triangle (Src/Core/triangle.h:43-57).
#pragma once
#include "common.cuh"
#include <limits.h>

namespace crt {

constexpr int kLeafMaxCount = 15;
constexpr int kStackSize = 64;
constexpr int kSentinel = INT_MIN;  // never a valid link: first < 2^27 - 1
constexpr float kTriTMax = 1e8f;    // Triangle::IsIntersect default tMax

// Grid of the 16-bit quantised nodes of one scene (bvh16.cuh): per axis
// the scale s = 2^e and the biased origin p'.
struct QuantGrid {
    float s[3], p[3];
};

struct BvhView {
    const float4 *nodes;   // 4 float4 per node
    const float4 *tris;    // 3 float4 per triangle
    int num_tris;
    const float4 *wnodes;  // 8-wide quantised nodes, 4 float4 each (bvh8.cuh)
    const int *wlinks;     // 8 child links per wide node
    int num_nodes;         // binary nodes (bound of interior links)
    int *err;              // device error word (kErrTraversalBounds), or null
    const float4 *cnodes;  // the binary nodes with 16-bit quantised boxes, 2 float4 each (bvh16.cuh)
    QuantGrid grid;
};

#ifdef __CUDACC__
// Records a traversal that met an index outside the tree (the traversal
// then stops instead of reading out of bounds).
__device__ __forceinline__ void report_traversal_bounds(const BvhView &bvh) {
    if (bvh.err) atomicOr(bvh.err, kErrTraversalBounds);
}
#endif

__host__ __device__ __forceinline__ int leaf_link(int first, int count) { return ~((first << 4) | count); }

#ifdef __CUDACC__

struct Hit {
    float t;
    int slot;  // triangle slot in leaf order (-1 = miss)
    float b1, b2;
};

// Triangle::IsIntersect (Src/Core/triangle.cu:100-133) with tMin = 0 and
// tMax = 1e8 as BVH::IsIntersect passes them (Src/Core/bvh.cu:271):
// back faces culled (det <= 0), reciprocal of the determinant correctly
// rounded (the reference divides 1.f by a double and rounds to float, which
// is the same value), strict t < closest so ties keep the first triangle
// visited. Returns true and updates `hit` when accepted.
// kCull = false accepts both facings (det != 0), as a rasteriser without
// face culling sees the nearest surface (used for the G-buffer only).
// intersect_triangle_e takes the edges e1 = v1 - v0, e2 = v2 - v0 already
// formed; intersect_triangle forms them from the three vertices. (One
// predicate over all quantities instead of the early returns measured 4-6%
// slower on a 1.3M-triangle scene and on the Cornell box.)
template <bool kCull = true>
__device__ __forceinline__ bool intersect_triangle_e(V3 o, V3 d, V3 v0, V3 e1, V3 e2, int slot, Hit &hit) {
    V3 s = vsub(o, v0);
    V3 s1 = vcross(d, e2);
    V3 s2 = vcross(s, e1);
    float det = vdot(e1, s1);
    if (kCull ? (det == 0.f || det < 0.f) : det == 0.f) return false;
    float inv = rrcp(det);
    float t = rmul(inv, vdot(s2, e2));
    if (t >= hit.t) return false;
    float b1 = rmul(inv, vdot(s1, s));
    if (b1 < 0.f || b1 > 1.f) return false;
    float b2 = rmul(inv, vdot(s2, d));
    if (b2 < 0.f || radd(b1, b2) > 1.f) return false;
    if (t < 0.f || t > kTriTMax) return false;
    hit.t = t;
    hit.slot = slot;
    hit.b1 = b1;
    hit.b2 = b2;
    return true;
}

template <bool kCull = true>
__device__ __forceinline__ bool intersect_triangle(V3 o, V3 d, float4 a, float4 b, float4 c,
                                                   int slot, Hit &hit) {
    const V3 v0 = v3(a.x, a.y, a.z);
    return intersect_triangle_e<kCull>(o, d, v0, vsub(v3(b.x, b.y, b.z), v0), vsub(v3(c.x, c.y, c.z), v0), slot, hit);
}

// Conservative slab test of one child box. Returns entry distance in `tnear`.
// lo/hi include the ray interval [tmin, closest]; the padding keeps the test
// conservative against rounding so a different tree cannot cull the box of
// the reference's closest triangle.
__device__ __forceinline__ bool slab(float lox, float hix, float loy, float hiy, float loz, float hiz,
                                     V3 o, V3 inv, float tmin, float tmax, float &tnear) {
    float tx0 = (lox - o.x) * inv.x, tx1 = (hix - o.x) * inv.x;
    float ty0 = (loy - o.y) * inv.y, ty1 = (hiy - o.y) * inv.y;
    float tz0 = (loz - o.z) * inv.z, tz1 = (hiz - o.z) * inv.z;
    float lo = fmaxf(fmaxf(fminf(tx0, tx1), fminf(ty0, ty1)), fmaxf(fminf(tz0, tz1), tmin));
    float hi = fminf(fminf(fmaxf(tx0, tx1), fmaxf(ty0, ty1)), fminf(fmaxf(tz0, tz1), tmax));
    tnear = lo;
    return lo <= hi * 1.00000095f;
}

// Closest hit with the reference's semantics (BVH::IsIntersect,
// Src/Core/bvh.cu:253-306): boxes pruned by [tmin, closest], triangles
// accepted on [0, 1e8] with closest initialised to tmax. When t_exit > 0 the
// traversal stops at the first accepted hit with t < t_exit (used by the
// shadow predicate, whose answer is fixed once such a hit exists).
// One 64 B interior node (child boxes n0, n1 and n2.xy / n2.zw, child links
// n3.xy) as two 32 B read-only loads: nodes sit 64 B apart from a 256 B-
// aligned allocation. Measured 1.3-1.5% faster than four 16 B loads in the
// standalone extend and shadow kernels (traverse.cuh), with identical
// results; in the renderer's stages (closest_hit below) it measured 0.5-1%
// slower per frame, so closest_hit keeps the 16 B loads.
__device__ __forceinline__ void load_node(const float4 *nd, float4 &n0, float4 &n1, float4 &n2, int4 &n3) {
    asm("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
        : "=f"(n0.x), "=f"(n0.y), "=f"(n0.z), "=f"(n0.w), "=f"(n1.x), "=f"(n1.y), "=f"(n1.z), "=f"(n1.w)
        : "l"(nd));
    asm("ld.global.nc.v8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
        : "=f"(n2.x), "=f"(n2.y), "=f"(n2.z), "=f"(n2.w), "=r"(n3.x), "=r"(n3.y), "=r"(n3.z), "=r"(n3.w)
        : "l"(nd + 2));
}

// Traversal stacks with one interface: reset / empty / push / pop of 32-bit
// entries, at most kStackSize of them (the builder's depth bound). The
// stack object holds only scalars, so it lives in registers; the entries
// that live in local memory are in a separate array of kLocal words that
// the traversal declares and passes to push / pop.
//
// LocalStack: every entry in that local array (L1-cached; local stores
// are written through to L2).
struct LocalStack {
    static constexpr int kLocal = kStackSize;
    int sp;
    __device__ __forceinline__ void reset() { sp = 0; }
    __device__ __forceinline__ bool empty() const { return sp == 0; }
    __device__ __forceinline__ void push(unsigned v, unsigned *lm) { lm[sp++] = v; }
    __device__ __forceinline__ unsigned pop(unsigned *lm) { return lm[--sp]; }
};

// ShortStack: the top kShort entries (a power of two) in shared memory, one
// column per thread (`col` = &smem[threadIdx.x], `stride` = words per
// level = threads per block), so the 32 lanes of a warp touch 32 different
// banks at every level; deeper entries spill to the local array, oldest
// first.
template <int kShort>
struct ShortStack {
    static constexpr int kLocal = kStackSize - kShort;
    unsigned *col;
    int stride;
    int sp;
    __device__ __forceinline__ void reset() { sp = 0; }
    __device__ __forceinline__ bool empty() const { return sp == 0; }
    __device__ __forceinline__ void push(unsigned v, unsigned *lm) {
        unsigned *slot = col + (sp & (kShort - 1)) * stride;
        if (sp >= kShort) lm[sp - kShort] = *slot;
        *slot = v;
        ++sp;
    }
    __device__ __forceinline__ unsigned pop(unsigned *lm) {
        --sp;
        unsigned *slot = col + (sp & (kShort - 1)) * stride;
        const unsigned v = *slot;
        if (sp >= kShort) *slot = lm[sp - kShort];
        return v;
    }
};

// --- 16-bit quantised nodes (layout and grid: bvh16.cuh) ---

// 2^23 + the low (kHi = 0) or high (kHi = 1) 16 bits of w, as a float.
template <int kHi>
__device__ __forceinline__ float q16_biased(unsigned w) {
    return __uint_as_float(__byte_perm(w, 0x4B000000u, kHi ? 0x7432u : 0x7410u));
}

// One 32 B quantised node: the two child boxes decoded to floats and the
// links, in the float node's register layout (n0, n1: x/y bounds of child
// 0 and 1; n2: z bounds of both; n3: links).
__device__ __forceinline__ void load_node16(const float4 *cn, int node, const QuantGrid &g, float4 &n0, float4 &n1,
                                            float4 &n2, int4 &n3) {
    unsigned w[8];
    asm("ld.global.nc.v8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
        : "=r"(w[0]), "=r"(w[1]), "=r"(w[2]), "=r"(w[3]), "=r"(w[4]), "=r"(w[5]), "=r"(w[6]), "=r"(w[7])
        : "l"(cn + 2 * (size_t)node));
    // child c, component j (0-5: lo x y z, hi x y z) is index 6c + j
#define CRT_Q16(I) q16_biased<(I)&1>(w[(I) >> 1])
    n0 = make_float4(fmaf(CRT_Q16(0), g.s[0], g.p[0]), fmaf(CRT_Q16(3), g.s[0], g.p[0]),
                     fmaf(CRT_Q16(1), g.s[1], g.p[1]), fmaf(CRT_Q16(4), g.s[1], g.p[1]));
    n1 = make_float4(fmaf(CRT_Q16(6), g.s[0], g.p[0]), fmaf(CRT_Q16(9), g.s[0], g.p[0]),
                     fmaf(CRT_Q16(7), g.s[1], g.p[1]), fmaf(CRT_Q16(10), g.s[1], g.p[1]));
    n2 = make_float4(fmaf(CRT_Q16(2), g.s[2], g.p[2]), fmaf(CRT_Q16(5), g.s[2], g.p[2]),
                     fmaf(CRT_Q16(8), g.s[2], g.p[2]), fmaf(CRT_Q16(11), g.s[2], g.p[2]));
#undef CRT_Q16
    n3 = make_int4((int)w[6], (int)w[7], 0, 0);
}


template <bool kEarlyExit, bool kCull = true, bool kQuant = false, class Stack>
__device__ __forceinline__ Hit closest_hit_st(const BvhView &bvh, Stack &st, V3 o, V3 d, float tmin, float tmax,
                                              float t_exit = 0.f);

// closest_hit with the whole stack in local memory.
template <bool kEarlyExit, bool kCull = true>
__device__ __forceinline__ Hit closest_hit(const BvhView &bvh, V3 o, V3 d, float tmin, float tmax,
                                           float t_exit = 0.f) {
    LocalStack st;
    return closest_hit_st<kEarlyExit, kCull>(bvh, st, o, d, tmin, tmax, t_exit);
}

// The ordered traversal over a given stack (far child pushed, near child
// descended first; the empty stack ends it), over the float nodes or, with
// kQuant, their 16-bit quantised copy.
template <bool kEarlyExit, bool kCull, bool kQuant, class Stack>
__device__ __forceinline__ Hit closest_hit_st(const BvhView &bvh, Stack &st, V3 o, V3 d, float tmin, float tmax,
                                              float t_exit) {
    Hit hit;
    hit.t = tmax;
    hit.slot = -1;
    hit.b1 = hit.b2 = 0.f;
    V3 inv = v3(rrcp(d.x), rrcp(d.y), rrcp(d.z));
    unsigned lm[Stack::kLocal];
    st.reset();
    int link = 0;  // root interior node
    while (link != kSentinel) {
        // Descend interior nodes until a leaf link or an empty stack.
        while (link >= 0) {
            if (link >= bvh.num_nodes) {
                report_traversal_bounds(bvh);
                return hit;
            }
            float4 n0, n1, n2;
            int4 n3;
            if (kQuant) {
                load_node16(bvh.cnodes, link, bvh.grid, n0, n1, n2, n3);
            } else {
                const float4 *n = bvh.nodes + 4 * (size_t)link;
                n0 = __ldg(n + 0);
                n1 = __ldg(n + 1);
                n2 = __ldg(n + 2);
                n3 = __ldg(reinterpret_cast<const int4 *>(n + 3));
            }
            float t0, t1;
            bool h0 = slab(n0.x, n0.y, n0.z, n0.w, n2.x, n2.y, o, inv, tmin, hit.t, t0);
            bool h1 = slab(n1.x, n1.y, n1.z, n1.w, n2.z, n2.w, o, inv, tmin, hit.t, t1);
            if (h0 && h1) {
                int near = n3.x, far = n3.y;
                if (t1 < t0) { near = n3.y; far = n3.x; }
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
        // Leaf.
        int code = ~link;
        int first = code >> 4, count = code & 15;
        if (first + count > bvh.num_tris) {
            report_traversal_bounds(bvh);
            return hit;
        }
        for (int k = 0; k < count; ++k) {
            int slot = first + k;
            const float4 *tp = bvh.tris + 3 * (size_t)slot;
            float4 a = __ldg(tp + 0), b = __ldg(tp + 1), c = __ldg(tp + 2);
            bool acc = intersect_triangle<kCull>(o, d, a, b, c, slot, hit);
            if (kEarlyExit && acc && hit.t < t_exit) return hit;
        }
        link = st.empty() ? kSentinel : (int)st.pop(lm);
    }
    return hit;
}

// Warp-coherent closest hit: the 32 lanes of a warp traverse the tree as
// one packet (for the extend stage's primary rays, which sit in pixel
// order). Every lane of the current node's mask tests the node's two child
// boxes against its own ray interval [tmin, own closest]; the warp descends
// into a child that some lane hit (the one most of the lanes hitting both
// reach first) and pushes the other, with the mask of lanes that hit it,
// onto a stack of (link, mask) entries kept for the warp in shared memory
// (ws_link / ws_mask, kStackSize entries each, touched by lane 0 only and
// broadcast by shuffles). A leaf's triangles are tested by the lanes of its
// mask. Each lane prunes and tests exactly as closest_hit<false> does on its
// own ray; it may enter boxes its own ray would not, which only adds
// triangle tests whose accepted hits are real intersections, so its closest
// hit is closest_hit's up to the choice between triangles at equal t. All
// 32 lanes call it together; lanes with `active` false only vote.
template <bool kCull = true>
__device__ __forceinline__ Hit closest_hit_warp(const BvhView &bvh, int *ws_link, unsigned *ws_mask, bool active, V3 o,
                                                V3 d, float tmin, float tmax) {
    Hit hit;
    hit.t = tmax;
    hit.slot = -1;
    hit.b1 = hit.b2 = 0.f;
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const unsigned lane_bit = 1u << lane;
    const V3 inv = v3(rrcp(d.x), rrcp(d.y), rrcp(d.z));
    unsigned mask = __ballot_sync(full, active);
    int link = 0, sp = 0;  // warp-uniform: current link, stack depth
    while (mask) {
        bool pop = true;
        if (link >= 0) {
            if (link >= bvh.num_nodes) {
                report_traversal_bounds(bvh);
                return hit;
            }
            float4 n0, n1, n2;
            int4 n3;
            load_node(bvh.nodes + 4 * (size_t)link, n0, n1, n2, n3);
            float t0 = 0.f, t1 = 0.f;
            bool h0 = false, h1 = false;
            if (mask & lane_bit) {
                h0 = slab(n0.x, n0.y, n0.z, n0.w, n2.x, n2.y, o, inv, tmin, hit.t, t0);
                h1 = slab(n1.x, n1.y, n1.z, n1.w, n2.z, n2.w, o, inv, tmin, hit.t, t1);
            }
            const unsigned m0 = __ballot_sync(full, h0), m1 = __ballot_sync(full, h1);
            if (m0 && m1) {
                const unsigned near1 = __ballot_sync(full, h0 && h1 && t1 < t0);
                const bool go1 = 2 * __popc(near1) > __popc(m0 & m1);
                if (sp >= kStackSize) {
                    report_traversal_bounds(bvh);
                    return hit;
                }
                if (lane == 0) {
                    ws_link[sp] = go1 ? n3.x : n3.y;
                    ws_mask[sp] = go1 ? m0 : m1;
                }
                ++sp;
                link = go1 ? n3.y : n3.x;
                mask = go1 ? m1 : m0;
                pop = false;
            } else if (m0 | m1) {
                link = m0 ? n3.x : n3.y;
                mask = m0 ? m0 : m1;
                pop = false;
            }
        } else {
            const int code = ~link;
            const int first = code >> 4, count = code & 15;
            if (first + count > bvh.num_tris) {
                report_traversal_bounds(bvh);
                return hit;
            }
            if (mask & lane_bit)
                for (int k = 0; k < count; ++k) {
                    const int slot = first + k;
                    const float4 *tp = bvh.tris + 3 * (size_t)slot;
                    const float4 a = __ldg(tp + 0), b = __ldg(tp + 1), c = __ldg(tp + 2);
                    intersect_triangle<kCull>(o, d, a, b, c, slot, hit);
                }
        }
        if (pop) {
            if (sp == 0) break;
            --sp;
            int l = 0;
            unsigned mk = 0;
            if (lane == 0) {
                l = ws_link[sp];
                mk = ws_mask[sp];
            }
            link = __shfl_sync(full, l, 0);
            mask = __shfl_sync(full, mk, 0);
        }
    }
    return hit;
}

__device__ __forceinline__ int tri_prim(const BvhView &bvh, int slot) {
    return __float_as_int(__ldg(bvh.tris + 3 * (size_t)slot).w);
}

#endif  // __CUDACC__

}  // namespace crt
