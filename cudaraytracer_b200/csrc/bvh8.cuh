// 8-wide BVH with 8-bit quantised child boxes, and its traversal.
//
// The binary tree of bvh_build.cu is collapsed into nodes of up to eight
// children (bvh8.cu). Per wide node, in HBM:
//   nodes: 64 B = 4 x float4, read as two 32 B loads
//     [0] px', py', pz' (float), w = ex | ey << 8 | ez << 16 | valid << 24
//     [1] qlo_x[8] qlo_y[8]   (bytes, child slot j at byte j)
//     [2] qlo_z[8] qhi_x[8]
//     [3] qhi_y[8] qhi_z[8]
//   links: 32 B = 8 x int per node, the child in each slot: >= 0 a wide node,
//     < 0 a leaf ~((first << 4) | count) of the binary tree's leaf-ordered
//     triangles (count 1..8).
// A child bound decodes as fmaf(2^23 + q, 2^(e-127), p') with one rounding:
// (2^23 + q) is the float whose low mantissa byte is q (one byte permute),
// the product by a power of two is exact, and p' is chosen by the builder.
// The builder evaluates the same fmaf and picks every byte so the decoded
// box contains the child's float box; the slab test (bvh.cuh) is monotone in
// the box bounds, so every box the binary traversal accepts is accepted
// here too, and closest hits stay those of the triangle test itself.
// The 8 children sit in slots by octant: the child in slot s lies towards
// corner s (bit 2 = +x, bit 1 = +y, bit 0 = +z) of the node; a ray whose
// direction has sign bits `oct` visits slot k ^ oct in order k = 0..7,
// nearest corner first (the ordering of Ylitie, Karras and Laine, "Efficient
// Incoherent Ray Traversal on GPUs Through Compressed Wide BVHs", HPG 2017).
// The reference traverses a binary tree of 32 B nodes (Src/Core/bvh.cu:253).
#pragma once
#include "bvh.cuh"
#include <vector>

namespace crt {

constexpr int kBvh8MaxDepth = 64;

#ifdef __CUDACC__

// 2^23 + the j-th byte of w, as a float (j in 0..3, compile-time).
template <int j>
__device__ __forceinline__ float q_biased(unsigned w) {
    return __uint_as_float(__byte_perm(w, 0x4B000000u, 0x7440u | j));
}

// Tests the eight child boxes of wide node `node` against the ray interval
// [tmin, tmax]. Returns the hit children as bits k = slot ^ oct.
__device__ __forceinline__ unsigned visit8(const float4 *nodes, int node, V3 o, V3 inv, float tmin, float tmax,
                                           unsigned oct) {
    const float4 *nd = nodes + 4 * (size_t)node;
    float4 h;
    uint4 b1, b2, b3;
    asm("ld.global.nc.v8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
        : "=f"(h.x), "=f"(h.y), "=f"(h.z), "=f"(h.w), "=r"(b1.x), "=r"(b1.y), "=r"(b1.z), "=r"(b1.w)
        : "l"(nd));
    asm("ld.global.nc.v8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
        : "=r"(b2.x), "=r"(b2.y), "=r"(b2.z), "=r"(b2.w), "=r"(b3.x), "=r"(b3.y), "=r"(b3.z), "=r"(b3.w)
        : "l"(nd + 2));
    const unsigned hw = __float_as_uint(h.w);
    const float sx = __uint_as_float((hw & 0xffu) << 23);
    const float sy = __uint_as_float(((hw >> 8) & 0xffu) << 23);
    const float sz = __uint_as_float(((hw >> 16) & 0xffu) << 23);
    const unsigned valid = hw >> 24;
    unsigned mask = 0;
#define CRT_VISIT_CHILD(J, LX, LY, LZ, HX, HY, HZ)                                                              \
    {                                                                                                         \
        float t_;                                                                                             \
        const bool hit_ = slab(fmaf(q_biased<(J)&3>(LX), sx, h.x), fmaf(q_biased<(J)&3>(HX), sx, h.x),       \
                               fmaf(q_biased<(J)&3>(LY), sy, h.y), fmaf(q_biased<(J)&3>(HY), sy, h.y),       \
                               fmaf(q_biased<(J)&3>(LZ), sz, h.z), fmaf(q_biased<(J)&3>(HZ), sz, h.z), o, inv, \
                               tmin, tmax, t_);                                                               \
        if (hit_ && (valid & (1u << (J)))) mask |= 1u << ((J) ^ oct);                                         \
    }
    CRT_VISIT_CHILD(0, b1.x, b1.z, b2.x, b2.z, b3.x, b3.z)
    CRT_VISIT_CHILD(1, b1.x, b1.z, b2.x, b2.z, b3.x, b3.z)
    CRT_VISIT_CHILD(2, b1.x, b1.z, b2.x, b2.z, b3.x, b3.z)
    CRT_VISIT_CHILD(3, b1.x, b1.z, b2.x, b2.z, b3.x, b3.z)
    CRT_VISIT_CHILD(4, b1.y, b1.w, b2.y, b2.w, b3.y, b3.w)
    CRT_VISIT_CHILD(5, b1.y, b1.w, b2.y, b2.w, b3.y, b3.w)
    CRT_VISIT_CHILD(6, b1.y, b1.w, b2.y, b2.w, b3.y, b3.w)
    CRT_VISIT_CHILD(7, b1.y, b1.w, b2.y, b2.w, b3.y, b3.w)
#undef CRT_VISIT_CHILD
    return mask;
}

// The eight child links of wide node `node` (one 32 B read-only load).
__device__ __forceinline__ void load_links8(const int *links, int node, int (&lk)[8]) {
    asm("ld.global.nc.v8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
        : "=r"(lk[0]), "=r"(lk[1]), "=r"(lk[2]), "=r"(lk[3]), "=r"(lk[4]), "=r"(lk[5]), "=r"(lk[6]), "=r"(lk[7])
        : "l"(links + 8 * (size_t)node));
}

// lk[s] for a run-time slot s without indexing registers dynamically.
__device__ __forceinline__ int select_link(const int (&lk)[8], unsigned s) {
    const int a = (s & 1) ? lk[1] : lk[0], b = (s & 1) ? lk[3] : lk[2];
    const int c = (s & 1) ? lk[5] : lk[4], d = (s & 1) ? lk[7] : lk[6];
    const int e = (s & 2) ? b : a, f = (s & 2) ? d : c;
    return (s & 4) ? f : e;
}

__device__ __forceinline__ unsigned ray_octant(V3 d) {
    return (d.x < 0.f ? 4u : 0u) | (d.y < 0.f ? 2u : 0u) | (d.z < 0.f ? 1u : 0u);
}

// Finds the next leaf of an ordered traversal. `cur` holds the current
// wide node and its children still to visit; returns a leaf link (< 0), or
// 0 when the stack is exhausted. With kRegLinks the links of the node last
// visited are fetched with its boxes and kept in registers (lk, valid while
// `fresh`), so descending into its children needs no further load; links of
// nodes popped from the stack are read from memory.
template <int kShort, bool kRegLinks = false>
__device__ __forceinline__ int next_leaf8(const BvhView &bvh, unsigned &cur, ShortStack<kShort> &st, unsigned *lm, V3 o,
                                          V3 inv, float tmin, float tmax, unsigned oct, int (&lk)[8], bool &fresh) {
    while (true) {
        unsigned m = cur & 0xffu;
        if (m == 0) {
            if (st.empty()) return 0;
            cur = st.pop(lm);
            m = cur & 0xffu;
            fresh = false;
        }
        const unsigned k = __ffs(m) - 1;
        cur &= ~(1u << k);
        const int link = (kRegLinks && fresh) ? select_link(lk, k ^ oct)
                                              : __ldg(bvh.wlinks + 8 * (size_t)(cur >> 8) + (k ^ oct));
        if (link < 0) return link;
        if (cur & 0xffu) st.push(cur, lm);
        if (kRegLinks) {
            load_links8(bvh.wlinks, link, lk);
            fresh = true;
        }
        cur = ((unsigned)link << 8) | visit8(bvh.wnodes, link, o, inv, tmin, tmax, oct);
    }
}

// closest_hit (bvh.cuh) over the 8-wide tree: the same semantics (boxes
// pruned by [tmin, closest], triangles accepted on [0, 1e8], strict t <
// closest, early exit at an accepted hit with t < t_exit when kEarlyExit).
template <bool kEarlyExit, int kShort, bool kCull = true>
__device__ __forceinline__ Hit closest_hit8(const BvhView &bvh, ShortStack<kShort> &st, V3 o, V3 d, float tmin,
                                            float tmax, float t_exit = 0.f) {
    Hit hit;
    hit.t = tmax;
    hit.slot = -1;
    hit.b1 = hit.b2 = 0.f;
    const V3 inv = v3(rrcp(d.x), rrcp(d.y), rrcp(d.z));
    const unsigned oct = ray_octant(d);
    st.reset();
    unsigned lm[ShortStack<kShort>::kLocal];
    unsigned cur = visit8(bvh.wnodes, 0, o, inv, tmin, hit.t, oct);
    int lk[8];
    bool fresh = false;
    while (true) {
        const int leaf = next_leaf8<kShort>(bvh, cur, st, lm, o, inv, tmin, hit.t, oct, lk, fresh);
        if (leaf == 0) break;
        const int code = ~leaf;
        const int first = code >> 4, count = code & 15;
        for (int k = 0; k < count; ++k) {
            const int slot = first + k;
            const float4 *tp = bvh.tris + 3 * (size_t)slot;
            const float4 a = __ldg(tp + 0), b = __ldg(tp + 1), c = __ldg(tp + 2);
            const bool acc = intersect_triangle<kCull>(o, d, a, b, c, slot, hit);
            if (kEarlyExit && acc && hit.t < t_exit) return hit;
        }
    }
    return hit;
}

#endif  // __CUDACC__

// Host: collapses the binary tree (num_nodes x 4 float4 in the bvh.cuh
// layout, root at 0) into the 8-wide layout above. Appends to `nodes` (4
// float4 per node) and `links` (8 ints per node); returns the wide depth.
int collapse_bvh8(const float4 *bin_nodes, int64_t num_nodes, std::vector<float4> &nodes, std::vector<int> &links);
// Device: builds b.wnodes / b.wlinks from b.nodes (bvh8.cu).
struct BvhBuffers;
void build_bvh8(BvhBuffers &b, cudaStream_t stream);

}  // namespace crt
