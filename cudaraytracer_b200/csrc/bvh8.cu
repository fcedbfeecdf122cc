// Collapse of the binary BVH into the 8-wide quantised layout of bvh8.cuh.
//
// Each wide node starts from the two children of a binary node and opens
// the interior child of largest surface area until it holds eight children
// or only leaves remain (the greedy collapse of the wide-BVH literature;
// the SAH-optimal variant is not needed for the bound it gives here). The
// children are placed into slots by octant, and their boxes are quantised
// per axis to bytes on a power-of-two grid whose decoded value is checked
// against the float box with the same fmaf the kernels evaluate.
#include "bvh8.cuh"
#include "bvh_build.h"
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

namespace crt {
namespace {

struct Child {
    int link;
    float lo[3], hi[3];
};

inline int f2i(float f) {
    int i;
    std::memcpy(&i, &f, 4);
    return i;
}
inline float u2f(unsigned u) {
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}

void read_children(const float4 *n, Child c[2]) {
    c[0] = Child{f2i(n[3].x), {n[0].x, n[0].z, n[2].x}, {n[0].y, n[0].w, n[2].y}};
    c[1] = Child{f2i(n[3].y), {n[1].x, n[1].z, n[2].z}, {n[1].y, n[1].w, n[2].w}};
}

bool empty_leaf(int link) { return link < 0 && ((~link) & 15) == 0; }

double half_area(const Child &c) {
    double dx = std::max(0.0, (double)c.hi[0] - c.lo[0]);
    double dy = std::max(0.0, (double)c.hi[1] - c.lo[1]);
    double dz = std::max(0.0, (double)c.hi[2] - c.lo[2]);
    return dx * dy + dy * dz + dz * dx;
}

// The value the kernels decode for byte q: fmaf(2^23 + q, s, pp).
inline float decode(int q, float s, float pp) { return std::fmaf(8388608.0f + (float)q, s, pp); }

struct AxisQuant {
    float pp;
    unsigned ebias;
    unsigned char qlo[8], qhi[8];
};

// Quantises the children's [lo, hi] on one axis: the decoded bytes satisfy
// decode(qlo) <= lo and decode(qhi) >= hi for every child.
AxisQuant quantise_axis(const std::vector<Child> &ch, int axis) {
    float L = INFINITY, H = -INFINITY;
    for (const Child &c : ch) {
        L = std::min(L, c.lo[axis]);
        H = std::max(H, c.hi[axis]);
    }
    CRT_CHECK(std::isfinite(L) && std::isfinite(H), CRT_ERR_INVALID, "BVH8: non-finite bounds");
    const double ext = (double)H - (double)L;
    int e = ext > 0.0 ? (int)std::ceil(std::log2(ext / 250.0)) : -126;
    e = std::max(-126, std::min(e, 100));
    for (;; ++e) {
        CRT_CHECK(e <= 100, CRT_ERR_INVALID, "BVH8: cannot quantise a child box");
        AxisQuant a;
        a.ebias = (unsigned)(e + 127);
        const float s = u2f(a.ebias << 23);
        float pp = L - 8388608.0f * s;
        while (decode(0, s, pp) > L) pp = std::nextafter(pp, -INFINITY);
        a.pp = pp;
        bool ok = true;
        for (size_t j = 0; j < ch.size() && ok; ++j) {
            const float lo = ch[j].lo[axis], hi = ch[j].hi[axis];
            int q = (int)std::floor(((double)lo - (double)L) / (double)s);
            q = std::max(0, std::min(q, 255));
            while (q > 0 && decode(q, s, pp) > lo) --q;
            while (q < 255 && decode(q + 1, s, pp) <= lo) ++q;
            int r = (int)std::ceil(((double)hi - (double)L) / (double)s);
            r = std::max(0, std::min(r, 255));
            while (r < 255 && decode(r, s, pp) < hi) ++r;
            while (r > 0 && decode(r - 1, s, pp) >= hi) --r;
            if (decode(q, s, pp) > lo || decode(r, s, pp) < hi) {
                ok = false;
                break;
            }
            a.qlo[j] = (unsigned char)q;
            a.qhi[j] = (unsigned char)r;
        }
        if (ok) return a;
    }
}

struct Collapser {
    const float4 *bin;
    int64_t nbin;
    std::vector<float4> &nodes;
    std::vector<int> &links;
    int depth = 0;

    // Emits the wide node whose children are the binary node `b`'s subtree
    // frontier; returns its index.
    int emit(int b, int level) {
        CRT_CHECK(b >= 0 && b < nbin, CRT_ERR_INVALID, "BVH8: binary link out of range");
        CRT_CHECK(level < kBvh8MaxDepth - 1, CRT_ERR_CAPACITY, "BVH8: tree deeper than the traversal stack");
        depth = std::max(depth, level + 1);
        std::vector<Child> ch;
        ch.reserve(8);
        Child c2[2];
        read_children(bin + 4 * (size_t)b, c2);
        for (const Child &c : c2)
            if (!empty_leaf(c.link)) ch.push_back(c);
        while (ch.size() < 8) {
            int best = -1;
            double best_a = -1.0;
            for (size_t i = 0; i < ch.size(); ++i)
                if (ch[i].link >= 0 && half_area(ch[i]) > best_a) {
                    best_a = half_area(ch[i]);
                    best = (int)i;
                }
            if (best < 0) break;
            CRT_CHECK(ch[best].link < nbin, CRT_ERR_INVALID, "BVH8: binary link out of range");
            read_children(bin + 4 * (size_t)ch[best].link, c2);
            ch.erase(ch.begin() + best);
            for (const Child &c : c2)
                if (!empty_leaf(c.link)) ch.push_back(c);
        }
        // slots by octant: child towards corner s of the node's centre
        float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (const Child &c : ch)
            for (int k = 0; k < 3; ++k) {
                lo[k] = std::min(lo[k], c.lo[k]);
                hi[k] = std::max(hi[k], c.hi[k]);
            }
        int slot_of[8] = {-1, -1, -1, -1, -1, -1, -1, -1};
        std::vector<Child> slotted(8, Child{0, {0, 0, 0}, {0, 0, 0}});
        unsigned valid = 0;
        {
            bool used_child[8] = {false, false, false, false, false, false, false, false};
            for (size_t round = 0; round < ch.size(); ++round) {
                double best = -INFINITY;
                int bc = -1, bs = -1;
                for (size_t i = 0; i < ch.size(); ++i) {
                    if (used_child[i]) continue;
                    double off[3];
                    for (int k = 0; k < 3; ++k)
                        off[k] = 0.5 * ((double)ch[i].lo[k] + ch[i].hi[k]) - 0.5 * ((double)lo[k] + hi[k]);
                    for (int s = 0; s < 8; ++s) {
                        if (slot_of[s] >= 0) continue;
                        double score = (s & 4 ? off[0] : -off[0]) + (s & 2 ? off[1] : -off[1]) +
                                       (s & 1 ? off[2] : -off[2]);
                        if (score > best) {
                            best = score;
                            bc = (int)i;
                            bs = s;
                        }
                    }
                }
                used_child[bc] = true;
                slot_of[bs] = bc;
                slotted[bs] = ch[bc];
                valid |= 1u << bs;
            }
        }
        // quantise over the slotted children (empty slots decode from 0)
        std::vector<Child> filled;
        int fill_slot[8];
        for (int s = 0; s < 8; ++s)
            if (valid & (1u << s)) {
                fill_slot[filled.size()] = s;
                filled.push_back(slotted[s]);
            }
        AxisQuant q[3] = {quantise_axis(filled, 0), quantise_axis(filled, 1), quantise_axis(filled, 2)};
        unsigned char bytes[6][8];
        std::memset(bytes, 0, sizeof(bytes));
        for (size_t i = 0; i < filled.size(); ++i) {
            const int s = fill_slot[i];
            for (int k = 0; k < 3; ++k) {
                bytes[k][s] = q[k].qlo[i];
                bytes[3 + k][s] = q[k].qhi[i];
            }
        }
        const int me = (int)(nodes.size() / 4);
        CRT_CHECK(me < (1 << 24), CRT_ERR_CAPACITY, "BVH8: more than 2^24 wide nodes");
        nodes.resize(nodes.size() + 4);
        links.resize(links.size() + 8, 0);
        float4 *nd = &nodes[4 * (size_t)me];
        const unsigned w = q[0].ebias | (q[1].ebias << 8) | (q[2].ebias << 16) | (valid << 24);
        nd[0] = make_float4(q[0].pp, q[1].pp, q[2].pp, u2f(w));
        unsigned words[12];
        std::memcpy(words, bytes, sizeof(words));
        // [1] qlo_x qlo_y  [2] qlo_z qhi_x  [3] qhi_y qhi_z (slot j at byte j)
        nd[1] = make_float4(u2f(words[0]), u2f(words[1]), u2f(words[2]), u2f(words[3]));
        nd[2] = make_float4(u2f(words[4]), u2f(words[5]), u2f(words[6]), u2f(words[7]));
        nd[3] = make_float4(u2f(words[8]), u2f(words[9]), u2f(words[10]), u2f(words[11]));
        for (int s = 0; s < 8; ++s) {
            if (!(valid & (1u << s))) continue;
            const int l = slotted[s].link;
            const int wl = l >= 0 ? emit(l, level + 1) : l;
            links[8 * (size_t)me + s] = wl;
        }
        return me;
    }
};

}  // namespace

int collapse_bvh8(const float4 *bin_nodes, int64_t num_nodes, std::vector<float4> &nodes, std::vector<int> &links) {
    CRT_CHECK(num_nodes >= 1, CRT_ERR_INVALID, "BVH8: empty binary tree");
    nodes.clear();
    links.clear();
    nodes.reserve((size_t)num_nodes / 2 * 4);
    links.reserve((size_t)num_nodes / 2 * 8);
    Collapser c{bin_nodes, num_nodes, nodes, links};
    c.emit(0, 0);
    return c.depth;
}

void build_bvh8(BvhBuffers &b, cudaStream_t stream) {
    std::vector<float4> bin((size_t)b.num_nodes * 4);
    CRT_CUDA(cudaMemcpyAsync(bin.data(), b.nodes, bin.size() * sizeof(float4), cudaMemcpyDeviceToHost, stream));
    CRT_CUDA(cudaStreamSynchronize(stream));
    std::vector<float4> nodes;
    std::vector<int> links;
    b.wide_depth = collapse_bvh8(bin.data(), b.num_nodes, nodes, links);
    b.num_wide_nodes = (int64_t)(nodes.size() / 4);
    CRT_CUDA(cudaMalloc(&b.wnodes, nodes.size() * sizeof(float4)));
    CRT_CUDA(cudaMalloc(&b.wlinks, links.size() * sizeof(int)));
    CRT_CUDA(cudaMemcpyAsync(b.wnodes, nodes.data(), nodes.size() * sizeof(float4), cudaMemcpyHostToDevice, stream));
    CRT_CUDA(cudaMemcpyAsync(b.wlinks, links.data(), links.size() * sizeof(int), cudaMemcpyHostToDevice, stream));
    CRT_CUDA(cudaStreamSynchronize(stream));
}

}  // namespace crt
