// On-device binned-SAH BVH build.
//
// Replaces the reference's host recursion (BVH::RecursiveBuild,
// Src/Core/bvh.cu:44-175: 12 buckets on the largest centroid axis, leaves of
// at most 4, one `new` per node) and its flattening/upload (FlattenBVHTree,
// Src/Core/bvh.cu:186-206; CreateBVH, :308-314).
//
// Scheme (all on the device, deterministic):
//  * "large" tasks (> kSmallTask primitives) are split breadth-first, one
//    level per round: a binning kernel over 4096-primitive chunks (shared
//    memory bins merged with global atomics), one thread per task evaluating
//    the SAH over 3 axes x 15 candidate planes, and a stable chunked
//    partition (per-chunk counts, host prefix, block-local ranks).
//  * "small" tasks (<= kSmallTask) are finished by one 256-thread block each,
//    depth-first with a shared-memory task stack, binning + SAH + stable
//    partition per node in shared memory.
//  * a gather kernel writes the triangles in leaf order (48 B each).
// Min/max reductions are order-independent and all partitions are stable, so
// the tree (and thus tie-breaking between equal-t triangles) is reproducible.
#include "bvh_build.h"
#include <vector>
#include <algorithm>
#include <cstring>
#include <chrono>
#include <cstdlib>

namespace crt {
namespace {

constexpr int NB = 16;             // bins per axis
constexpr int kSmallTask = 2048;   // largest task finished by one block
constexpr int kChunk = 4096;       // primitives per block in the large phase
constexpr int kBlock = 256;
constexpr int kMaxLeafSAH = 8;     // largest leaf the SAH may choose
constexpr int kMedianDepth = 36;   // below this depth, split by index median
// Traversal step cost relative to one triangle test: 3 (leaves of 4.5
// triangles on average on the icosphere field, 293k nodes for 1.31M
// triangles) measured 6% faster shadow queries than 1 (1.7 per leaf, 764k
// nodes), extend within 1.5%; higher costs were not faster.
constexpr float kCostTrav = 3.0f;
constexpr float kCostTri = 1.0f;

// The SAH's leaf decision in the small phase: traversal cost relative to
// one triangle test, and the largest leaf it may form (1..kMaxLeafSAH).
// Defaults kCostTrav and kMaxLeafSAH; CRT_SAH_TRAV and CRT_SAH_MAX_LEAF
// override them at build time (for measuring other tree shapes).
struct SahParams {
    float cost_trav;
    int max_leaf;
};

SahParams sah_params() {
    SahParams p{kCostTrav, kMaxLeafSAH};
    if (const char *e = getenv("CRT_SAH_TRAV")) {
        const float v = (float)atof(e);
        if (v > 0.f && v < 100.f) p.cost_trav = v;
    }
    if (const char *e = getenv("CRT_SAH_MAX_LEAF")) {
        const int v = atoi(e);
        if (v >= 1 && v <= kMaxLeafSAH) p.max_leaf = v;
    }
    return p;
}

struct Task {
    int start, count, link_slot, depth;
    float blo[3], bhi[3];  // bounds of the primitives
    float clo[3], chi[3];  // bounds of their centroids
};

struct Bins {  // keys are order-preserving ints of floats
    int cnt[3][NB];
    int b[3][NB][6];  // prim bounds lo xyz, hi xyz
    int c[3][NB][6];  // centroid bounds lo xyz, hi xyz
};

struct Decision {
    int mode;   // 0 leaf, 1 sah, 2 median
    int axis, split, nleft;
    Task child[2];
};

__host__ __device__ inline int f2key(float f) {
#ifdef __CUDA_ARCH__
    int i = __float_as_int(f);
#else
    int i;
    std::memcpy(&i, &f, 4);
#endif
    return i >= 0 ? i : i ^ 0x7FFFFFFF;
}
__host__ __device__ inline float key2f(int k) {
    int i = k >= 0 ? k : k ^ 0x7FFFFFFF;
#ifdef __CUDA_ARCH__
    return __int_as_float(i);
#else
    float f;
    std::memcpy(&f, &i, 4);
    return f;
#endif
}

__device__ __forceinline__ float bin_scale(float lo, float hi) {
    float ext = hi - lo;
    return ext > 0.f ? (float)NB / ext : 0.f;
}
__device__ __forceinline__ int bin_of(float c, float lo, float scale) {
    int b = (int)((c - lo) * scale);
    return b < 0 ? 0 : (b >= NB ? NB - 1 : b);
}
__device__ __forceinline__ float half_area(float lx, float ly, float lz, float hx, float hy, float hz) {
    if (lx > hx || ly > hy || lz > hz) return 0.f;
    float ex = hx - lx, ey = hy - ly, ez = hz - lz;
    return ex * ey + ey * ez + ez * ex;
}

__device__ __forceinline__ void load_prim(const float4 *plo, const float4 *phi, int p, float lo[3], float hi[3],
                                          float c[3]) {
    float4 a = __ldg(plo + p), b = __ldg(phi + p);
    lo[0] = a.x; lo[1] = a.y; lo[2] = a.z;
    hi[0] = b.x; hi[1] = b.y; hi[2] = b.z;
    c[0] = 0.5f * (a.x + b.x);
    c[1] = 0.5f * (a.y + b.y);
    c[2] = 0.5f * (a.z + b.z);
}

__device__ void bins_clear(Bins &bn, int tid, int nthreads) {
    int *cnt = &bn.cnt[0][0];
    int *b = &bn.b[0][0][0];
    int *c = &bn.c[0][0][0];
    for (int i = tid; i < 3 * NB; i += nthreads) cnt[i] = 0;
    for (int i = tid; i < 3 * NB * 6; i += nthreads) {
        int lohi = i % 6;
        int v = lohi < 3 ? INT_MAX : INT_MIN;
        b[i] = v;
        c[i] = v;
    }
}

__device__ __forceinline__ void bins_add(Bins &bn, const float lo[3], const float hi[3], const float c[3],
                                         const float clo[3], const float sc[3]) {
    int kl[3] = {f2key(lo[0]), f2key(lo[1]), f2key(lo[2])};
    int kh[3] = {f2key(hi[0]), f2key(hi[1]), f2key(hi[2])};
    int kc[3] = {f2key(c[0]), f2key(c[1]), f2key(c[2])};
    for (int a = 0; a < 3; ++a) {
        int b = bin_of(c[a], clo[a], sc[a]);
        atomicAdd(&bn.cnt[a][b], 1);
        for (int k = 0; k < 3; ++k) {
            atomicMin(&bn.b[a][b][k], kl[k]);
            atomicMax(&bn.b[a][b][3 + k], kh[k]);
            atomicMin(&bn.c[a][b][k], kc[k]);
            atomicMax(&bn.c[a][b][3 + k], kc[k]);
        }
    }
}

// Best split plane of one axis from its bins: bins 0..split go left.
__device__ void eval_axis(const Bins &bn, int a, float &best_cost, int &best_split) {
    float rarea[NB];
    int rcnt[NB];
    int lx = INT_MAX, ly = INT_MAX, lz = INT_MAX, hx = INT_MIN, hy = INT_MIN, hz = INT_MIN, n = 0;
    for (int i = NB - 1; i >= 1; --i) {
        lx = min(lx, bn.b[a][i][0]); ly = min(ly, bn.b[a][i][1]); lz = min(lz, bn.b[a][i][2]);
        hx = max(hx, bn.b[a][i][3]); hy = max(hy, bn.b[a][i][4]); hz = max(hz, bn.b[a][i][5]);
        n += bn.cnt[a][i];
        rcnt[i] = n;
        rarea[i] = n ? half_area(key2f(lx), key2f(ly), key2f(lz), key2f(hx), key2f(hy), key2f(hz)) : 0.f;
    }
    best_cost = INFINITY;
    best_split = -1;
    lx = ly = lz = INT_MAX;
    hx = hy = hz = INT_MIN;
    n = 0;
    for (int i = 0; i < NB - 1; ++i) {
        lx = min(lx, bn.b[a][i][0]); ly = min(ly, bn.b[a][i][1]); lz = min(lz, bn.b[a][i][2]);
        hx = max(hx, bn.b[a][i][3]); hy = max(hy, bn.b[a][i][4]); hz = max(hz, bn.b[a][i][5]);
        n += bn.cnt[a][i];
        if (n == 0 || rcnt[i + 1] == 0) continue;
        float cost = half_area(key2f(lx), key2f(ly), key2f(lz), key2f(hx), key2f(hy), key2f(hz)) * n +
                     rarea[i + 1] * rcnt[i + 1];
        if (cost < best_cost) {
            best_cost = cost;
            best_split = i;
        }
    }
}

// Child task bounds from the bins of a chosen (axis, split).
__device__ void child_from_bins(const Bins &bn, int a, int split, bool right, Task &t) {
    int bl[3] = {INT_MAX, INT_MAX, INT_MAX}, bh[3] = {INT_MIN, INT_MIN, INT_MIN};
    int cl[3] = {INT_MAX, INT_MAX, INT_MAX}, ch[3] = {INT_MIN, INT_MIN, INT_MIN};
    int n = 0;
    int i0 = right ? split + 1 : 0, i1 = right ? NB : split + 1;
    for (int i = i0; i < i1; ++i) {
        n += bn.cnt[a][i];
        for (int k = 0; k < 3; ++k) {
            bl[k] = min(bl[k], bn.b[a][i][k]);
            bh[k] = max(bh[k], bn.b[a][i][3 + k]);
            cl[k] = min(cl[k], bn.c[a][i][k]);
            ch[k] = max(ch[k], bn.c[a][i][3 + k]);
        }
    }
    t.count = n;
    for (int k = 0; k < 3; ++k) {
        t.blo[k] = key2f(bl[k]);
        t.bhi[k] = key2f(bh[k]);
        t.clo[k] = key2f(cl[k]);
        t.chi[k] = key2f(ch[k]);
    }
}

__device__ void write_node(float4 *nodes, int id, const Task &l, const Task &r) {
    float4 *n = nodes + 4 * (size_t)id;
    n[0] = make_float4(l.blo[0], l.bhi[0], l.blo[1], l.bhi[1]);
    n[1] = make_float4(r.blo[0], r.bhi[0], r.blo[1], r.bhi[1]);
    n[2] = make_float4(l.blo[2], l.bhi[2], r.blo[2], r.bhi[2]);
    n[3] = make_float4(__int_as_float(kSentinel), __int_as_float(kSentinel), 0.f, 0.f);
}

__device__ __forceinline__ void write_link(float4 *nodes, int slot, int value) {
    if (slot >= 0) reinterpret_cast<int *>(nodes)[slot] = value;
}

// ---------------------------------------------------------------------------
// Setup: per-primitive bounds, identity permutation, root bounds.
// ---------------------------------------------------------------------------
__global__ void k_prim_bounds(const float *verts, int n, float4 *plo, float4 *phi, int *idx, int *root_keys) {
    __shared__ int s[12];
    if (threadIdx.x < 12) s[threadIdx.x] = (threadIdx.x % 6) < 3 ? INT_MAX : INT_MIN;
    __syncthreads();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float *v = verts + 9 * (size_t)i;
        float lo[3], hi[3], c[3];
        for (int k = 0; k < 3; ++k) {
            // Bounds3D(v0, v1, v2) = Min(v0, Min(v1, v2)) (Src/Core/bounds.h:20-24).
            lo[k] = fminf(v[k], fminf(v[3 + k], v[6 + k]));
            hi[k] = fmaxf(v[k], fmaxf(v[3 + k], v[6 + k]));
            c[k] = 0.5f * (lo[k] + hi[k]);
        }
        plo[i] = make_float4(lo[0], lo[1], lo[2], 0.f);
        phi[i] = make_float4(hi[0], hi[1], hi[2], 0.f);
        idx[i] = i;
        for (int k = 0; k < 3; ++k) {
            atomicMin(&s[k], f2key(lo[k]));
            atomicMax(&s[3 + k], f2key(hi[k]));
            atomicMin(&s[6 + k], f2key(c[k]));
            atomicMax(&s[9 + k], f2key(c[k]));
        }
    }
    __syncthreads();
    if (threadIdx.x < 12) {
        if ((threadIdx.x % 6) < 3)
            atomicMin(&root_keys[threadIdx.x], s[threadIdx.x]);
        else
            atomicMax(&root_keys[threadIdx.x], s[threadIdx.x]);
    }
}

// ---------------------------------------------------------------------------
// Large phase.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kBlock) k_bin_large(const Task *tasks, const int *chunk_task, const int *chunk_begin,
                                                      const int *idx, const float4 *plo, const float4 *phi,
                                                      Bins *bins) {
    __shared__ Bins sb;
    int c = blockIdx.x;
    int ti = chunk_task[c];
    const Task &t = tasks[ti];
    int begin = chunk_begin[c];
    int end = min(begin + kChunk, t.start + t.count);
    bins_clear(sb, threadIdx.x, blockDim.x);
    __syncthreads();
    float sc[3] = {bin_scale(t.clo[0], t.chi[0]), bin_scale(t.clo[1], t.chi[1]), bin_scale(t.clo[2], t.chi[2])};
    for (int i = begin + threadIdx.x; i < end; i += blockDim.x) {
        float lo[3], hi[3], cc[3];
        load_prim(plo, phi, idx[i], lo, hi, cc);
        bins_add(sb, lo, hi, cc, t.clo, sc);
    }
    __syncthreads();
    Bins &g = bins[ti];
    for (int i = threadIdx.x; i < 3 * NB; i += blockDim.x) {
        int v = (&sb.cnt[0][0])[i];
        if (v) atomicAdd(&g.cnt[0][0] + i, v);
    }
    for (int i = threadIdx.x; i < 3 * NB * 6; i += blockDim.x) {
        bool lo = (i % 6) < 3;
        int vb = (&sb.b[0][0][0])[i], vc = (&sb.c[0][0][0])[i];
        if (lo) {
            if (vb != INT_MAX) atomicMin(&g.b[0][0][0] + i, vb);
            if (vc != INT_MAX) atomicMin(&g.c[0][0][0] + i, vc);
        } else {
            if (vb != INT_MIN) atomicMax(&g.b[0][0][0] + i, vb);
            if (vc != INT_MIN) atomicMax(&g.c[0][0][0] + i, vc);
        }
    }
}

__global__ void k_bins_init(Bins *bins, int ntasks) {
    int total = ntasks * (int)(sizeof(Bins) / 4);
    int *p = reinterpret_cast<int *>(bins);
    const int per = sizeof(Bins) / 4;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        int w = i % per;
        if (w < 3 * NB) {
            p[i] = 0;
        } else {
            int j = (w - 3 * NB) % 6;
            p[i] = j < 3 ? INT_MAX : INT_MIN;
        }
    }
}

__global__ void k_split_large(const Task *tasks, int ntasks, const Bins *bins, float4 *nodes, int *node_counter,
                              Decision *dec) {
    int ti = blockIdx.x * blockDim.x + threadIdx.x;
    if (ti >= ntasks) return;
    const Task t = tasks[ti];
    const Bins &bn = bins[ti];
    Decision d;
    d.mode = 2;
    d.axis = -1;
    d.split = -1;
    if (t.depth < kMedianDepth) {
        float best = INFINITY;
        for (int a = 0; a < 3; ++a) {
            float cst;
            int sp;
            eval_axis(bn, a, cst, sp);
            if (sp >= 0 && cst < best) {
                best = cst;
                d.axis = a;
                d.split = sp;
            }
        }
        if (d.axis >= 0) d.mode = 1;
    }
    int id = atomicAdd(node_counter, 1);
    write_link(nodes, t.link_slot, id);
    Task l, r;
    if (d.mode == 1) {
        child_from_bins(bn, d.axis, d.split, false, l);
        child_from_bins(bn, d.axis, d.split, true, r);
    } else {
        // Index median with the parent's bounds (conservative; rare).
        l = t;
        r = t;
        l.count = t.count / 2;
        r.count = t.count - l.count;
    }
    l.start = t.start;
    r.start = t.start + l.count;
    l.depth = r.depth = t.depth + 1;
    l.link_slot = id * 16 + 12;
    r.link_slot = id * 16 + 13;
    write_node(nodes, id, l, r);
    d.nleft = l.count;
    d.child[0] = l;
    d.child[1] = r;
    dec[ti] = d;
}

__device__ __forceinline__ bool goes_left(const Decision &d, const Task &t, int pos, const float4 *plo,
                                          const float4 *phi, int p) {
    if (d.mode != 1) return pos < t.start + d.nleft;
    float a = d.axis == 0 ? 0.5f * (__ldg(&plo[p].x) + __ldg(&phi[p].x))
              : d.axis == 1 ? 0.5f * (__ldg(&plo[p].y) + __ldg(&phi[p].y))
                            : 0.5f * (__ldg(&plo[p].z) + __ldg(&phi[p].z));
    return bin_of(a, t.clo[d.axis], bin_scale(t.clo[d.axis], t.chi[d.axis])) <= d.split;
}

// Block-wide exclusive scan of one int per thread (kBlock threads).
__device__ int block_exclusive_scan(int v, int *s_warp, int &total) {
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int x = v;
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[w] = x;
    __syncthreads();
    if (w == 0) {
        int nw = blockDim.x >> 5;
        int s = lane < nw ? s_warp[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < nw) s_warp[lane] = s;
    }
    __syncthreads();
    int warp_prefix = w ? s_warp[w - 1] : 0;
    total = s_warp[(blockDim.x >> 5) - 1];
    __syncthreads();
    return warp_prefix + x - v;
}

constexpr int kPer = kChunk / kBlock;  // 16 primitives per thread, contiguous

__global__ void __launch_bounds__(kBlock) k_count_large(const Task *tasks, const Decision *dec, const int *chunk_task,
                                                        const int *chunk_begin, const int *idx, const float4 *plo,
                                                        const float4 *phi, int *chunk_left) {
    __shared__ int s_warp[32];
    int c = blockIdx.x;
    int ti = chunk_task[c];
    const Task &t = tasks[ti];
    const Decision &d = dec[ti];
    int begin = chunk_begin[c];
    int end = min(begin + kChunk, t.start + t.count);
    int mine = 0;
    int i0 = begin + threadIdx.x * kPer;
    for (int k = 0; k < kPer; ++k) {
        int i = i0 + k;
        if (i < end && goes_left(d, t, i, plo, phi, idx[i])) ++mine;
    }
    int total;
    block_exclusive_scan(mine, s_warp, total);
    if (threadIdx.x == 0) chunk_left[c] = total;
}

__global__ void __launch_bounds__(kBlock) k_scatter_large(const Task *tasks, const Decision *dec,
                                                          const int *chunk_task, const int *chunk_begin,
                                                          const int *chunk_left_off, const int *idx,
                                                          const float4 *plo, const float4 *phi, int *tmp) {
    __shared__ int s_warp[32];
    int c = blockIdx.x;
    int ti = chunk_task[c];
    const Task &t = tasks[ti];
    const Decision &d = dec[ti];
    int begin = chunk_begin[c];
    int end = min(begin + kChunk, t.start + t.count);
    int i0 = begin + threadIdx.x * kPer;
    int flags = 0, mine = 0;
    for (int k = 0; k < kPer; ++k) {
        int i = i0 + k;
        if (i < end && goes_left(d, t, i, plo, phi, idx[i])) {
            flags |= 1 << k;
            ++mine;
        }
    }
    int total;
    int loff = block_exclusive_scan(mine, s_warp, total);
    int chunk_l = chunk_left_off[c];
    int chunk_r = (begin - t.start) - chunk_l;  // right elements in earlier chunks
    int thread_first = i0 - begin;
    int l = t.start + chunk_l + loff;
    int r = t.start + d.nleft + chunk_r + (thread_first - loff);
    for (int k = 0; k < kPer; ++k) {
        int i = i0 + k;
        if (i >= end) break;
        int p = idx[i];
        if (flags & (1 << k))
            tmp[l++] = p;
        else
            tmp[r++] = p;
    }
}

__global__ void k_copy_range(const int *chunk_task, const int *chunk_begin, const Task *tasks, const int *tmp,
                             int *idx) {
    int c = blockIdx.x;
    const Task &t = tasks[chunk_task[c]];
    int begin = chunk_begin[c];
    int end = min(begin + kChunk, t.start + t.count);
    for (int i = begin + threadIdx.x; i < end; i += blockDim.x) idx[i] = tmp[i];
}

// ---------------------------------------------------------------------------
// Small phase: one block per task, depth-first in shared memory.
// ---------------------------------------------------------------------------
struct SmallShared {
    Task stack[72];
    Task cur;
    Bins bins;
    float axis_cost[3];
    int axis_split[3];
    int sp;
    int mode, axis, split, nleft;
    int red[2][12];
    int s_warp[32];
    int lbase, rbase;
    int tmp[kSmallTask];
};

__global__ void __launch_bounds__(kBlock) k_small(const Task *tasks, int *idx, const float4 *plo, const float4 *phi,
                                                  float4 *nodes, int *node_counter, int *max_depth, int *error_flag,
                                                  SahParams sah) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SmallShared &S = *reinterpret_cast<SmallShared *>(smem_raw);
    const int tid = threadIdx.x;
    if (tid == 0) {
        S.stack[0] = tasks[blockIdx.x];
        S.sp = 1;
    }
    __syncthreads();
    while (true) {
        if (tid == 0) {
            if (S.sp == 0)
                S.cur.count = -1;
            else
                S.cur = S.stack[--S.sp];
        }
        __syncthreads();
        const Task t = S.cur;
        if (t.count < 0) break;
        bool can_bin = t.count > 1 && t.depth < kMedianDepth;
        if (can_bin) {
            bins_clear(S.bins, tid, blockDim.x);
            __syncthreads();
            float sc[3] = {bin_scale(t.clo[0], t.chi[0]), bin_scale(t.clo[1], t.chi[1]),
                           bin_scale(t.clo[2], t.chi[2])};
            for (int e = tid; e < t.count; e += blockDim.x) {
                float lo[3], hi[3], c[3];
                load_prim(plo, phi, idx[t.start + e], lo, hi, c);
                bins_add(S.bins, lo, hi, c, t.clo, sc);
            }
            __syncthreads();
            if (tid < 3) eval_axis(S.bins, tid, S.axis_cost[tid], S.axis_split[tid]);
            __syncthreads();
        }
        if (tid == 0) {
            int axis = -1, split = -1;
            float best = INFINITY;
            if (can_bin) {
                for (int a = 0; a < 3; ++a)
                    if (S.axis_split[a] >= 0 && S.axis_cost[a] < best) {
                        best = S.axis_cost[a];
                        axis = a;
                        split = S.axis_split[a];
                    }
            }
            int mode;
            float area = half_area(t.blo[0], t.blo[1], t.blo[2], t.bhi[0], t.bhi[1], t.bhi[2]);
            float leaf_cost = kCostTri * t.count;
            float split_cost = axis >= 0 ? sah.cost_trav + kCostTri * (area > 0.f ? best / area : (float)t.count)
                                         : INFINITY;
            if (t.count <= 1 || (t.count <= sah.max_leaf && leaf_cost <= split_cost))
                mode = 0;
            else if (axis >= 0)
                mode = 1;
            else if (t.count <= kMaxLeafSAH)
                mode = 0;
            else
                mode = 2;
            S.mode = mode;
            S.axis = axis;
            S.split = split;
            S.nleft = mode == 1 ? 0 : t.count / 2;
            if (mode == 1)
                for (int i = 0; i <= split; ++i) S.nleft += S.bins.cnt[axis][i];
            S.lbase = 0;
            S.rbase = 0;
            if (mode == 0) write_link(nodes, t.link_slot, leaf_link(t.start, t.count));
            if (mode == 2)
                for (int k = 0; k < 12; ++k) {
                    S.red[0][k] = (k % 6) < 3 ? INT_MAX : INT_MIN;
                    S.red[1][k] = (k % 6) < 3 ? INT_MAX : INT_MIN;
                }
        }
        __syncthreads();
        const int mode = S.mode;
        if (mode == 0) continue;  // leaf written; pop next (loop top syncs)
        if (mode == 1) {
            // Stable partition through shared tmp, 256 elements per round.
            const int axis = S.axis, split = S.split, nleft = S.nleft;
            float sc = bin_scale(t.clo[axis], t.chi[axis]);
            for (int base = 0; base < t.count; base += blockDim.x) {
                int e = base + tid;
                int p = 0;
                bool left = false;
                bool valid = e < t.count;
                if (valid) {
                    p = idx[t.start + e];
                    float lo[3], hi[3], c[3];
                    load_prim(plo, phi, p, lo, hi, c);
                    left = bin_of(c[axis], t.clo[axis], sc) <= split;
                }
                int total;
                int lrank = block_exclusive_scan(left ? 1 : 0, S.s_warp, total);
                if (valid) {
                    int pos = left ? S.lbase + lrank : nleft + S.rbase + (e - base) - lrank;
                    if (pos >= 0 && pos < t.count) S.tmp[pos] = p;
                }
                int nvalid = min((int)blockDim.x, t.count - base);
                __syncthreads();
                if (tid == 0) {
                    S.lbase += total;
                    S.rbase += nvalid - total;
                }
                __syncthreads();
            }
            if (tid == 0 && S.lbase != nleft) atomicExch(error_flag, 1);
            __syncthreads();
            if (*(volatile int *)error_flag == 0)
                for (int e = tid; e < t.count; e += blockDim.x) idx[t.start + e] = S.tmp[e];
        } else {
            // Index median: exact bounds of both halves.
            const int nleft = S.nleft;
            for (int e = tid; e < t.count; e += blockDim.x) {
                float lo[3], hi[3], c[3];
                load_prim(plo, phi, idx[t.start + e], lo, hi, c);
                int side = e < nleft ? 0 : 1;
                for (int k = 0; k < 3; ++k) {
                    atomicMin(&S.red[side][k], f2key(lo[k]));
                    atomicMax(&S.red[side][3 + k], f2key(hi[k]));
                    atomicMin(&S.red[side][6 + k], f2key(c[k]));
                    atomicMax(&S.red[side][9 + k], f2key(c[k]));
                }
            }
        }
        __syncthreads();
        if (tid == 0) {
            Task l, r;
            if (mode == 1) {
                child_from_bins(S.bins, S.axis, S.split, false, l);
                child_from_bins(S.bins, S.axis, S.split, true, r);
            } else {
                l.count = S.nleft;
                r.count = t.count - S.nleft;
                Task *ch[2] = {&l, &r};
                for (int s = 0; s < 2; ++s)
                    for (int k = 0; k < 3; ++k) {
                        ch[s]->blo[k] = key2f(S.red[s][k]);
                        ch[s]->bhi[k] = key2f(S.red[s][3 + k]);
                        ch[s]->clo[k] = key2f(S.red[s][6 + k]);
                        ch[s]->chi[k] = key2f(S.red[s][9 + k]);
                    }
            }
            int id = atomicAdd(node_counter, 1);
            write_link(nodes, t.link_slot, id);
            l.start = t.start;
            r.start = t.start + l.count;
            l.depth = r.depth = t.depth + 1;
            l.link_slot = id * 16 + 12;
            r.link_slot = id * 16 + 13;
            write_node(nodes, id, l, r);
            atomicMax(max_depth, t.depth + 1);
            S.stack[S.sp++] = r;
            S.stack[S.sp++] = l;
        }
        __syncthreads();
    }
}

__global__ void k_gather_tris(const float *verts, const int *idx, int n, float4 *tris) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        int p = idx[s];
        const float *v = verts + 9 * (size_t)p;
        tris[3 * (size_t)s + 0] = make_float4(v[0], v[1], v[2], __int_as_float(p));
        tris[3 * (size_t)s + 1] = make_float4(v[3], v[4], v[5], 0.f);
        tris[3 * (size_t)s + 2] = make_float4(v[6], v[7], v[8], 0.f);
    }
}

__global__ void k_prim_slot(const int *idx, int n, int *slot_of_prim) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) slot_of_prim[idx[s]] = s;
}

// Single-leaf tree for tiny scenes (n <= kMaxLeafSAH): root with the whole
// soup in child 0 and an empty leaf in child 1.
__global__ void k_tiny_root(float4 *nodes, const int *root_keys, int n) {
    float lo[3], hi[3];
    for (int k = 0; k < 3; ++k) {
        lo[k] = key2f(root_keys[k]);
        hi[k] = key2f(root_keys[3 + k]);
    }
    nodes[0] = make_float4(lo[0], hi[0], lo[1], hi[1]);
    nodes[1] = make_float4(lo[0], hi[0], lo[1], hi[1]);
    nodes[2] = make_float4(lo[2], hi[2], lo[2], hi[2]);
    nodes[3] = make_float4(__int_as_float(leaf_link(0, n)), __int_as_float(leaf_link(0, 0)), 0.f, 0.f);
}

template <class T>
struct DevBuf {
    T *p = nullptr;
    explicit DevBuf(size_t n) {
        if (n) CRT_CUDA(cudaMalloc(&p, n * sizeof(T)));
    }
    ~DevBuf() {
        if (p) cudaFree(p);
    }
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
};

}  // namespace

void build_bvh(const float *d_verts, int n, cudaStream_t stream, BvhBuffers &out) {
    CRT_CHECK(n > 0, CRT_ERR_INVALID, "scene has no triangles");
    CRT_CHECK(n < (1 << 27) - 1, CRT_ERR_CAPACITY, "more than 2^27-2 triangles");
    cudaEvent_t e0, e1;
    CRT_CUDA(cudaEventCreate(&e0));
    CRT_CUDA(cudaEventCreate(&e1));
    CRT_CUDA(cudaEventRecord(e0, stream));

    DevBuf<float4> plo(n), phi(n);
    DevBuf<int> idx(n), tmp(n), root_keys(12), counters(3);
    int max_nodes = std::max(1, n - 1);
    CRT_CUDA(cudaMalloc(&out.nodes, (size_t)max_nodes * 4 * sizeof(float4)));
    CRT_CUDA(cudaMalloc(&out.tris, (size_t)n * 3 * sizeof(float4)));
    CRT_CUDA(cudaMalloc(&out.slot_of_prim, (size_t)n * sizeof(int)));

    int init_keys[12];
    for (int k = 0; k < 12; ++k) init_keys[k] = (k % 6) < 3 ? INT_MAX : INT_MIN;
    CRT_CUDA(cudaMemcpyAsync(root_keys.p, init_keys, sizeof(init_keys), cudaMemcpyHostToDevice, stream));
    CRT_CUDA(cudaMemsetAsync(counters.p, 0, 3 * sizeof(int), stream));
    int grid = std::min((n + kBlock - 1) / kBlock, 148 * 8);
    k_prim_bounds<<<grid, kBlock, 0, stream>>>(d_verts, n, plo.p, phi.p, idx.p, root_keys.p);
    CRT_CUDA(cudaGetLastError());
    int keys[12];
    CRT_CUDA(cudaMemcpyAsync(keys, root_keys.p, sizeof(keys), cudaMemcpyDeviceToHost, stream));
    CRT_CUDA(cudaStreamSynchronize(stream));
    for (int k = 0; k < 3; ++k) {
        out.bounds_min[k] = key2f(keys[k]);
        out.bounds_max[k] = key2f(keys[3 + k]);
    }
    out.depth = 1;

    if (n <= kMaxLeafSAH) {
        k_tiny_root<<<1, 1, 0, stream>>>(out.nodes, root_keys.p, n);
        CRT_CUDA(cudaGetLastError());
        out.num_nodes = 1;
    } else {
        Task root;
        root.start = 0;
        root.count = n;
        root.link_slot = -1;
        root.depth = 0;
        for (int k = 0; k < 3; ++k) {
            root.blo[k] = key2f(keys[k]);
            root.bhi[k] = key2f(keys[3 + k]);
            root.clo[k] = key2f(keys[6 + k]);
            root.chi[k] = key2f(keys[9 + k]);
        }
        std::vector<Task> large, small;
        (root.count > kSmallTask ? large : small).push_back(root);
        int max_depth_host = 0;
        while (!large.empty()) {
            int nt = (int)large.size();
            std::vector<int> ctask, cbegin;
            for (int i = 0; i < nt; ++i)
                for (int b = large[i].start; b < large[i].start + large[i].count; b += kChunk) {
                    ctask.push_back(i);
                    cbegin.push_back(b);
                }
            int nc = (int)ctask.size();
            DevBuf<Task> d_tasks(nt);
            DevBuf<Bins> d_bins(nt);
            DevBuf<Decision> d_dec(nt);
            DevBuf<int> d_ctask(nc), d_cbegin(nc), d_cleft(nc), d_cloff(nc);
            CRT_CUDA(cudaMemcpyAsync(d_tasks.p, large.data(), nt * sizeof(Task), cudaMemcpyHostToDevice, stream));
            CRT_CUDA(cudaMemcpyAsync(d_ctask.p, ctask.data(), nc * sizeof(int), cudaMemcpyHostToDevice, stream));
            CRT_CUDA(cudaMemcpyAsync(d_cbegin.p, cbegin.data(), nc * sizeof(int), cudaMemcpyHostToDevice, stream));
            k_bins_init<<<std::min(nt * 8, 1024), 256, 0, stream>>>(d_bins.p, nt);
            k_bin_large<<<nc, kBlock, 0, stream>>>(d_tasks.p, d_ctask.p, d_cbegin.p, idx.p, plo.p, phi.p, d_bins.p);
            k_split_large<<<(nt + 127) / 128, 128, 0, stream>>>(d_tasks.p, nt, d_bins.p, out.nodes, counters.p,
                                                                 d_dec.p);
            k_count_large<<<nc, kBlock, 0, stream>>>(d_tasks.p, d_dec.p, d_ctask.p, d_cbegin.p, idx.p, plo.p, phi.p,
                                                    d_cleft.p);
            CRT_CUDA(cudaGetLastError());
            std::vector<Decision> dec(nt);
            std::vector<int> cleft(nc), cloff(nc);
            CRT_CUDA(cudaMemcpyAsync(dec.data(), d_dec.p, nt * sizeof(Decision), cudaMemcpyDeviceToHost, stream));
            CRT_CUDA(cudaMemcpyAsync(cleft.data(), d_cleft.p, nc * sizeof(int), cudaMemcpyDeviceToHost, stream));
            CRT_CUDA(cudaStreamSynchronize(stream));
            int run = 0;
            for (int c = 0; c < nc; ++c) {
                if (c == 0 || ctask[c] != ctask[c - 1]) run = 0;
                cloff[c] = run;
                run += cleft[c];
                if (c == nc - 1 || ctask[c + 1] != ctask[c])
                    CRT_CHECK(run == dec[ctask[c]].nleft, CRT_ERR_CUDA,
                              "BVH build: partition count disagrees with the SAH bins");
            }
            CRT_CUDA(cudaMemcpyAsync(d_cloff.p, cloff.data(), nc * sizeof(int), cudaMemcpyHostToDevice, stream));
            k_scatter_large<<<nc, kBlock, 0, stream>>>(d_tasks.p, d_dec.p, d_ctask.p, d_cbegin.p, d_cloff.p, idx.p,
                                                      plo.p, phi.p, tmp.p);
            k_copy_range<<<nc, kBlock, 0, stream>>>(d_ctask.p, d_cbegin.p, d_tasks.p, tmp.p, idx.p);
            CRT_CUDA(cudaGetLastError());
            CRT_CUDA(cudaStreamSynchronize(stream));
            std::vector<Task> next;
            for (int i = 0; i < nt; ++i)
                for (int s = 0; s < 2; ++s) {
                    const Task &c = dec[i].child[s];
                    max_depth_host = std::max(max_depth_host, c.depth);
                    (c.count > kSmallTask ? next : small).push_back(c);
                }
            large.swap(next);
        }
        CRT_CUDA(cudaMemcpyAsync(counters.p + 1, &max_depth_host, sizeof(int), cudaMemcpyHostToDevice, stream));
        if (!small.empty()) {
            DevBuf<Task> d_small(small.size());
            CRT_CUDA(cudaMemcpyAsync(d_small.p, small.data(), small.size() * sizeof(Task), cudaMemcpyHostToDevice,
                                     stream));
            size_t smem = sizeof(SmallShared);
            CRT_CUDA(cudaFuncSetAttribute(k_small, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            k_small<<<(int)small.size(), kBlock, smem, stream>>>(d_small.p, idx.p, plo.p, phi.p, out.nodes,
                                                                counters.p, counters.p + 1, counters.p + 2,
                                                                sah_params());
            CRT_CUDA(cudaGetLastError());
            CRT_CUDA(cudaStreamSynchronize(stream));
        }
        int cnt[3];
        CRT_CUDA(cudaMemcpyAsync(cnt, counters.p, sizeof(cnt), cudaMemcpyDeviceToHost, stream));
        CRT_CUDA(cudaStreamSynchronize(stream));
        CRT_CHECK(cnt[2] == 0, CRT_ERR_CUDA, "BVH build: partition count disagrees with the SAH bins");
        CRT_CHECK(cnt[0] <= max_nodes && cnt[1] < kStackSize - 2, CRT_ERR_CAPACITY, "BVH build: node or depth bound");
        out.num_nodes = cnt[0];
        out.depth = cnt[1];
    }
    k_gather_tris<<<grid, kBlock, 0, stream>>>(d_verts, idx.p, n, out.tris);
    k_prim_slot<<<grid, kBlock, 0, stream>>>(idx.p, n, out.slot_of_prim);
    CRT_CUDA(cudaGetLastError());
    CRT_CUDA(cudaEventRecord(e1, stream));
    CRT_CUDA(cudaEventSynchronize(e1));
    CRT_CUDA(cudaEventElapsedTime(&out.build_ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    out.num_tris = n;
    // the 16-bit quantised copy of the nodes (bvh16.cuh), one kernel
    build_bvh16(out, out.err, stream);
    CRT_CUDA(cudaStreamSynchronize(stream));
    // The 8-wide quantised tree is built only on request (CRT_BVH8=1): its
    // traversal measured slower than the binary one on the icosphere field.
    const char *w8 = getenv("CRT_BVH8");
    if (w8 && w8[0] == '1') {
        const auto w0 = std::chrono::steady_clock::now();
        build_bvh8(out, stream);
        out.wide_build_ms = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - w0).count();
    }
}

void free_bvh(BvhBuffers &b) {
    if (b.nodes) cudaFree(b.nodes);
    if (b.tris) cudaFree(b.tris);
    if (b.slot_of_prim) cudaFree(b.slot_of_prim);
    if (b.wnodes) cudaFree(b.wnodes);
    if (b.wlinks) cudaFree(b.wlinks);
    if (b.cnodes) cudaFree(b.cnodes);
    b = BvhBuffers();
}

}  // namespace crt
