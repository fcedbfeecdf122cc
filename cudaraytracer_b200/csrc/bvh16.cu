// Compression of the binary BVH's float child boxes into the 16-bit grid
// of bvh16.cuh, on the device, one thread per node.
#include "bvh16.cuh"
#include "bvh_build.h"
#include <cmath>
#include <cstring>

namespace crt {
namespace {

constexpr int kQMax = 65535;

inline float u2f_host(unsigned u) {
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}

__host__ __device__ __forceinline__ float qdecode(int q, float s, float p) {
    return fmaf(8388608.0f + (float)q, s, p);
}

// Largest q in [0, kQMax] with decode(q) <= v (decode(0) <= the grid origin
// <= v by construction), or smallest q with decode(q) >= v. A guess from
// the linear map is refined by a few steps; should that not settle, the
// grid ends are conservative by construction.
__device__ __forceinline__ unsigned quantise(float v, bool upper, float s, float p, float L) {
    int q = (int)floorf((v - L) / s);
    q = max(0, min(q, kQMax));
    if (!upper) {
        for (int k = 0; k < 4 && q > 0 && qdecode(q, s, p) > v; ++k) --q;
        for (int k = 0; k < 4 && q < kQMax && qdecode(q + 1, s, p) <= v; ++k) ++q;
        if (qdecode(q, s, p) > v) q = 0;
    } else {
        ++q;
        q = min(q, kQMax);
        for (int k = 0; k < 4 && q < kQMax && qdecode(q, s, p) < v; ++k) ++q;
        for (int k = 0; k < 4 && q > 0 && qdecode(q - 1, s, p) >= v; ++k) --q;
        if (qdecode(q, s, p) < v) q = kQMax;
    }
    return (unsigned)q;
}

__global__ void k_compress_nodes(const float4 *nodes, int64_t n, QuantGrid g, float L0, float L1, float L2,
                                 float4 *out, int *err) {
    const float Lx[3] = {L0, L1, L2};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float4 a = nodes[4 * i], b = nodes[4 * i + 1], c = nodes[4 * i + 2], d = nodes[4 * i + 3];
        // child c, component j (lo x y z, hi x y z) -> index 6c + j
        const float v[12] = {a.x, a.z, c.x, a.y, a.w, c.y, b.x, b.z, c.z, b.y, b.w, c.w};
        unsigned q[12];
        bool ok = true;
#pragma unroll
        for (int k = 0; k < 12; ++k) {
            const int ax = k % 3;
            const bool upper = (k % 6) >= 3;
            q[k] = quantise(v[k], upper, g.s[ax], g.p[ax], Lx[ax]);
            const float dv = qdecode((int)q[k], g.s[ax], g.p[ax]);
            ok = ok && (upper ? dv >= v[k] : dv <= v[k]);
        }
        if (!ok && err) atomicOr(err, kErrTraversalBounds);
        unsigned w[8];
#pragma unroll
        for (int k = 0; k < 6; ++k) w[k] = q[2 * k] | (q[2 * k + 1] << 16);
        w[6] = __float_as_uint(d.x);
        w[7] = __float_as_uint(d.y);
        out[2 * i] = make_float4(__uint_as_float(w[0]), __uint_as_float(w[1]), __uint_as_float(w[2]),
                                 __uint_as_float(w[3]));
        out[2 * i + 1] = make_float4(__uint_as_float(w[4]), __uint_as_float(w[5]), __uint_as_float(w[6]),
                                     __uint_as_float(w[7]));
    }
}

}  // namespace

QuantGrid quant_grid(const float lo[3], const float hi[3]) {
    QuantGrid g;
    for (int a = 0; a < 3; ++a) {
        const float L = lo[a], H = hi[a];
        CRT_CHECK(std::isfinite(L) && std::isfinite(H) && H >= L, CRT_ERR_INVALID, "BVH grid: bad scene bounds");
        const double ext = (double)H - (double)L;
        int e = ext > 0.0 ? (int)std::ceil(std::log2(ext / 65000.0)) : -126;
        e = std::max(-126, std::min(e, 100));
        for (;; ++e) {
            CRT_CHECK(e <= 100, CRT_ERR_INVALID, "BVH grid: cannot cover the scene bounds");
            const float s = u2f_host((unsigned)(e + 127) << 23);
            float p = L - 8388608.0f * s;
            while (qdecode(0, s, p) > L) p = std::nextafter(p, -INFINITY);
            if (qdecode(kQMax, s, p) >= H) {
                g.s[a] = s;
                g.p[a] = p;
                break;
            }
        }
    }
    return g;
}

void build_bvh16(BvhBuffers &b, int *err, cudaStream_t stream) {
    b.grid = quant_grid(b.bounds_min, b.bounds_max);
    CRT_CUDA(cudaMalloc(&b.cnodes, (size_t)b.num_nodes * 2 * sizeof(float4)));
    const int grid = (int)std::min<int64_t>((b.num_nodes + 255) / 256, 148 * 8);
    k_compress_nodes<<<std::max(grid, 1), 256, 0, stream>>>(b.nodes, b.num_nodes, b.grid, b.bounds_min[0],
                                                            b.bounds_min[1], b.bounds_min[2], b.cnodes, err);
    CRT_CUDA(cudaGetLastError());
}

}  // namespace crt
