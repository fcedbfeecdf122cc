// Standalone extend (closest-hit) and shadow (Light::Visible) kernels over
// ray batches in HBM.
//
// Extend replaces IntersectionKernel's traversal (Src/Core/renderer.cuh:132
// -> TraceRay :124 -> BVH::IsIntersect Src/Core/bvh.cu:253): one ray per
// thread, 32 B in (two float4 loads), 16 B out (one float4 store), node
// boxes and triangles through the read-only path.
#include "trace.cuh"

namespace crt {

constexpr int kTraceBlock = 128;

__global__ void __launch_bounds__(kTraceBlock) k_trace_closest(BvhView bvh, const float4 *__restrict__ rays,
                                                               int64_t n, float4 *__restrict__ hits) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        float4 r0 = __ldg(rays + 2 * i), r1 = __ldg(rays + 2 * i + 1);
        Hit h = closest_hit<false>(bvh, v3(r0.x, r0.y, r0.z), v3(r1.x, r1.y, r1.z), r0.w, r1.w);
        int prim = h.slot >= 0 ? tri_prim(bvh, h.slot) : -1;
        hits[i] = make_float4(h.t, __int_as_float(prim), h.b1, h.b2);
    }
}

__global__ void __launch_bounds__(kTraceBlock) k_trace_shadow(BvhView bvh, const float4 *__restrict__ q, int64_t n,
                                                              uint8_t *__restrict__ occ) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        float4 a = __ldg(q + 3 * i), b = __ldg(q + 3 * i + 1), c = __ldg(q + 3 * i + 2);
        bool vis = visible(bvh, v3(a.x, a.y, a.z), v3(a.w, b.x, b.y), v3(b.z, b.w, c.x), v3(c.y, c.z, c.w));
        occ[i] = vis ? 0 : 1;
    }
}

static int trace_grid(int64_t n) {
    int64_t blocks = (n + kTraceBlock - 1) / kTraceBlock;
    const int64_t cap = 148LL * 16 * 64;  // grid-stride beyond this
    return (int)(blocks < cap ? (blocks > 0 ? blocks : 1) : cap);
}

void launch_trace_closest(const BvhView &bvh, const float4 *d_rays, int64_t n, float4 *d_hits, cudaStream_t s) {
    if (n <= 0) return;
    k_trace_closest<<<trace_grid(n), kTraceBlock, 0, s>>>(bvh, d_rays, n, d_hits);
    CRT_CUDA(cudaGetLastError());
}

void launch_trace_shadow(const BvhView &bvh, const float *d_q, int64_t n, uint8_t *d_occ, cudaStream_t s) {
    if (n <= 0) return;
    k_trace_shadow<<<trace_grid(n), kTraceBlock, 0, s>>>(bvh, reinterpret_cast<const float4 *>(d_q), n, d_occ);
    CRT_CUDA(cudaGetLastError());
}

}  // namespace crt
