// Ray-query device functions shared by the standalone trace kernels and the
// wavefront shade stage.
#pragma once
#include "bvh.cuh"
#include "bvh8.cuh"

namespace crt {

#ifdef __CUDACC__

// Hit point of a closest-hit record: b0*v0 + b1*v1 + b2*v2 with
// b0 = 1 - b1 - b2, evaluated in the reference's order
// (Src/Core/triangle.cu:121-127).
__device__ __forceinline__ V3 hit_point(const BvhView &bvh, const Hit &h) {
    const float4 *tp = bvh.tris + 3 * (size_t)h.slot;
    float4 a = __ldg(tp + 0), b = __ldg(tp + 1), c = __ldg(tp + 2);
    float b0 = rsub(rsub(1.f, h.b1), h.b2);
    return V3{radd(radd(rmul(b0, a.x), rmul(h.b1, b.x)), rmul(h.b2, c.x)),
              radd(radd(rmul(b0, a.y), rmul(h.b1, b.y)), rmul(h.b2, c.y)),
              radd(radd(rmul(b0, a.z), rmul(h.b1, b.z)), rmul(h.b2, c.z))};
}

// Light::Visible (Src/Core/light.cu:5-27). Both endpoints are pushed 1e-4
// along their normals; the ray runs from the light point toward the shading
// point starting 1e-2 along it, with box tMin 1e-6. The point is occluded iff
// the closest hit lies more than 0.1 from the shading point AND its distance
// to the light differs from the sample distance by more than 0.1. (The
// reference compares float distances with the double 0.1, i.e. x >= 0.1f.)
// Any accepted hit with t < t_exit already fixes the answer to "occluded"
// (the closest hit is then at least as near, hence more than 0.1 short of the
// shading point on both tests), so traversal stops there.
struct ShadowRay {
    V3 h, l, o, dir;
    float sd, t_exit;
};

__device__ __forceinline__ void shadow_ray_init(ShadowRay &r, V3 hp, V3 hn, V3 lp, V3 ln) {
    r.h = vadd(hp, vscale(hn, 1e-4f));
    r.l = vadd(lp, vscale(ln, 1e-4f));
    V3 diff = vsub(r.h, r.l);
    r.sd = vnorm(diff);
    r.dir = vnormalized(diff);
    r.o = vadd(r.l, vscale(r.dir, 1e-2f));
    r.t_exit = r.sd * 0.9999f - 0.1101f;
}

// The predicate from the closest hit of closest_hit<true>(bvh, r.o, r.dir,
// 1e-6, 1e8, r.t_exit).
__device__ __forceinline__ bool shadow_ray_visible(const ShadowRay &r, const BvhView &bvh, const Hit &hit) {
    if (hit.slot < 0) return true;
    if (hit.t < r.t_exit) return false;
    V3 thp = hit_point(bvh, hit);
    float td = vnorm(vsub(thp, r.l));
    if (vnorm(vsub(r.h, thp)) >= 0.1f && fabsf(rsub(td, r.sd)) >= 0.1f) return false;
    return true;
}

__device__ __forceinline__ bool visible(const BvhView &bvh, V3 hp, V3 hn, V3 lp, V3 ln) {
    ShadowRay r;
    shadow_ray_init(r, hp, hn, lp, ln);
    Hit hit = closest_hit<true>(bvh, r.o, r.dir, 1e-6f, 1e8f, r.t_exit);
    return shadow_ray_visible(r, bvh, hit);
}

// visible() over the 8-wide tree with a short stack (bvh8.cuh).
template <int kShort>
__device__ __forceinline__ bool visible8(const BvhView &bvh, ShortStack<kShort> &st, V3 hp, V3 hn, V3 lp, V3 ln) {
    ShadowRay r;
    shadow_ray_init(r, hp, hn, lp, ln);
    Hit hit = closest_hit8<true, kShort>(bvh, st, r.o, r.dir, 1e-6f, 1e8f, r.t_exit);
    return shadow_ray_visible(r, bvh, hit);
}

#endif

// Host launchers (trace.cu).
void launch_trace_closest(const BvhView &bvh, const float4 *d_rays, int64_t n, float4 *d_hits, cudaStream_t s);
void launch_trace_shadow(const BvhView &bvh, const float *d_q, int64_t n, uint8_t *d_occ, cudaStream_t s);

}  // namespace crt
