/*
 * Oracle: CPU restatement of DarrenChen-CN/CudaRayTracer's render-path
 * arithmetic, written from the reference's behaviour. Test infrastructure
 * only -- the CUDA kernels are checked against it; nothing in the product
 * path calls it. Built with -ffp-contract=off so every float operation
 * rounds once, in the order of the reference's Eigen expressions:
 *   dot(a,b)   = a0*b0 + (a1*b1 + a2*b2)
 *   cross(a,b) = (a1*b2 - a2*b1, a2*b0 - a0*b2, a0*b1 - a1*b0)
 * Its results are pinned against the reference's own host-compiled code
 * (oracle/_ref) by tests/test_oracle_pin.py.
 */
#include "crt_oracle.h"
#include <math.h>
#include <string.h>
#include <float.h>
#include "par.h"

typedef struct { float x, y, z; } v3;

static inline v3 mk(float x, float y, float z) { v3 r = {x, y, z}; return r; }
static inline v3 sub(v3 a, v3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 add(v3 a, v3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 scale(v3 a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
static inline float dot(v3 a, v3 b) { return a.x * b.x + (a.y * b.y + a.z * b.z); }
static inline v3 cross(v3 a, v3 b) {
    return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline float norm(v3 a) { return sqrtf(dot(a, a)); }
static inline v3 normalized(v3 a) {
    float z = dot(a, a);
    if (z > 0.f) {
        float s = sqrtf(z);
        return mk(a.x / s, a.y / s, a.z / s);
    }
    return a;
}
static inline v3 ld3(const float *p) { return mk(p[0], p[1], p[2]); }


/* Triangle::IsIntersect (Src/Core/triangle.cu:100-133) with tMin = 0,
 * tMax = 1e8 (the defaults BVH traversal passes, Src/Core/bvh.cu:271).
 * det is a float dot product; the reference divides 1.f by it in double and
 * rounds to float, which equals the correctly rounded float reciprocal. */
int oracle_tri_isect(const float *v, const float *o_, const float *d_, float closest, float *t_out, float *b1_out,
                     float *b2_out) {
    v3 v0 = ld3(v), v1 = ld3(v + 3), v2 = ld3(v + 6), o = ld3(o_), d = ld3(d_);
    v3 e1 = sub(v1, v0), e2 = sub(v2, v0), s = sub(o, v0);
    v3 s1 = cross(d, e2), s2 = cross(s, e1);
    float det = dot(e1, s1);
    if (det == 0.f || det < 0.f) return 0;
    float inv = (float)(1.0 / (double)det);
    float t = inv * dot(s2, e2);
    if (t >= closest) return 0;
    float b1 = inv * dot(s1, s);
    if (b1 < 0.f || b1 > 1.f) return 0;
    float b2 = inv * dot(s2, d);
    if (b2 < 0.f || b1 + b2 > 1.f) return 0;
    if (t < 0.f || t > 1e8f) return 0;
    *t_out = t;
    *b1_out = b1;
    *b2_out = b2;
    return 1;
}

/* Closest hit by testing every triangle in index order: the minimum-t
 * triangle, ties resolved to the lowest index (first visited). The box tMin
 * of BVH::IsIntersect (Src/Core/bvh.cu:283-284) only prunes boxes and has no
 * brute-force counterpart; closest starts at tMax (:263). */
int oracle_closest_brute(const float *verts, long ntris, const float *o_, const float *d_, float tmax, float *t,
                         float *b1, float *b2) {
    v3 o = ld3(o_), d = ld3(d_);
    int prim = -1;
    float best = tmax, tb1 = 0.f, tb2 = 0.f;
    float oo[3] = {o.x, o.y, o.z}, dd[3] = {d.x, d.y, d.z};
    for (long k = 0; k < ntris; ++k) {
        float tt, u, w;
        if (oracle_tri_isect(verts + 9 * k, oo, dd, best, &tt, &u, &w)) {
            best = tt;
            prim = (int)k;
            tb1 = u;
            tb2 = w;
        }
    }
    *t = best;
    *b1 = tb1;
    *b2 = tb2;
    return prim;
}

typedef struct {
    const float *verts;
    long ntris;
    const float *in;
    float *out;
    double *out_t;
    int32_t *out_prim;
    uint8_t *out_u8;
} job_ctx;

static void trace_brute_body(long i, void *c_) {
    job_ctx *c = (job_ctx *)c_;
    const float *r = c->in + 8 * i;
    float t, b1, b2;
    int prim = oracle_closest_brute(c->verts, c->ntris, r, r + 4, r[7], &t, &b1, &b2);
    float *o = c->out + 4 * i;
    o[0] = t;
    memcpy(&o[1], &prim, 4);
    o[2] = prim >= 0 ? b1 : 0.f;
    o[3] = prim >= 0 ? b2 : 0.f;
}

void oracle_trace_brute(const float *verts, long ntris, const float *rays, long n, float *out, int nthreads) {
    job_ctx c = {verts, ntris, rays, out, 0, 0, 0};
    par_for(n, 64, nthreads, trace_brute_body, &c);
}

/* The same acceptance predicate evaluated in double precision: culling on
 * det <= 0, barycentrics in [0,1] with b1 + b2 <= 1, 0 <= t <= 1e8, strict
 * t < closest. Adjudicates float disagreements and near-ties. */
static void trace_fp64_body(long i, void *c_) {
    job_ctx *c = (job_ctx *)c_;
    const float *verts = c->verts;
    long ntris = c->ntris;
    {
        const float *r = c->in + 8 * i;
        double o[3] = {r[0], r[1], r[2]}, d[3] = {r[4], r[5], r[6]};
        double best = r[7];
        int prim = -1;
        for (long k = 0; k < ntris; ++k) {
            const float *v = verts + 9 * k;
            double e1[3], e2[3], s[3], s1[3], s2[3];
            for (int q = 0; q < 3; ++q) {
                e1[q] = (double)v[3 + q] - v[q];
                e2[q] = (double)v[6 + q] - v[q];
                s[q] = o[q] - v[q];
            }
            s1[0] = d[1] * e2[2] - d[2] * e2[1];
            s1[1] = d[2] * e2[0] - d[0] * e2[2];
            s1[2] = d[0] * e2[1] - d[1] * e2[0];
            s2[0] = s[1] * e1[2] - s[2] * e1[1];
            s2[1] = s[2] * e1[0] - s[0] * e1[2];
            s2[2] = s[0] * e1[1] - s[1] * e1[0];
            double det = e1[0] * s1[0] + e1[1] * s1[1] + e1[2] * s1[2];
            if (!(det > 0.0)) continue;
            double t = (s2[0] * e2[0] + s2[1] * e2[1] + s2[2] * e2[2]) / det;
            if (t >= best) continue;
            double b1 = (s1[0] * s[0] + s1[1] * s[1] + s1[2] * s[2]) / det;
            if (b1 < 0.0 || b1 > 1.0) continue;
            double b2 = (s2[0] * d[0] + s2[1] * d[1] + s2[2] * d[2]) / det;
            if (b2 < 0.0 || b1 + b2 > 1.0) continue;
            if (t < 0.0 || t > 1e8) continue;
            best = t;
            prim = (int)k;
        }
        c->out_t[i] = best;
        c->out_prim[i] = prim;
    }
}

void oracle_trace_fp64(const float *verts, long ntris, const float *rays, long n, double *out_t, int32_t *out_prim,
                       int nthreads) {
    job_ctx c = {verts, ntris, rays, 0, out_t, out_prim, 0};
    par_for(n, 64, nthreads, trace_fp64_body, &c);
}

/* Light::Visible (Src/Core/light.cu:5-27): offset both endpoints 1e-4 along
 * their normals, cast from the light point toward the shading point starting
 * 1e-2 along the ray; occluded iff the closest hit is more than 0.1 from the
 * shading point and its light distance differs from the sample distance by
 * more than 0.1 (float distances compared with the double 0.1). */
int oracle_visible_one(const float *verts, long ntris, const float *a) {
    v3 h = add(ld3(a), scale(ld3(a + 3), 1e-4f));
    v3 l = add(ld3(a + 6), scale(ld3(a + 9), 1e-4f));
    v3 diff = sub(h, l);
    float sd = norm(diff);
    v3 dir = normalized(diff);
    v3 o = add(l, scale(dir, 1e-2f));
    float t, b1, b2;
    float oo[3] = {o.x, o.y, o.z}, dd[3] = {dir.x, dir.y, dir.z};
    int prim = oracle_closest_brute(verts, ntris, oo, dd, 1e8f, &t, &b1, &b2);
    if (prim < 0) return 1;
    const float *v = verts + 9 * prim;
    float b0 = (1.f - b1) - b2;
    v3 p = add(add(scale(ld3(v), b0), scale(ld3(v + 3), b1)), scale(ld3(v + 6), b2));
    float td = norm(sub(p, l));
    if ((double)norm(sub(h, p)) > 1e-1 && (double)fabsf(td - sd) > 1e-1) return 0;
    return 1;
}

static void visible_body(long i, void *c_) {
    job_ctx *c = (job_ctx *)c_;
    c->out_u8[i] = oracle_visible_one(c->verts, c->ntris, c->in + 12 * i) ? 0 : 1;
}

void oracle_visible(const float *verts, long ntris, const float *q, long n, uint8_t *occluded, int nthreads) {
    job_ctx c = {verts, ntris, q, 0, 0, 0, occluded};
    par_for(n, 64, nthreads, visible_body, &c);
}
