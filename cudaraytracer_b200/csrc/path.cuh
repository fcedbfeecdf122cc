// Per-path device code shared by the wavefront kernels (render.cu, the
// multi-view batch and the multi-scene server): SoA path-state encoding,
// pixel accumulation, warp-aggregated queue allocation and one shading step
// (PathTracing, Src/Core/renderer.cuh:170-422).
#pragma once
#include "render_kernels.cuh"

namespace crt {
// ---------------------------------------------------------------------------
// device: path state
// ---------------------------------------------------------------------------

struct PathState {
    V3 o, d, w, dc, ic;
    float pdf;
    uint32_t pixel;
    bool first, spec;
    Pcg32 rng;
};


__device__ __forceinline__ PathState load_path(const QueueView &q, int i) {
    float4 a = q.p[0][i], b = q.p[1][i], c = q.p[2][i], d = q.p[3][i], e = q.p[4][i];
    PathState s;
    s.o = V3{a.x, a.y, a.z};
    s.pdf = a.w;
    s.d = V3{b.x, b.y, b.z};
    uint32_t meta = __float_as_uint(b.w);
    s.pixel = meta & kPixelMask;
    s.first = (meta & kFirst) != 0;
    s.spec = (meta & kSpec) != 0;
    s.w = V3{c.x, c.y, c.z};
    s.dc = V3{c.w, d.x, d.y};
    s.ic = V3{d.z, d.w, e.x};
    s.rng.state = ((uint64_t)__float_as_uint(e.z) << 32) | __float_as_uint(e.y);
    s.rng.inc = ((uint64_t)s.pixel << 1) | 1u;
    return s;
}

// `tag` fills the spare word of plane 4 (the multi-scene server keeps the
// path's scene and request there; 0 elsewhere).
__device__ __forceinline__ void store_path(const QueueView &q, int i, const PathState &s, uint32_t tag = 0) {
    uint32_t meta = s.pixel | (s.first ? kFirst : 0u) | (s.spec ? kSpec : 0u);
    q.p[0][i] = make_float4(s.o.x, s.o.y, s.o.z, s.pdf);
    q.p[1][i] = make_float4(s.d.x, s.d.y, s.d.z, __uint_as_float(meta));
    q.p[2][i] = make_float4(s.w.x, s.w.y, s.w.z, s.dc.x);
    q.p[3][i] = make_float4(s.dc.y, s.dc.z, s.ic.x, s.ic.y);
    q.p[4][i] = make_float4(s.ic.z, __uint_as_float((uint32_t)s.rng.state), __uint_as_float((uint32_t)(s.rng.state >> 32)),
                            __uint_as_float(tag));
}


// AccumulateColor (renderer.cuh:117-122) for a terminated path, plus the
// per-pixel sum of squares of the sample value (for z-tests).
__device__ __forceinline__ void accumulate(const AccumView &a, uint32_t pixel, V3 dc, V3 ic) {
    atomicAdd(a.direct + pixel, make_float4(dc.x, dc.y, dc.z, 0.f));
    atomicAdd(a.indirect + pixel, make_float4(ic.x, ic.y, ic.z, 0.f));
    if (a.sumsq) {
        float r = dc.x + ic.x, g = dc.y + ic.y, b = dc.z + ic.z;
        atomicAdd(a.sumsq + pixel, make_float4(r * r, g * g, b * b, 1.f));
    }
}

// Warp-aggregated slot allocation: one atomic per converged group of lanes.
__device__ __forceinline__ int warp_alloc(int *counter, bool want) {
    unsigned active = __activemask();
    unsigned m = __ballot_sync(active, want);
    if (m == 0) return -1;
    int lane = threadIdx.x & 31;
    int leader = __ffs(m) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(counter, __popc(m));
    base = __shfl_sync(active, base, leader);
    return want ? base + __popc(m & ((1u << lane) - 1u)) : -1;
}

// The path that shade thread t visits: the hits (other materials, then
// subsurface) or the misses of the shade order.
__device__ __forceinline__ int shade_hit_index(const ShadeOrder &o, int t, int nhit) {
    return __ldg(o.idx + (t < nhit ? t : o.cap + (t - nhit)));
}
__device__ __forceinline__ int shade_miss_index(const ShadeOrder &o, int t) { return __ldg(o.idx + (o.cap - 1 - t)); }

// Places path i, whose closest hit is in slot (< 0: a miss), into the shade
// order (every lane of the warp calls it).
__device__ __forceinline__ void shade_order_put(const ShadeOrder &o, int *counters, int slot, int i) {
    const bool hit = slot >= 0;
    const int ms = warp_alloc(&counters[kMissCounter], !hit);
    if (!o.cls) {  // no subsurface material in the scene (uniform branch)
        const int hs = warp_alloc(&counters[kHitCounter], hit);
        o.idx[hit ? hs : o.cap - 1 - ms] = i;
        return;
    }
    const bool sss = hit && o.cls[slot];
    const int hs = warp_alloc(&counters[kHitCounter], hit && !sss);
    const int ss = warp_alloc(&counters[kSssCounter], sss);
    o.idx[sss ? o.cap + ss : (hit ? hs : o.cap - 1 - ms)] = i;
}

struct NeeRecord {
    V3 hp, hn, lp, ln, C;
    bool direct;
    bool valid;
};

enum StepResult { kContinue = 0, kTerminate = 1 };

// NEE toward one light: sample it, evaluate the contribution as if visible
// and leave the visibility test (Light::Visible) to the shadow kernel.
__device__ __forceinline__ bool nee_sample(const SceneView &s, Pcg32 &rng, int &lid, LightSample &ls, float &sel_pdf) {
    if (s.num_lights == 0) return false;  // LightManager::SampleLight returns nullptr
    lid = (int)(pcg32_uniform(rng) * s.num_lights);
    if (lid == s.num_lights) lid = s.num_lights - 1;
    sel_pdf = 1.0f / s.num_lights;
    light_sample_point(s, s.lights[lid], rng, ls);
    return true;
}

// ProbeOutgongingPoint (material.cu:405-441): two probe rays along -n and +n
// through the displaced point, the nearer hit wins.
static __device__ __noinline__ void sss_probe(const SceneView &s, V3 hitPoint, V3 normal, float distance, float angle,
                                          V3 &outP, V3 &outN) {
    V3 pn = normalized(normal), t, b;
    create_onb(pn, t, b);
    V3 off = distance * (cosf(angle) * t + sinf(angle) * b);
    outP = hitPoint + off;
    float ro = fmaxf(distance, 1e-3f);
    float tmin = 1e-4f, tmax = fmaxf(distance * 2.f, 1e-2f);
    V3 fo = outP + pn * ro, bo = outP - pn * ro;
    Hit fh = closest_hit<false>(s.bvh, fo, -pn, tmin, tmax);
    Hit bh = closest_hit<false>(s.bvh, bo, pn, tmin, tmax);
    const Hit *use = nullptr;
    if (fh.slot >= 0 && bh.slot >= 0)
        use = fh.t <= bh.t ? &fh : &bh;
    else if (fh.slot >= 0)
        use = &fh;
    else if (bh.slot >= 0)
        use = &bh;
    if (use) {
        outP = hit_point(s.bvh, *use);
        const float4 *tp = s.bvh.tris + 3 * (size_t)use->slot;
        float4 a = __ldg(tp), bb = __ldg(tp + 1), c = __ldg(tp + 2);
        V3 v0{a.x, a.y, a.z};
        outN = vnormalized(vcross(vsub(V3{bb.x, bb.y, bb.z}, v0), vsub(V3{c.x, c.y, c.z}, v0)));
    } else {
        outP = hitPoint;
        outN = pn;
    }
}

// PathTracing (renderer.cuh:170-422) for one path at its closest hit.
__device__ inline StepResult path_step(const SceneView &s, const StepParams &sp, PathState &ps, const Hit &h, NeeRecord &nee) {
    nee.valid = false;
    const bool rr_on = sp.bounce >= sp.rr_start;
    // IntersectionInfo of Triangle::IsIntersect (triangle.cu:121-130)
    const float4 *tp = s.bvh.tris + 3 * (size_t)h.slot;
    float4 ta = __ldg(tp), tb = __ldg(tp + 1), tc = __ldg(tp + 2);
    int prim = __float_as_int(ta.w);
    V3 v0{ta.x, ta.y, ta.z}, v1{tb.x, tb.y, tb.z}, v2{tc.x, tc.y, tc.z};
    V3 hitPoint = hit_point(s.bvh, h);
    V3 infoNormal = vnormalized(vcross(vsub(v1, v0), vsub(v2, v0)));
    const float4 *ap = s.attr + 4 * (size_t)prim;
    float4 A0 = __ldg(ap), A1 = __ldg(ap + 1), A2 = __ldg(ap + 2), A3 = __ldg(ap + 3);
    float b0 = rsub(rsub(1.f, h.b1), h.b2);
    V3 sn = normalized((b0 * V3{A0.x, A0.y, A0.z} + h.b1 * V3{A1.x, A1.y, A1.z}) + h.b2 * V3{A2.x, A2.y, A2.z});
    const DMesh &M = s.meshes[__float_as_int(A3.w)];
    DMaterial mat = s.materials[M.material];
    if (mat.tex >= 0 && (mat.type == MAT_DIFFUSE || mat.type == MAT_PBR || mat.type == MAT_SUBSURFACE)) {
        // Texture::Sample (texture.cu:243-252) at the interpolated texCoord
        // (triangle.cu:128): u, v clamped to [0, 0.999999], v flipped; it
        // replaces basecolor where the reference reads its diffuse texture
        // (material.cu:70, 211, 246, 283, 336).
        float tu = (b0 * A0.w + h.b1 * A2.w) + h.b2 * A3.y;
        float tv = (b0 * A1.w + h.b1 * A3.x) + h.b2 * A3.z;
        tu = fminf(fmaxf(tu, 0.0f), 0.999999f);
        tv = fminf(fmaxf(tv, 0.0f), 0.999999f);
        const float4 tc = tex2D<float4>(s.textures[mat.tex], tu, 1.0f - tv);
        mat.base[0] = tc.x;
        mat.base[1] = tc.y;
        mat.base[2] = tc.z;
    }

    V3 geomNormal = normalized(infoNormal);
    V3 hitNormal = (double)sqnorm(sn) > kEpsD ? normalized(sn) : geomNormal;
    if (dot(hitNormal, geomNormal) < 0.f) hitNormal = -hitNormal;
    V3 wo = -ps.d;

    if (mat.type == MAT_LIGHT) {  // renderer.cuh:192-216
        V3 ke = ld3(mat.ke);
        if (ps.first) {
            ps.dc = ps.dc + ke;
            ps.first = false;
            return kTerminate;
        } else if (ps.spec) {
            ps.ic = ps.ic + mul(ps.w, ke);
        } else {
            float pdfLight = 0.f;  // a light material on a mesh that is not a light: no MIS
            if (M.light >= 0) pdfLight = light_solid_angle_pdf(s, s.lights[M.light], ps.o, hitPoint, infoNormal);
            float mw = mis_weight(ps.pdf, pdfLight);
            ps.ic = ps.ic + mul(ps.w, ke) * mw;
        }
        return kTerminate;
    }

    if (mat.type == MAT_DIELECTRIC) {  // renderer.cuh:218-240
        V3 dwi, dw;
        float dpdf = 1.0f;
        sample_dielectric(mat, wo, hitNormal, dwi, dpdf, dw, ps.rng);
        ps.pdf = dpdf;
        ps.o = hitPoint + dwi * 1e-4f;
        ps.d = dwi;
        ps.w = mul(ps.w, dw);
        float p = pcg32_uniform(ps.rng);
        if (rr_on && p > sp.rr) return kTerminate;
        if (rr_on) ps.w = ps.w / sp.rr;
        ps.first = false;
        ps.spec = true;
        return kContinue;
    }

    if (mat.type != MAT_SUBSURFACE) {  // renderer.cuh:242-289
        int lid;
        LightSample ls;
        float sel;
        if (nee_sample(s, ps.rng, lid, ls, sel)) {
            const DLight &L = s.lights[lid];
            V3 dirWi = normalized(ls.position - hitPoint);
            float pdfLight = light_solid_angle_pdf(s, L, hitPoint, ls.position, ls.normal);
            pdfLight *= sel;
            float cosT = dot(hitNormal, dirWi);
            V3 brdf = mat_eval(mat, wo, hitNormal, dirWi);
            V3 dirL = (mul(light_emission(s, L, dirWi), brdf) * cosT) / pdfLight;
            float pdfB = mat_pdf(mat, wo, hitNormal, dirWi);
            float mw = mis_weight(pdfLight, pdfB);
            nee.C = mw * mul(ps.w, dirL);
            nee.hp = hitPoint;
            nee.hn = infoNormal;
            nee.lp = ls.position;
            nee.ln = ls.normal;
            nee.direct = ps.first;
            nee.valid = nee.C.x != 0.f || nee.C.y != 0.f || nee.C.z != 0.f;
        }
        V3 iwi;
        float ipdf;
        mat_sample(mat, wo, hitNormal, iwi, ipdf, ps.rng);
        V3 brdf = mat_eval(mat, wo, hitNormal, iwi);
        ps.pdf = ipdf;
        ps.o = hitPoint;
        ps.d = iwi;
        float c = dot(hitNormal, iwi);
        if (!((double)ipdf < kEpsD || c < 0))
            ps.w = (mul(ps.w, brdf) * c) / ipdf;
        else
            return kTerminate;
    } else {  // subsurface, renderer.cuh:290-404
        float FIn = fresnel_mat(mat, wo, hitNormal);
        float reflectProb = clampf(0.02f, 0.98f, FIn);
        float transmitProb = fmaxf(1.f - reflectProb, 1e-6f);
        float ev = pcg32_uniform(ps.rng);
        if (ev < reflectProb) {
            V3 rd;
            if (mat.roughness > 1e-3f) {
                float r1 = pcg32_uniform(ps.rng), r2 = pcg32_uniform(ps.rng);
                float a = fmaxf(mat.roughness * mat.roughness, 0.02f);
                float phi = (float)(2.0 * kPiD * (double)r1);
                float cosT = sqrtf((1.0f - r2) / (1.0f + (a * a - 1.0f) * r2));
                float sinT = sqrtf(fmaxf(0.0f, 1.0f - cosT * cosT));
                V3 hw = local_to_world(V3{sinT * cosf(phi), sinT * sinf(phi), cosT}, hitNormal);
                rd = normalized(reflect(-wo, hw));
                if (dot(rd, hitNormal) <= 0.0f) rd = normalized(reflect(-wo, hitNormal));
            } else {
                rd = normalized(reflect(-wo, hitNormal));
            }
            ps.o = hitPoint + rd * 1e-4f;
            ps.d = rd;
            ps.w = mul(ps.w, V3{FIn, FIn, FIn}) / reflectProb;
            ps.pdf = 1.0f;
            float p = pcg32_uniform(ps.rng);
            if (rr_on && p > sp.rr) return kTerminate;
            if (rr_on) ps.w = ps.w / sp.rr;
            ps.first = false;
            ps.spec = true;
            return kContinue;
        }
        // SampleSpatialDiffusionProfile (material.cu:343-368)
        float distance;
        int ch = (int)(pcg32_uniform(ps.rng) * 3);
        ch = (int)clampf(0.f, 2.f, (float)ch);
        float d = mat.scatter[ch];
        if (d < 1e-6f) {
            distance = 0.f;
        } else {
            float r1 = pcg32_uniform(ps.rng);
            if (r1 < 0.5f) {
                r1 = r1 * 2.f;
                distance = -d * logf(1.f - r1);
            } else {
                r1 = (r1 - 0.5f) * 2.f;
                distance = -3.f * d * logf(1.f - r1);
            }
        }
        float angle = (float)((double)(pcg32_uniform(ps.rng) * 2.f) * kPiD);
        V3 outP, outN;
        sss_probe(s, hitPoint, geomNormal, distance, angle, outP, outN);
        float sd = norm(outP - hitPoint);
        float spatialPdf = sd < 1e-6f ? 0.f : burley_pdf(mat, sd);
        if ((double)spatialPdf < kEpsD) return kTerminate;
        V3 prof{0.f, 0.f, 0.f};
        if (!(sd < 1e-6f)) prof = mul(albedo_of(mat), V3{burley(mat, sd, 0), burley(mat, sd, 1), burley(mat, sd, 2)}) / kPiF;
        ps.w = mul(mul(ps.w, V3{1.f - FIn, 1.f - FIn, 1.f - FIn}), prof) / (transmitProb * spatialPdf);
        int lid;
        LightSample ls;
        float sel;
        if (nee_sample(s, ps.rng, lid, ls, sel)) {
            const DLight &L = s.lights[lid];
            V3 dirWi = normalized(ls.position - outP);
            float ftout = 1 - fresnel_mat(mat, dirWi, outN);
            float pdfLight = light_solid_angle_pdf(s, L, outP, ls.position, ls.normal);
            pdfLight *= sel;
            float cosT = dot(outN, dirWi);
            if (cosT > 0.f && (double)pdfLight > kEpsD) {
                V3 dirL = (mul(light_emission(s, L, dirWi), V3{1.f, 1.f, 1.f} / kPiF) * cosT) / pdfLight;
                float pdfB = (float)((double)cosT / kPiD);
                float mw = mis_weight(pdfLight, pdfB);
                nee.C = (mw * mul(ps.w, dirL)) * ftout;
                nee.hp = outP;
                nee.hn = outN;
                nee.lp = ls.position;
                nee.ln = ls.normal;
                nee.direct = ps.first;
                nee.valid = nee.C.x != 0.f || nee.C.y != 0.f || nee.C.z != 0.f;
            }
        }
        V3 odir;
        float opdf;
        sample_diffuse(outN, odir, opdf, ps.rng);
        float cosOut = dot(outN, odir);
        float ftout = 1 - fresnel_mat(mat, odir, outN);
        if ((double)opdf < kEpsD || cosOut < 0.f) return kTerminate;
        ps.o = outP + outN * 1e-4f;
        ps.d = odir;
        ps.w = ps.w * ftout;
        ps.pdf = opdf;
    }
    // Russian roulette (renderer.cuh:407-420)
    float p = pcg32_uniform(ps.rng);
    if (rr_on && p > sp.rr) return kTerminate;
    if (rr_on) ps.w = ps.w / sp.rr;
    ps.first = false;
    ps.spec = false;
    return kContinue;
}

}  // namespace crt
