// Device-side restatement of the reference's shading model: camera rays,
// materials (Lambertian, GGX "PBR", dielectric, Burley subsurface), lights
// (uniform light choice, mesh area lights, environment map), MIS and the
// per-hit path-tracing step. Each function names the reference routine it
// follows; expression order and the places where the reference computes in
// double (its PI = 3.1415926 and eps = 1e-6 are double literals) are kept.
#pragma once
#include "trace.cuh"
#include "rng.cuh"
#include "scene_data.h"

namespace crt {

constexpr double kPiD = 3.1415926;       // PI (Src/Core/global.h:6)
constexpr float kPiF = 3.1415926f;       // PI after Eigen's scalar promotion
constexpr double kEpsD = 1e-6;           // eps (Src/Core/global.h:5)
constexpr float kFloatMax = 3.40282e+38f;  // FLOATMAX (Src/Core/global.h:7)

struct EnvView {
    cudaTextureObject_t tex;
    int w, h;
    const float *ucdf;        // w*h, per-row normalised prefix sums
    const float *vcdf;        // h, normalised prefix of row sums
    const float2 *row_alias;  // h: (probability, alias row)
    const float2 *col_alias;  // w*h: (probability, alias column)
};

struct SceneView {
    BvhView bvh;
    const int *slot_of_prim;
    const float4 *attr;  // 4 per primitive: (n0, u0) (n1, v0) (n2, u1) (v1, u2, v2, mesh)
    const DMesh *meshes;
    const DMaterial *materials;
    const DLight *lights;
    int num_lights;
    int env_light;
    EnvView env;
    float center[3];
    float diag;
    const cudaTextureObject_t *textures;  // DMaterial::tex indexes this
    const uint8_t *slot_class;             // per triangle slot: 1 = subsurface material (shade order); null
                                           // when the scene has no subsurface material
};

#ifdef __CUDACC__

// --- small vector helpers (plain float arithmetic) --------------------------
// The large shading functions the shade stage calls from two or three
// sites each: inlined (default) or, with CRT_SHADE_NOINLINE, compiled once
// per translation unit and called. Out of line measured 2% faster on the
// 1080p icosphere frame (a smaller instruction footprint for the
// fetch-bound shade kernels) but 7% slower on the Cornell-box batch (call
// overhead on short diffuse paths), so they stay inlined.
#ifdef CRT_SHADE_NOINLINE
#define CRT_SHADE_FN static __device__ __noinline__
#else
#define CRT_SHADE_FN __device__ __forceinline__
#endif

__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V3 operator-(V3 a) { return V3{-a.x, -a.y, -a.z}; }
__device__ __forceinline__ V3 operator*(V3 a, float s) { return V3{a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ V3 operator*(float s, V3 a) { return V3{a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ V3 operator/(V3 a, float s) { return V3{a.x / s, a.y / s, a.z / s}; }
__device__ __forceinline__ V3 mul(V3 a, V3 b) { return V3{a.x * b.x, a.y * b.y, a.z * b.z}; }
__device__ __forceinline__ float dot(V3 a, V3 b) { return a.x * b.x + (a.y * b.y + a.z * b.z); }
__device__ __forceinline__ V3 cross(V3 a, V3 b) {
    return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ float sqnorm(V3 a) { return dot(a, a); }
__device__ __forceinline__ float norm(V3 a) { return sqrtf(sqnorm(a)); }
__device__ __forceinline__ V3 normalized(V3 a) {
    float z = sqnorm(a);
    if (z > 0.f) {
        float s = sqrtf(z);
        return V3{a.x / s, a.y / s, a.z / s};
    }
    return a;
}
__device__ __forceinline__ V3 ld3(const float *p) { return V3{p[0], p[1], p[2]}; }

// Clamp(a, b, c) clamps c to [a, b] (Src/Utils/mathutil.cu:68-75).
__device__ __forceinline__ float clampf(float a, float b, float c) { return c < a ? a : (c > b ? b : c); }
// Luminance, Rec.709 (Src/Utils/mathutil.cu:143-146).
__device__ __forceinline__ float luminance(V3 c) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; }
// Reflect (Src/Utils/mathutil.cu:139-141).
__device__ __forceinline__ V3 reflect(V3 I, V3 N) { return I - (2.0f * dot(I, N)) * N; }
// Lerp (Src/Utils/mathutil.cu:135-137).
__device__ __forceinline__ V3 lerp(V3 a, V3 b, float t) { return a * (1.0f - t) + b * t; }

// LocalToWorld (Src/Utils/mathutil.cu:48-60).
__device__ __forceinline__ V3 local_to_world(V3 v, V3 normal) {
    V3 n = normalized(normal);
    V3 up = fabsf(n.x) > fabsf(n.y) ? V3{0.f, 1.f, 0.f} : V3{1.f, 0.f, 0.f};
    V3 a = normalized(cross(up, n));
    V3 b = normalized(cross(n, a));
    return (a * v.x + b * v.y) + n * v.z;
}

// CreateONB (Src/Utils/mathutil.cu:148-155).
__device__ __forceinline__ void create_onb(V3 n, V3 &t, V3 &b) {
    t = fabsf(n.x) > fabsf(n.y) ? normalized(V3{-n.z, 0.f, n.x}) : normalized(V3{0.f, n.z, -n.y});
    b = normalized(cross(n, t));
}

// MISWeight, power heuristic with exponent 2 (Src/Core/renderer.cuh:165-168).
__device__ __forceinline__ float mis_weight(float a, float b) {
    float t1 = powf(a, 2.f), t2 = powf(b, 2.f);
    return t1 / (t1 + t2);
}

// --- materials (Src/Core/material.cu) ---------------------------------------

// FresnelDielectric (material.cu:121-142).
__device__ __forceinline__ float fresnel_dielectric(float cosI, float etaI, float etaT) {
    cosI = clampf(-1.0f, 1.0f, cosI);
    bool entering = cosI > 0.0f;
    if (!entering) {
        float t = etaI;
        etaI = etaT;
        etaT = t;
        cosI = fabsf(cosI);
    }
    float sinI = sqrtf(fmaxf(0.0f, 1.0f - cosI * cosI));
    float sinT = etaI / etaT * sinI;
    if (sinT >= 1.0f) return 1.0f;
    float cosT = sqrtf(fmaxf(0.0f, 1.0f - sinT * sinT));
    float rpar = ((etaT * cosI) - (etaI * cosT)) / ((etaT * cosI) + (etaI * cosT));
    float rper = ((etaI * cosI) - (etaT * cosT)) / ((etaI * cosI) + (etaT * cosT));
    return 0.5f * (rpar * rpar + rper * rper);
}

// Fresnel (material.cu:116-119): reflectance for cos = n.wi, eta 1 -> ior.
CRT_SHADE_FN float fresnel_mat(const DMaterial &m, V3 wi, V3 n) {
    return fresnel_dielectric(dot(n, wi), 1.0f, m.ior);
}

// RefractDirection (material.cu:144-153).
__device__ __forceinline__ bool refract_dir(V3 incident, V3 n, float eta, V3 &out) {
    float cosI = fmaxf(0.0f, -dot(incident, n));
    float sin2T = eta * eta * fmaxf(0.0f, 1.0f - cosI * cosI);
    if (sin2T >= 1.0f) return false;
    float cosT = sqrtf(fmaxf(0.0f, 1.0f - sin2T));
    out = eta * incident + (eta * cosI - cosT) * n;
    return true;
}

// SampleDielectric (material.cu:155-192). wi points toward the viewer.
CRT_SHADE_FN void sample_dielectric(const DMaterial &m, V3 wi, V3 normal, V3 &wo, float &pdf, V3 &weight,
                                                  Pcg32 &rng) {
    V3 incident = -normalized(wi);
    V3 on = normalized(normal);
    float etaI = 1.0f, etaT = m.ior;
    if (dot(incident, on) > 0.0f) {
        on = -on;
        float t = etaI;
        etaI = etaT;
        etaT = t;
    }
    float cosI = fmaxf(0.0f, -dot(incident, on));
    float F = fresnel_dielectric(cosI, etaI, etaT);
    float r = pcg32_uniform(rng);
    if (r < F) {
        wo = normalized(reflect(incident, on));
        pdf = fmaxf(F, 1e-6f);
        weight = V3{1.f, 1.f, 1.f};
        return;
    }
    V3 refr;
    if (!refract_dir(incident, on, etaI / etaT, refr)) {
        wo = normalized(reflect(incident, on));
        pdf = 1.0f;
        weight = V3{1.f, 1.f, 1.f};
        return;
    }
    wo = normalized(refr);
    pdf = fmaxf(1.0f - F, 1e-6f);
    weight = lerp(V3{1.f, 1.f, 1.f}, ld3(m.base), m.transmission);
}

// DistributionGGX (material.cu:96-107); the reference multiplies by PI in double.
__device__ __forceinline__ float ggx_d(float roughness, V3 wi, V3 n, V3 wo) {
    V3 h = normalized(wi + wo);
    float NdotH = fmaxf(dot(n, h), 0.f);
    float alpha = roughness * roughness;
    float alpha2 = alpha * alpha;
    float NdotH2 = NdotH * NdotH;
    float denom = (NdotH2 * (alpha2 - 1.f) + 1.f);
    double dd = kPiD * denom * denom;
    return (float)(alpha2 / dd);
}

__device__ __forceinline__ V3 albedo_of(const DMaterial &m) { return ld3(m.base); }

// EvaluateDiffuse (material.cu:66-74): kd / PI when wo faces the normal.
__device__ __forceinline__ V3 eval_diffuse(const DMaterial &m, V3 n, V3 wo) {
    if (dot(wo, n) > 0.f) return albedo_of(m) / kPiF;
    return V3{0.f, 0.f, 0.f};
}
// PdfDiffuse (material.cu:76-82).
__device__ __forceinline__ float pdf_diffuse(V3 n, V3 wo) {
    float c = dot(wo, n);
    return c > 0.f ? (float)((double)c / kPiD) : 0.f;
}
// SampleDiffuse (material.cu:84-92): cosine lobe via theta = acos(1-2u)/2.
__device__ __forceinline__ void sample_diffuse(V3 n, V3 &wo, float &pdf, Pcg32 &rng) {
    float t1 = pcg32_uniform(rng), t2 = pcg32_uniform(rng);
    float theta = (float)(0.5 * (double)acosf(1.f - 2.f * t1));
    float phi = (float)(2.0 * kPiD * (double)t2);
    float x = sinf(theta) * cosf(phi), y = sinf(theta) * sinf(phi), z = cosf(theta);
    wo = local_to_world(V3{x, y, z}, n);
    pdf = pdf_diffuse(n, wo);
}

// EvaluatePBR (material.cu:205-241).
__device__ __forceinline__ V3 eval_pbr(const DMaterial &m, V3 wi, V3 n, V3 wo) {
    float NdotV = fmaxf(dot(n, wi), 0.0f), NdotL = fmaxf(dot(n, wo), 0.0f);
    if (NdotL <= 0.0f || NdotV <= 0.0f) return V3{0.f, 0.f, 0.f};
    V3 albedo = albedo_of(m);
    V3 F0 = lerp(V3{0.04f, 0.04f, 0.04f}, albedo, m.metallic);
    float D = ggx_d(m.roughness, wi, n, wo);
    // GeometrySchlickGGX (material.cu:194-203)
    float r = m.roughness + 1.f, k = (r * r) / 8.f;
    float G = (NdotV / (NdotV * (1.f - k) + k)) * (NdotL / (NdotL * (1.f - k) + k));
    // FresnelSchlick (material.cu:109-114)
    V3 h = normalized(wi + wo);
    float HdotV = fmaxf(dot(h, wi), 0.f);
    float f5 = powf(1.f - HdotV, 5.f);
    V3 F = F0 + (V3{1.f, 1.f, 1.f} - F0) * f5;
    V3 spec = (F * (D * G)) / (4.0f * NdotV * NdotL + 0.0001f);
    V3 kd = (V3{1.f, 1.f, 1.f} - F) * (1.0f - m.metallic);
    V3 diff = (dot(wi, n) > 0.f && dot(wo, n) > 0.f) ? mul(kd, albedo) / kPiF : V3{0.f, 0.f, 0.f};
    return diff + spec;
}

// P_spec of PdfPBR / SamplePBR (material.cu:250-258, 287-295).
__device__ __forceinline__ float pbr_pspec(const DMaterial &m, V3 wi, V3 n) {
    V3 albedo = albedo_of(m);
    V3 F0 = lerp(V3{0.04f, 0.04f, 0.04f}, albedo, m.metallic);
    float NdotV = fmaxf(dot(n, wi), 0.0f);
    V3 Fa = F0 + (V3{1.f, 1.f, 1.f} - F0) * powf(1.0f - NdotV, 5.0f);
    float s = luminance(Fa), d = luminance(albedo) * (1.0f - m.metallic);
    float p = fmaxf(s / (s + d), 1e-6f);
    return clampf(0.01f, 0.99f, p);
}

// PdfPBR (material.cu:243-278).
__device__ __forceinline__ float pdf_pbr(const DMaterial &m, V3 wi, V3 n, V3 wo) {
    float ps = pbr_pspec(m, wi, n);
    float NdotL = fmaxf(dot(n, wo), 0.0f);
    if (NdotL <= 0.0f) return 0.f;
    V3 h = normalized(wi + wo);
    float VdotH = fmaxf(dot(wi, h), 1e-6f), NdotH = fmaxf(dot(n, h), 1e-6f);
    float D = ggx_d(m.roughness, wi, n, wo);
    float pspec = (D * NdotH) / (4.0f * VdotH);
    float pdiff = (float)((double)NdotL / kPiD);
    return ps * pspec + (1.0f - ps) * pdiff;
}

// SamplePBR (material.cu:280-324): draws r1, r2, choice in that order.
__device__ __forceinline__ void sample_pbr(const DMaterial &m, V3 wi, V3 n, V3 &wo, float &pdf, Pcg32 &rng) {
    float ps = pbr_pspec(m, wi, n);
    float r1 = pcg32_uniform(rng), r2 = pcg32_uniform(rng), ch = pcg32_uniform(rng);
    float phi = (float)(2.0 * kPiD * (double)r1);
    if (ch < ps) {
        float a = m.roughness * m.roughness;
        float cosT = sqrtf((1.0f - r2) / (1.0f + (a * a - 1.0f) * r2));
        float sinT = sqrtf(fmaxf(0.0f, 1.0f - cosT * cosT));
        V3 hw = local_to_world(V3{sinT * cosf(phi), sinT * sinf(phi), cosT}, n);
        wo = normalized(reflect(-wi, hw));
    } else {
        float cosT = sqrtf(r2), sinT = sqrtf(1.0f - r2);
        wo = local_to_world(V3{sinT * cosf(phi), sinT * sinf(phi), cosT}, n);
    }
    pdf = pdf_pbr(m, wi, n, wo);
}

// Material::Evaluate / Pdf / Sample dispatch (material.cu:14-64).
CRT_SHADE_FN V3 mat_eval(const DMaterial &m, V3 wi, V3 n, V3 wo) {
    if (m.type == MAT_PBR) return eval_pbr(m, wi, n, wo);
    if (m.type == MAT_DIELECTRIC) return V3{0.f, 0.f, 0.f};
    return eval_diffuse(m, n, wo);
}
CRT_SHADE_FN float mat_pdf(const DMaterial &m, V3 wi, V3 n, V3 wo) {
    if (m.type == MAT_PBR) return pdf_pbr(m, wi, n, wo);
    if (m.type == MAT_DIELECTRIC) return 0.f;
    return pdf_diffuse(n, wo);
}
CRT_SHADE_FN void mat_sample(const DMaterial &m, V3 wi, V3 n, V3 &wo, float &pdf, Pcg32 &rng) {
    if (m.type == MAT_PBR)
        sample_pbr(m, wi, n, wo, pdf, rng);
    else
        sample_diffuse(n, wo, pdf, rng);
}

// BurleyDiffusionProfile (material.cu:380-392); the divisor is in double.
__device__ __forceinline__ float burley(const DMaterial &m, float r, int c) {
    float d = m.scatter[c];
    if (r < 1e-6f || d < 1e-6f) return 0.f;
    float e1 = expf(-r / d), e2 = expf(-r / (3 * d));
    return (float)((double)(e1 + e2) / (8.0 * kPiD * (double)d * (double)r));
}
// PdfBurleyDiffusionProfile (material.cu:394-400).
__device__ __forceinline__ float burley_pdf(const DMaterial &m, float r) {
    return (burley(m, r, 0) + burley(m, r, 1) + burley(m, r, 2)) / 3.f;
}

// --- environment map (Src/Core/texture.cu) -----------------------------------

// HDRTexture::SamplePDF (texture.cu:155-166): uv-space pdf p * W * H.
__device__ __forceinline__ float env_sample_pdf(const EnvView &e, float u, float v) {
    u = clampf(0.0f, 0.999999f, u);
    v = clampf(0.0f, 0.999999f, v);
    int ui = min((int)(u * e.w), e.w - 1), vi = min((int)(v * e.h), e.h - 1);
    float prow = vi == 0 ? __ldg(e.vcdf) : __ldg(e.vcdf + vi) - __ldg(e.vcdf + vi - 1);
    const float *row = e.ucdf + (size_t)vi * e.w;
    float pcol = ui == 0 ? __ldg(row) : __ldg(row + ui) - __ldg(row + ui - 1);
    float p = prow * pcol;
    return p * e.w * e.h;
}

// Texel choice of HDRTexture::Sample (texture.cu:112-153) by alias tables
// that carry exactly the CDFs' discrete distribution (row = vCDF[y] -
// vCDF[y-1], column = uCDF[y][x] - uCDF[y][x-1]); one uniform per axis, row
// first, as the reference's two binary searches. Returns texel centres.
__device__ __forceinline__ void env_sample_uv(const EnvView &e, Pcg32 &rng, float &u, float &v) {
    float rv = pcg32_uniform(rng);
    float fy = rv * e.h;
    int y = min((int)fy, e.h - 1);
    float2 ra = __ldg(e.row_alias + y);
    if (fy - y >= ra.x) y = __float_as_int(ra.y);
    float ru = pcg32_uniform(rng);
    float fx = ru * e.w;
    int x = min((int)fx, e.w - 1);
    float2 ca = __ldg(e.col_alias + (size_t)y * e.w + x);
    if (fx - x >= ca.x) x = __float_as_int(ca.y);
    u = ((float)x + 0.5f) / (float)e.w;
    v = ((float)y + 0.5f) / (float)e.h;
}

// Light::Emission for the environment (light.cu:141-155): u = phi/2pi,
// v = theta/pi, hardware bilinear fetch (wrap u, clamp v).
CRT_SHADE_FN V3 env_emission(const EnvView &e, V3 wi) {
    float theta = acosf(wi.y);
    float phi = atan2f(wi.x, wi.z);
    if (phi < 0) phi = (float)((double)phi + 2.0 * kPiD);
    float u = (float)((double)phi / (2.0 * kPiD));
    float v = (float)((double)theta / kPiD);
    float4 c = tex2D<float4>(e.tex, u, v);
    return V3{c.x, c.y, c.z};
}

// --- lights (Src/Core/light.cu, lightmanager.cu) -----------------------------

struct LightSample {
    V3 position, normal;
};

// Triangle::Sample (triangle.cu:135-143): fold (u,v) when u+v > 1.
__device__ __forceinline__ void sample_triangle(const SceneView &s, int prim, Pcg32 &rng, LightSample &ls) {
    float u = pcg32_uniform(rng), v = pcg32_uniform(rng);
    if (u + v > 1) {
        u = 1 - u;
        v = 1 - v;
    }
    int slot = __ldg(s.slot_of_prim + prim);
    const float4 *tp = s.bvh.tris + 3 * (size_t)slot;
    float4 a = __ldg(tp), b = __ldg(tp + 1), c = __ldg(tp + 2);
    V3 v0{a.x, a.y, a.z}, v1{b.x, b.y, b.z}, v2{c.x, c.y, c.z};
    float w = 1 - u - v;
    ls.position = (w * v0 + u * v1) + v * v2;
    // Triangle::normal = normalize((v1-v0) x (v2-v0)) (triangle.cu:6-9)
    ls.normal = vnormalized(vcross(vsub(v1, v0), vsub(v2, v0)));
}

// Light::SamplePoint (light.cu:29-41).
CRT_SHADE_FN void light_sample_point(const SceneView &s, const DLight &L, Pcg32 &rng,
                                                   LightSample &ls) {
    if (L.type == LIGHT_AREA) {
        // SampleAreaLight (light.cu:60-69): triangle uniform by index.
        const DMesh &m = s.meshes[L.mesh];
        int t = (int)(pcg32_uniform(rng) * m.count);
        if (t == m.count) t = m.count - 1;
        sample_triangle(s, m.start + t, rng, ls);
    } else {
        // SampleEnvLight (light.cu:91-107).
        float u, v;
        env_sample_uv(s.env, rng, u, v);
        float theta = (float)((double)(u * 2.f) * kPiD);
        float phi = acosf(1.f - 2.f * v);
        V3 dir{sinf(phi) * sinf(theta), cosf(phi), sinf(phi) * cosf(theta)};
        V3 c{s.center[0], s.center[1], s.center[2]};
        ls.position = c + (dir * 2.f) * s.diag;
        ls.normal = -dir;
    }
}

// Light::SampleSolidAnglePDF (light.cu:50-58) with origin = the shading point.
CRT_SHADE_FN float light_solid_angle_pdf(const SceneView &s, const DLight &L, V3 origin, V3 lp,
                                                       V3 ln) {
    if (L.type == LIGHT_AREA) {
        // SampleAreaLightSolidAnglePDF (light.cu:79-89)
        V3 wi = normalized(origin - lp);
        float d2 = sqnorm(origin - lp);
        float c = fmaxf(dot(ln, wi), 1e-6f);
        return d2 / (s.meshes[L.mesh].area * c);
    }
    // SampleEnvLightSolidAnglePDF (light.cu:125-139): flipped v, uv-space pdf.
    V3 dir = normalized(lp - origin);
    float theta = acosf(dir.y);
    float phi = atan2f(dir.x, dir.z);
    if (phi < 0) phi = (float)((double)phi + 2.0 * kPiD);
    float u = (float)((double)phi / (2.0 * kPiD));
    float v = (float)(1.0 - (double)theta / kPiD);
    return env_sample_pdf(s.env, u, v);
}

// Light::Emission (light.cu:141-155).
CRT_SHADE_FN V3 light_emission(const SceneView &s, const DLight &L, V3 wi) {
    if (L.type == LIGHT_ENV) return env_emission(s.env, wi);
    return ld3(L.emission);
}

#endif  // __CUDACC__

}  // namespace crt
