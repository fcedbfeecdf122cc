/*
 * Oracle renderer: CPU restatement of the reference's path tracer
 * (DarrenChen-CN/CudaRayTracer, Src/Core/renderer.cuh:96-440 with the
 * material, light, texture and camera routines it calls), driven by the
 * same per-path PCG32 streams as the CUDA renderer, so the two can be
 * compared pixel by pixel at low sample counts. Test infrastructure only.
 *
 * Closest hits are brute force in primitive order. The environment map is
 * fetched with CUDA's documented bilinear filtering (8-bit fractional
 * weights, wrap in u, clamp in v, normalised coordinates). Expressions that
 * the reference evaluates in double (its PI = 3.1415926 and eps = 1e-6 are
 * double literals) are evaluated in double here too.
 */
#include "crt_oracle.h"
#include "par.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define PI_D 3.1415926
#define PI_F 3.1415926f
#define EPS_D 1e-6

typedef struct { float x, y, z; } vec;

static inline vec V(float x, float y, float z) { vec r = {x, y, z}; return r; }
static inline vec vadd(vec a, vec b) { return V(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline vec vsub(vec a, vec b) { return V(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline vec vneg(vec a) { return V(-a.x, -a.y, -a.z); }
static inline vec vs(vec a, float s) { return V(a.x * s, a.y * s, a.z * s); }
static inline vec vdivs(vec a, float s) { return V(a.x / s, a.y / s, a.z / s); }
static inline vec vmul(vec a, vec b) { return V(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline float vdot(vec a, vec b) { return a.x * b.x + (a.y * b.y + a.z * b.z); }
static inline vec vcross(vec a, vec b) {
    return V(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline float vsq(vec a) { return vdot(a, a); }
static inline float vlen(vec a) { return sqrtf(vsq(a)); }
static inline vec vnorm(vec a) {
    float z = vsq(a);
    if (z > 0.f) {
        float s = sqrtf(z);
        return V(a.x / s, a.y / s, a.z / s);
    }
    return a;
}
static inline vec L3(const float *p) { return V(p[0], p[1], p[2]); }
static inline float clampf3(float a, float b, float c) { return c < a ? a : (c > b ? b : c); }
static inline float luminance(vec c) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; }
static inline vec reflectv(vec I, vec N) { return vsub(I, vs(N, 2.0f * vdot(I, N))); }
static inline vec lerpv(vec a, vec b, float t) { return vadd(vs(a, 1.0f - t), vs(b, t)); }

/* ---- PCG32, identical to the CUDA renderer's ---------------------------- */
typedef struct { unsigned long long state, inc; } pcg;
static inline unsigned int pcg_next(pcg *r) {
    unsigned long long old = r->state;
    r->state = old * 6364136223846793005ULL + r->inc;
    unsigned int xs = (unsigned int)(((old >> 18u) ^ old) >> 27u);
    unsigned int rot = (unsigned int)(old >> 59u);
    return (xs >> rot) | (xs << ((0u - rot) & 31u));
}
static inline pcg pcg_seed(unsigned long long seed, unsigned int pixel, unsigned int sample) {
    pcg r;
    r.state = 0u;
    r.inc = ((unsigned long long)pixel << 1u) | 1u;
    pcg_next(&r);
    r.state += seed * 0x9E3779B97F4A7C15ULL + (unsigned long long)sample * 0xD1B54A32D192ED03ULL;
    pcg_next(&r);
    return r;
}
static inline float U(pcg *r) { return (float)((pcg_next(r) >> 8) + 1u) * (1.0f / 16777216.0f); }

/* ---- scene context ---------------------------------------------------------- */
typedef struct {
    const oracle_scene *s;
    float *ucdf, *vcdf, *ra, *ca;
    float center[3], diag;
} ctx_t;

enum { M_LIGHT = 0, M_DIFFUSE = 1, M_PBR = 2, M_DIELECTRIC = 3, M_SUBSURFACE = 4 };

typedef struct {
    int type;
    vec base, ke;
    float rough, metal, trans;
    float scatter[3];
    float ior;
} mat_t;

/* tex2D<float4> of a uchar4 texture read as normalised float (byte / 255),
 * linear filtering with 8-bit fractional weights, wrap u / clamp v. */
static vec tex_fetch(const ctx_t *c, int t, float u, float v) {
    int W = c->s->tex_w[t], H = c->s->tex_h[t];
    const unsigned char *e = c->s->tex[t];
    float x = (u - floorf(u)) * W, y = v * H;
    float xb = x - 0.5f, yb = y - 0.5f;
    int i = (int)floorf(xb), j = (int)floorf(yb);
    float a = floorf((xb - i) * 256.f + 0.5f) / 256.f, b = floorf((yb - j) * 256.f + 0.5f) / 256.f;
    int i0 = ((i % W) + W) % W, i1 = (((i + 1) % W) + W) % W;
    int j0 = j < 0 ? 0 : (j >= H ? H - 1 : j), j1 = j + 1 < 0 ? 0 : (j + 1 >= H ? H - 1 : j + 1);
    const unsigned char *t00 = e + 4 * ((size_t)j0 * W + i0), *t10 = e + 4 * ((size_t)j0 * W + i1);
    const unsigned char *t01 = e + 4 * ((size_t)j1 * W + i0), *t11 = e + 4 * ((size_t)j1 * W + i1);
    float r[3];
    for (int k = 0; k < 3; ++k)
        r[k] = (1 - a) * (1 - b) * (t00[k] / 255.f) + a * (1 - b) * (t10[k] / 255.f) + (1 - a) * b * (t01[k] / 255.f) +
               a * b * (t11[k] / 255.f);
    return V(r[0], r[1], r[2]);
}

static mat_t get_mat(const ctx_t *c, int i) {
    const float *m = c->s->materials + 16 * i;
    mat_t r;
    r.type = (int)m[0];
    r.base = L3(m + 1);
    r.ke = L3(m + 4);
    r.rough = m[7];
    r.metal = m[8];
    r.trans = m[9];
    r.scatter[0] = m[10];
    r.scatter[1] = m[11];
    r.scatter[2] = m[12];
    r.ior = m[13];
    return r;
}

/* LocalToWorld (Src/Utils/mathutil.cu:48-60) */
static vec local_to_world(vec v, vec normal) {
    vec n = vnorm(normal);
    vec up = fabsf(n.x) > fabsf(n.y) ? V(0.f, 1.f, 0.f) : V(1.f, 0.f, 0.f);
    vec a = vnorm(vcross(up, n));
    vec b = vnorm(vcross(n, a));
    return vadd(vadd(vs(a, v.x), vs(b, v.y)), vs(n, v.z));
}

/* CreateONB (Src/Utils/mathutil.cu:148-155) */
static void create_onb(vec n, vec *t, vec *b) {
    *t = fabsf(n.x) > fabsf(n.y) ? vnorm(V(-n.z, 0.f, n.x)) : vnorm(V(0.f, n.z, -n.y));
    *b = vnorm(vcross(n, *t));
}

static float mis(float a, float b) {
    float t1 = powf(a, 2.f), t2 = powf(b, 2.f);
    return t1 / (t1 + t2);
}

/* FresnelDielectric (Src/Core/material.cu:121-142) */
static float fresnel_diel(float cosI, float etaI, float etaT) {
    cosI = clampf3(-1.0f, 1.0f, cosI);
    if (!(cosI > 0.0f)) {
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
static float fresnel_mat(const mat_t *m, vec wi, vec n) { return fresnel_diel(vdot(n, wi), 1.0f, m->ior); }

/* SampleDielectric (Src/Core/material.cu:155-192) */
static void sample_dielectric(const mat_t *m, vec wi, vec normal, vec *wo, float *pdf, vec *w, pcg *rng) {
    vec inc = vneg(vnorm(wi)), on = vnorm(normal);
    float etaI = 1.0f, etaT = m->ior;
    if (vdot(inc, on) > 0.0f) {
        on = vneg(on);
        float t = etaI;
        etaI = etaT;
        etaT = t;
    }
    float cosI = fmaxf(0.0f, -vdot(inc, on));
    float F = fresnel_diel(cosI, etaI, etaT);
    float r = U(rng);
    if (r < F) {
        *wo = vnorm(reflectv(inc, on));
        *pdf = fmaxf(F, 1e-6f);
        *w = V(1.f, 1.f, 1.f);
        return;
    }
    float eta = etaI / etaT;
    float c = fmaxf(0.0f, -vdot(inc, on));
    float s2 = eta * eta * fmaxf(0.0f, 1.0f - c * c);
    if (s2 >= 1.0f) {
        *wo = vnorm(reflectv(inc, on));
        *pdf = 1.0f;
        *w = V(1.f, 1.f, 1.f);
        return;
    }
    float ct = sqrtf(fmaxf(0.0f, 1.0f - s2));
    vec refr = vadd(vs(inc, eta), vs(on, eta * c - ct));
    *wo = vnorm(refr);
    *pdf = fmaxf(1.0f - F, 1e-6f);
    *w = lerpv(V(1.f, 1.f, 1.f), m->base, m->trans);
}

/* DistributionGGX (Src/Core/material.cu:96-107) */
static float ggx_d(float rough, vec wi, vec n, vec wo) {
    vec h = vnorm(vadd(wi, wo));
    float NdotH = fmaxf(vdot(n, h), 0.f);
    float a = rough * rough, a2 = a * a, NdotH2 = NdotH * NdotH;
    float den = (NdotH2 * (a2 - 1.f) + 1.f);
    double dd = PI_D * den * den;
    return (float)(a2 / dd);
}

static vec eval_pbr(const mat_t *m, vec wi, vec n, vec wo) {
    float NdotV = fmaxf(vdot(n, wi), 0.0f), NdotL = fmaxf(vdot(n, wo), 0.0f);
    if (NdotL <= 0.0f || NdotV <= 0.0f) return V(0.f, 0.f, 0.f);
    vec F0 = lerpv(V(0.04f, 0.04f, 0.04f), m->base, m->metal);
    float D = ggx_d(m->rough, wi, n, wo);
    float r = m->rough + 1.f, k = (r * r) / 8.f;
    float G = (NdotV / (NdotV * (1.f - k) + k)) * (NdotL / (NdotL * (1.f - k) + k));
    vec h = vnorm(vadd(wi, wo));
    float HdotV = fmaxf(vdot(h, wi), 0.f);
    float f5 = powf(1.f - HdotV, 5.f);
    vec F = vadd(F0, vs(vsub(V(1.f, 1.f, 1.f), F0), f5));
    vec spec = vdivs(vs(F, D * G), 4.0f * NdotV * NdotL + 0.0001f);
    vec kd = vs(vsub(V(1.f, 1.f, 1.f), F), 1.0f - m->metal);
    vec diff = (vdot(wi, n) > 0.f && vdot(wo, n) > 0.f) ? vdivs(vmul(kd, m->base), PI_F) : V(0.f, 0.f, 0.f);
    return vadd(diff, spec);
}

static float pbr_pspec(const mat_t *m, vec wi, vec n) {
    vec F0 = lerpv(V(0.04f, 0.04f, 0.04f), m->base, m->metal);
    float NdotV = fmaxf(vdot(n, wi), 0.0f);
    vec Fa = vadd(F0, vs(vsub(V(1.f, 1.f, 1.f), F0), powf(1.0f - NdotV, 5.0f)));
    float s = luminance(Fa), d = luminance(m->base) * (1.0f - m->metal);
    float p = fmaxf(s / (s + d), 1e-6f);
    return clampf3(0.01f, 0.99f, p);
}

static float pdf_pbr(const mat_t *m, vec wi, vec n, vec wo) {
    float ps = pbr_pspec(m, wi, n);
    float NdotL = fmaxf(vdot(n, wo), 0.0f);
    if (NdotL <= 0.0f) return 0.f;
    vec h = vnorm(vadd(wi, wo));
    float VdotH = fmaxf(vdot(wi, h), 1e-6f), NdotH = fmaxf(vdot(n, h), 1e-6f);
    float D = ggx_d(m->rough, wi, n, wo);
    float pspec = (D * NdotH) / (4.0f * VdotH);
    float pdiff = (float)((double)NdotL / PI_D);
    return ps * pspec + (1.0f - ps) * pdiff;
}

static float pdf_diffuse(vec n, vec wo) {
    float c = vdot(wo, n);
    return c > 0.f ? (float)((double)c / PI_D) : 0.f;
}

static void sample_diffuse(vec n, vec *wo, float *pdf, pcg *rng) {
    float t1 = U(rng), t2 = U(rng);
    float theta = (float)(0.5 * (double)acosf(1.f - 2.f * t1));
    float phi = (float)(2.0 * PI_D * (double)t2);
    float x = sinf(theta) * cosf(phi), y = sinf(theta) * sinf(phi), z = cosf(theta);
    *wo = local_to_world(V(x, y, z), n);
    *pdf = pdf_diffuse(n, *wo);
}

static void sample_pbr(const mat_t *m, vec wi, vec n, vec *wo, float *pdf, pcg *rng) {
    float ps = pbr_pspec(m, wi, n);
    float r1 = U(rng), r2 = U(rng), ch = U(rng);
    float phi = (float)(2.0 * PI_D * (double)r1);
    if (ch < ps) {
        float a = m->rough * m->rough;
        float cosT = sqrtf((1.0f - r2) / (1.0f + (a * a - 1.0f) * r2));
        float sinT = sqrtf(fmaxf(0.0f, 1.0f - cosT * cosT));
        vec hw = local_to_world(V(sinT * cosf(phi), sinT * sinf(phi), cosT), n);
        *wo = vnorm(reflectv(vneg(wi), hw));
    } else {
        float cosT = sqrtf(r2), sinT = sqrtf(1.0f - r2);
        *wo = local_to_world(V(sinT * cosf(phi), sinT * sinf(phi), cosT), n);
    }
    *pdf = pdf_pbr(m, wi, n, *wo);
}

static vec mat_eval(const mat_t *m, vec wi, vec n, vec wo) {
    if (m->type == M_PBR) return eval_pbr(m, wi, n, wo);
    if (m->type == M_DIELECTRIC) return V(0.f, 0.f, 0.f);
    return vdot(wo, n) > 0.f ? vdivs(m->base, PI_F) : V(0.f, 0.f, 0.f);
}
static float mat_pdf(const mat_t *m, vec wi, vec n, vec wo) {
    if (m->type == M_PBR) return pdf_pbr(m, wi, n, wo);
    if (m->type == M_DIELECTRIC) return 0.f;
    return pdf_diffuse(n, wo);
}
static void mat_sample(const mat_t *m, vec wi, vec n, vec *wo, float *pdf, pcg *rng) {
    if (m->type == M_PBR)
        sample_pbr(m, wi, n, wo, pdf, rng);
    else
        sample_diffuse(n, wo, pdf, rng);
}

static float burley(const mat_t *m, float r, int c) {
    float d = m->scatter[c];
    if (r < 1e-6f || d < 1e-6f) return 0.f;
    float e1 = expf(-r / d), e2 = expf(-r / (3 * d));
    return (float)((double)(e1 + e2) / (8.0 * PI_D * (double)d * (double)r));
}
static float burley_pdf(const mat_t *m, float r) { return (burley(m, r, 0) + burley(m, r, 1) + burley(m, r, 2)) / 3.f; }

/* ---- environment map -------------------------------------------------------- */

static void build_alias(const double *w, int n, float *out) {
    double sum = 0;
    for (int i = 0; i < n; ++i) sum += w[i];
    double *p = (double *)malloc(sizeof(double) * n);
    int *small = (int *)malloc(sizeof(int) * n), *large = (int *)malloc(sizeof(int) * n);
    int *alias = (int *)malloc(sizeof(int) * n);
    float *prob = (float *)malloc(sizeof(float) * n);
    int ns = 0, nl = 0;
    for (int i = 0; i < n; ++i) {
        p[i] = sum > 0 ? w[i] * n / sum : 1.0;
        if (p[i] < 1.0)
            small[ns++] = i;
        else
            large[nl++] = i;
        prob[i] = 1.f;
        alias[i] = i;
    }
    while (ns > 0 && nl > 0) {
        int s = small[--ns];
        int l = large[nl - 1];
        prob[s] = (float)p[s];
        alias[s] = l;
        p[l] = (p[l] + p[s]) - 1.0;
        if (p[l] < 1.0) {
            --nl;
            small[ns++] = l;
        }
    }
    for (int i = 0; i < n; ++i) {
        out[2 * i] = prob[i];
        memcpy(&out[2 * i + 1], &alias[i], 4);
    }
    /* remaining large/small items keep probability 1 */
    for (int k = 0; k < nl; ++k) out[2 * large[k]] = 1.f;
    for (int k = 0; k < ns; ++k) out[2 * small[k]] = 1.f;
    free(p);
    free(small);
    free(large);
    free(alias);
    free(prob);
}

/* HDRTexture::Load CDFs (Src/Core/texture.cu:40-83) + alias tables. */
void oracle_env_tables(const float *env, int W, int H, float *u, float *v, float *ra, float *ca) {
    for (int y = 0; y < H; ++y) {
        float vsum = 0.0f;
        for (int x = 0; x < W; ++x) {
            size_t i = (size_t)y * W + x;
            float lum = 0.2126f * env[4 * i] + 0.7152f * env[4 * i + 1] + 0.0722f * env[4 * i + 2];
            float theta = (float)((double)(((float)y + 0.5f) / (float)H) * PI_D);
            lum *= sinf(theta);
            vsum += lum;
            u[i] = vsum;
        }
        v[y] = vsum;
    }
    for (int y = 0; y < H; ++y) {
        float rs = v[y];
        for (int x = 0; x < W; ++x) {
            size_t i = (size_t)y * W + x;
            u[i] = rs > 0.0f ? u[i] / rs : 0.0f;
        }
    }
    for (int i = 1; i < H; ++i) v[i] += v[i - 1];
    float tot = v[H - 1];
    for (int i = 0; i < H; ++i) v[i] = tot > 0.0f ? v[i] / tot : 0.0f;
    double *w = (double *)malloc(sizeof(double) * (W > H ? W : H));
    for (int y = 0; y < H; ++y) w[y] = y == 0 ? v[0] : (double)(v[y] - v[y - 1]);
    build_alias(w, H, ra);
    for (int y = 0; y < H; ++y) {
        const float *row = u + (size_t)y * W;
        for (int x = 0; x < W; ++x) w[x] = x == 0 ? row[0] : (double)(row[x] - row[x - 1]);
        build_alias(w, W, ca + 2 * (size_t)y * W);
    }
    free(w);
}

static float env_sample_pdf(const ctx_t *c, float u, float v) {
    int W = c->s->env_w, H = c->s->env_h;
    u = clampf3(0.0f, 0.999999f, u);
    v = clampf3(0.0f, 0.999999f, v);
    int ui = (int)(u * W), vi = (int)(v * H);
    if (ui > W - 1) ui = W - 1;
    if (vi > H - 1) vi = H - 1;
    float prow = vi == 0 ? c->vcdf[0] : c->vcdf[vi] - c->vcdf[vi - 1];
    const float *row = c->ucdf + (size_t)vi * W;
    float pcol = ui == 0 ? row[0] : row[ui] - row[ui - 1];
    float p = prow * pcol;
    return p * W * H;
}

static void env_sample_uv(const ctx_t *c, pcg *rng, float *u, float *v) {
    int W = c->s->env_w, H = c->s->env_h;
    float rv = U(rng);
    float fy = rv * H;
    int y = (int)fy;
    if (y > H - 1) y = H - 1;
    if (fy - y >= c->ra[2 * y]) memcpy(&y, &c->ra[2 * y + 1], 4);
    float ru = U(rng);
    float fx = ru * W;
    int x = (int)fx;
    if (x > W - 1) x = W - 1;
    const float *e = c->ca + 2 * ((size_t)y * W + x);
    if (fx - x >= e[0]) memcpy(&x, &e[1], 4);
    *u = ((float)x + 0.5f) / (float)W;
    *v = ((float)y + 0.5f) / (float)H;
}

/* tex2D<float4> with linear filtering, wrap u / clamp v, normalised coords. */
static vec env_fetch(const ctx_t *c, float u, float v) {
    int W = c->s->env_w, H = c->s->env_h;
    float x = (u - floorf(u)) * W, y = v * H;
    float xb = x - 0.5f, yb = y - 0.5f;
    int i = (int)floorf(xb), j = (int)floorf(yb);
    float a = floorf((xb - i) * 256.f + 0.5f) / 256.f, b = floorf((yb - j) * 256.f + 0.5f) / 256.f;
    int i0 = ((i % W) + W) % W, i1 = (((i + 1) % W) + W) % W;
    int j0 = j < 0 ? 0 : (j >= H ? H - 1 : j), j1 = j + 1 < 0 ? 0 : (j + 1 >= H ? H - 1 : j + 1);
    const float *e = c->s->env;
    const float *t00 = e + 4 * ((size_t)j0 * W + i0), *t10 = e + 4 * ((size_t)j0 * W + i1);
    const float *t01 = e + 4 * ((size_t)j1 * W + i0), *t11 = e + 4 * ((size_t)j1 * W + i1);
    float r[3];
    for (int k = 0; k < 3; ++k)
        r[k] = (1 - a) * (1 - b) * t00[k] + a * (1 - b) * t10[k] + (1 - a) * b * t01[k] + a * b * t11[k];
    return V(r[0], r[1], r[2]);
}

static vec env_emission(const ctx_t *c, vec wi) {
    float theta = acosf(wi.y);
    float phi = atan2f(wi.x, wi.z);
    if (phi < 0) phi = (float)((double)phi + 2.0 * PI_D);
    float u = (float)((double)phi / (2.0 * PI_D));
    float v = (float)((double)theta / PI_D);
    return env_fetch(c, u, v);
}

/* ---- lights ----------------------------------------------------------------- */
typedef struct { vec p, n; } lsample;

static void light_sample_point(const ctx_t *c, int lid, pcg *rng, lsample *ls) {
    const float *L = c->s->lights + 8 * lid;
    if ((int)L[0] == 0) { /* area */
        const float *m = c->s->meshes + 8 * (int)L[1];
        int count = (int)m[3], start = (int)m[2];
        int t = (int)(U(rng) * count);
        if (t == count) t = count - 1;
        float u = U(rng), v = U(rng);
        if (u + v > 1) {
            u = 1 - u;
            v = 1 - v;
        }
        const float *tv = c->s->verts + 9 * (size_t)(start + t);
        vec v0 = L3(tv), v1 = L3(tv + 3), v2 = L3(tv + 6);
        float w = 1 - u - v;
        ls->p = vadd(vadd(vs(v0, w), vs(v1, u)), vs(v2, v));
        ls->n = vnorm(vcross(vsub(v1, v0), vsub(v2, v0)));
    } else { /* env */
        float u, v;
        env_sample_uv(c, rng, &u, &v);
        float theta = (float)((double)(u * 2.f) * PI_D);
        float phi = acosf(1.f - 2.f * v);
        vec dir = V(sinf(phi) * sinf(theta), cosf(phi), sinf(phi) * cosf(theta));
        ls->p = vadd(V(c->center[0], c->center[1], c->center[2]), vs(vs(dir, 2.f), c->diag));
        ls->n = vneg(dir);
    }
}

static float light_pdf(const ctx_t *c, int lid, vec origin, vec lp, vec ln) {
    const float *L = c->s->lights + 8 * lid;
    if ((int)L[0] == 0) {
        vec wi = vnorm(vsub(origin, lp));
        float d2 = vsq(vsub(origin, lp));
        float cc = fmaxf(vdot(ln, wi), 1e-6f);
        return d2 / (c->s->meshes[8 * (int)L[1] + 4] * cc);
    }
    vec dir = vnorm(vsub(lp, origin));
    float theta = acosf(dir.y);
    float phi = atan2f(dir.x, dir.z);
    if (phi < 0) phi = (float)((double)phi + 2.0 * PI_D);
    float u = (float)((double)phi / (2.0 * PI_D));
    float v = (float)(1.0 - (double)theta / PI_D);
    return env_sample_pdf(c, u, v);
}

static vec light_emission(const ctx_t *c, int lid, vec wi) {
    const float *L = c->s->lights + 8 * lid;
    if ((int)L[0] == 2) return env_emission(c, wi);
    return L3(L + 2);
}

/* ---- geometry ------------------------------------------------------------- */
typedef struct {
    int prim;
    float t, b1, b2;
} hit_t;

static hit_t closest(const ctx_t *c, vec o, vec d, float tmax) {
    float oo[3] = {o.x, o.y, o.z}, dd[3] = {d.x, d.y, d.z};
    hit_t h;
    h.prim = oracle_closest_brute(c->s->verts, c->s->ntris, oo, dd, tmax, &h.t, &h.b1, &h.b2);
    return h;
}

static vec hit_point(const ctx_t *c, hit_t h) {
    const float *v = c->s->verts + 9 * (size_t)h.prim;
    float b0 = (1.f - h.b1) - h.b2;
    return vadd(vadd(vs(L3(v), b0), vs(L3(v + 3), h.b1)), vs(L3(v + 6), h.b2));
}

static vec face_normal(const ctx_t *c, int prim) {
    const float *v = c->s->verts + 9 * (size_t)prim;
    return vnorm(vcross(vsub(L3(v + 3), L3(v)), vsub(L3(v + 6), L3(v))));
}

static int visible(const ctx_t *c, vec hp, vec hn, vec lp, vec ln) {
    float q[12] = {hp.x, hp.y, hp.z, hn.x, hn.y, hn.z, lp.x, lp.y, lp.z, ln.x, ln.y, ln.z};
    return oracle_visible_one(c->s->verts, c->s->ntris, q);
}

/* ---- the path ---------------------------------------------------------------- */
typedef struct {
    vec o, d, w, dc, ic;
    float pdf;
    int first, spec;
    pcg rng;
} path_t;

static int sample_light(const ctx_t *c, pcg *rng, int *lid, lsample *ls, float *sel) {
    int n = c->s->nlights;
    if (n == 0) return 0;
    *lid = (int)(U(rng) * n);
    if (*lid == n) *lid = n - 1;
    *sel = 1.0f / n;
    light_sample_point(c, *lid, rng, ls);
    return 1;
}

/* PathTracing (Src/Core/renderer.cuh:170-422); returns 1 to continue. */
static int path_step(const ctx_t *c, int bounce, path_t *ps, hit_t h) {
    const oracle_scene *s = c->s;
    const int rr_on = bounce >= s->rr_start;
    int prim = h.prim;
    vec hitPoint = hit_point(c, h);
    vec infoNormal = face_normal(c, prim);
    const float *nn = s->normals + 9 * (size_t)prim;
    float b0 = (1.f - h.b1) - h.b2;
    vec sn = vnorm(vadd(vadd(vs(L3(nn), b0), vs(L3(nn + 3), h.b1)), vs(L3(nn + 6), h.b2)));
    const float *M = s->meshes + 8 * s->prim_mesh[prim];
    mat_t mat = get_mat(c, (int)M[0]);
    {   /* diffuse texture (Texture::Sample, texture.cu:243-252): clamped uv, v flipped */
        int ti = (int)s->materials[16 * (int)M[0] + 14];
        if (ti >= 0 && ti < s->ntex && (mat.type == M_DIFFUSE || mat.type == M_PBR || mat.type == M_SUBSURFACE)) {
            const float *uv = s->uvs + 6 * (size_t)prim;
            float tu = (b0 * uv[0] + h.b1 * uv[2]) + h.b2 * uv[4];
            float tv = (b0 * uv[1] + h.b1 * uv[3]) + h.b2 * uv[5];
            tu = tu < 0.f ? 0.f : (tu > 0.999999f ? 0.999999f : tu);
            tv = tv < 0.f ? 0.f : (tv > 0.999999f ? 0.999999f : tv);
            mat.base = tex_fetch(c, ti, tu, 1.0f - tv);
        }
    }
    int mesh_light = (int)M[1];

    vec geomNormal = vnorm(infoNormal);
    vec hitNormal = (double)vsq(sn) > EPS_D ? vnorm(sn) : geomNormal;
    if (vdot(hitNormal, geomNormal) < 0.f) hitNormal = vneg(hitNormal);
    vec wo = vneg(ps->d);

    if (mat.type == M_LIGHT) {
        if (ps->first) {
            ps->dc = vadd(ps->dc, mat.ke);
            ps->first = 0;
            return 0;
        } else if (ps->spec) {
            ps->ic = vadd(ps->ic, vmul(ps->w, mat.ke));
        } else {
            float pdfLight = 0.f;
            if (mesh_light >= 0) pdfLight = light_pdf(c, mesh_light, ps->o, hitPoint, infoNormal);
            float mw = mis(ps->pdf, pdfLight);
            ps->ic = vadd(ps->ic, vs(vmul(ps->w, mat.ke), mw));
        }
        return 0;
    }
    if (mat.type == M_DIELECTRIC) {
        vec dwi, dw;
        float dp = 1.0f;
        sample_dielectric(&mat, wo, hitNormal, &dwi, &dp, &dw, &ps->rng);
        ps->pdf = dp;
        ps->o = vadd(hitPoint, vs(dwi, 1e-4f));
        ps->d = dwi;
        ps->w = vmul(ps->w, dw);
        float p = U(&ps->rng);
        if (rr_on && p > s->rr) return 0;
        if (rr_on) ps->w = vdivs(ps->w, s->rr);
        ps->first = 0;
        ps->spec = 1;
        return 1;
    }
    if (mat.type != M_SUBSURFACE) {
        int lid;
        lsample ls;
        float sel;
        if (sample_light(c, &ps->rng, &lid, &ls, &sel)) {
            vec dirWi = vnorm(vsub(ls.p, hitPoint));
            float pdfLight = light_pdf(c, lid, hitPoint, ls.p, ls.n);
            pdfLight *= sel;
            float cosT = vdot(hitNormal, dirWi);
            vec brdf = mat_eval(&mat, wo, hitNormal, dirWi);
            vec dirL = vdivs(vs(vmul(light_emission(c, lid, dirWi), brdf), cosT), pdfLight);
            float pdfB = mat_pdf(&mat, wo, hitNormal, dirWi);
            float mw = mis(pdfLight, pdfB);
            vec C = vs(vmul(ps->w, dirL), mw);
            if ((C.x != 0.f || C.y != 0.f || C.z != 0.f) && visible(c, hitPoint, infoNormal, ls.p, ls.n)) {
                if (ps->first)
                    ps->dc = vadd(ps->dc, C);
                else
                    ps->ic = vadd(ps->ic, C);
            }
        }
        vec iwi;
        float ipdf;
        mat_sample(&mat, wo, hitNormal, &iwi, &ipdf, &ps->rng);
        vec brdf = mat_eval(&mat, wo, hitNormal, iwi);
        ps->pdf = ipdf;
        ps->o = hitPoint;
        ps->d = iwi;
        float cc = vdot(hitNormal, iwi);
        if (!((double)ipdf < EPS_D || cc < 0))
            ps->w = vdivs(vs(vmul(ps->w, brdf), cc), ipdf);
        else
            return 0;
    } else {
        float FIn = fresnel_mat(&mat, wo, hitNormal);
        float reflectProb = clampf3(0.02f, 0.98f, FIn);
        float transmitProb = fmaxf(1.f - reflectProb, 1e-6f);
        float ev = U(&ps->rng);
        if (ev < reflectProb) {
            vec rd;
            if (mat.rough > 1e-3f) {
                float r1 = U(&ps->rng), r2 = U(&ps->rng);
                float a = fmaxf(mat.rough * mat.rough, 0.02f);
                float phi = (float)(2.0 * PI_D * (double)r1);
                float cosT = sqrtf((1.0f - r2) / (1.0f + (a * a - 1.0f) * r2));
                float sinT = sqrtf(fmaxf(0.0f, 1.0f - cosT * cosT));
                vec hw = local_to_world(V(sinT * cosf(phi), sinT * sinf(phi), cosT), hitNormal);
                rd = vnorm(reflectv(vneg(wo), hw));
                if (vdot(rd, hitNormal) <= 0.0f) rd = vnorm(reflectv(vneg(wo), hitNormal));
            } else {
                rd = vnorm(reflectv(vneg(wo), hitNormal));
            }
            ps->o = vadd(hitPoint, vs(rd, 1e-4f));
            ps->d = rd;
            ps->w = vdivs(vmul(ps->w, V(FIn, FIn, FIn)), reflectProb);
            ps->pdf = 1.0f;
            float p = U(&ps->rng);
            if (rr_on && p > s->rr) return 0;
            if (rr_on) ps->w = vdivs(ps->w, s->rr);
            ps->first = 0;
            ps->spec = 1;
            return 1;
        }
        float distance;
        int ch = (int)(U(&ps->rng) * 3);
        ch = (int)clampf3(0.f, 2.f, (float)ch);
        float d = mat.scatter[ch];
        if (d < 1e-6f) {
            distance = 0.f;
        } else {
            float r1 = U(&ps->rng);
            if (r1 < 0.5f) {
                r1 = r1 * 2.f;
                distance = -d * logf(1.f - r1);
            } else {
                r1 = (r1 - 0.5f) * 2.f;
                distance = -3.f * d * logf(1.f - r1);
            }
        }
        float angle = (float)((double)(U(&ps->rng) * 2.f) * PI_D);
        /* ProbeOutgongingPoint (Src/Core/material.cu:405-441) */
        vec pn = vnorm(geomNormal), t, b;
        create_onb(pn, &t, &b);
        vec outP = vadd(hitPoint, vs(vadd(vs(t, cosf(angle)), vs(b, sinf(angle))), distance));
        float ro = fmaxf(distance, 1e-3f), tmax = fmaxf(distance * 2.f, 1e-2f);
        hit_t fh = closest(c, vadd(outP, vs(pn, ro)), vneg(pn), tmax);
        hit_t bh = closest(c, vsub(outP, vs(pn, ro)), pn, tmax);
        const hit_t *use = 0;
        if (fh.prim >= 0 && bh.prim >= 0)
            use = fh.t <= bh.t ? &fh : &bh;
        else if (fh.prim >= 0)
            use = &fh;
        else if (bh.prim >= 0)
            use = &bh;
        vec outN;
        if (use) {
            outP = hit_point(c, *use);
            outN = face_normal(c, use->prim);
        } else {
            outP = hitPoint;
            outN = pn;
        }
        float sd = vlen(vsub(outP, hitPoint));
        float spatialPdf = sd < 1e-6f ? 0.f : burley_pdf(&mat, sd);
        if ((double)spatialPdf < EPS_D) return 0;
        vec prof = V(0.f, 0.f, 0.f);
        if (!(sd < 1e-6f)) prof = vdivs(vmul(mat.base, V(burley(&mat, sd, 0), burley(&mat, sd, 1), burley(&mat, sd, 2))), PI_F);
        ps->w = vdivs(vmul(vmul(ps->w, V(1.f - FIn, 1.f - FIn, 1.f - FIn)), prof), transmitProb * spatialPdf);
        int lid;
        lsample ls;
        float sel;
        if (sample_light(c, &ps->rng, &lid, &ls, &sel)) {
            vec dirWi = vnorm(vsub(ls.p, outP));
            float ftout = 1 - fresnel_mat(&mat, dirWi, outN);
            float pdfLight = light_pdf(c, lid, outP, ls.p, ls.n);
            pdfLight *= sel;
            float cosT = vdot(outN, dirWi);
            if (cosT > 0.f && (double)pdfLight > EPS_D) {
                vec dirL = vdivs(vs(vmul(light_emission(c, lid, dirWi), vdivs(V(1.f, 1.f, 1.f), PI_F)), cosT), pdfLight);
                float pdfB = (float)((double)cosT / PI_D);
                float mw = mis(pdfLight, pdfB);
                vec C = vs(vs(vmul(ps->w, dirL), mw), ftout);
                if ((C.x != 0.f || C.y != 0.f || C.z != 0.f) && visible(c, outP, outN, ls.p, ls.n)) {
                    if (ps->first)
                        ps->dc = vadd(ps->dc, C);
                    else
                        ps->ic = vadd(ps->ic, C);
                }
            }
        }
        vec odir;
        float opdf;
        sample_diffuse(outN, &odir, &opdf, &ps->rng);
        float cosOut = vdot(outN, odir);
        float ftout = 1 - fresnel_mat(&mat, odir, outN);
        if ((double)opdf < EPS_D || cosOut < 0.f) return 0;
        ps->o = vadd(outP, vs(outN, 1e-4f));
        ps->d = odir;
        ps->w = vs(ps->w, ftout);
        ps->pdf = opdf;
    }
    float p = U(&ps->rng);
    if (rr_on && p > s->rr) return 0;
    if (rr_on) ps->w = vdivs(ps->w, s->rr);
    ps->first = 0;
    ps->spec = 0;
    return 1;
}

typedef struct {
    const ctx_t *c;
    int first_sample, spp;
    float *direct, *indirect, *sumsq;
} job_t;

static void pixel_body(long pixel, void *j_) {
    const job_t *j = (const job_t *)j_;
    const ctx_t *c = j->c;
    const oracle_scene *s = c->s;
    int px = (int)(pixel % s->width), py = (int)(pixel / s->width);
    for (int k = 0; k < j->spp; ++k) {
        path_t ps;
        ps.rng = pcg_seed(s->seed, (unsigned)pixel, (unsigned)(j->first_sample + k));
        float u0 = U(&ps.rng), u1 = U(&ps.rng);
        vec pp = vadd(vadd(L3(s->cam_ld), vs(L3(s->cam_du), (float)px + u0)), vs(L3(s->cam_dv), (float)py + u1));
        ps.o = L3(s->cam_pos);
        ps.d = vnorm(vsub(pp, ps.o));
        ps.w = V(1.f, 1.f, 1.f);
        ps.dc = ps.ic = V(0.f, 0.f, 0.f);
        ps.pdf = 0.f;
        ps.first = 1;
        ps.spec = 0;
        int done = 0;
        for (int b = 0; b < s->max_bounces && !done; ++b) {
            hit_t h = closest(c, ps.o, ps.d, 1e8f);
            if (h.prim < 0) {
                if (s->env_light >= 0) {
                    vec bg = env_emission(c, ps.d);
                    if (ps.first)
                        ps.dc = vadd(ps.dc, vmul(ps.w, bg));
                    else
                        ps.ic = vadd(ps.ic, vmul(ps.w, bg));
                }
                done = 1;
                break;
            }
            if (!path_step(c, b, &ps, h)) done = 1;
        }
        if (!done) continue; /* alive after max_bounces: dropped */
        float *D = j->direct + 4 * pixel, *I = j->indirect + 4 * pixel;
        D[0] += ps.dc.x;
        D[1] += ps.dc.y;
        D[2] += ps.dc.z;
        I[0] += ps.ic.x;
        I[1] += ps.ic.y;
        I[2] += ps.ic.z;
        if (j->sumsq) {
            float *Q = j->sumsq + 4 * pixel;
            float r = ps.dc.x + ps.ic.x, g = ps.dc.y + ps.ic.y, bb = ps.dc.z + ps.ic.z;
            Q[0] += r * r;
            Q[1] += g * g;
            Q[2] += bb * bb;
            Q[3] += 1.f;
        }
    }
}

void oracle_render(const oracle_scene *s, int first_sample, int spp, float *direct, float *indirect, float *sumsq,
                   int nthreads) {
    ctx_t c;
    memset(&c, 0, sizeof(c));
    c.s = s;
    if (s->env_light >= 0) {
        size_t W = s->env_w, H = s->env_h;
        c.ucdf = (float *)malloc(sizeof(float) * W * H);
        c.vcdf = (float *)malloc(sizeof(float) * H);
        c.ra = (float *)malloc(sizeof(float) * 2 * H);
        c.ca = (float *)malloc(sizeof(float) * 2 * W * H);
        oracle_env_tables(s->env, (int)W, (int)H, c.ucdf, c.vcdf, c.ra, c.ca);
    }
    float lo[3] = {3.4e38f, 3.4e38f, 3.4e38f}, hi[3] = {-3.4e38f, -3.4e38f, -3.4e38f};
    for (long i = 0; i < 3 * s->ntris; ++i)
        for (int k = 0; k < 3; ++k) {
            float x = s->verts[3 * i + k];
            lo[k] = x < lo[k] ? x : lo[k];
            hi[k] = x > hi[k] ? x : hi[k];
        }
    float e[3];
    for (int k = 0; k < 3; ++k) {
        c.center[k] = (lo[k] + hi[k]) * 0.5f;
        e[k] = hi[k] - lo[k];
    }
    c.diag = sqrtf(e[0] * e[0] + (e[1] * e[1] + e[2] * e[2]));
    job_t j = {&c, first_sample, spp, direct, indirect, sumsq};
    par_for((long)s->width * s->height, 16, nthreads, pixel_body, &j);
    free(c.ucdf);
    free(c.vcdf);
    free(c.ra);
    free(c.ca);
}
