// Harness around the reference's own code (DarrenChen-CN/CudaRayTracer),
// compiled as host C++ from the reference tree by oracle/Makefile into
// oracle/_ref/libcrtref.so. It exposes the reference's closest-hit query
// (BVH::BVH + BVH::IsIntersect, Src/Core/bvh.cu:9,253) and its visibility
// predicate (Light::Visible, Src/Core/light.cu:5) behind a small C ABI so
// tests can pin the CPU restatement (oracle/crt_oracle.c) and the CUDA
// kernels against the reference itself. Test infrastructure only.
#include "bvh.h"
#include "light.h"
#include "sampler.h"
#include <atomic>
#include <thread>
#include <cstring>
#include <cstdio>
#include <vector>

// Host replacement for Src/Core/sampler.cu, whose constructor launches a
// kernel: one XORWOW state per index, curand_init(seed, idx, 0)
// (Src/Core/sampler.cu:29-36), uniform draws as in :17-27.
Sampler::Sampler(int seed_, int numPixels_) : seed(seed_), numPixels(numPixels_) {
    devStates = new curandState[numPixels_];
    for (int i = 0; i < numPixels_; ++i) curand_init(seed_, i, 0, &devStates[i]);
}
Sampler::~Sampler() {
    delete[] devStates;
    devStates = nullptr;
}
float Sampler::Get1D(int idx) { return curand_uniform(&devStates[idx]); }
Vec2f Sampler::Get2D(int idx) {
    float u = curand_uniform(&devStates[idx]);
    float v = curand_uniform(&devStates[idx]);
    return Vec2f(u, v);
}

namespace {
// Dynamic parallel-for over [0, n) on std::thread (no OpenMP runtime here).
template <class F>
void parallel_for(long n, int nthreads, F &&body) {
    if (nthreads <= 0) nthreads = (int)std::thread::hardware_concurrency();
    if (nthreads <= 0) nthreads = 1;
    std::atomic<long> next(0);
    const long chunk = 256;
    auto work = [&] {
        for (;;) {
            long b = next.fetch_add(chunk);
            if (b >= n) break;
            long e = b + chunk < n ? b + chunk : n;
            for (long i = b; i < e; ++i) body(i);
        }
    };
    std::vector<std::thread> th;
    for (int t = 1; t < nthreads; ++t) th.emplace_back(work);
    work();
    for (auto &x : th) x.join();
}

struct RefScene {
    std::vector<Triangle> tris;
    BVH *bvh = nullptr;
};

// Triangle with primitive index in meshID and texture coordinates
// (0,0), (1,0), (0,1) so the interpolated texCoord returns (b1, b2).
Triangle make_triangle(const float *v, int prim) {
    Vertex a, b, c;
    a.position = Vec3f(v[0], v[1], v[2]);
    b.position = Vec3f(v[3], v[4], v[5]);
    c.position = Vec3f(v[6], v[7], v[8]);
    Vec3f n = (b.position - a.position).cross(c.position - a.position).normalized();
    a.normal = b.normal = c.normal = n;
    a.texCoord = Vec2f(0.f, 0.f);
    b.texCoord = Vec2f(1.f, 0.f);
    c.texCoord = Vec2f(0.f, 1.f);
    a.barycentricCoords = Vec3f(1, 0, 0);
    b.barycentricCoords = Vec3f(0, 1, 0);
    c.barycentricCoords = Vec3f(0, 0, 1);
    return Triangle(a, b, c, prim);
}
}  // namespace

extern "C" {

void *ref_scene_from_triangles(const float *verts, long n) {
    auto *s = new RefScene();
    s->tris.reserve(n);
    for (long i = 0; i < n; ++i) s->tris.push_back(make_triangle(verts + 9 * i, (int)i));
    std::vector<Triangle> work(s->tris);
    s->bvh = new BVH(work.data(), (int)n, 4, SAH);
    // Host copies stand in for the device arrays CreateBVH would upload.
    s->bvh->orderedTriangles = s->bvh->hostOrderedTriangles;
    s->bvh->linearNodes = s->bvh->hostLinearNodes;
    fflush(stdout);
    return s;
}

void ref_scene_free(void *h) {
    auto *s = static_cast<RefScene *>(h);
    if (!s) return;
    s->bvh->orderedTriangles = nullptr;
    s->bvh->linearNodes = nullptr;
    delete s->bvh;
    delete s;
}

void ref_bvh_stats(void *h, int *nodes, int *depth) {
    auto *s = static_cast<RefScene *>(h);
    *nodes = s->bvh->totalNode;
    *depth = s->bvh->maxDepth;
}

// rays: n x 8 floats (o, tmin, d, tmax); out: n x 4 (t, prim bits, b1, b2).
void ref_trace_closest(void *h, const float *rays, long n, float *out, int nthreads) {
    auto *s = static_cast<RefScene *>(h);
    parallel_for(n, nthreads, [&](long i) {
        const float *r = rays + 8 * i;
        Ray ray(Vec3f(r[0], r[1], r[2]), Vec3f(r[4], r[5], r[6]));
        IntersectionInfo info;
        info.hitTime = FLOATMAX;
        info.hit = false;
        bool hit = s->bvh->IsIntersect(ray, info, r[3], r[7]);
        float *o = out + 4 * i;
        int prim = hit ? info.meshID : -1;
        o[0] = info.hitTime;
        std::memcpy(&o[1], &prim, 4);
        o[2] = hit ? info.texCoord(0) : 0.f;
        o[3] = hit ? info.texCoord(1) : 0.f;
    });
}

// q: n x 12 floats (p, n, light p, light n); occluded[i] = !Visible.
void ref_visible(void *h, const float *q, long n, unsigned char *occluded, int nthreads) {
    auto *s = static_cast<RefScene *>(h);
    parallel_for(n, nthreads, [&](long i) {
        const float *a = q + 12 * i;
        IntersectionInfo info;
        info.hitPoint = Vec3f(a[0], a[1], a[2]);
        info.normal = Vec3f(a[3], a[4], a[5]);
        TriangleSampleInfo li;
        li.position = Vec3f(a[6], a[7], a[8]);
        li.normal = Vec3f(a[9], a[10], a[11]);
        Light light;
        occluded[i] = light.Visible(info, li, s->bvh) ? 0 : 1;
    });
}

}  // extern "C"
