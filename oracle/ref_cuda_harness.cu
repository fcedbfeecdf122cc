// Headless CUDA build of the reference's traversal (DarrenChen-CN/
// CudaRayTracer): its BVH (host build + CreateBVH upload, Src/Core/bvh.cu:9,
// 308) and its device closest-hit query and visibility test
// (BVH::IsIntersect, Src/Core/bvh.cu:253; Light::Visible,
// Src/Core/light.cu:5), compiled with nvcc for sm_100a from the reference
// tree by oracle/Makefile (upstream flags: -O3, separable compilation).
// One thread per ray, as the reference's IntersectionKernel
// (Src/Core/renderer.cuh:132-163) launches it. Used to time the reference's
// GPU traversal beside the product kernels; test/bench infrastructure only.
#include "bvh.h"
#include "light.h"
#include <cstdio>
#include <vector>

namespace {
struct RefCudaScene {
    BVH *host = nullptr;
    BVH *dev = nullptr;
};

__global__ void k_ref_trace(BVH *bvh, const float4 *rays, long n, float4 *out) {
    long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 a = rays[2 * i], b = rays[2 * i + 1];
    Ray ray(Vec3f(a.x, a.y, a.z), Vec3f(b.x, b.y, b.z));
    IntersectionInfo info;
    info.hitTime = FLOATMAX;
    info.hit = false;
    bool hit = bvh->IsIntersect(ray, info, a.w, b.w);
    int prim = hit ? info.meshID : -1;
    out[i] = make_float4(info.hitTime, __int_as_float(prim), hit ? info.texCoord(0) : 0.f,
                         hit ? info.texCoord(1) : 0.f);
}

__global__ void k_ref_visible(BVH *bvh, const float *q, long n, unsigned char *occ) {
    long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float *a = q + 12 * i;
    IntersectionInfo info;
    info.hitPoint = Vec3f(a[0], a[1], a[2]);
    info.normal = Vec3f(a[3], a[4], a[5]);
    TriangleSampleInfo li;
    li.position = Vec3f(a[6], a[7], a[8]);
    li.normal = Vec3f(a[9], a[10], a[11]);
    Light light;
    occ[i] = light.Visible(info, li, bvh) ? 0 : 1;
}
}  // namespace

extern "C" {

void *refcuda_scene_from_triangles(const float *verts, long n) {
    std::vector<Triangle> tris;
    tris.reserve(n);
    for (long i = 0; i < n; ++i) {
        const float *v = verts + 9 * i;
        Vertex a, b, c;
        a.position = Vec3f(v[0], v[1], v[2]);
        b.position = Vec3f(v[3], v[4], v[5]);
        c.position = Vec3f(v[6], v[7], v[8]);
        Vec3f nrm = (b.position - a.position).cross(c.position - a.position).normalized();
        a.normal = b.normal = c.normal = nrm;
        a.texCoord = Vec2f(0.f, 0.f);
        b.texCoord = Vec2f(1.f, 0.f);
        c.texCoord = Vec2f(0.f, 1.f);
        tris.push_back(Triangle(a, b, c, (int)i));
    }
    auto *s = new RefCudaScene();
    s->host = new BVH(tris.data(), (int)n, 4, SAH);
    cudaMalloc(&s->dev, sizeof(BVH));
    CreateBVH(s->host, s->dev);
    fflush(stdout);
    return s;
}

void refcuda_scene_free(void *h) {
    auto *s = static_cast<RefCudaScene *>(h);
    if (!s) return;
    cudaFree(s->dev);
    delete s->host;  // frees its device arrays too
    delete s;
}

int refcuda_trace(void *h, const float *d_rays, long n, float *d_out, void *stream) {
    auto *s = static_cast<RefCudaScene *>(h);
    if (n <= 0) return 0;
    k_ref_trace<<<(unsigned)((n + 127) / 128), 128, 0, (cudaStream_t)stream>>>(
        s->dev, (const float4 *)d_rays, n, (float4 *)d_out);
    return (int)cudaGetLastError();
}

int refcuda_visible(void *h, const float *d_q, long n, unsigned char *d_occ, void *stream) {
    auto *s = static_cast<RefCudaScene *>(h);
    if (n <= 0) return 0;
    k_ref_visible<<<(unsigned)((n + 127) / 128), 128, 0, (cudaStream_t)stream>>>(s->dev, d_q, n, d_occ);
    return (int)cudaGetLastError();
}

}  // extern "C"
