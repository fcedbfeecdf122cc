// Host stand-ins for the CUDA runtime calls the reference's sources make, so
// its scene, texture and BVH code runs unmodified on the CPU inside
// oracle/_ref: device allocations become host allocations, copies become
// memcpy, and texture objects fetch from host arrays with CUDA's documented
// addressing (wrap / clamp, normalised or texel coordinates) and filtering
// (nearest, or bilinear with 8-bit fractional weights; CUDA C Programming
// Guide, "Texture Fetching"). Test infrastructure only.
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <mutex>
#include <vector>

struct cudaArray {
    cudaChannelFormatDesc desc;
    size_t w, h, elem;
    std::vector<unsigned char> data;
};

namespace {
struct HostTex {
    cudaArray *arr;
    cudaTextureDesc td;
};
std::mutex g_mu;
std::vector<HostTex> g_tex;  // handle = index + 1

size_t elem_size(const cudaChannelFormatDesc &d) { return (size_t)(d.x + d.y + d.z + d.w) / 8; }

float frac_fixed8(float f) { return std::floor(f * 256.f + 0.5f) / 256.f; }

int address(int i, int n, cudaTextureAddressMode m) {
    if (m == cudaAddressModeWrap) {
        i %= n;
        return i < 0 ? i + n : i;
    }
    return i < 0 ? 0 : (i >= n ? n - 1 : i);
}

// Texel fetch as 4 floats (float / normalised uchar / raw ushort).
void texel(const HostTex &t, int x, int y, float out[4]) {
    const cudaArray *a = t.arr;
    const unsigned char *p = a->data.data() + ((size_t)y * a->w + x) * a->elem;
    if (a->desc.f == cudaChannelFormatKindFloat) {
        std::memcpy(out, p, 16);
    } else if (a->elem == 4) {
        for (int k = 0; k < 4; ++k)
            out[k] = t.td.readMode == cudaReadModeNormalizedFloat ? p[k] / 255.f : (float)p[k];
    } else {
        unsigned short s[4];
        std::memcpy(s, p, 8);
        for (int k = 0; k < 4; ++k) out[k] = (float)s[k];
    }
}

void fetch(cudaTextureObject_t obj, float x, float y, float out[4]) {
    HostTex t;
    {
        std::lock_guard<std::mutex> g(g_mu);
        t = g_tex.at(obj - 1);
    }
    const int W = (int)t.arr->w, H = (int)t.arr->h;
    cudaTextureAddressMode mx = t.td.addressMode[0], my = t.td.addressMode[1];
    if (t.td.normalizedCoords) {
        if (mx == cudaAddressModeWrap) x = x - std::floor(x);
        if (my == cudaAddressModeWrap) y = y - std::floor(y);
        x *= W;
        y *= H;
    }
    if (t.td.filterMode == cudaFilterModePoint) {
        texel(t, address((int)std::floor(x), W, mx), address((int)std::floor(y), H, my), out);
        return;
    }
    float xb = x - 0.5f, yb = y - 0.5f;
    int i = (int)std::floor(xb), j = (int)std::floor(yb);
    float a = frac_fixed8(xb - i), b = frac_fixed8(yb - j);
    float t00[4], t10[4], t01[4], t11[4];
    texel(t, address(i, W, mx), address(j, H, my), t00);
    texel(t, address(i + 1, W, mx), address(j, H, my), t10);
    texel(t, address(i, W, mx), address(j + 1, H, my), t01);
    texel(t, address(i + 1, W, mx), address(j + 1, H, my), t11);
    for (int k = 0; k < 4; ++k)
        out[k] = (1 - a) * (1 - b) * t00[k] + a * (1 - b) * t10[k] + (1 - a) * b * t01[k] + a * b * t11[k];
}
}  // namespace

template <>
float4 tex2D<float4>(cudaTextureObject_t obj, float x, float y) {
    float v[4];
    fetch(obj, x, y, v);
    return make_float4(v[0], v[1], v[2], v[3]);
}

template <>
ushort4 tex2D<ushort4>(cudaTextureObject_t obj, float x, float y) {
    float v[4];
    fetch(obj, x, y, v);
    return make_ushort4((unsigned short)v[0], (unsigned short)v[1], (unsigned short)v[2], (unsigned short)v[3]);
}

extern "C" {

cudaError_t cudaMalloc(void **p, size_t n) {
    *p = std::calloc(1, n ? n : 1);
    return *p ? cudaSuccess : cudaErrorMemoryAllocation;
}
cudaError_t cudaFree(void *p) {
    std::free(p);
    return cudaSuccess;
}
cudaError_t cudaMemcpy(void *dst, const void *src, size_t n, cudaMemcpyKind) {
    std::memmove(dst, src, n);
    return cudaSuccess;
}
cudaError_t cudaMemset(void *dst, int v, size_t n) {
    std::memset(dst, v, n);
    return cudaSuccess;
}
cudaError_t cudaDeviceSynchronize(void) { return cudaSuccess; }
cudaError_t cudaGetLastError(void) { return cudaSuccess; }
const char *cudaGetErrorString(cudaError_t) { return "host runtime"; }

struct cudaChannelFormatDesc cudaCreateChannelDesc(int x, int y, int z, int w, enum cudaChannelFormatKind f) {
    cudaChannelFormatDesc d;
    d.x = x;
    d.y = y;
    d.z = z;
    d.w = w;
    d.f = f;
    return d;
}

cudaError_t cudaMallocArray(cudaArray_t *arr, const struct cudaChannelFormatDesc *desc, size_t w, size_t h,
                            unsigned int) {
    auto *a = new cudaArray();
    a->desc = *desc;
    a->w = w;
    a->h = h ? h : 1;
    a->elem = elem_size(*desc);
    a->data.assign(a->w * a->h * a->elem, 0);
    *arr = a;
    return cudaSuccess;
}
cudaError_t cudaMemcpyToArray(cudaArray_t dst, size_t wOffset, size_t hOffset, const void *src, size_t count,
                              enum cudaMemcpyKind) {
    size_t off = (hOffset * dst->w + wOffset) * dst->elem;
    std::memcpy(dst->data.data() + off, src, count);
    return cudaSuccess;
}
cudaError_t cudaFreeArray(cudaArray_t a) {
    delete a;
    return cudaSuccess;
}
cudaError_t cudaCreateTextureObject(cudaTextureObject_t *obj, const struct cudaResourceDesc *rd,
                                    const struct cudaTextureDesc *td, const struct cudaResourceViewDesc *) {
    std::lock_guard<std::mutex> g(g_mu);
    g_tex.push_back(HostTex{rd->res.array.array, *td});
    *obj = g_tex.size();
    return cudaSuccess;
}
cudaError_t cudaDestroyTextureObject(cudaTextureObject_t) { return cudaSuccess; }

}  // extern "C"
