// Kernel-predicting denoiser (KPCN): a 3-level U-Net (32/64/96 channels,
// 3x3 convolutions on the tensor cores, conv.cu) that predicts a 5x5
// per-pixel filter, applied to the noisy radiance. Trained on the GPU with
// the project's own forward and backward kernels (relMSE loss, Adam on FP32
// master weights). The reference has no learned denoiser: its only filter is
// SVGF (Src/Core/renderer.cuh:442-954), which stays the fallback.
//
// Network (NHWC BF16 activations, channel counts padded to multiples of 16):
//   e0a 16->32, e0b 32->32                     full resolution
//   pool, e1a 32->64, e1b 64->64               1/2
//   pool, e2a 64->96, e2b 96->96               1/4
//   up(e2b) ++ e1b -> d1a 160->64, d1b 64->64  1/2
//   up(d1b) ++ e0b -> d0a 96->32, d0b 32->32   full
//   out 32->32 (25 used): filter logits (FP32)
// Every conv but `out` is followed by ReLU; pooling is 2x2 averaging,
// upsampling nearest. Input features (16 channels): log(1 + radiance) (3),
// albedo (3), shading normal (3), linear depth (1), motion (2),
// 1 / sqrt(spp) (1), zeros (3).
// Output: softmax over the 25 logits weights the 5x5 neighbourhood of the
// noisy radiance (clamped at the image border).
//
// Loss: relMSE = mean over pixels and RGB of (out - ref)^2 / (ref^2 + 0.01).
#include "api_internal.h"
#include <algorithm>
#include <cmath>
#include <memory>
#include <cstring>
#include <random>
#include <vector>

namespace crt {
namespace {

constexpr int kLayers = 11;
constexpr int kFeat = 16;
constexpr int kTaps5 = 25;
constexpr int kOutC = 32;
constexpr float kRelEps = 0.01f;

struct LayerSpec {
    int cin, cout, cin_real;
    bool relu;
};
// e0a e0b e1a e1b e2a e2b d1a d1b d0a d0b out
constexpr LayerSpec kSpec[kLayers] = {{16, 32, 13, true},  {32, 32, 32, true},   {32, 64, 32, true}, {64, 64, 64, true},
                                      {64, 96, 64, true},  {96, 96, 96, true},   {160, 64, 160, true},
                                      {64, 64, 64, true},  {96, 32, 96, true},   {32, 32, 32, true}, {32, 32, 32, false}};
enum { E0A, E0B, E1A, E1B, E2A, E2B, D1A, D1B, D0A, D0B, OUT };

__device__ __forceinline__ void load8(const __nv_bfloat16 *p, float (&v)[8]) {
    uint4 u = *reinterpret_cast<const uint4 *>(p);
    const __nv_bfloat16 *b = reinterpret_cast<const __nv_bfloat16 *>(&u);
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = __bfloat162float(b[i]);
}
__device__ __forceinline__ void store8(__nv_bfloat16 *p, const float (&v)[8]) {
    uint4 u;
    __nv_bfloat16 *b = reinterpret_cast<__nv_bfloat16 *>(&u);
#pragma unroll
    for (int i = 0; i < 8; ++i) b[i] = __float2bfloat16_rn(v[i]);
    *reinterpret_cast<uint4 *>(p) = u;
}

// 2x2 average pooling: out [n][h/2][w/2][C].
__global__ void k_avgpool2(const __nv_bfloat16 *in, __nv_bfloat16 *out, int n, int h, int w, int C) {
    const int oh = h / 2, ow = w / 2, G = C / 8;
    const int64_t total = (int64_t)n * oh * ow * G;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int g = (int)(i % G);
        const int64_t q = i / G;
        const int x = (int)(q % ow), y = (int)((q / ow) % oh), b = (int)(q / ((int64_t)ow * oh));
        float s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int dy = 0; dy < 2; ++dy)
            for (int dx = 0; dx < 2; ++dx) {
                float v[8];
                load8(in + (((int64_t)b * h + 2 * y + dy) * w + 2 * x + dx) * C + g * 8, v);
                for (int k = 0; k < 8; ++k) s[k] += v[k];
            }
        for (int k = 0; k < 8; ++k) s[k] *= 0.25f;
        store8(out + q * C + g * 8, s);
    }
}

// out[p] = concat(up2(low)[p] (Ca), skip[p] (Cb)), 8 channels (16 B) per
// thread step; index arithmetic in I (32-bit whenever the element count
// allows: the divisions are most of the work).
template <class I>
__device__ __forceinline__ void up_concat(const __nv_bfloat16 *low, const __nv_bfloat16 *skip, __nv_bfloat16 *out,
                                          int n, int h, int w, int Ca, int Cb) {
    const int C = Ca + Cb, G = C / 8;
    const I total = (I)n * h * w * G;
    for (I i = blockIdx.x * (I)blockDim.x + threadIdx.x; i < total; i += (I)gridDim.x * blockDim.x) {
        const int g = (int)(i % G);
        const I p = i / G;
        const int x = (int)(p % w), y = (int)((p / w) % h), b = (int)(p / ((I)w * h));
        const __nv_bfloat16 *src = g * 8 < Ca
                                       ? low + (((int64_t)b * (h / 2) + y / 2) * (w / 2) + x / 2) * Ca + g * 8
                                       : skip + (int64_t)p * Cb + (g * 8 - Ca);
        *reinterpret_cast<uint4 *>(out + (int64_t)p * C + g * 8) = *reinterpret_cast<const uint4 *>(src);
    }
}

__global__ void k_up_concat(const __nv_bfloat16 *low, const __nv_bfloat16 *skip, __nv_bfloat16 *out, int n, int h,
                            int w, int Ca, int Cb) {
    if ((int64_t)n * h * w * ((Ca + Cb) / 8) < (int64_t)INT32_MAX - (int64_t)gridDim.x * blockDim.x)
        up_concat<int>(low, skip, out, n, h, w, Ca, Cb);
    else
        up_concat<int64_t>(low, skip, out, n, h, w, Ca, Cb);
}

// Adjoint of up2 on the first Ca channels of gcat: glow[q] = sum of the 2x2
// children.
__global__ void k_down_sum(const __nv_bfloat16 *gcat, int Cc, __nv_bfloat16 *glow, int n, int h, int w, int Ca) {
    const int oh = h / 2, ow = w / 2, G = Ca / 8;
    const int64_t total = (int64_t)n * oh * ow * G;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int g = (int)(i % G);
        const int64_t q = i / G;
        const int x = (int)(q % ow), y = (int)((q / ow) % oh), b = (int)(q / ((int64_t)ow * oh));
        float s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int dy = 0; dy < 2; ++dy)
            for (int dx = 0; dx < 2; ++dx) {
                float v[8];
                load8(gcat + (((int64_t)b * h + 2 * y + dy) * w + 2 * x + dx) * Cc + g * 8, v);
                for (int k = 0; k < 8; ++k) s[k] += v[k];
            }
        store8(glow + q * Ca + g * 8, s);
    }
}

// Gradient of a ReLU output that feeds both a skip connection and a pooling:
// out[p] = (gskip[p] + gpool[p / 2] / 4) * (act[p] > 0), with gskip read from
// channels [off, off + C) of a concat gradient of Cc channels.
__global__ void k_unpool_add_mask(const __nv_bfloat16 *gcat, int Cc, int off, const __nv_bfloat16 *gpool,
                                  const __nv_bfloat16 *act, __nv_bfloat16 *out, int n, int h, int w, int C) {
    const int G = C / 8;
    const int64_t total = (int64_t)n * h * w * G;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int g = (int)(i % G);
        const int64_t p = i / G;
        const int x = (int)(p % w), y = (int)((p / w) % h), b = (int)(p / ((int64_t)w * h));
        float a[8], s[8], u[8];
        load8(gcat + p * Cc + off + g * 8, s);
        load8(gpool + (((int64_t)b * (h / 2) + y / 2) * (w / 2) + x / 2) * C + g * 8, u);
        load8(act + p * C + g * 8, a);
        float o[8];
        for (int k = 0; k < 8; ++k) o[k] = a[k] > 0.f ? s[k] + 0.25f * u[k] : 0.f;
        store8(out + p * C + g * 8, o);
    }
}

// db[o] += sum_p g[p][o].
__global__ void k_bias_grad(const __nv_bfloat16 *g, float *db, int64_t P, int N) {
    __shared__ float acc[256];
    for (int i = threadIdx.x; i < N; i += blockDim.x) acc[i] = 0.f;
    __syncthreads();
    const int G = N / 8;
    const int64_t total = P * G;
    float s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    int mygroup = -1;
    // each thread keeps one channel group; the stride is a multiple of G
    const int64_t stride = (int64_t)gridDim.x * blockDim.x / G * G;
    const int64_t start = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (stride > 0 && start < stride) {
        mygroup = (int)(start % G);
        for (int64_t i = start; i < total; i += stride) {
            float v[8];
            load8(g + i * 8, v);  // (p, group) -> p * N + group * 8 = i * 8
            for (int k = 0; k < 8; ++k) s[k] += v[k];
        }
    }
    if (mygroup >= 0)
        for (int k = 0; k < 8; ++k) atomicAdd(&acc[mygroup * 8 + k], s[k]);
    __syncthreads();
    for (int i = threadIdx.x; i < N; i += blockDim.x) atomicAdd(db + i, acc[i]);
}

struct FeatureArgs {
    const float4 *direct, *indirect;
    float inv_spp;
    const ushort4 *normal_mat, *bary_mesh;
    const float4 *motion_depth;
    const DMaterial *materials;
    int num_materials;
    float depth_scale;
    __nv_bfloat16 *features;  // [P][16]
    float4 *noisy;            // [P]
    int64_t P;
};

__global__ void k_features(FeatureArgs a) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < a.P; p += (int64_t)gridDim.x * blockDim.x) {
        const float4 d = a.direct[p], id = a.indirect[p];
        const float r = (d.x + id.x) * a.inv_spp, g = (d.y + id.y) * a.inv_spp, b = (d.z + id.z) * a.inv_spp;
        a.noisy[p] = make_float4(r, g, b, 0.f);
        float f[16];
        for (int k = 0; k < 16; ++k) f[k] = 0.f;
        f[0] = log1pf(fmaxf(r, 0.f));
        f[1] = log1pf(fmaxf(g, 0.f));
        f[2] = log1pf(fmaxf(b, 0.f));
        f[12] = sqrtf(a.inv_spp);  // noise level of the estimate
        const ushort4 bm = a.bary_mesh[p];
        if (bm.w != 0) {  // a primary hit (mesh id + 1)
            const ushort4 nm = a.normal_mat[p];
            const float4 md = a.motion_depth[p];
            const int mat = nm.w;
            if (mat >= 0 && mat < a.num_materials) {
                const DMaterial &m = a.materials[mat];
                if (m.type == MAT_LIGHT) {
                    f[3] = f[4] = f[5] = 1.f;
                } else {
                    f[3] = m.base[0];
                    f[4] = m.base[1];
                    f[5] = m.base[2];
                }
            }
            f[6] = nm.x * (2.f / 65535.f) - 1.f;
            f[7] = nm.y * (2.f / 65535.f) - 1.f;
            f[8] = nm.z * (2.f / 65535.f) - 1.f;
            f[9] = md.z / a.depth_scale;
            f[10] = md.x;
            f[11] = md.y;
        }
        float lo[8], hi[8];
        for (int k = 0; k < 8; ++k) {
            lo[k] = f[k];
            hi[k] = f[8 + k];
        }
        store8(a.features + p * kFeat, lo);
        store8(a.features + p * kFeat + 8, hi);
    }
}

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// Softmax over the 25 logits of one pixel (its 32-float row, 16-byte
// aligned), weights in w. The row is read as 7 float4 loads (28 floats),
// not 25 scalar loads that each touch a sector per lane.
__device__ __forceinline__ void filter_weights(const float *logits, float (&w)[kTaps5]) {
    float l[28];
    const float4 *lp = reinterpret_cast<const float4 *>(logits);
#pragma unroll
    for (int j = 0; j < 7; ++j) {
        const float4 v = lp[j];
        l[4 * j] = v.x;
        l[4 * j + 1] = v.y;
        l[4 * j + 2] = v.z;
        l[4 * j + 3] = v.w;
    }
    float mx = l[0];
#pragma unroll
    for (int k = 1; k < kTaps5; ++k) mx = fmaxf(mx, l[k]);
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < kTaps5; ++k) {
        w[k] = expf(l[k] - mx);
        s += w[k];
    }
    const float inv = 1.f / s;
#pragma unroll
    for (int k = 0; k < kTaps5; ++k) w[k] *= inv;
}

// out[p] = sum_k w_k(p) * noisy[clamp(p + off5(k))].
__global__ void k_apply_filter(const float *logits, const float4 *noisy, float4 *out, int n, int h, int w) {
    const int64_t P = (int64_t)n * h * w;
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < P; p += (int64_t)gridDim.x * blockDim.x) {
        const int x = (int)(p % w), y = (int)((p / w) % h);
        const int64_t base = p - (int64_t)y * w - x;
        float wt[kTaps5];
        filter_weights(logits + p * kOutC, wt);
        float r = 0.f, g = 0.f, b = 0.f;
#pragma unroll
        for (int k = 0; k < kTaps5; ++k) {
            const int sy = clampi(y + k / 5 - 2, 0, h - 1), sx = clampi(x + k % 5 - 2, 0, w - 1);
            const float4 v = noisy[base + (int64_t)sy * w + sx];
            r += wt[k] * v.x;
            g += wt[k] * v.y;
            b += wt[k] * v.z;
        }
        out[p] = make_float4(r, g, b, 0.f);
    }
}

// Loss and its gradient w.r.t. the logits (BF16, 32 channels, 25..31 zero).
__global__ void k_filter_loss_grad(const float *logits, const float4 *noisy, const float4 *ref, __nv_bfloat16 *dlogits,
                                   float *loss_sum, int n, int h, int w, float scale) {
    __shared__ float red[256];
    const int64_t P = (int64_t)n * h * w;
    float lsum = 0.f;
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < P; p += (int64_t)gridDim.x * blockDim.x) {
        const int x = (int)(p % w), y = (int)((p / w) % h);
        const int64_t base = p - (int64_t)y * w - x;
        float wt[kTaps5];
        filter_weights(logits + p * kOutC, wt);
        float4 nv[kTaps5];
        float o[3] = {0.f, 0.f, 0.f};
        for (int k = 0; k < kTaps5; ++k) {
            const int sy = clampi(y + k / 5 - 2, 0, h - 1), sx = clampi(x + k % 5 - 2, 0, w - 1);
            nv[k] = noisy[base + (int64_t)sy * w + sx];
            o[0] += wt[k] * nv[k].x;
            o[1] += wt[k] * nv[k].y;
            o[2] += wt[k] * nv[k].z;
        }
        const float4 rf = ref[p];
        const float rr[3] = {rf.x, rf.y, rf.z};
        float go[3];
        for (int c = 0; c < 3; ++c) {
            const float e = o[c] - rr[c], den = rr[c] * rr[c] + kRelEps;
            lsum += e * e / den;
            go[c] = 2.f * e / den * scale;
        }
        float dw[kTaps5], dot = 0.f;
        for (int k = 0; k < kTaps5; ++k) {
            dw[k] = go[0] * nv[k].x + go[1] * nv[k].y + go[2] * nv[k].z;
            dot += wt[k] * dw[k];
        }
        float gl[kOutC];
        for (int k = 0; k < kOutC; ++k) gl[k] = k < kTaps5 ? wt[k] * (dw[k] - dot) : 0.f;
        for (int q = 0; q < kOutC / 8; ++q) {
            float v[8];
            for (int k = 0; k < 8; ++k) v[k] = gl[q * 8 + k];
            store8(dlogits + p * kOutC + q * 8, v);
        }
    }
    red[threadIdx.x] = lsum;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) atomicAdd(loss_sum, red[0]);
}

// Adam on a flat FP32 parameter range.
__global__ void k_adam(float *w, const float *g, float *m, float *v, int64_t n, float lr, float b1, float b2, float eps,
                       float c1, float c2) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi, vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

// FP32 master weights [9][O][C] -> BF16 copy and the per-tap transpose.
__global__ void k_weights_bf16(const float *w, __nv_bfloat16 *wb, __nv_bfloat16 *wtb, int O, int C) {
    const int total = 9 * O * C;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const int c = i % C, o = (i / C) % O, t = i / (C * O);
        const __nv_bfloat16 b = __float2bfloat16_rn(w[i]);
        wb[i] = b;
        wtb[((size_t)t * C + c) * O + o] = b;
    }
}

int grid_for(int64_t work, int block = 256) {
    int64_t g = (work + block - 1) / block;
    return (int)std::max<int64_t>(1, std::min<int64_t>(g, 148 * 32));
}

}  // namespace
}  // namespace crt

using namespace crt;

struct crt_kpcn {
    struct Layer {
        int cin, cout;
        bool relu;
        size_t woff, boff;  // offsets into the flat parameter arrays
        __nv_bfloat16 *wb = nullptr, *wtb = nullptr;
    };
    crt_ctx *ctx = nullptr;
    Layer L[kLayers];
    size_t nparams = 0;
    float *params = nullptr, *grads = nullptr, *adam_m = nullptr, *adam_v = nullptr;
    __nv_bfloat16 *wbuf = nullptr;  // BF16 weights and transposes
    int64_t step = 0;
    // activation / gradient buffers: the current (n, h, w) and the pixel
    // count the buffers hold (a smaller batch or image reuses them)
    int n = 0, h = 0, w = 0;
    size_t cap_px = 0;
    std::vector<void *> bufs;
    __nv_bfloat16 *act[kLayers] = {};
    __nv_bfloat16 *pool0 = nullptr, *pool1 = nullptr, *cat1 = nullptr, *cat0 = nullptr;
    float *logits = nullptr;
    float *loss = nullptr;
    // gradient buffers
    __nv_bfloat16 *gl = nullptr, *ga = nullptr, *gb = nullptr, *gcat = nullptr, *gpool = nullptr, *gsk = nullptr;
    float4 *tmp_out = nullptr;

    ~crt_kpcn() {
        free_buffers();
        for (void *p : {(void *)params, (void *)grads, (void *)adam_m, (void *)adam_v, (void *)wbuf})
            if (p) cudaFree(p);
    }
    void free_buffers() {
        for (void *p : bufs) cudaFree(p);
        bufs.clear();
        n = h = w = 0;
        cap_px = 0;
    }
    template <class T>
    T *alloc(size_t count) {
        void *p = nullptr;
        CRT_CUDA(cudaMalloc(&p, count * sizeof(T)));
        bufs.push_back(p);
        return static_cast<T *>(p);
    }
    void ensure(int n_, int h_, int w_) {
        CRT_CHECK(n_ > 0 && h_ > 0 && w_ > 0 && h_ % 4 == 0 && w_ % 4 == 0, CRT_ERR_INVALID,
                  "kpcn: image height and width must be multiples of 4");
        // every buffer is a per-pixel plane of the full, half or quarter
        // resolution, so buffers for cap_px pixels hold any n * h * w <= cap_px
        const size_t P0 = (size_t)n_ * h_ * w_, P1 = P0 / 4, P2 = P0 / 16;
        if (P0 <= cap_px) {
            n = n_;
            h = h_;
            w = w_;
            return;
        }
        CRT_CUDA(cudaDeviceSynchronize());
        free_buffers();
        const size_t P[kLayers] = {P0, P0, P1, P1, P2, P2, P1, P1, P0, P0, P0};
        for (int i = 0; i < OUT; ++i) act[i] = alloc<__nv_bfloat16>(P[i] * L[i].cout);
        pool0 = alloc<__nv_bfloat16>(P1 * 32);
        pool1 = alloc<__nv_bfloat16>(P2 * 64);
        cat1 = alloc<__nv_bfloat16>(P1 * 160);
        cat0 = alloc<__nv_bfloat16>(P0 * 96);
        logits = alloc<float>(P0 * kOutC);
        loss = alloc<float>(1);
        gl = alloc<__nv_bfloat16>(P0 * kOutC);
        ga = alloc<__nv_bfloat16>(P0 * 96);
        gb = alloc<__nv_bfloat16>(P0 * 96);
        gcat = alloc<__nv_bfloat16>(P0 * 160);
        gpool = alloc<__nv_bfloat16>(P1 * 64);
        gsk = alloc<__nv_bfloat16>(P0 * 64);
        tmp_out = alloc<float4>(P0);
        n = n_;
        h = h_;
        w = w_;
        cap_px = P0;
    }
    void conv(int i, const __nv_bfloat16 *in, int ln, int lh, int lw, __nv_bfloat16 *out, float *out_f32,
              cudaStream_t s) {
        conv3x3_launch(in, L[i].wb, params + L[i].boff, nullptr, out, out_f32, ctx->d_err, ln, lh, lw, L[i].cin,
                       L[i].cout, false, L[i].relu, s);
    }
    void forward(const __nv_bfloat16 *feat, cudaStream_t s) {
        const int h1 = h / 2, w1 = w / 2, h2 = h / 4, w2 = w / 4;
        conv(E0A, feat, n, h, w, act[E0A], nullptr, s);
        conv(E0B, act[E0A], n, h, w, act[E0B], nullptr, s);
        k_avgpool2<<<grid_for((int64_t)n * h1 * w1 * 4), 256, 0, s>>>(act[E0B], pool0, n, h, w, 32);
        conv(E1A, pool0, n, h1, w1, act[E1A], nullptr, s);
        conv(E1B, act[E1A], n, h1, w1, act[E1B], nullptr, s);
        k_avgpool2<<<grid_for((int64_t)n * h2 * w2 * 8), 256, 0, s>>>(act[E1B], pool1, n, h1, w1, 64);
        conv(E2A, pool1, n, h2, w2, act[E2A], nullptr, s);
        conv(E2B, act[E2A], n, h2, w2, act[E2B], nullptr, s);
        k_up_concat<<<grid_for((int64_t)n * h1 * w1 * 20), 256, 0, s>>>(act[E2B], act[E1B], cat1, n, h1, w1, 96, 64);
        conv(D1A, cat1, n, h1, w1, act[D1A], nullptr, s);
        conv(D1B, act[D1A], n, h1, w1, act[D1B], nullptr, s);
        k_up_concat<<<grid_for((int64_t)n * h * w * 12), 256, 0, s>>>(act[D1B], act[E0B], cat0, n, h, w, 64, 32);
        conv(D0A, cat0, n, h, w, act[D0A], nullptr, s);
        conv(D0B, act[D0A], n, h, w, act[D0B], nullptr, s);
        conv(OUT, act[D0B], n, h, w, nullptr, logits, s);
        CRT_CUDA(cudaGetLastError());
    }
    // Gradients of layer i given the pre-activation output gradient g (BF16):
    // dW, db; and, when gin != null, the input gradient (masked by `mask`).
    void layer_backward(int i, const __nv_bfloat16 *in, const __nv_bfloat16 *g, int ln, int lh, int lw,
                        const __nv_bfloat16 *mask, __nv_bfloat16 *gin, cudaStream_t s) {
        conv3x3_wgrad_launch(in, g, grads + L[i].woff, ctx->d_err, ln, lh, lw, L[i].cin, L[i].cout, s);
        const int64_t P = (int64_t)ln * lh * lw;
        k_bias_grad<<<grid_for(P * L[i].cout / 8 / 16, 256), 256, 0, s>>>(g, grads + L[i].boff, P, L[i].cout);
        if (gin)
            conv3x3_launch(g, L[i].wtb, nullptr, mask, gin, nullptr, ctx->d_err, ln, lh, lw, L[i].cout, L[i].cin, true,
                           false, s);
    }
    void backward(const __nv_bfloat16 *feat, cudaStream_t s) {
        const int h1 = h / 2, w1 = w / 2, h2 = h / 4, w2 = w / 4;
        CRT_CUDA(cudaMemsetAsync(grads, 0, nparams * sizeof(float), s));
        // out: g = dlogits (gl); input d0b (ReLU output)
        layer_backward(OUT, act[D0B], gl, n, h, w, act[D0B], ga, s);            // ga = g(d0b pre)
        layer_backward(D0B, act[D0A], ga, n, h, w, act[D0A], gb, s);            // gb = g(d0a pre)
        layer_backward(D0A, cat0, gb, n, h, w, cat0, gcat, s);                  // gcat = g(cat0), masked
        k_down_sum<<<grid_for((int64_t)n * h1 * w1 * 8), 256, 0, s>>>(gcat, 96, ga, n, h, w, 64);  // ga = g(d1b pre)
        // keep g(e0b) skip part: gcat[..., 64:96] -> gsk (copy via unpool later); stash in gsk
        CRT_CUDA(cudaMemcpy2DAsync(gsk, 32 * sizeof(__nv_bfloat16), gcat + 64, 96 * sizeof(__nv_bfloat16),
                                   32 * sizeof(__nv_bfloat16), (size_t)n * h * w, cudaMemcpyDeviceToDevice, s));
        layer_backward(D1B, act[D1A], ga, n, h1, w1, act[D1A], gb, s);          // gb = g(d1a pre)
        layer_backward(D1A, cat1, gb, n, h1, w1, cat1, gcat, s);                // gcat = g(cat1) [160]
        k_down_sum<<<grid_for((int64_t)n * h2 * w2 * 12), 256, 0, s>>>(gcat, 160, ga, n, h1, w1, 96);  // g(e2b pre)
        layer_backward(E2B, act[E2A], ga, n, h2, w2, act[E2A], gb, s);          // gb = g(e2a pre)
        layer_backward(E2A, pool1, gb, n, h2, w2, nullptr, gpool, s);           // gpool = g(pool1)
        // g(e1b pre) = (gcat[..., 96:160] + up(gpool)/4) * (e1b > 0)
        k_unpool_add_mask<<<grid_for((int64_t)n * h1 * w1 * 8), 256, 0, s>>>(gcat, 160, 96, gpool, act[E1B], ga, n, h1,
                                                                               w1, 64);
        layer_backward(E1B, act[E1A], ga, n, h1, w1, act[E1A], gb, s);          // gb = g(e1a pre)
        layer_backward(E1A, pool0, gb, n, h1, w1, nullptr, gpool, s);           // gpool = g(pool0) [32]
        k_unpool_add_mask<<<grid_for((int64_t)n * h * w * 4), 256, 0, s>>>(gsk, 32, 0, gpool, act[E0B], ga, n, h, w,
                                                                             32);  // ga = g(e0b pre)
        layer_backward(E0B, act[E0A], ga, n, h, w, act[E0A], gb, s);            // gb = g(e0a pre)
        layer_backward(E0A, feat, gb, n, h, w, nullptr, nullptr, s);
        CRT_CUDA(cudaGetLastError());
    }
    void refresh_bf16(cudaStream_t s) {
        for (int i = 0; i < kLayers; ++i)
            k_weights_bf16<<<grid_for(9 * L[i].cout * L[i].cin), 256, 0, s>>>(params + L[i].woff, L[i].wb, L[i].wtb,
                                                                               L[i].cout, L[i].cin);
        CRT_CUDA(cudaGetLastError());
    }
};

extern "C" crt_status crt_kpcn_create(crt_ctx *ctx, uint64_t seed, crt_kpcn **out) {
    return guard([&] {
        CRT_CHECK(ctx && out, CRT_ERR_INVALID, "crt_kpcn_create: null argument");
        CRT_CUDA(cudaSetDevice(ctx->device));
        auto k = std::make_unique<crt_kpcn>();
        k->ctx = ctx;
        size_t off = 0, wbf = 0;
        for (int i = 0; i < kLayers; ++i) {
            k->L[i].cin = kSpec[i].cin;
            k->L[i].cout = kSpec[i].cout;
            k->L[i].relu = kSpec[i].relu;
            k->L[i].woff = off;
            off += (size_t)9 * kSpec[i].cout * kSpec[i].cin;
            k->L[i].boff = off;
            off += kSpec[i].cout;
            wbf += (size_t)2 * 9 * kSpec[i].cout * kSpec[i].cin;
        }
        k->nparams = off;
        CRT_CUDA(cudaMalloc(&k->params, off * sizeof(float)));
        CRT_CUDA(cudaMalloc(&k->grads, off * sizeof(float)));
        CRT_CUDA(cudaMalloc(&k->adam_m, off * sizeof(float)));
        CRT_CUDA(cudaMalloc(&k->adam_v, off * sizeof(float)));
        CRT_CUDA(cudaMalloc(&k->wbuf, wbf * sizeof(__nv_bfloat16)));
        CRT_CUDA(cudaMemset(k->adam_m, 0, off * sizeof(float)));
        CRT_CUDA(cudaMemset(k->adam_v, 0, off * sizeof(float)));
        size_t bo = 0;
        for (int i = 0; i < kLayers; ++i) {
            const size_t sz = (size_t)9 * kSpec[i].cout * kSpec[i].cin;
            k->L[i].wb = k->wbuf + bo;
            k->L[i].wtb = k->wbuf + bo + sz;
            bo += 2 * sz;
        }
        // He initialisation over the real input channels; the filter layer
        // starts small (near-uniform 5x5 box filter); biases zero; weights of
        // padded input or output channels zero.
        std::vector<float> h(off, 0.f);
        std::mt19937_64 rng(seed);
        std::normal_distribution<float> nd(0.f, 1.f);
        for (int i = 0; i < kLayers; ++i) {
            const LayerSpec &sp = kSpec[i];
            const int used_out = i == OUT ? kTaps5 : sp.cout;
            const float stdv = i == OUT ? 0.01f : std::sqrt(2.f / (9.f * sp.cin_real));
            for (int t = 0; t < 9; ++t)
                for (int o = 0; o < used_out; ++o)
                    for (int c = 0; c < sp.cin_real; ++c)
                        h[k->L[i].woff + ((size_t)t * sp.cout + o) * sp.cin + c] = stdv * nd(rng);
        }
        CRT_CUDA(cudaMemcpy(k->params, h.data(), off * sizeof(float), cudaMemcpyHostToDevice));
        k->refresh_bf16(ctx->stream);
        CRT_CUDA(cudaStreamSynchronize(ctx->stream));
        *out = k.release();
    });
}

extern "C" void crt_kpcn_free(crt_kpcn *k) {
    if (!k) return;
    cudaSetDevice(k->ctx->device);
    delete k;
}

extern "C" crt_status crt_kpcn_num_params(const crt_kpcn *k, int64_t *n) {
    return guard([&] {
        CRT_CHECK(k && n, CRT_ERR_INVALID, "crt_kpcn_num_params: null argument");
        *n = (int64_t)k->nparams;
    });
}

extern "C" crt_status crt_kpcn_get_params(crt_kpcn *k, float *host) {
    return guard([&] {
        CRT_CHECK(k && host, CRT_ERR_INVALID, "crt_kpcn_get_params: null argument");
        CRT_CUDA(cudaSetDevice(k->ctx->device));
        CRT_CUDA(cudaDeviceSynchronize());
        CRT_CUDA(cudaMemcpy(host, k->params, k->nparams * sizeof(float), cudaMemcpyDeviceToHost));
    });
}

extern "C" crt_status crt_kpcn_set_params(crt_kpcn *k, const float *host) {
    return guard([&] {
        CRT_CHECK(k && host, CRT_ERR_INVALID, "crt_kpcn_set_params: null argument");
        CRT_CUDA(cudaSetDevice(k->ctx->device));
        CRT_CUDA(cudaDeviceSynchronize());
        CRT_CUDA(cudaMemcpy(k->params, host, k->nparams * sizeof(float), cudaMemcpyHostToDevice));
        k->refresh_bf16(k->ctx->stream);
        CRT_CUDA(cudaStreamSynchronize(k->ctx->stream));
    });
}

extern "C" crt_status crt_kpcn_features(crt_scene *scene, const crt_gbuffer *gb, const float *d_direct,
                                        const float *d_indirect, int32_t spp, int64_t pixels, float depth_scale,
                                        void *d_features, float *d_noisy, void *stream) {
    return guard([&] {
        CRT_CHECK(scene && scene->renderable && gb && d_direct && d_indirect && d_features && d_noisy && spp > 0 &&
                      pixels > 0 && depth_scale > 0.f,
                  CRT_ERR_INVALID, "crt_kpcn_features: bad argument");
        CRT_CUDA(cudaSetDevice(scene->ctx->device));
        cudaStream_t s = stream ? (cudaStream_t)stream : scene->ctx->stream;
        FeatureArgs a;
        a.direct = (const float4 *)d_direct;
        a.indirect = (const float4 *)d_indirect;
        a.inv_spp = 1.f / (float)spp;
        a.normal_mat = (const ushort4 *)gb->normal_mat;
        a.bary_mesh = (const ushort4 *)gb->bary_mesh;
        a.motion_depth = (const float4 *)gb->motion_depth;
        a.materials = scene->rd.materials;
        a.num_materials = scene->rd.num_materials;
        a.depth_scale = depth_scale;
        a.features = (__nv_bfloat16 *)d_features;
        a.noisy = (float4 *)d_noisy;
        a.P = pixels;
        k_features<<<grid_for(pixels), 256, 0, s>>>(a);
        CRT_CUDA(cudaGetLastError());
    });
}

extern "C" crt_status crt_kpcn_forward(crt_kpcn *k, int32_t n, int32_t h, int32_t w, const void *d_features,
                                       const float *d_noisy, float *d_out, void *stream) {
    return guard([&] {
        CRT_CHECK(k && d_features && d_noisy && d_out, CRT_ERR_INVALID, "crt_kpcn_forward: null argument");
        CRT_CUDA(cudaSetDevice(k->ctx->device));
        cudaStream_t s = stream ? (cudaStream_t)stream : k->ctx->stream;
        k->ensure(n, h, w);
        k->forward((const __nv_bfloat16 *)d_features, s);
        k_apply_filter<<<grid_for((int64_t)n * h * w), 256, 0, s>>>(k->logits, (const float4 *)d_noisy,
                                                                      (float4 *)d_out, n, h, w);
        CRT_CUDA(cudaGetLastError());
    });
}

// Forward + relMSE loss + backward; gradients land in the gradient buffer.
// With lr > 0 an Adam step follows. *loss (host) = the batch loss.
extern "C" crt_status crt_kpcn_train_step(crt_kpcn *k, int32_t n, int32_t h, int32_t w, const void *d_features,
                                          const float *d_noisy, const float *d_target, float lr, float *loss,
                                          void *stream) {
    return guard([&] {
        CRT_CHECK(k && d_features && d_noisy && d_target, CRT_ERR_INVALID, "crt_kpcn_train_step: null argument");
        CRT_CUDA(cudaSetDevice(k->ctx->device));
        cudaStream_t s = stream ? (cudaStream_t)stream : k->ctx->stream;
        k->ensure(n, h, w);
        const __nv_bfloat16 *feat = (const __nv_bfloat16 *)d_features;
        k->forward(feat, s);
        const int64_t P = (int64_t)n * h * w;
        CRT_CUDA(cudaMemsetAsync(k->loss, 0, sizeof(float), s));
        k_filter_loss_grad<<<grid_for(P), 256, 0, s>>>(k->logits, (const float4 *)d_noisy, (const float4 *)d_target,
                                                         k->gl, k->loss, n, h, w, 1.f / (3.f * (float)P));
        k->backward(feat, s);
        if (lr > 0.f) {
            k->step += 1;
            const float b1 = 0.9f, b2 = 0.999f;
            const float c1 = 1.f - std::pow(b1, (float)k->step), c2 = 1.f - std::pow(b2, (float)k->step);
            k_adam<<<grid_for((int64_t)k->nparams), 256, 0, s>>>(k->params, k->grads, k->adam_m, k->adam_v,
                                                                  (int64_t)k->nparams, lr, b1, b2, 1e-8f, c1, c2);
            k->refresh_bf16(s);
        }
        CRT_CUDA(cudaGetLastError());
        if (loss) {
            float l = 0.f;
            CRT_CUDA(cudaMemcpyAsync(&l, k->loss, sizeof(float), cudaMemcpyDeviceToHost, s));
            CRT_CUDA(cudaStreamSynchronize(s));
            *loss = l / (3.f * (float)P);
        }
    });
}

extern "C" crt_status crt_kpcn_get_grads(crt_kpcn *k, float *host) {
    return guard([&] {
        CRT_CHECK(k && host, CRT_ERR_INVALID, "crt_kpcn_get_grads: null argument");
        CRT_CUDA(cudaSetDevice(k->ctx->device));
        CRT_CUDA(cudaDeviceSynchronize());
        CRT_CUDA(cudaMemcpy(host, k->grads, k->nparams * sizeof(float), cudaMemcpyDeviceToHost));
    });
}

// Copies an internal tensor for tests: 0..9 layer activations, 10 logits
// (FP32), 11 pool0, 12 pool1, 13 cat1, 14 cat0.
extern "C" crt_status crt_kpcn_debug_tensor(crt_kpcn *k, int32_t which, void *host, int64_t bytes) {
    return guard([&] {
        CRT_CHECK(k && host && k->n > 0, CRT_ERR_INVALID, "crt_kpcn_debug_tensor: nothing computed yet");
        CRT_CUDA(cudaSetDevice(k->ctx->device));
        CRT_CUDA(cudaDeviceSynchronize());
        const size_t P0 = (size_t)k->n * k->h * k->w, P1 = P0 / 4, P2 = P0 / 16;
        const size_t P[kLayers] = {P0, P0, P1, P1, P2, P2, P1, P1, P0, P0, P0};
        const void *src = nullptr;
        size_t sz = 0;
        if (which >= 0 && which < OUT) {
            src = k->act[which];
            sz = P[which] * k->L[which].cout * 2;
        } else if (which == 10) {
            src = k->logits;
            sz = P0 * kOutC * 4;
        } else if (which == 11) {
            src = k->pool0;
            sz = P1 * 32 * 2;
        } else if (which == 12) {
            src = k->pool1;
            sz = P2 * 64 * 2;
        } else if (which == 13) {
            src = k->cat1;
            sz = P1 * 160 * 2;
        } else if (which == 14) {
            src = k->cat0;
            sz = P0 * 96 * 2;
        }
        CRT_CHECK(src && (int64_t)sz == bytes, CRT_ERR_INVALID, "crt_kpcn_debug_tensor: bad tensor or size");
        CRT_CUDA(cudaMemcpy(host, src, sz, cudaMemcpyDeviceToHost));
    });
}
