// 3x3 convolutions (stride 1, zero padding 1) on NHWC BF16 activations as
// implicit GEMMs on the sm_100a tensor cores (tcgen05.mma kind::f16, BF16 x
// BF16 -> FP32 in TMEM). These are the dense contractions of the learned
// kernel-predicting denoiser (kpcn.cu); the reference has no learned part.
//
// Forward and data gradient share one kernel: output pixel tile (M = 128
// pixels) x all output channels (N), K = 9 taps x C input channels.
//   forward : out[p, n] = sum_{t, c} in[p + off(t), c] * w[t][n][c]
//   data grad: out[p, n] = sum_{t, c} g[p - off(t), c] * wt[t][n][c]
//             (wt = w transposed per tap, flip = 1)
// The input is staged per (tile, channel chunk) as three halo regions with
// 16 B cp.async copies (zero-filled outside the image) in the K-major
// core-matrix layout of tc.cuh; every tap's A operand is a shifted
// descriptor into them, B the tap's weight slice (resident in shared memory
// when the layer's weights fit). Producer warps, one MMA-issuing thread and
// epilogue warps hand stages and the two TMEM accumulator slots to each
// other through mbarriers, so copies, MMAs and the epilogue of the previous
// tile overlap. The epilogue reads the FP32 accumulators from TMEM (one
// pixel per thread) and applies bias + ReLU (forward) or the ReLU mask of
// the layer below (data gradient), writing BF16 (or FP32) NHWC.
//
// The weight gradient is a second kernel: rows M = (tap, c) (9C rows in
// 128-row tiles), columns N = output channels, K = pixels split across
// CTAs; both operands MN-major, partial sums added to FP32 dW with atomics.
#include "api_internal.h"
#include "tc.cuh"
#include <algorithm>

namespace crt {
namespace {

constexpr int kBM = 128;      // pixels (or (tap, c) rows) per tile
constexpr int kThreads = 128;      // weight-gradient kernel
constexpr int kConvThreads = 288;  // forward / data-gradient kernel: 4 producer, 4 epilogue, 1 MMA warp
constexpr int kStages = 4;
constexpr int kWgradBK = 64;  // pixels per weight-gradient K step

struct ConvArgs {
    const __nv_bfloat16 *in;    // [P][C]
    const __nv_bfloat16 *wgt;   // [9][N][C]
    const float *bias;          // [N] or null
    const __nv_bfloat16 *mask;  // [P][N] or null: out *= (mask > 0)
    __nv_bfloat16 *out;         // [P][N] or null
    float *out_f32;             // [P][N] or null
    int *err;
    int nimg, h, wd, C, N, KC;
    int flip, relu;
};

__device__ __forceinline__ uint32_t tmem_cols(int n) {
    uint32_t c = 32;
    while ((int)c < n) c <<= 1;
    return c;
}

constexpr int kHalo = kBM + 2;  // rows of one halo region

// Position q of the padded linear image space (rows of W + 2: columns W and
// W + 1 are zero padding, column W + 1 doubling as column -1 of the next
// row; row 0 and one row after every image are zero rows) -> NHWC pixel
// index, or -1 for padding.
// (32-bit arithmetic: the host refuses images whose padded space reaches 2^31.)
__device__ __forceinline__ int padded_to_pixel(int q, int W, int H, int NR) {
    if (q < 0) return -1;
    const int Wp = W + 2;
    const int R = q / Wp;
    const int x = q - R * Wp;
    if (x >= W || R < 1 || R > NR - 2) return -1;
    const int rr = R - 1;
    const int b = rr / (H + 1);
    const int r = rr - b * (H + 1);
    if (r >= H) return -1;
    return (b * H + r) * W + x;
}

// One CTA walks its tiles of 128 consecutive padded positions. Per tile and
// channel chunk of KC, a stage holds three halo regions (input rows shifted
// by -1, 0, +1; 130 positions each: the tile plus one on either side) and,
// unless the weights are resident, the chunk of all 9 taps' weights. Tap
// (dy, dx) is then the MMA whose A operand starts dx + 1 rows (16 B each)
// into region dy + 1: no per-tap gather.
// Warp roles (no block-wide barrier inside the tile loop):
//   warps 0-3  producers: cp.async the halo (and streamed weights) of step s
//              into stage s % kS; once a step's copies have landed they
//              make them visible to the tensor core (proxy fence) and
//              arrive on full[stage]. kS - 2 steps stay in flight.
//   warp 8     one thread issues the step's 9 taps x KC/16 MMAs into one of
//              two TMEM accumulator slots and commits them to empty[stage]
//              (the stage may be refilled) and, after a tile's last chunk,
//              to tfull[slot].
//   warps 4-7  epilogue: TMEM lane quarter (warp % 4), one pixel per thread:
//              bias / ReLU / mask, BF16 or FP32 NHWC stores; then arrive on
//              tempty[slot] so the MMAs of tile + 2 may overwrite the slot.
// Every wait is bounded and also ends when another role has given up.
// kResident: the layer's weights (all taps, all channel chunks) are loaded
// into shared memory once per CTA; stages then hold only halo regions.
template <int kS, bool kResident>
__global__ void __launch_bounds__(kConvThreads, 1) k_conv3x3(ConvArgs a) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ uint64_t full[kS], empty[kS], tfull[2], tempty[2], mma_done;
    __shared__ uint32_t tmem_slot;
    __shared__ int abort_flag;
    __shared__ int hpix[3 * kHalo];  // pixel index (or -1) of each halo row of the producers' tile
    __shared__ float sbias[256];
    constexpr int kLag = kS - 2;     // producer steps in flight before a step is signalled
    constexpr int kProd = 128, kEpi0 = 4, kMmaWarp = 8;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int C = a.C, N = a.N, KC = a.KC, W = a.wd, H = a.h;
    const int Wp = W + 2, NR = a.nimg * (H + 1) + 1;
    const int qbeg = Wp, qend = Wp * (NR - 1);
    const int ntiles = (qend - qbeg + kBM - 1) / kBM;
    const int chunks = C / KC, KG = KC / 8, kg_shift = KG == 8 ? 3 : KG == 4 ? 2 : 1;
    const uint32_t lbo_a = kHalo * 16, region_bytes = KG * lbo_a, a_bytes = 3 * region_bytes;
    const uint32_t lbo_b = (uint32_t)N * 16, tap_bytes = KG * lbo_b, b_bytes = 9 * tap_bytes;
    const uint32_t stage_bytes = kResident ? a_bytes : a_bytes + b_bytes;
    // resident weights: [chunk][tap][k group][n], then the stages
    unsigned char *const wres = smem_raw;
    unsigned char *const stages = smem_raw + (kResident ? (size_t)chunks * b_bytes : 0);
    const uint32_t ncols = tmem_cols(2 * N);
    const int my_tiles = blockIdx.x < ntiles ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
    volatile int *abort = &abort_flag;

    if (tid == 0) {
        for (int i = 0; i < kS; ++i) {
            tc::mbar_init(&full[i], kProd);
            tc::mbar_init(&empty[i], 1);
        }
        for (int i = 0; i < 2; ++i) {
            tc::mbar_init(&tfull[i], 1);
            tc::mbar_init(&tempty[i], 128);
        }
        tc::mbar_init(&mma_done, 1);
        abort_flag = 0;
        tc::fence_mbar_init();
    }
    for (int n = tid; n < N; n += kConvThreads) sbias[n] = a.bias ? a.bias[n] : 0.f;
    if (warp == kMmaWarp) tc::tmem_alloc(&tmem_slot, ncols);
    if (kResident) {
        for (int pr = tid; pr < chunks * 9 * N * KG; pr += kConvThreads) {
            const int kg = pr & (KG - 1), row = pr >> kg_shift;
            const int ch = row / (9 * N), rest = row - ch * 9 * N, t = rest / N, n = rest - t * N;
            tc::cp_async16(wres + ch * b_bytes + t * tap_bytes + kg * lbo_b + n * 16,
                           a.wgt + ((size_t)t * N + n) * C + ch * KC + kg * 8, 16u);
        }
        tc::cp_async_commit();
        tc::cp_async_wait_all();
        tc::fence_proxy_async();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tmem_slot;

    if (warp < kEpi0) {
        // ---- producers ----
        const int ptid = tid;
        int s = 0;
        for (int tl = 0; tl < my_tiles; ++tl) {
            const int t0 = qbeg + (blockIdx.x + tl * gridDim.x) * kBM;
            tc::named_sync(1, kProd);  // the previous tile's rows are no longer read
            for (int pr = ptid; pr < 3 * kHalo; pr += kProd) {
                const int r = pr / kHalo, j = pr - r * kHalo;
                hpix[pr] = padded_to_pixel(t0 + (r - 1) * Wp + j - 1, W, H, NR);
            }
            tc::named_sync(1, kProd);
            for (int chunk = 0; chunk < chunks; ++chunk, ++s) {
                const int st = s % kS, c0 = chunk * KC;
                if (s >= kS && !tc::mbar_wait_or_abort(&empty[st], ((s / kS) - 1) & 1, abort)) {
                    // another role gave up: keep the loop (and its named
                    // barriers) uniform over the producer warps, copy nothing
                } else if (!*abort) {
                    unsigned char *sa = stages + st * stage_bytes;
                    // halo: consecutive threads copy consecutive 16 B of one pixel
                    for (int it = ptid; it < 3 * kHalo * KG; it += kProd) {
                        const int kg = it & (KG - 1), pr = it >> kg_shift;
                        const int r = pr / kHalo, j = pr - r * kHalo, p = hpix[pr];
                        const __nv_bfloat16 *src = p >= 0 ? a.in + (size_t)p * C + c0 + kg * 8 : a.in;
                        tc::cp_async16(sa + r * region_bytes + kg * lbo_a + j * 16, src, p >= 0 ? 16u : 0u);
                    }
                    if (!kResident) {
                        unsigned char *sb = sa + a_bytes;
                        for (int it = ptid; it < 9 * N * KG; it += kProd) {
                            const int kg = it & (KG - 1), row = it >> kg_shift, t = row / N, n = row - t * N;
                            tc::cp_async16(sb + t * tap_bytes + kg * lbo_b + n * 16,
                                           a.wgt + ((size_t)t * N + n) * C + c0 + kg * 8, 16u);
                        }
                    }
                }
                tc::cp_async_commit();
                if (s >= kLag) {
                    tc::cp_async_wait<kLag>();
                    tc::fence_proxy_async();
                    tc::mbar_arrive(&full[(s - kLag) % kS]);
                }
            }
        }
        tc::cp_async_wait_all();
        tc::fence_proxy_async();
        for (int s2 = s > kLag ? s - kLag : 0; s2 < s; ++s2) tc::mbar_arrive(&full[s2 % kS]);
    } else if (warp < kMmaWarp) {
        // ---- epilogue ----
        const int etid = tid - kEpi0 * 32;  // = 32 * (warp % 4) + lane: this thread's TMEM lane
        for (int tl = 0; tl < my_tiles; ++tl) {
            const int slot = tl & 1;
            if (!tc::mbar_wait_or_abort(&tfull[slot], (tl >> 1) & 1, abort)) break;
            tc::fence_after_sync();
            const int64_t p = padded_to_pixel(qbeg + (blockIdx.x + tl * gridDim.x) * kBM + etid, W, H, NR);
            const uint32_t lane_base = tmem + ((uint32_t)(etid & ~31) << 16) + slot * N;
            for (int n0 = 0; n0 < N; n0 += 16) {
                float v[16];
                tc::tmem_ld16(lane_base + n0, v);
                if (p < 0) continue;
                for (int i = 0; i < 16; ++i) v[i] += sbias[n0 + i];
                if (a.relu)
                    for (int i = 0; i < 16; ++i) v[i] = fmaxf(v[i], 0.f);
                if (a.mask) {
                    const uint4 *mp = reinterpret_cast<const uint4 *>(a.mask + p * N + n0);
                    uint4 mv[2] = {mp[0], mp[1]};
                    const __nv_bfloat16 *mb = reinterpret_cast<const __nv_bfloat16 *>(mv);
                    for (int i = 0; i < 16; ++i)
                        if (!(__bfloat162float(mb[i]) > 0.f)) v[i] = 0.f;
                }
                if (a.out) {
                    uint4 ov[2];
                    __nv_bfloat16 *ob = reinterpret_cast<__nv_bfloat16 *>(ov);
                    for (int i = 0; i < 16; ++i) ob[i] = __float2bfloat16_rn(v[i]);
                    uint4 *op = reinterpret_cast<uint4 *>(a.out + p * N + n0);
                    op[0] = ov[0];
                    op[1] = ov[1];
                }
                if (a.out_f32) {
                    float4 *op = reinterpret_cast<float4 *>(a.out_f32 + p * N + n0);
                    for (int i = 0; i < 4; ++i) op[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
                }
            }
            tc::fence_before_sync();
            tc::mbar_arrive(&tempty[slot]);  // this slot's TMEM reads are done
        }
    } else if ((tid & 31) == 0) {
        // ---- MMA issuer ----
        const uint32_t idesc = tc::idesc_bf16(kBM, N, false, false);
        int s = 0;
        for (int tl = 0; tl < my_tiles && !*abort; ++tl) {
            const int slot = tl & 1;
            if (tl >= 2 && !tc::mbar_wait_or_abort(&tempty[slot], ((tl >> 1) - 1) & 1, abort)) break;
            tc::fence_after_sync();
            bool ok = true;
            for (int chunk = 0; chunk < chunks; ++chunk, ++s) {
                const int st = s % kS;
                if (!tc::mbar_wait_or_abort(&full[st], (s / kS) & 1, abort)) {
                    ok = false;
                    break;
                }
                tc::fence_after_sync();
                const uint32_t sa = tc::smem_addr(stages + st * stage_bytes);
                const uint32_t sb = kResident ? tc::smem_addr(wres + chunk * b_bytes) : sa + a_bytes;
                for (int tap = 0; tap < 9; ++tap) {
                    int sy = tap / 3 - 1, sx = tap % 3 - 1;
                    if (a.flip) {
                        sy = -sy;
                        sx = -sx;
                    }
                    for (int jj = 0; jj < KG / 2; ++jj)
                        tc::mma_bf16(tmem + slot * N,
                                     tc::smem_desc(sa + (sy + 1) * region_bytes + 2 * jj * lbo_a + (sx + 1) * 16, lbo_a, 128),
                                     tc::smem_desc(sb + tap * tap_bytes + 2 * jj * lbo_b, lbo_b, 128), idesc,
                                     chunk > 0 || tap > 0 || jj > 0);
                }
                tc::mma_commit(tc::smem_addr(&empty[st]));
                if (chunk == chunks - 1) tc::mma_commit(tc::smem_addr(&tfull[slot]));
            }
            if (!ok) break;
        }
        // every MMA issued has finished before TMEM is released
        tc::mma_commit(tc::smem_addr(&mma_done));
        tc::mbar_wait(&mma_done, 0);
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (tid == 0 && abort_flag) atomicExch(a.err, 1);
    if (warp == kMmaWarp) tc::tmem_dealloc(tmem, ncols);
}

struct WgradArgs {
    const __nv_bfloat16 *in;   // [P][C] layer input
    const __nv_bfloat16 *g;    // [P][N] gradient of the layer's pre-activation output
    float *dw;                 // [9][N][C], accumulated
    int *err;
    int nimg, h, wd, C, N;
    int pix_per_cta;           // multiple of kWgradBK
};

// dW[t][n][c] += sum_p in[p + off(t), c] * g[p, n] over this CTA's pixels.
// Tile rows m = t * C + c (blockIdx.y selects 128 of them), columns n.
__global__ void __launch_bounds__(kThreads) k_conv3x3_wgrad(WgradArgs a) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ uint64_t bars[kStages + 1];
    __shared__ uint32_t tmem_slot;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int C = a.C, N = a.N;
    const int P = a.nimg * a.h * a.wd, HW = a.h * a.wd;
    const int rows = 9 * C, m0 = blockIdx.y * kBM;
    const int k0 = blockIdx.x * a.pix_per_cta, k1 = min(P, k0 + a.pix_per_cta);
    const int steps = (k1 - k0 + kWgradBK - 1) / kWgradBK;
    const uint32_t a_bytes = kBM * kWgradBK * 2, b_bytes = (uint32_t)N * kWgradBK * 2;
    const uint32_t stage_bytes = a_bytes + b_bytes;
    const uint32_t sbo = 128, lbo_a = (kBM / 8) * 128, lbo_b = (uint32_t)(N / 8) * 128;
    const uint32_t idesc = tc::idesc_bf16(kBM, N, true, true);
    const uint32_t ncols = tmem_cols(N);
    if (steps <= 0) return;

    if (tid == 0) {
        for (int s = 0; s <= kStages; ++s) tc::mbar_init(&bars[s], 1);
        tc::fence_mbar_init();
    }
    if (warp == 0) tc::tmem_alloc(&tmem_slot, ncols);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tmem_slot;
    bool failed = false;

    for (int s = 0; s < steps + kStages - 1; ++s) {
        bool ok = true;
        if (s < steps) {
            const uint32_t st = s % kStages;
            if (s >= kStages) ok = tc::mbar_wait(&bars[st], ((s / kStages) - 1) & 1);
            unsigned char *sa = smem_raw + st * stage_bytes, *sb = sa + a_bytes;
            const int kb = k0 + s * kWgradBK;
            // A: 16 row groups x 64 pixels, one 16 B vector (8 channels of one tap) each
            for (int v = tid; v < (kBM / 8) * kWgradBK; v += kThreads) {
                const int k = v % kWgradBK, mg = v / kWgradBK;
                const int m = m0 + mg * 8, p = kb + k;
                bool valid = m < rows && p < k1;
                const __nv_bfloat16 *src = a.in;
                if (valid) {
                    const int tap = m / C, c0 = m - tap * C;
                    const int b = p / HW, r = p - b * HW, y = r / a.wd, x = r - y * a.wd;
                    const int sy = y + tap / 3 - 1, sx = x + tap % 3 - 1;
                    valid = sy >= 0 && sy < a.h && sx >= 0 && sx < a.wd;
                    if (valid) src = a.in + (size_t)(b * HW + sy * a.wd + sx) * C + c0;
                }
                tc::cp_async16(sa + mg * sbo + (k >> 3) * lbo_a + (k & 7) * 16, src, valid ? 16u : 0u);
            }
            // B: N/8 column groups x 64 pixels
            for (int v = tid; v < (N / 8) * kWgradBK; v += kThreads) {
                const int k = v % kWgradBK, ng = v / kWgradBK;
                const int p = kb + k;
                const bool valid = p < k1;
                const __nv_bfloat16 *src = valid ? a.g + (size_t)p * N + ng * 8 : a.g;
                tc::cp_async16(sb + ng * sbo + (k >> 3) * lbo_b + (k & 7) * 16, src, valid ? 16u : 0u);
            }
        }
        tc::cp_async_commit();
        const int c = s - (kStages - 1);
        if (c >= 0) {
            tc::cp_async_wait<kStages - 1>();
            tc::fence_proxy_async();
            if (__syncthreads_or(!ok)) {
                failed = true;
                break;
            }
            if (tid == 0) {
                const uint32_t st = c % kStages;
                const uint32_t sa = tc::smem_addr(smem_raw + st * stage_bytes), sb = sa + a_bytes;
                tc::fence_after_sync();
                for (int j = 0; j < kWgradBK / 16; ++j)
                    tc::mma_bf16(tmem, tc::smem_desc(sa + 2 * j * lbo_a, lbo_a, sbo),
                                 tc::smem_desc(sb + 2 * j * lbo_b, lbo_b, sbo), idesc, c > 0 || j > 0);
                tc::mma_commit(tc::smem_addr(&bars[st]));
            }
        } else if (__syncthreads_or(!ok)) {
            failed = true;
            break;
        }
    }
    if (!failed) {
        if (tid == 0) tc::mma_commit(tc::smem_addr(&bars[kStages]));
        const bool ok = tc::mbar_wait(&bars[kStages], 0);
        if (__syncthreads_or(!ok)) {
            failed = true;
        } else {
            tc::fence_after_sync();
            const int m = m0 + tid;
            const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
            for (int n0 = 0; n0 < N; n0 += 16) {
                float v[16];
                tc::tmem_ld16(lane_base + n0, v);
                if (m < rows) {
                    const int tap = m / C, c = m - tap * C;
                    float *dst = a.dw + ((size_t)tap * N + n0) * C + c;
                    for (int i = 0; i < 16; ++i) atomicAdd(dst + (size_t)i * C, v[i]);
                }
            }
        }
    }
    if (failed && tid == 0) atomicExch(a.err, 1);
    tc::cp_async_wait_all();
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, ncols);
}

int g_sms = 0;

int sm_count() {
    if (!g_sms) {
        int dev;
        CRT_CUDA(cudaGetDevice(&dev));
        CRT_CUDA(cudaDeviceGetAttribute(&g_sms, cudaDevAttrMultiProcessorCount, dev));
    }
    return g_sms;
}

int host_tmem_cols(int n) {
    int c = 32;
    while (c < n) c <<= 1;
    return c;
}

}  // namespace

void conv3x3_check(int C, int N) {
    CRT_CHECK(C > 0 && C % 16 == 0 && C <= 512, CRT_ERR_INVALID, "conv3x3: input channels must be a multiple of 16");
    CRT_CHECK(N >= 16 && N % 16 == 0 && N <= 256, CRT_ERR_INVALID,
              "conv3x3: output channels must be a multiple of 16 in [16, 256]");
}

// out = conv3x3(in) (+ bias, ReLU) or the data gradient (flip = 1, weights
// transposed per tap, optional ReLU mask of the layer below).
void conv3x3_launch(const __nv_bfloat16 *in, const __nv_bfloat16 *wgt, const float *bias, const __nv_bfloat16 *mask,
                    __nv_bfloat16 *out, float *out_f32, int *err, int nimg, int h, int w, int C, int N, bool flip,
                    bool relu, cudaStream_t s) {
    conv3x3_check(C, N);
    const int64_t P = (int64_t)nimg * h * w;
    CRT_CHECK(P > 0 && P < (1LL << 31) - kBM, CRT_ERR_INVALID, "conv3x3: bad image size");
    ConvArgs a;
    a.in = in;
    a.wgt = wgt;
    a.bias = bias;
    a.mask = mask;
    a.out = out;
    a.out_f32 = out_f32;
    a.err = err;
    a.nimg = nimg;
    a.h = h;
    a.wd = w;
    a.C = C;
    a.N = N;
    a.flip = flip ? 1 : 0;
    a.relu = relu ? 1 : 0;
    // Weights resident in shared memory when they fit next to 4 or 5 halo
    // stages, else streamed per stage with 3 or 4 stages; the largest
    // channel chunk KC of 64, 32, 16 dividing C that fits wins, then the
    // deeper pipeline.
    const size_t kSmemCap = 220 * 1024;
    const size_t wbytes = (size_t)9 * N * C * 2;
    auto a_stage = [&](int kc) { return (size_t)kc * 3 * kHalo * 2; };
    bool resident = false;
    int stages = 0;
    a.KC = 0;
    for (int kc : {64, 32, 16})
        for (int ns : {5, 4})
            if (!a.KC && C % kc == 0 && wbytes + ns * a_stage(kc) <= kSmemCap) {
                a.KC = kc;
                stages = ns;
                resident = true;
            }
    for (int kc : {64, 32, 16})
        for (int ns : {4, 3})
            if (!a.KC && C % kc == 0 && ns * (a_stage(kc) + (size_t)18 * N * kc) <= kSmemCap) {
                a.KC = kc;
                stages = ns;
            }
    CRT_CHECK(a.KC > 0, CRT_ERR_INVALID, "conv3x3: tile does not fit shared memory");
    const size_t smem = resident ? wbytes + stages * a_stage(a.KC) : stages * (a_stage(a.KC) + (size_t)18 * N * a.KC);
    const void *kfn = resident ? (stages == 5 ? (const void *)k_conv3x3<5, true> : (const void *)k_conv3x3<4, true>)
                               : (stages == 4 ? (const void *)k_conv3x3<4, false> : (const void *)k_conv3x3<3, false>);
    CRT_CUDA(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    CRT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, kConvThreads, smem));
    per_sm = std::max(1, std::min(per_sm, 512 / host_tmem_cols(2 * N)));
    const int64_t padded = (int64_t)(w + 2) * (nimg * (int64_t)(h + 1) + 1);
    CRT_CHECK(padded < (1LL << 31) - 4 * kBM, CRT_ERR_INVALID, "conv3x3: image too large");
    const int64_t tiles = ((int64_t)(w + 2) * (nimg * (int64_t)(h + 1) - 1) + kBM - 1) / kBM;
    const int grid = (int)std::min<int64_t>(tiles, (int64_t)sm_count() * per_sm);
    void *args[] = {&a};
    CRT_CUDA(cudaLaunchKernel(kfn, dim3(grid), dim3(kConvThreads), args, smem, s));
    CRT_CUDA(cudaGetLastError());
}

// dw[9][N][C] += weight gradient of a 3x3 conv with input `in` [P][C] and
// pre-activation output gradient `g` [P][N].
void conv3x3_wgrad_launch(const __nv_bfloat16 *in, const __nv_bfloat16 *g, float *dw, int *err, int nimg, int h, int w,
                          int C, int N, cudaStream_t s) {
    conv3x3_check(C, N);
    const int64_t P = (int64_t)nimg * h * w;
    CRT_CHECK(P > 0 && P < (1LL << 31) - kWgradBK, CRT_ERR_INVALID, "conv3x3_wgrad: bad image size");
    WgradArgs a;
    a.in = in;
    a.g = g;
    a.dw = dw;
    a.err = err;
    a.nimg = nimg;
    a.h = h;
    a.wd = w;
    a.C = C;
    a.N = N;
    const int mtiles = (9 * C + kBM - 1) / kBM;
    const size_t smem = (size_t)kStages * (kBM * kWgradBK * 2 + (size_t)N * kWgradBK * 2);
    CRT_CHECK(smem <= 200 * 1024, CRT_ERR_INVALID, "conv3x3_wgrad: tile does not fit shared memory");
    CRT_CUDA(cudaFuncSetAttribute(k_conv3x3_wgrad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    CRT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_conv3x3_wgrad, kThreads, smem));
    per_sm = std::max(1, std::min(per_sm, 512 / host_tmem_cols(N)));
    // enough pixel splits for about two waves, at least 8 K steps per CTA
    const int64_t want = std::max<int64_t>(1, 2LL * sm_count() * per_sm / mtiles);
    int64_t ppc = (P + want - 1) / want;
    ppc = std::max<int64_t>(ppc, 8 * kWgradBK);
    ppc = (ppc + kWgradBK - 1) / kWgradBK * kWgradBK;
    a.pix_per_cta = (int)ppc;
    dim3 grid((unsigned)((P + ppc - 1) / ppc), (unsigned)mtiles);
    k_conv3x3_wgrad<<<grid, kThreads, smem, s>>>(a);
    CRT_CUDA(cudaGetLastError());
}

}  // namespace crt

using namespace crt;

extern "C" crt_status crt_check_device_errors(crt_ctx *ctx) {
    return guard([&] {
        CRT_CHECK(ctx, CRT_ERR_INVALID, "crt_check_device_errors: null context");
        CRT_CUDA(cudaSetDevice(ctx->device));
        int e = 0;
        CRT_CUDA(cudaDeviceSynchronize());
        CRT_CUDA(cudaMemcpy(&e, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost));
        if (e) {
            CRT_CUDA(cudaMemset(ctx->d_err, 0, sizeof(int)));
            throw Error(CRT_ERR_TIMEOUT, "a tensor-core kernel gave up waiting on an mbarrier");
        }
    });
}

extern "C" crt_status crt_conv3x3_forward(crt_ctx *ctx, const void *d_in, int32_t n, int32_t h, int32_t w,
                                          int32_t cin, const void *d_weights, const float *d_bias, int32_t cout,
                                          int32_t relu, void *d_out_bf16, float *d_out_f32, void *stream) {
    return guard([&] {
        CRT_CHECK(ctx && d_in && d_weights && (d_out_bf16 || d_out_f32), CRT_ERR_INVALID,
                  "crt_conv3x3_forward: null argument");
        CRT_CUDA(cudaSetDevice(ctx->device));
        cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
        conv3x3_launch((const __nv_bfloat16 *)d_in, (const __nv_bfloat16 *)d_weights, d_bias, nullptr,
                       (__nv_bfloat16 *)d_out_bf16, d_out_f32, ctx->d_err, n, h, w, cin, cout, false, relu != 0, s);
    });
}

extern "C" crt_status crt_conv3x3_backward_data(crt_ctx *ctx, const void *d_grad_out, int32_t n, int32_t h, int32_t w,
                                                int32_t cout, const void *d_weights_t, int32_t cin, const void *d_mask,
                                                void *d_grad_in, void *stream) {
    return guard([&] {
        CRT_CHECK(ctx && d_grad_out && d_weights_t && d_grad_in, CRT_ERR_INVALID,
                  "crt_conv3x3_backward_data: null argument");
        CRT_CUDA(cudaSetDevice(ctx->device));
        cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
        conv3x3_launch((const __nv_bfloat16 *)d_grad_out, (const __nv_bfloat16 *)d_weights_t, nullptr,
                       (const __nv_bfloat16 *)d_mask, (__nv_bfloat16 *)d_grad_in, nullptr, ctx->d_err, n, h, w, cout,
                       cin, true, false, s);
    });
}

extern "C" crt_status crt_conv3x3_backward_weights(crt_ctx *ctx, const void *d_in, const void *d_grad_out, int32_t n,
                                                   int32_t h, int32_t w, int32_t cin, int32_t cout, float *d_grad_w,
                                                   void *stream) {
    return guard([&] {
        CRT_CHECK(ctx && d_in && d_grad_out && d_grad_w, CRT_ERR_INVALID,
                  "crt_conv3x3_backward_weights: null argument");
        CRT_CUDA(cudaSetDevice(ctx->device));
        cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
        conv3x3_wgrad_launch((const __nv_bfloat16 *)d_in, (const __nv_bfloat16 *)d_grad_out, d_grad_w, ctx->d_err, n,
                             h, w, cin, cout, s);
    });
}
