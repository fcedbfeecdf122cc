// 3x3 convolutions (stride 1, zero padding 1) on NHWC BF16 activations as
// implicit GEMMs on the sm_100a tensor cores (tcgen05.mma kind::f16, BF16 x
// BF16 -> FP32 in TMEM). These are the dense contractions of the learned
// kernel-predicting denoiser (kpcn.cu); the reference has no learned part.
//
//   forward : out[p, n] = sum_{t, c} in[p + off(t), c] * w[t][n][c]
//   data grad: out[p, n] = sum_{t, c} g[p - off(t), c] * wt[t][n][c]
//             (wt = w transposed per tap, flip = 1)
//   weights  : dW[t][n][c] += sum_p in[p + off(t), c] * g[p, n]
//
// Three kernels:
//   k_conv3x3             forward and data gradient: output channels as the
//                         MMA's M, 256 (or 128) pixels of one image row as
//                         its N; input rows TMA-loaded in swizzled layouts,
//                         the 9 taps as row-shifted descriptors; a ring of
//                         input rows per column strip (ring mode) or
//                         three-row stages per tile (step mode, weights
//                         resident or streamed).
//   k_conv3x3_wgrad_ring  weight gradient on the same row ring, MN-major,
//                         accumulators resident in TMEM over each CTA's
//                         pixel range.
//   k_conv3x3_wgrad       weight gradient for layers whose ring does not fit
//                         shared memory: (tap, channel) row tiles x output
//                         channels, pixels split over CTAs, cp.async-staged
//                         MN-major operands, FP32 atomics into dW.
#include "api_internal.h"
#include "tc.cuh"
#include <algorithm>
#include <cudaTypedefs.h>
#include <type_traits>

namespace crt {
namespace {

constexpr int kBM = 128;           // k_conv3x3_wgrad: (tap, c) rows per tile
constexpr int kThreads = 128;      // k_conv3x3_wgrad
constexpr int kFwdThreads = 320;  // forward / data gradient: TMA warp, MMA warp, 8 epilogue warps
constexpr int kMaxStages = 5;
constexpr int kStages = 4;         // k_conv3x3_wgrad pipeline depth
constexpr int kWgradBK = 64;       // k_conv3x3_wgrad: pixels per K step

struct ConvArgs {
    const float *bias;          // [N] or null
    const __nv_bfloat16 *mask;  // [P][N] or null: out *= (mask > 0)
    __nv_bfloat16 *out;         // [P][N] or null
    float *out_f32;             // [P][N] or null
    int *err;
    int nimg, h, wd, C, N;
    int KC, RB;                 // channel chunk and its row bytes in shared memory (2 KC, the swizzle span)
    int NP, MB, M;              // pixels per tile (the MMA's N), 128-row blocks of output channels, MMA M
    int stages, resident, flip, relu;
    uint32_t region_bytes;      // one halo row: NP + 2 pixels x RB, rounded up to 1 KB
    uint32_t wchunk_bytes;      // weights of one channel chunk: [KC / 8][9][N][16 B]
    uint32_t stage_bytes, wres_bytes;
};

__device__ __forceinline__ uint32_t tmem_cols(int n) {
    uint32_t c = 32;
    while ((int)c < n) c <<= 1;
    return c;
}

// Forward and data gradient with the output channels on the MMA's M side
// (M = 64 for up to 64 channels, else 128-row blocks; rows past N read
// neighbouring weights and their results are never read back) and NP = 256
// (or 128) pixels of one image row on its N side. One tcgen05.mma costs
// about the same issue time whatever its shape, so the wide N = 256 tile is
// what keeps the tensor core busy.
//
// A tile is pixels x0 .. x0 + NP - 1 of row y of image b. Per channel chunk
// of KC a stage holds the three input rows y - 1, y, y + 1, columns
// x0 - 1 .. x0 + NP, each written by TMA (an NP-wide box and a 2-wide edge
// box, zero-filled outside the image) in the swizzled K-major layout with
// RB = 2 KC bytes per pixel row. Tap (dy, dx) is the MMA whose B operand
// starts dx + 1 rows into row buffer dy + 1: no gather (the swizzle is a
// function of the absolute shared-memory address, so shifted starts read
// the rows TMA wrote). The weights (A, [chunk][k group][tap][n][16 B], no
// swizzle) are loaded by TMA once per CTA when they fit next to the stages,
// else per stage.
// Warp roles (no block-wide barrier inside the tile loop):
//   warp 0     one thread issues the TMA loads of step s into stage s % S
//              (after the MMAs of step s - S released it) with the bytes
//              it expects on full[stage].
//   warp 1     the whole warp runs the MMA loop, one elected lane issues the
//              step's 9 taps x KC / 16 x MB MMAs into one of two TMEM
//              accumulator slots and commits them to empty[stage] and,
//              after a tile's last chunk, to tfull[slot].
//   warps 2-9  epilogue: TMEM lane quarter warp % 4, half (warp - 2) / 4 of
//              the tile's pixels; bias / ReLU in FP32, BF16 staged through
//              shared memory into 16 B stores (ReLU mask applied there).
//              Then arrive on tempty[slot].
// Every wait is bounded and also ends when another role has given up.
// kKS = KC / 16 (K steps per tap) and kMB are compile-time so that the MMA
// warp's loop unrolls into base descriptors plus precomputed offsets: the
// issue loop, not the tensor core, is otherwise the bottleneck.
template <int kKS, int kMB, bool kRing>
__global__ void __launch_bounds__(kFwdThreads, 1)
    k_conv3x3(const __grid_constant__ CUtensorMap map_in, const __grid_constant__ CUtensorMap map_edge,
              const __grid_constant__ CUtensorMap map_w, ConvArgs a) {
    extern __shared__ unsigned char smem_raw[];
    __shared__ uint64_t full[kMaxStages], empty[kMaxStages], tfull[2], tempty[2], wbar, mma_done;
    __shared__ uint32_t tmem_slot;
    __shared__ int abort_flag;
    __shared__ int mma_pace;
    __shared__ __align__(16) __nv_bfloat16 ostage[8][16 * 32];  // per epilogue warp: 16 pixels x 32 channels
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    constexpr int KC = 16 * kKS, RB = 2 * KC, KG = KC / 8, MB = kMB;
    const int C = a.C, N = a.N, W = a.wd, H = a.h, NP = a.NP, S = a.stages;
    const int chunks = C / KC;
    const int ntx = (W + NP - 1) / NP, ntiles = a.nimg * H * ntx;
    const uint32_t region_bytes = a.region_bytes, stage_bytes = a.stage_bytes, wchunk_bytes = a.wchunk_bytes;
    const uint32_t tap_bytes = (uint32_t)N * 16, wkg_bytes = 9 * tap_bytes;
    // 1 KB aligned: TMA swizzle atoms and the descriptors' address phase
    unsigned char *const base = reinterpret_cast<unsigned char *>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
    unsigned char *const wres = base;
    unsigned char *const stages = base + a.wres_bytes;
    const uint32_t slot_cols = (uint32_t)(MB * NP), ncols = tmem_cols(2 * MB * NP);
    // Step mode: tiles blockIdx.x, + gridDim.x, ... in (image, row, x tile)
    // order. Ring mode: a contiguous range of tiles in (image, x tile, row)
    // order, so consecutive tiles are consecutive rows of one column strip.
    const int t_beg = kRing ? (int)((int64_t)ntiles * blockIdx.x / gridDim.x) : 0;
    const int my_tiles = kRing ? (int)((int64_t)ntiles * (blockIdx.x + 1) / gridDim.x) - t_beg
                               : (blockIdx.x < ntiles ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0);
    auto tile_of = [&](int tl, int &b, int &y, int &x0) {
        if (kRing) {
            const int t = t_beg + tl, r2 = t / H;
            y = t - r2 * H;
            x0 = (r2 % ntx) * NP;
            b = r2 / ntx;
        } else {
            const int t = blockIdx.x + tl * gridDim.x, by = t / ntx;
            x0 = (t - by * ntx) * NP;
            y = by % H;
            b = by / H;
        }
    };
    volatile int *abort = &abort_flag;

    if (tid == 0) {
        for (int i = 0; i < S; ++i) {
            tc::mbar_init(&full[i], 1);
            tc::mbar_init(&empty[i], 1);
        }
        for (int i = 0; i < 2; ++i) {
            tc::mbar_init(&tfull[i], 1);
            tc::mbar_init(&tempty[i], 256);
        }
        tc::mbar_init(&wbar, 1);
        tc::mbar_init(&mma_done, 1);
        abort_flag = 0;
        mma_pace = 0;
        tc::fence_mbar_init();
    }
    if (warp == 1) tc::tmem_alloc(&tmem_slot, ncols);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            // ---- TMA producer ----
            if (a.resident) {
                tc::mbar_arrive_expect_tx(&wbar, chunks * wchunk_bytes);
                for (int ch = 0; ch < chunks; ++ch)
                    for (int kg = 0; kg < KG; ++kg)
                        tc::tma_load_3d(wres + ch * wchunk_bytes + kg * wkg_bytes, &map_w, ch * KC + kg * 8, 0, 0,
                                        &wbar);
            }
            int s = 0;
            if (kRing) {
                // one row buffer (all channel chunks) per load; a column
                // strip's first tile loads rows y - 1, y, y + 1, every later
                // tile only row y + 1
                const uint32_t tx = (uint32_t)chunks * (NP + 2) * RB;
                for (int tl = 0; tl < my_tiles && !*abort; ++tl) {
                    int b, y, x0;
                    tile_of(tl, b, y, x0);
                    const bool seg = tl == 0 || y == 0;
                    bool ok = true;
                    for (int yy = seg ? y - 1 : y + 1; yy <= y + 1; ++yy, ++s) {
                        const int st = s % S;
                        if (s >= S && !tc::mbar_wait_or_abort(&empty[st], ((s / S) - 1) & 1, abort)) {
                            ok = false;
                            break;
                        }
                        unsigned char *sa = stages + st * stage_bytes;
                        tc::mbar_arrive_expect_tx(&full[st], tx);
                        for (int ch = 0; ch < chunks; ++ch) {
                            tc::tma_load_4d(sa + ch * region_bytes, &map_in, ch * KC, x0 - 1, yy, b, &full[st]);
                            tc::tma_load_4d(sa + ch * region_bytes + NP * RB, &map_edge, ch * KC, x0 - 1 + NP, yy, b,
                                            &full[st]);
                        }
                    }
                    if (!ok) break;
                }
            } else {
                const uint32_t tx = 3u * (NP + 2) * RB + (a.resident ? 0u : wchunk_bytes);
                for (int tl = 0; tl < my_tiles && !*abort; ++tl) {
                    int b, y, x0;
                    tile_of(tl, b, y, x0);
                    bool ok = true;
                    for (int ch = 0; ch < chunks; ++ch, ++s) {
                        const int st = s % S;
                        if (s >= S && !tc::mbar_wait_or_abort(&empty[st], ((s / S) - 1) & 1, abort)) {
                            ok = false;
                            break;
                        }
                        unsigned char *sa = stages + st * stage_bytes;
                        tc::mbar_arrive_expect_tx(&full[st], tx);
                        for (int r = 0; r < 3; ++r) {
                            tc::tma_load_4d(sa + r * region_bytes, &map_in, ch * KC, x0 - 1, y + r - 1, b, &full[st]);
                            tc::tma_load_4d(sa + r * region_bytes + NP * RB, &map_edge, ch * KC, x0 - 1 + NP,
                                            y + r - 1, b, &full[st]);
                        }
                        if (!a.resident)
                            for (int kg = 0; kg < KG; ++kg)
                                tc::tma_load_3d(sa + 3 * region_bytes + kg * wkg_bytes, &map_w, ch * KC + kg * 8, 0, 0,
                                                &full[st]);
                    }
                    if (!ok) break;
                }
            }
            // no TMA write may land after the CTA has exited: wait for the
            // last phase issued on every stage (immediate when consumed)
            for (int st = 0; st < S && st < s; ++st) {
                const int last = s - 1 - ((s - 1 - st) % S);
                tc::mbar_wait(&full[st], (last / S) & 1);
            }
            if (a.resident) tc::mbar_wait(&wbar, 0);
        }
    } else if (warp == 1) {
        // ---- MMA issuer: the whole warp runs the loop, one lane issues ----
        // Descriptor offsets (16 B units in the start-address field, which
        // never carries: shared addresses stay below 256 KB) of the 9 taps:
        // B = row buffer r shifted by c rows; A = the tap's weight slice
        // (mirrored taps for the data gradient).
        const uint32_t idesc = tc::idesc_bf16(a.M, NP, false, false);
        uint32_t boff[9], aoff[9];
#pragma unroll
        for (int t = 0; t < 9; ++t) {
            const int r = t / 3, c = t % 3, tap = a.flip ? 8 - t : t;
            boff[t] = (r * region_bytes + c * RB) >> 4;
            aoff[t] = (tap * tap_bytes) >> 4;
        }
        const uint64_t bdesc0 = tc::smem_desc_sw(tc::smem_addr(stages), RB);
        const uint64_t adesc0 = tc::smem_desc(tc::smem_addr(a.resident ? wres : stages + 3 * region_bytes), wkg_bytes, 128);
        const uint32_t stage16 = stage_bytes >> 4, wchunk16 = wchunk_bytes >> 4, kstep_a16 = (2 * wkg_bytes) >> 4;
        int s = 0;
        bool run = !a.resident || tc::mbar_wait_or_abort_warp(&wbar, 0, abort);
        if (kRing) {
            // rows top, top + 1, top + 2 of the load sequence; after the
            // tile, row `top` is released (all three at a strip's end)
            int top = 0;
            for (int tl = 0; tl < my_tiles && run; ++tl) {
                int b, y, x0;
                tile_of(tl, b, y, x0);
                if (tl == 0 || y == 0) {
                    top = s;
                    s += 3;
                } else {
                    top += 1;
                    s += 1;
                }
                const int slot = tl & 1;
                if (tl >= 2 && !tc::mbar_wait_or_abort_warp(&tempty[slot], ((tl >> 1) - 1) & 1, abort)) break;
                tc::fence_after_sync();
                const uint32_t d = tmem + slot * slot_cols;
                for (int r = 0; r < 3 && run; ++r) {
                    const int ld = top + r, st = ld % S;
                    if (!tc::mbar_wait_or_abort_warp(&full[st], (ld / S) & 1, abort)) {
                        run = false;
                        break;
                    }
                    tc::fence_after_sync();
                    const uint64_t bd = bdesc0 + st * stage16;
                    for (int ch = 0; ch < chunks; ++ch) {
                        const uint64_t bdc = bd + ((ch * region_bytes) >> 4);
                        const uint64_t adc = adesc0 + ch * wchunk16;
#pragma unroll
                        for (int c = 0; c < 3; ++c)
#pragma unroll
                            for (int kk = 0; kk < kKS; ++kk)
#pragma unroll
                                for (int mb = 0; mb < kMB; ++mb)
                                    tc::mma_bf16_warp(d + mb * NP, adc + aoff[3 * r + c] + kk * kstep_a16 + mb * 128,
                                                      bdc + ((c * RB) >> 4) + kk * 2, idesc,
                                                      r > 0 || ch > 0 || c > 0 || kk > 0);
                    }
                    // A shared-memory atomic by the issuing lane after each
                    // row of MMAs. Measured on B200: without it the kernel
                    // takes 2.3x as long (0.56 against 0.24 ms at 1920x1080,
                    // 64 -> 64); a plain store, a tcgen05 fence, a sleep of
                    // up to 60 ns or a spinning test_wait do not help.
                    if (lane == 0) atomicAdd(&mma_pace, 1);
                }
                if (!run) break;
                const bool strip_ends = tl + 1 == my_tiles || y + 1 == H;
                for (int r = 0; r < (strip_ends ? 3 : 1); ++r) tc::mma_commit_warp(tc::smem_addr(&empty[(top + r) % S]));
                tc::mma_commit_warp(tc::smem_addr(&tfull[slot]));
            }
        } else {
            for (int tl = 0; tl < my_tiles && run; ++tl) {
                const int slot = tl & 1;
                if (tl >= 2 && !tc::mbar_wait_or_abort_warp(&tempty[slot], ((tl >> 1) - 1) & 1, abort)) break;
                tc::fence_after_sync();
                const uint32_t d = tmem + slot * slot_cols;
                for (int ch = 0; ch < chunks; ++ch, ++s) {
                    const int st = s % S;
                    if (!tc::mbar_wait_or_abort_warp(&full[st], (s / S) & 1, abort)) {
                        run = false;
                        break;
                    }
                    tc::fence_after_sync();
                    const uint64_t bd = bdesc0 + st * stage16;
                    const uint64_t ad = adesc0 + (a.resident ? ch * wchunk16 : st * stage16);
#pragma unroll
                    for (int t = 0; t < 9; ++t)
#pragma unroll
                        for (int kk = 0; kk < kKS; ++kk)
#pragma unroll
                            for (int mb = 0; mb < kMB; ++mb)
                                tc::mma_bf16_warp(d + mb * NP, ad + aoff[t] + kk * kstep_a16 + mb * 128, bd + boff[t] + kk * 2,
                                                  idesc, ch > 0 || t > 0 || kk > 0);
                    if (lane == 0) atomicAdd(&mma_pace, 1);  // see the ring-mode loop
                    tc::mma_commit_warp(tc::smem_addr(&empty[st]));
                    if (ch == chunks - 1) tc::mma_commit_warp(tc::smem_addr(&tfull[slot]));
                }
            }
        }
        // every MMA issued has finished before TMEM is released
        tc::mma_commit_warp(tc::smem_addr(&mma_done));
        if (lane == 0) tc::mbar_wait(&mma_done, 0);
        __syncwarp();
    } else {
        // ---- epilogue ----
        // TMEM lane quarter q holds channels q * cpq .. + cpq - 1 of each
        // 128-row block in its first cpq lanes (M = 128: 32 per quarter;
        // M = 64: rows 16 q .. 16 q + 15 sit in lanes 32 q .. 32 q + 15).
        // Per 16-pixel chunk the warp converts its channels to BF16 (bias,
        // ReLU), stages them as [pixel][channel] in shared memory and writes
        // 16 B pieces (8 channels of one pixel; the ReLU mask applied there).
        const int q = warp & 3, half = (warp - 2) >> 2;
        const int cpq = a.M == 64 ? 16 : 32, pieces = 16 * cpq / 8;
        const int cbeg = half * (NP / 2), cend = cbeg + NP / 2;
        __nv_bfloat16 *const os = ostage[warp - 2];
        for (int tl = 0; tl < my_tiles; ++tl) {
            const int slot = tl & 1;
            if (!tc::mbar_wait_or_abort(&tfull[slot], (tl >> 1) & 1, abort)) break;
            tc::fence_after_sync();
            int b, y, x0;
            tile_of(tl, b, y, x0);
            const size_t row_pix = ((size_t)b * H + y) * W;
            for (int mb = 0; mb < MB; ++mb) {
                const int cq = mb * 128 + q * cpq;  // first channel of this quarter
                if (cq >= N) continue;             // warp-uniform: no channels here
                const int co = cq + lane;
                const bool cvalid = lane < cpq && co < N;
                const float bias = (a.bias && cvalid) ? a.bias[co] : 0.f;
                const uint32_t taddr = tmem + ((uint32_t)(q * 32) << 16) + slot * slot_cols + mb * NP;
                for (int col = cbeg; col < cend && x0 + col < W; col += 16) {
                    float v[16];
                    tc::tmem_ld16(taddr + col, v);
#pragma unroll
                    for (int i = 0; i < 16; ++i) {
                        v[i] += bias;
                        if (a.relu) v[i] = fmaxf(v[i], 0.f);
                    }
                    if (a.out_f32 && cvalid)
#pragma unroll
                        for (int i = 0; i < 16; ++i)
                            if (x0 + col + i < W) a.out_f32[(row_pix + x0 + col + i) * N + co] = v[i];
                    if (!a.out) continue;
                    if (lane < cpq)
#pragma unroll
                        for (int i = 0; i < 16; ++i) os[i * cpq + lane] = __float2bfloat16_rn(v[i]);
                    __syncwarp();
                    for (int j = lane; j < pieces; j += 32) {
                        const int px = j / (cpq / 8), part = j - px * (cpq / 8);
                        const int c8 = cq + part * 8;
                        if (x0 + col + px < W && c8 < N) {
                            uint4 val = *reinterpret_cast<const uint4 *>(os + px * cpq + part * 8);
                            const size_t o = (row_pix + x0 + col + px) * N + c8;
                            if (a.mask) {
                                const uint4 mv = *reinterpret_cast<const uint4 *>(a.mask + o);
                                const __nv_bfloat16 *mb16 = reinterpret_cast<const __nv_bfloat16 *>(&mv);
                                __nv_bfloat16 *vb = reinterpret_cast<__nv_bfloat16 *>(&val);
                                for (int e = 0; e < 8; ++e)
                                    if (!(__bfloat162float(mb16[e]) > 0.f)) vb[e] = __float2bfloat16_rn(0.f);
                            }
                            *reinterpret_cast<uint4 *>(a.out + o) = val;
                        }
                    }
                    __syncwarp();
                }
            }
            tc::fence_before_sync();
            tc::mbar_arrive(&tempty[slot]);  // this slot's TMEM reads are done
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (tid == 0 && abort_flag) atomicOr(a.err, kErrWaitGaveUp);
    if (warp == 1) tc::tmem_dealloc(tmem, ncols);
}

// ---- weight gradient on the row ring ----
//
// dW[t][n][c] += sum_p in[p + off(t)][c] * g[p][n] as one GEMM per CTA with
// rows (tap, channel), columns n and K = the CTA's pixels, accumulated in
// TMEM over its whole contiguous range of row tiles (same order as the
// forward's ring mode: consecutive rows of one column strip).
// A = the input rows of the ring, read MN-major: a 128-row block is the
// channel chunk (KC channels per 2 KC-byte swizzled row) of 128 / KC
// dx-adjacent taps of one input row; consecutive taps are the same rows
// shifted by one pixel, i.e. MN groups one row apart (LBO = one row). Taps
// past the third and channels past C fill the block's spare rows; their
// results are not read. B = the output gradient tile (NP pixels x N
// channels, TMA-loaded, MN-major). Blocks of one CTA group: TMEM holds
// (blocks per group) x N columns; with more blocks than fit, the grid is
// split into groups that each accumulate a subset and read all inputs.
struct WgradRingArgs {
    float *dw;  // [9][N][C], accumulated
    int *err;
    int nimg, h, wd, C, N;
    int NP, R;  // pixels per tile, ring rows
    int G, blocks_per_group, total_blocks;
    uint32_t region_bytes, row_bytes;     // input: one channel chunk of a ring row, one ring row
    uint32_t gregion_bytes, gtile_bytes;  // gradient: one channel group of a tile, one tile
};

template <int kKS, int kGS>  // input chunk KC = 16 kKS, gradient channel group 16 kGS
__global__ void __launch_bounds__(kFwdThreads, 1)
    k_conv3x3_wgrad_ring(const __grid_constant__ CUtensorMap map_in, const __grid_constant__ CUtensorMap map_edge,
                         const __grid_constant__ CUtensorMap map_g, WgradRingArgs a) {
    extern __shared__ unsigned char smem_raw[];
    __shared__ uint64_t full[kMaxStages], empty[kMaxStages], gfull[2], gempty[2], mma_done;
    __shared__ uint32_t tmem_slot;
    __shared__ int abort_flag, mma_pace;
    constexpr int KC = 16 * kKS, RB = 2 * KC, GKC = 16 * kGS, RBG = 2 * GKC;
    constexpr int TPB = KC == 64 ? 2 : 3;  // valid taps (dx) per 128-row block
    constexpr int BPD = KC == 64 ? 2 : 1;  // blocks per (input row, channel chunk)
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int C = a.C, N = a.N, W = a.wd, H = a.h, NP = a.NP, S = a.R;
    const int chunks = C / KC, ggroups = N / GKC;
    const int ntx = (W + NP - 1) / NP, ntiles = a.nimg * H * ntx;
    const int grp = blockIdx.x % a.G, ctas = gridDim.x / a.G, ci = blockIdx.x / a.G;
    const int b_beg = grp * a.blocks_per_group, b_end = min(a.total_blocks, b_beg + a.blocks_per_group);
    const int t_beg = (int)((int64_t)ntiles * ci / ctas);
    const int my_tiles = (int)((int64_t)ntiles * (ci + 1) / ctas) - t_beg;
    const uint32_t ncols = tmem_cols(a.blocks_per_group * N);
    unsigned char *const base = reinterpret_cast<unsigned char *>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
    unsigned char *const ring = base;
    unsigned char *const gbuf = base + (size_t)S * a.row_bytes;
    auto tile_of = [&](int tl, int &b, int &y, int &x0) {
        const int t = t_beg + tl, r2 = t / H;
        y = t - r2 * H;
        x0 = (r2 % ntx) * NP;
        b = r2 / ntx;
    };
    volatile int *abort = &abort_flag;

    if (tid == 0) {
        for (int i = 0; i < S; ++i) {
            tc::mbar_init(&full[i], 1);
            tc::mbar_init(&empty[i], 1);
        }
        for (int i = 0; i < 2; ++i) {
            tc::mbar_init(&gfull[i], 1);
            tc::mbar_init(&gempty[i], 1);
        }
        tc::mbar_init(&mma_done, 1);
        abort_flag = 0;
        mma_pace = 0;
        tc::fence_mbar_init();
    }
    if (warp == 1) tc::tmem_alloc(&tmem_slot, ncols);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            // ---- TMA producer: ring rows (as the forward's ring mode) and
            // one gradient tile per row tile (two buffers) ----
            const uint32_t tx_row = (uint32_t)chunks * (NP + 2) * RB, tx_g = (uint32_t)ggroups * NP * RBG;
            int s = 0, tl = 0;
            for (; tl < my_tiles && !*abort; ++tl) {
                int b, y, x0;
                tile_of(tl, b, y, x0);
                const bool seg = tl == 0 || y == 0;
                bool ok = true;
                for (int yy = seg ? y - 1 : y + 1; yy <= y + 1; ++yy, ++s) {
                    const int st = s % S;
                    if (s >= S && !tc::mbar_wait_or_abort(&empty[st], ((s / S) - 1) & 1, abort)) {
                        ok = false;
                        break;
                    }
                    unsigned char *sa = ring + (size_t)st * a.row_bytes;
                    tc::mbar_arrive_expect_tx(&full[st], tx_row);
                    for (int ch = 0; ch < chunks; ++ch) {
                        tc::tma_load_4d(sa + ch * a.region_bytes, &map_in, ch * KC, x0 - 1, yy, b, &full[st]);
                        tc::tma_load_4d(sa + ch * a.region_bytes + NP * RB, &map_edge, ch * KC, x0 - 1 + NP, yy, b,
                                        &full[st]);
                    }
                }
                if (!ok) break;
                const int gs = tl & 1;
                if (tl >= 2 && !tc::mbar_wait_or_abort(&gempty[gs], ((tl >> 1) - 1) & 1, abort)) break;
                unsigned char *gb = gbuf + (size_t)gs * a.gtile_bytes;
                tc::mbar_arrive_expect_tx(&gfull[gs], tx_g);
                for (int gg = 0; gg < ggroups; ++gg)
                    tc::tma_load_4d(gb + gg * a.gregion_bytes, &map_g, gg * GKC, x0, y, b, &gfull[gs]);
                // (a break above leaves this tile's gradient unissued: tl is
                // then not counted below)
            }
            // no TMA write may land after the CTA has exited
            for (int st = 0; st < S && st < s; ++st) {
                const int last = s - 1 - ((s - 1 - st) % S);
                tc::mbar_wait(&full[st], (last / S) & 1);
            }
            for (int t2 = tl > 2 ? tl - 2 : 0; t2 < tl; ++t2) tc::mbar_wait(&gfull[t2 & 1], (t2 >> 1) & 1);
        }
    } else if (warp == 1) {
        // ---- MMA issuer (whole warp, one elected lane issues) ----
        const uint32_t idesc = tc::idesc_bf16(128, N, true, true);
        const uint32_t ring_addr = tc::smem_addr(ring), gbuf_addr = tc::smem_addr(gbuf);
        const int ksteps = NP / 16;
        int s = 0, top = 0;
        bool run = true;
        for (int tl = 0; tl < my_tiles && run; ++tl) {
            int b, y, x0;
            tile_of(tl, b, y, x0);
            if (tl == 0 || y == 0) {
                top = s;
                s += 3;
            } else {
                top += 1;
                s += 1;
            }
            const int gs = tl & 1;
            if (!tc::mbar_wait_or_abort_warp(&gfull[gs], (tl >> 1) & 1, abort)) break;
            tc::fence_after_sync();
            const uint64_t bd0 = tc::smem_desc_sw(gbuf_addr + gs * a.gtile_bytes, RBG, a.gregion_bytes);
            for (int ri = 0; ri < 3 && run; ++ri) {
                const int ld = top + ri, st = ld % S;
                if (!tc::mbar_wait_or_abort_warp(&full[st], (ld / S) & 1, abort)) {
                    run = false;
                    break;
                }
                tc::fence_after_sync();
                for (int ch = 0; ch < chunks; ++ch)
#pragma unroll
                    for (int bb = 0; bb < BPD; ++bb) {
                        const int blk = (ri * chunks + ch) * BPD + bb;
                        if (blk < b_beg || blk >= b_end) continue;
                        const uint32_t d = tmem + (uint32_t)(blk - b_beg) * N;
                        const uint64_t ad0 = tc::smem_desc_sw(
                            ring_addr + st * a.row_bytes + ch * a.region_bytes + bb * TPB * RB, RB, RB);
                        for (int kk = 0; kk < ksteps; ++kk)
                            tc::mma_bf16_warp(d, ad0 + ((kk * 16 * RB) >> 4), bd0 + ((kk * 16 * RBG) >> 4), idesc,
                                              tl > 0 || kk > 0);
                    }
                if (lane == 0) atomicAdd(&mma_pace, 1);  // see k_conv3x3's ring loop
            }
            if (!run) break;
            const bool strip_ends = tl + 1 == my_tiles || y + 1 == H;
            for (int r = 0; r < (strip_ends ? 3 : 1); ++r) tc::mma_commit_warp(tc::smem_addr(&empty[(top + r) % S]));
            tc::mma_commit_warp(tc::smem_addr(&gempty[gs]));
        }
        tc::mma_commit_warp(tc::smem_addr(&mma_done));
        if (lane == 0) tc::mbar_wait(&mma_done, 0);
        __syncwarp();
    } else {
        // ---- epilogue: add the accumulators into dW ----
        const int q = warp & 3, half = (warp - 2) >> 2, r = q * 32 + lane;
        const bool ok = tc::mbar_wait_or_abort(&mma_done, 0, abort);
        tc::fence_after_sync();
        if (ok && my_tiles > 0 && !*abort)
            for (int blk = b_beg + half; blk < b_end; blk += 2) {
                const int bb = blk % BPD, rc = blk / BPD, ch = rc % chunks, ri = rc / chunks;
                const int gtap = bb * TPB + r / KC, c = ch * KC + r % KC;
                const bool valid = r / KC < TPB && gtap < 3;
                const int t = ri * 3 + gtap;
                const uint32_t taddr = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(blk - b_beg) * N;
                for (int n0 = 0; n0 < N; n0 += 16) {
                    float v[16];
                    tc::tmem_ld16(taddr + n0, v);
                    if (valid)
#pragma unroll
                        for (int i = 0; i < 16; ++i) atomicAdd(a.dw + ((size_t)t * N + n0 + i) * C + c, v[i]);
                }
            }
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (tid == 0 && abort_flag) atomicOr(a.err, kErrWaitGaveUp);
    if (warp == 1) tc::tmem_dealloc(tmem, ncols);
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
    if (failed && tid == 0) atomicOr(a.err, kErrWaitGaveUp);
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

// cuTensorMapEncodeTiled from the driver, found once through the runtime
// (the library links no driver library).
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        CRT_CUDA(cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &f, 12000, cudaEnableDefault, &q));
        CRT_CHECK(f && q == cudaDriverEntryPointSuccess, CRT_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
        fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
    }
    return fn;
}

void encode_map(CUtensorMap *m, const void *ptr, cuuint32_t rank, const cuuint64_t *dims,
                const cuuint64_t *strides_bytes, const cuuint32_t *box, CUtensorMapSwizzle swz) {
    const cuuint32_t ones[5] = {1, 1, 1, 1, 1};
    const CUresult r = tensor_map_encoder()(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, rank, const_cast<void *>(ptr), dims,
                                            strides_bytes, box, ones, CU_TENSOR_MAP_INTERLEAVE_NONE, swz,
                                            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    CRT_CHECK(r == CUDA_SUCCESS, CRT_ERR_CUDA, "conv3x3: tensor map encoding failed");
}

size_t round1k(size_t v) { return (v + 1023) & ~(size_t)1023; }

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
    CRT_CHECK(nimg > 0 && h > 0 && w > 0 && P < (1LL << 31), CRT_ERR_INVALID, "conv3x3: bad image size");
    CRT_CHECK((reinterpret_cast<uintptr_t>(in) & 15) == 0 && (reinterpret_cast<uintptr_t>(wgt) & 15) == 0,
              CRT_ERR_INVALID, "conv3x3: input and weights must be 16-byte aligned");
    CRT_CHECK((!out || (reinterpret_cast<uintptr_t>(out) & 15) == 0) &&
                  (!out_f32 || (reinterpret_cast<uintptr_t>(out_f32) & 3) == 0) &&
                  (!mask || (reinterpret_cast<uintptr_t>(mask) & 15) == 0),
              CRT_ERR_INVALID, "conv3x3: output and mask must be 16-byte aligned");
    ConvArgs a;
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
    // Tile: 256 pixels (one MMA of N = 256) unless the image is at most 128
    // wide or there are more than 128 output channels (two 128-row M
    // blocks; the TMEM then holds 2 slots x 2 x 128 columns).
    a.MB = N > 128 ? 2 : 1;
    a.M = N <= 64 ? 64 : 128;  // M = 64 spreads the channels over all four TMEM lane quarters
    a.NP = (a.MB == 2 || w <= 128) ? 128 : 256;
    const size_t kCap = 220 * 1024 - 1024 - 2048 - 8192;  // minus base alignment, over-read pad, epilogue staging
    const size_t wbytes = round1k((size_t)9 * N * C * 2);
    auto region = [&](int rb) { return round1k((size_t)(a.NP + 2) * rb); };
    a.KC = 0;
    a.stages = 0;
    a.resident = 0;
    bool ring = false;
    // Ring mode (preferred): resident weights and a ring of 4 or 5 input
    // rows, each holding all channels in chunks of the widest KC dividing C;
    // every input row is then loaded once per column strip.
    {
        const int kc = C % 64 == 0 ? 64 : C % 32 == 0 ? 32 : 16;
        const size_t row = (size_t)(C / kc) * region(2 * kc);
        for (int ns : {5, 4})
            if (!a.KC && wbytes + ns * row <= kCap) {
                a.KC = kc;
                a.stages = ns;
                a.resident = 1;
                ring = true;
            }
    }
    // Step mode: a stage is one channel chunk of the three rows of one tile.
    // Row bytes RB = 2 KC of 128, 64 or 32 (the TMA swizzle span); weights
    // resident when they fit next to at least 3 stages (widest chunk first,
    // then the deepest pipeline), else streamed with every stage.
    for (int rb : {128, 64, 32})
        for (int ns : {5, 4, 3})
            if (!a.KC && C % (rb / 2) == 0 && wbytes + ns * 3 * region(rb) <= kCap) {
                a.KC = rb / 2;
                a.stages = ns;
                a.resident = 1;
            }
    // (a pipeline of 3 or 4 stages at any chunk width first: the streamed
    // weights dominate a stage; two stages only for the widest layers)
    for (int ns : {4, 3, 2})
        for (int rb : {128, 64, 32})
            if (!a.KC && (ns >= 3 || rb == 32) && C % (rb / 2) == 0 &&
                ns * (3 * region(rb) + round1k((size_t)(rb / 16) * 9 * N * 16)) <= kCap) {
                a.KC = rb / 2;
                a.stages = ns;
            }
    CRT_CHECK(a.KC > 0, CRT_ERR_INVALID, "conv3x3: tile does not fit shared memory");
    a.RB = 2 * a.KC;
    a.region_bytes = (uint32_t)region(a.RB);
    a.wchunk_bytes = (uint32_t)((a.KC / 8) * 9 * N * 16);
    a.stage_bytes = (uint32_t)(ring ? (size_t)(C / a.KC) * a.region_bytes
                                    : 3 * a.region_bytes + (a.resident ? 0 : round1k(a.wchunk_bytes)));
    a.wres_bytes = a.resident ? (uint32_t)round1k((size_t)(C / a.KC) * a.wchunk_bytes) : 0u;
    const size_t smem = 1024 + a.wres_bytes + (size_t)a.stages * a.stage_bytes + 2048;

    // input [nimg][h][w][C] as 4D (C, w, h, nimg); weights [9][N][C] as 3D (C, N, 9)
    CUtensorMap map_in, map_edge, map_w;
    const CUtensorMapSwizzle swz = a.RB == 128 ? CU_TENSOR_MAP_SWIZZLE_128B
                                   : a.RB == 64 ? CU_TENSOR_MAP_SWIZZLE_64B
                                                : CU_TENSOR_MAP_SWIZZLE_32B;
    const cuuint64_t dims[4] = {(cuuint64_t)C, (cuuint64_t)w, (cuuint64_t)h, (cuuint64_t)nimg};
    const cuuint64_t strides[3] = {(cuuint64_t)C * 2, (cuuint64_t)w * C * 2, (cuuint64_t)h * w * C * 2};
    const cuuint32_t box[4] = {(cuuint32_t)a.KC, (cuuint32_t)a.NP, 1, 1};
    const cuuint32_t box_edge[4] = {(cuuint32_t)a.KC, 2, 1, 1};
    encode_map(&map_in, in, 4, dims, strides, box, swz);
    encode_map(&map_edge, in, 4, dims, strides, box_edge, swz);
    const cuuint64_t wdims[3] = {(cuuint64_t)C, (cuuint64_t)N, 9};
    const cuuint64_t wstrides[2] = {(cuuint64_t)C * 2, (cuuint64_t)N * C * 2};
    const cuuint32_t wbox[3] = {8, (cuuint32_t)N, 9};
    encode_map(&map_w, wgt, 3, wdims, wstrides, wbox, CU_TENSOR_MAP_SWIZZLE_NONE);

    using Kfn = void (*)(CUtensorMap, CUtensorMap, CUtensorMap, ConvArgs);
    const Kfn kfns[2][2][3] = {{{k_conv3x3<1, 1, false>, k_conv3x3<2, 1, false>, k_conv3x3<4, 1, false>},
                                {k_conv3x3<1, 2, false>, k_conv3x3<2, 2, false>, k_conv3x3<4, 2, false>}},
                               {{k_conv3x3<1, 1, true>, k_conv3x3<2, 1, true>, k_conv3x3<4, 1, true>},
                                {k_conv3x3<1, 2, true>, k_conv3x3<2, 2, true>, k_conv3x3<4, 2, true>}}};
    const Kfn kfn = kfns[ring ? 1 : 0][a.MB - 1][a.KC == 16 ? 0 : a.KC == 32 ? 1 : 2];
    CRT_CUDA(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    CRT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, kFwdThreads, smem));
    per_sm = std::max(1, std::min(per_sm, 512 / host_tmem_cols(2 * a.MB * a.NP)));
    const int64_t tiles = (int64_t)nimg * h * ((w + a.NP - 1) / a.NP);
    const int grid = (int)std::min<int64_t>(tiles, (int64_t)sm_count() * per_sm);
    kfn<<<grid, kFwdThreads, smem, s>>>(map_in, map_edge, map_w, a);
    CRT_CUDA(cudaGetLastError());
}

// dw[9][N][C] += weight gradient of a 3x3 conv with input `in` [P][C] and
// pre-activation output gradient `g` [P][N].
namespace {
// Weight gradient on the row ring when the ring and two gradient tiles fit
// in shared memory; returns false (nothing launched) otherwise.
bool wgrad_ring_launch(const __nv_bfloat16 *in, const __nv_bfloat16 *g, float *dw, int *err, int nimg, int h, int w,
                       int C, int N, cudaStream_t s) {
    if ((reinterpret_cast<uintptr_t>(in) & 15) || (reinterpret_cast<uintptr_t>(g) & 15)) return false;
    const int KC = C % 64 == 0 ? 64 : C % 32 == 0 ? 32 : 16, GKC = N % 64 == 0 ? 64 : N % 32 == 0 ? 32 : 16;
    const int RB = 2 * KC, RBG = 2 * GKC;
    WgradRingArgs a;
    a.dw = dw;
    a.err = err;
    a.nimg = nimg;
    a.h = h;
    a.wd = w;
    a.C = C;
    a.N = N;
    a.total_blocks = 3 * (C / KC) * (KC == 64 ? 2 : 1);
    a.blocks_per_group = std::min(a.total_blocks, 512 / N);
    a.G = (a.total_blocks + a.blocks_per_group - 1) / a.blocks_per_group;
    const size_t kCap = 220 * 1024 - 1024;
    a.NP = 0;
    for (int np : {256, 128}) {
        if (a.NP || (np == 256 && w <= 128)) continue;
        const size_t region = round1k((size_t)(np + 2) * RB), row = (size_t)(C / KC) * region;
        const size_t gregion = round1k((size_t)np * RBG), gtile = (size_t)(N / GKC) * gregion;
        for (int ns : {5, 4})
            if (!a.NP && ns * row + 2 * gtile <= kCap) {
                a.NP = np;
                a.R = ns;
                a.region_bytes = (uint32_t)region;
                a.row_bytes = (uint32_t)row;
                a.gregion_bytes = (uint32_t)gregion;
                a.gtile_bytes = (uint32_t)gtile;
            }
    }
    if (!a.NP) return false;
    const size_t smem = 1024 + (size_t)a.R * a.row_bytes + 2 * (size_t)a.gtile_bytes;
    CUtensorMap map_in, map_edge, map_g;
    auto swz = [](int rb) {
        return rb == 128 ? CU_TENSOR_MAP_SWIZZLE_128B : rb == 64 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_32B;
    };
    const cuuint64_t dims[4] = {(cuuint64_t)C, (cuuint64_t)w, (cuuint64_t)h, (cuuint64_t)nimg};
    const cuuint64_t strides[3] = {(cuuint64_t)C * 2, (cuuint64_t)w * C * 2, (cuuint64_t)h * w * C * 2};
    const cuuint32_t box[4] = {(cuuint32_t)KC, (cuuint32_t)a.NP, 1, 1}, box_edge[4] = {(cuuint32_t)KC, 2, 1, 1};
    encode_map(&map_in, in, 4, dims, strides, box, swz(RB));
    encode_map(&map_edge, in, 4, dims, strides, box_edge, swz(RB));
    const cuuint64_t gdims[4] = {(cuuint64_t)N, (cuuint64_t)w, (cuuint64_t)h, (cuuint64_t)nimg};
    const cuuint64_t gstrides[3] = {(cuuint64_t)N * 2, (cuuint64_t)w * N * 2, (cuuint64_t)h * w * N * 2};
    const cuuint32_t gbox[4] = {(cuuint32_t)GKC, (cuuint32_t)a.NP, 1, 1};
    encode_map(&map_g, g, 4, gdims, gstrides, gbox, swz(RBG));
    using Kfn = void (*)(CUtensorMap, CUtensorMap, CUtensorMap, WgradRingArgs);
    const Kfn kfns[3][3] = {{k_conv3x3_wgrad_ring<1, 1>, k_conv3x3_wgrad_ring<1, 2>, k_conv3x3_wgrad_ring<1, 4>},
                            {k_conv3x3_wgrad_ring<2, 1>, k_conv3x3_wgrad_ring<2, 2>, k_conv3x3_wgrad_ring<2, 4>},
                            {k_conv3x3_wgrad_ring<4, 1>, k_conv3x3_wgrad_ring<4, 2>, k_conv3x3_wgrad_ring<4, 4>}};
    const Kfn kfn = kfns[KC == 16 ? 0 : KC == 32 ? 1 : 2][GKC == 16 ? 0 : GKC == 32 ? 1 : 2];
    CRT_CUDA(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int64_t tiles = (int64_t)nimg * h * ((w + a.NP - 1) / a.NP);
    const int ctas = (int)std::max<int64_t>(1, std::min<int64_t>(tiles, sm_count() / a.G > 0 ? sm_count() / a.G : 1));
    kfn<<<ctas * a.G, kFwdThreads, smem, s>>>(map_in, map_edge, map_g, a);
    CRT_CUDA(cudaGetLastError());
    return true;
}
}  // namespace

void conv3x3_wgrad_launch(const __nv_bfloat16 *in, const __nv_bfloat16 *g, float *dw, int *err, int nimg, int h, int w,
                          int C, int N, cudaStream_t s) {
    conv3x3_check(C, N);
    const int64_t P = (int64_t)nimg * h * w;
    CRT_CHECK(P > 0 && P < (1LL << 31) - kWgradBK, CRT_ERR_INVALID, "conv3x3_wgrad: bad image size");
    if (wgrad_ring_launch(in, g, dw, err, nimg, h, w, C, N, s)) return;
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
            if (e & kErrTraversalBounds)
                throw Error(CRT_ERR_CUDA, "a BVH traversal met an out-of-range node, leaf or stack depth and stopped");
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
