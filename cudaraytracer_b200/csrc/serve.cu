// Multi-scene render server: continuous batching of render requests over
// resident scenes in shared wavefronts.
//
// The reference renders one scene, one request at a time, behind global
// singletons (renderParam, Src/Core/scene.h:20-46; Renderer::RenderLoop,
// Src/Core/renderer.cuh:1106-1307). Here many loaded scenes stay resident
// on the device; render requests of any scene, resolution and spp are queued
// and admitted while a request slot and HBM budget (scenes + shared wavefront
// + the admitted requests' accumulators) allow. Each wavefront pass takes up
// to paths_per_pass paths from the admitted requests in admission order, so a
// request's tail shares a pass with the heads of the requests behind it, and
// requests that arrive while passes run join the next pass.
//
// Every path carries a tag (scene << 20 | request slot) in the spare word of
// its path state; the stage kernels look up the scene (BVH, materials,
// lights, environment) and the request (camera, seed, RR, depth,
// accumulators) per path. A path's PCG32 stream is keyed by (request seed,
// pixel, sample) and its per-path arithmetic is the single-scene renderer's
// (path.cuh), so a request's image is the same alone and in a mix, up to the
// order of the float atomics that add paths into its pixels.
#include "api_internal.h"
#include "path.cuh"
#include <algorithm>
#include <deque>
#include <map>
#include <unordered_map>

namespace crt {
namespace {

constexpr int kSlotBits = 20;
constexpr uint32_t kSlotMask = (1u << kSlotBits) - 1;
constexpr int kMaxScenes = 1 << (32 - kSlotBits);

struct ReqDesc {
    CamView cam;
    float4 *direct, *indirect;
    uint64_t seed;
    int pixels, max_bounces, rr_start;
    float rr;
};

// A run of consecutive wavefront entries taken from one request.
struct Segment {
    int64_t begin;  // first flattened path index (sample * pixels + pixel) in the request
    int prefix;     // first wavefront index of the run
    uint32_t tag;   // (scene << kSlotBits) | slot
};

__device__ __forceinline__ uint32_t path_tag(const QueueView &q, int i) { return __float_as_uint(q.p[4][i].w); }

// GenerateRayKernel + PinholeGeneratingRay (renderer.cuh:96-115,
// camera.cu:27-35) for the request that owns wavefront entry i.
__global__ void ks_raygen(const ReqDesc *reqs, const Segment *segs, int nseg, int n, QueueView q, int *counters) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) {
        counters[0] = n;
        counters[kHitCounter] = 0;
        counters[kMissCounter] = 0;
        counters[kSssCounter] = 0;
    }
    if (i >= n) return;
    int lo = 0, hi = nseg - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (segs[mid].prefix <= i)
            lo = mid;
        else
            hi = mid - 1;
    }
    const Segment sg = segs[lo];
    const ReqDesc &r = reqs[sg.tag & kSlotMask];
    const int64_t g = sg.begin + (i - sg.prefix);
    const uint32_t sample = (uint32_t)(g / r.pixels);
    const uint32_t pixel = (uint32_t)(g % r.pixels);
    const CamView &cam = r.cam;
    const int px = (int)pixel % cam.w, py = (int)pixel / cam.w;
    PathState s;
    s.rng = pcg32_seed(r.seed, pixel, sample);
    float u0 = pcg32_uniform(s.rng), u1 = pcg32_uniform(s.rng);
    V3 ld = ld3(cam.ld), du = ld3(cam.du), dv = ld3(cam.dv), pos = ld3(cam.pos);
    V3 pp = (ld + (px + u0) * du) + (py + u1) * dv;
    s.o = pos;
    s.d = normalized(pp - pos);
    s.w = V3{1.f, 1.f, 1.f};
    s.dc = s.ic = V3{0.f, 0.f, 0.f};
    s.pdf = 0.f;
    s.pixel = pixel;
    s.first = true;
    s.spec = false;
    store_path(q, i, s, sg.tag);
}

__global__ void __launch_bounds__(128) ks_extend(const SceneView *scenes, QueueView q, const int *n_in, float4 *hits,
                                                 int *counters, int out_idx, int mode, ShadeOrder ord) {
    __shared__ unsigned s_stack[kStageShort * 128];
    ShortStack<kStageShort> st;
    st.col = s_stack + threadIdx.x;
    st.stride = blockDim.x;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        counters[out_idx] = 0;
        counters[2] = 0;
        counters[3] = 0;
    }
    const int n = *n_in;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float4 a = q.p[0][i], b = q.p[1][i];
        const SceneView &sv = scenes[path_tag(q, i) >> kSlotBits];
        const BvhView bvh = sv.bvh;
        const V3 o{a.x, a.y, a.z}, d{b.x, b.y, b.z};
        Hit h = stage_closest<false>(bvh, st, mode, o, d, 0.f, kTriTMax);
        hits[i] = make_float4(h.t, __int_as_float(h.slot), h.b1, h.b2);
        ShadeOrder so = ord;
        so.cls = sv.slot_class;
        shade_order_put(so, counters, h.slot, i);  // the shade order (render_kernels.cuh)
    }
}

// The single-scene shade (k_shade in render.cu) with per-path scene and
// request. A path still alive after its request's last bounce is dropped
// with its pending NEE sample, as the reference drops survivors
// (renderer.cuh:1166-1193). As in render.cu, one launch over the shade
// order's hits (ks_shade, registers capped for 8 resident blocks per SM)
// and one over its misses (ks_shade_miss).
template <bool kMisses>
__device__ __forceinline__ void ks_shade_body(const SceneView *scenes, const ReqDesc *reqs, int bounce,
                                              const QueueView &qin, const float4 *hits, const int *n_in,
                                              const QueueView &qout, int *counters, int out_idx, const ShadowView &sh,
                                              float4 *term0, float4 *term1, const ShadeOrder &ord) {
    (void)n_in;
    const int nhit = counters[kHitCounter];
    const int t_end = kMisses ? counters[kMissCounter] : nhit + counters[kSssCounter];
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < t_end; t += gridDim.x * blockDim.x) {
        const int i = kMisses ? shade_miss_index(ord, t) : shade_hit_index(ord, t, nhit);
        PathState ps = load_path(qin, i);
        const uint32_t tag = path_tag(qin, i);
        const SceneView &s = scenes[tag >> kSlotBits];
        const ReqDesc &r = reqs[tag & kSlotMask];
        StepParams sp;
        sp.bounce = bounce;
        sp.rr = r.rr;
        sp.rr_start = r.rr_start;
        float4 hr = hits[i];
        Hit h;
        h.t = hr.x;
        h.slot = __float_as_int(hr.y);
        h.b1 = hr.z;
        h.b2 = hr.w;
        NeeRecord nee;
        nee.valid = false;
        StepResult res;
        if (kMisses) {
            if (s.env_light >= 0) {
                V3 bg = env_emission(s.env, ps.d);
                if (ps.first)
                    ps.dc = ps.dc + mul(ps.w, bg);
                else
                    ps.ic = ps.ic + mul(ps.w, bg);
            }
            res = kTerminate;
        } else {
            res = path_step(s, sp, ps, h, nee);
        }
        bool cont = res == kContinue;
        const bool drop = cont && bounce + 1 >= r.max_bounces;
        if (drop) {
            cont = false;
            nee.valid = false;
        }
        int slot = warp_alloc(&counters[out_idx], cont);
        if (cont) store_path(qout, slot, ps, tag);
        bool need_term = !cont && !drop && nee.valid;
        int tslot = warp_alloc(&counters[3], need_term);
        if (need_term) {
            term0[tslot] = make_float4(ps.dc.x, ps.dc.y, ps.dc.z, __uint_as_float(ps.pixel));
            term1[tslot] = make_float4(ps.ic.x, ps.ic.y, ps.ic.z, __uint_as_float(tag));
        } else if (!cont && !drop) {
            accumulate(AccumView{r.direct, r.indirect, nullptr}, ps.pixel, ps.dc, ps.ic);
        }
        int sslot = warp_alloc(&counters[2], nee.valid);
        if (nee.valid) {
            uint32_t target = cont ? (uint32_t)slot : (kTermBit | (uint32_t)tslot);
            if (nee.direct) target |= kDirectBit;
            sh.r[0][sslot] = make_float4(nee.hp.x, nee.hp.y, nee.hp.z, nee.hn.x);
            sh.r[1][sslot] = make_float4(nee.hn.y, nee.hn.z, nee.lp.x, nee.lp.y);
            sh.r[2][sslot] = make_float4(nee.lp.z, nee.ln.x, nee.ln.y, nee.ln.z);
            sh.r[3][sslot] = make_float4(nee.C.x, nee.C.y, nee.C.z, __uint_as_float(target));
        }
    }
}

__global__ void __launch_bounds__(128, 8) ks_shade(const SceneView *scenes, const ReqDesc *reqs, int bounce,
                                                QueueView qin, const float4 *hits, const int *n_in, QueueView qout,
                                                int *counters, int out_idx, ShadowView sh, float4 *term0,
                                                float4 *term1, ShadeOrder ord) {
    ks_shade_body<false>(scenes, reqs, bounce, qin, hits, n_in, qout, counters, out_idx, sh, term0, term1, ord);
}

__global__ void __launch_bounds__(128) ks_shade_miss(const SceneView *scenes, const ReqDesc *reqs, int bounce,
                                                     QueueView qin, const float4 *hits, const int *n_in,
                                                     QueueView qout, int *counters, int out_idx, ShadowView sh,
                                                     float4 *term0, float4 *term1, ShadeOrder ord) {
    ks_shade_body<true>(scenes, reqs, bounce, qin, hits, n_in, qout, counters, out_idx, sh, term0, term1, ord);
}

// Light::Visible for each deferred NEE sample against the scene of the path
// it belongs to; then as k_shadow in render.cu.
__global__ void __launch_bounds__(128) ks_shadow(const SceneView *scenes, const ReqDesc *reqs, ShadowView sh,
                                                 int *counters, QueueView qout, float4 *term0, float4 *term1,
                                                 int mode) {
    __shared__ unsigned s_stack[kStageShort * 128];
    ShortStack<kStageShort> st;
    st.col = s_stack + threadIdx.x;
    st.stride = blockDim.x;
    const int n = counters[2];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        counters[kHitCounter] = 0;  // the next bounce's shade order starts empty
        counters[kMissCounter] = 0;
        counters[kSssCounter] = 0;
    }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float4 d = sh.r[3][i];
        uint32_t target = __float_as_uint(d.w);
        uint32_t idx = target & kIndexMask;
        const bool term = (target & kTermBit) != 0;
        const uint32_t tag = term ? __float_as_uint(term1[idx].w) : path_tag(qout, idx);
        float4 a = sh.r[0][i], b = sh.r[1][i], c = sh.r[2][i];
        const BvhView bvh = scenes[tag >> kSlotBits].bvh;
        const V3 hp{a.x, a.y, a.z}, hn{a.w, b.x, b.y}, lp{b.z, b.w, c.x}, ln{c.y, c.z, c.w};
        const bool vis = stage_visible(bvh, st, mode, hp, hn, lp, ln);
        bool direct = (target & kDirectBit) != 0;
        V3 C{d.x, d.y, d.z};
        if (term) {
            float4 t0 = term0[idx], t1 = term1[idx];
            V3 dc{t0.x, t0.y, t0.z}, ic{t1.x, t1.y, t1.z};
            if (vis) {
                if (direct)
                    dc = dc + C;
                else
                    ic = ic + C;
            }
            const ReqDesc &r = reqs[tag & kSlotMask];
            accumulate(AccumView{r.direct, r.indirect, nullptr}, __float_as_uint(t0.w), dc, ic);
        } else if (vis) {
            if (direct) {
                float4 p2 = qout.p[2][idx], p3 = qout.p[3][idx];
                p2.w += C.x;
                p3.x += C.y;
                p3.y += C.z;
                qout.p[2][idx] = p2;
                qout.p[3][idx] = p3;
            } else {
                float4 p3 = qout.p[3][idx], p4 = qout.p[4][idx];
                p3.z += C.x;
                p3.w += C.y;
                p4.x += C.z;
                qout.p[3][idx] = p3;
                qout.p[4][idx] = p4;
            }
        }
    }
}

size_t scene_device_bytes(const Scene &sc) {
    const size_t n = (size_t)sc.bvh.num_tris;
    size_t b = (size_t)sc.bvh.num_nodes * 64 + n * 48 + n * 4;  // nodes, leaf-order triangles, slot_of_prim
    b += (size_t)sc.bvh.num_wide_nodes * (64 + 32);            // 8-wide nodes and their child links
    b += n * 36;                                              // input vertices
    b += n * 64;                                              // shading attributes
    b += sc.host.meshes.size() * sizeof(DMesh) + sc.host.materials.size() * sizeof(DMaterial) +
         sc.host.lights.size() * sizeof(DLight);
    for (const HostTexture &t : sc.host.textures) b += (size_t)t.width * t.height * 4;
    if (sc.host.env_light >= 0) {
        const size_t px = (size_t)sc.host.env_w * sc.host.env_h;
        b += px * 16 + px * 4 + (size_t)sc.host.env_h * 4 + (px + sc.host.env_h) * 8;  // texels, CDFs, alias tables
    }
    return b;
}

// Per wavefront path: two queues of 5 float4, the hit record, 4 shadow and
// 2 terminal float4, and two shade-order entries.
constexpr size_t kWavefrontBytesPerPath = 2 * 5 * 16 + 16 + 4 * 16 + 2 * 16 + 8;

}  // namespace
}  // namespace crt

using namespace crt;

struct crt_server {
    struct Request {
        int64_t id = 0;
        int scene = 0;
        int slot = -1;
        int state = CRT_REQ_QUEUED;
        ReqDesc desc{};
        int64_t total = 0, next = 0;
        size_t bytes = 0;
        float4 *buf = nullptr;  // direct then indirect, pixels float4 each
    };
    struct Pass {
        cudaEvent_t ev = nullptr;
        std::vector<int64_t> finishing;
    };

    crt_ctx *ctx = nullptr;
    crt_server_config cfg{};
    cudaStream_t stream = nullptr, copy_stream = nullptr;
    std::vector<crt_scene *> scenes;
    SceneView *d_scenes = nullptr;
    Wavefront wf;
    ReqDesc *d_reqs = nullptr, *h_reqs = nullptr;  // h_reqs: pinned staging, one entry per slot
    Segment *d_segs = nullptr, *h_segs = nullptr;  // (passes_in_flight + 1) tables of max_requests + 1 entries
    std::vector<cudaEvent_t> events;
    std::deque<Pass> inflight;
    int64_t pass_seq = 0, paths_done = 0, next_id = 1;
    std::deque<Request *> queued;
    std::vector<Request *> active;  // admitted, paths left to enqueue, admission order
    std::vector<Request *> order;   // scratch: active sorted by paths left
    std::unordered_map<int64_t, Request *> reqs;
    std::vector<int> free_slots;
    std::multimap<size_t, float4 *> pool;  // released accumulator buffers by size
    size_t bytes_scenes = 0, bytes_wavefront = 0, bytes_requests = 0, bytes_pool = 0;
    int64_t n_running = 0, n_done = 0;
    int g_ext = 0, g_sh = 0, g_sm = 0, g_sd = 0;

    ~crt_server() {
        if (stream) cudaStreamSynchronize(stream);
        for (auto &kv : reqs) {
            if (kv.second->buf) cudaFree(kv.second->buf);
            delete kv.second;
        }
        for (auto &kv : pool) cudaFree(kv.second);
        for (cudaEvent_t e : events) cudaEventDestroy(e);
        if (d_scenes) cudaFree(d_scenes);
        if (d_reqs) cudaFree(d_reqs);
        if (d_segs) cudaFree(d_segs);
        if (h_reqs) cudaFreeHost(h_reqs);
        if (h_segs) cudaFreeHost(h_segs);
        wf.release();
        if (stream) cudaStreamDestroy(stream);
        if (copy_stream) cudaStreamDestroy(copy_stream);
    }

    size_t bytes_held() const { return bytes_scenes + bytes_wavefront + bytes_requests + bytes_pool; }

    Request *find(int64_t id) {
        auto it = reqs.find(id);
        CRT_CHECK(it != reqs.end(), CRT_ERR_INVALID, "crt_server: unknown request id");
        return it->second;
    }

    // Accumulator buffer of `bytes` from the pool or a new allocation that
    // keeps the held total within the budget (pooled buffers are freed first).
    float4 *take_buffer(size_t bytes) {
        auto it = pool.find(bytes);
        if (it != pool.end()) {
            float4 *p = it->second;
            pool.erase(it);
            bytes_pool -= bytes;
            return p;
        }
        while (!pool.empty() && bytes_held() + bytes > (size_t)cfg.hbm_budget_bytes) {
            auto last = std::prev(pool.end());
            CRT_CUDA(cudaFree(last->second));
            bytes_pool -= last->first;
            pool.erase(last);
        }
        float4 *p = nullptr;
        CRT_CUDA(cudaMalloc(&p, bytes));
        return p;
    }

    bool try_admit(Request *r) {
        if (free_slots.empty()) return false;
        if (bytes_scenes + bytes_wavefront + bytes_requests + r->bytes > (size_t)cfg.hbm_budget_bytes) return false;
        r->buf = take_buffer(r->bytes);
        bytes_requests += r->bytes;
        r->slot = free_slots.back();
        free_slots.pop_back();
        const size_t px = (size_t)r->desc.pixels;
        r->desc.direct = r->buf;
        r->desc.indirect = r->buf + px;
        CRT_CUDA(cudaMemsetAsync(r->buf, 0, r->bytes, stream));
        h_reqs[r->slot] = r->desc;  // the slot's previous occupant finished and was released
        CRT_CUDA(cudaMemcpyAsync(d_reqs + r->slot, h_reqs + r->slot, sizeof(ReqDesc), cudaMemcpyHostToDevice, stream));
        r->state = CRT_REQ_RUNNING;
        ++n_running;
        if (r->total == 0) {
            r->state = CRT_REQ_DONE;  // nothing to render: done once the clear is ordered
            --n_running;
            ++n_done;
        } else {
            active.push_back(r);
        }
        return true;
    }

    int retire(bool wait) {
        int done = 0;
        while (!inflight.empty()) {
            Pass &p = inflight.front();
            cudaError_t e = wait && done == 0 ? cudaEventSynchronize(p.ev) : cudaEventQuery(p.ev);
            if (e == cudaErrorNotReady) break;
            CRT_CHECK(e == cudaSuccess, CRT_ERR_CUDA, std::string("crt_server: pass failed: ") + cudaGetErrorString(e));
            for (int64_t id : p.finishing) {
                Request *r = reqs.at(id);
                r->state = CRT_REQ_DONE;
                --n_running;
                ++n_done;
                ++done;
            }
            inflight.pop_front();
        }
        return done;
    }

    void enqueue_pass() {
        const int cap = cfg.paths_per_pass;
        const int table = (int)(pass_seq % (cfg.passes_in_flight + 1));
        // a pass holds at most one segment per admitted request, plus the
        // oldest request's second segment under shortest-first filling
        Segment *hs = h_segs + (size_t)table * (cfg.max_requests + 1);
        Segment *ds = d_segs + (size_t)table * (cfg.max_requests + 1);
        int n = 0, nseg = 0, max_b = 0;
        Pass pass;
        pass.ev = events[table];
        // one segment: the next `limit` (at most) paths of r
        auto add = [&](Request *r, int64_t limit) {
            const int64_t take = std::min<int64_t>(std::min<int64_t>(r->total - r->next, limit), cap - n);
            if (take <= 0) return;
            CRT_CHECK(nseg <= cfg.max_requests, CRT_ERR_CAPACITY, "crt_server: pass segment table full");
            hs[nseg].begin = r->next;
            hs[nseg].prefix = n;
            hs[nseg].tag = ((uint32_t)r->scene << kSlotBits) | (uint32_t)r->slot;
            ++nseg;
            r->next += take;
            n += (int)take;
            max_b = std::max(max_b, r->desc.max_bounces);
            if (r->next == r->total) pass.finishing.push_back(r->id);
        };
        if (cfg.schedule == CRT_SCHED_ADMISSION_ORDER) {
            for (size_t k = 0; k < active.size() && n < cap; ++k) add(active[k], cap);
        } else {
            // the oldest request's guaranteed share, then fewest paths left first
            add(active[0], cap / 2);
            order.assign(active.begin(), active.end());
            std::stable_sort(order.begin(), order.end(),
                             [](const Request *a, const Request *b) { return a->total - a->next < b->total - b->next; });
            for (size_t k = 0; k < order.size() && n < cap; ++k) add(order[k], cap);
        }
        active.erase(std::remove_if(active.begin(), active.end(), [](Request *r) { return r->next == r->total; }),
                     active.end());
        CRT_CUDA(cudaMemcpyAsync(ds, hs, sizeof(Segment) * nseg, cudaMemcpyHostToDevice, stream));
        QueueView q[2];
        for (int j = 0; j < 2; ++j)
            for (int c = 0; c < 5; ++c) q[j].p[c] = wf.q[j][c];
        ShadowView sh{{wf.shadow[0], wf.shadow[1], wf.shadow[2], wf.shadow[3]}};
        const ShadeOrder ord{wf.order, (int)wf.cap, nullptr};  // ks_extend takes each path's scene's classes
        ks_raygen<<<(n + 255) / 256, 256, 0, stream>>>(d_reqs, ds, nseg, n, q[0], wf.counters);
        const int smem = stage_traversal_env();
        for (int b = 0; b < max_b; ++b) {
            const int in = b & 1, out = 1 - in;
            ks_extend<<<g_ext, 128, 0, stream>>>(d_scenes, q[in], wf.counters + in, wf.hits, wf.counters, out, smem,
                                                 ord);
            ks_shade<<<g_sh, 128, 0, stream>>>(d_scenes, d_reqs, b, q[in], wf.hits, wf.counters + in, q[out],
                                               wf.counters, out, sh, wf.term[0], wf.term[1], ord);
            ks_shade_miss<<<g_sm, 128, 0, stream>>>(d_scenes, d_reqs, b, q[in], wf.hits, wf.counters + in, q[out],
                                                    wf.counters, out, sh, wf.term[0], wf.term[1], ord);
            ks_shadow<<<g_sd, 128, 0, stream>>>(d_scenes, d_reqs, sh, wf.counters, q[out], wf.term[0], wf.term[1],
                                                smem);
        }
        CRT_CUDA(cudaGetLastError());
        CRT_CUDA(cudaEventRecord(pass.ev, stream));
        inflight.push_back(std::move(pass));
        ++pass_seq;
        paths_done += n;
    }

    int step(bool wait) {
        int done = retire(false);
        while (!queued.empty() && try_admit(queued.front())) {
            if (queued.front()->state == CRT_REQ_DONE) ++done;
            queued.pop_front();
        }
        while ((int)inflight.size() < cfg.passes_in_flight && !active.empty()) enqueue_pass();
        if (wait && done == 0 && !inflight.empty()) {
            done += retire(true);
            while (!queued.empty() && try_admit(queued.front())) {
                if (queued.front()->state == CRT_REQ_DONE) ++done;
                queued.pop_front();
            }
            while ((int)inflight.size() < cfg.passes_in_flight && !active.empty()) enqueue_pass();
        }
        return done;
    }
};

extern "C" crt_status crt_server_create(crt_ctx *ctx, const crt_server_config *cfg, crt_server **out) {
    return guard([&] {
        CRT_CHECK(ctx && out, CRT_ERR_INVALID, "crt_server_create: null argument");
        *out = nullptr;
        CRT_CUDA(cudaSetDevice(ctx->device));
        std::unique_ptr<crt_server> s(new crt_server());
        s->ctx = ctx;
        crt_server_config c = cfg ? *cfg : crt_server_config{};
        if (c.hbm_budget_bytes <= 0) c.hbm_budget_bytes = (int64_t)150 << 30;
        if (c.paths_per_pass <= 0) c.paths_per_pass = 8 << 20;
        if (c.max_requests <= 0) c.max_requests = 4096;
        if (c.passes_in_flight <= 0) c.passes_in_flight = 2;
        CRT_CHECK(c.max_requests <= (1 << kSlotBits), CRT_ERR_INVALID, "crt_server_create: max_requests > 2^20");
        CRT_CHECK(c.paths_per_pass <= (int)kIndexMask, CRT_ERR_INVALID, "crt_server_create: paths_per_pass > 2^30");
        CRT_CHECK(c.passes_in_flight <= 64, CRT_ERR_INVALID, "crt_server_create: passes_in_flight > 64");
        CRT_CHECK(c.schedule == CRT_SCHED_SHORTEST_FIRST || c.schedule == CRT_SCHED_ADMISSION_ORDER, CRT_ERR_INVALID,
                  "crt_server_create: unknown schedule");
        s->cfg = c;
        s->bytes_wavefront = kWavefrontBytesPerPath * (size_t)c.paths_per_pass;
        CRT_CHECK(s->bytes_wavefront < (size_t)c.hbm_budget_bytes, CRT_ERR_CAPACITY,
                  "crt_server_create: the wavefront alone exceeds the HBM budget");
        CRT_CUDA(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
        CRT_CUDA(cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking));
        s->wf.reserve((size_t)c.paths_per_pass);
        CRT_CUDA(cudaMalloc(&s->d_scenes, sizeof(SceneView) * kMaxScenes));
        CRT_CUDA(cudaMalloc(&s->d_reqs, sizeof(ReqDesc) * c.max_requests));
        CRT_CUDA(cudaHostAlloc(&s->h_reqs, sizeof(ReqDesc) * c.max_requests, cudaHostAllocDefault));
        const size_t nseg = (size_t)(c.passes_in_flight + 1) * (c.max_requests + 1);
        CRT_CUDA(cudaMalloc(&s->d_segs, sizeof(Segment) * nseg));
        CRT_CUDA(cudaHostAlloc(&s->h_segs, sizeof(Segment) * nseg, cudaHostAllocDefault));
        s->events.resize(c.passes_in_flight + 1);
        for (auto &e : s->events) CRT_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        for (int i = c.max_requests - 1; i >= 0; --i) s->free_slots.push_back(i);
        s->g_ext = persistent_grid((const void *)ks_extend, 128);
        s->g_sh = persistent_grid((const void *)ks_shade, 128);
        s->g_sm = persistent_grid((const void *)ks_shade_miss, 128);
        s->g_sd = persistent_grid((const void *)ks_shadow, 128);
        *out = s.release();
    });
}

extern "C" void crt_server_free(crt_server *srv) {
    if (!srv) return;
    cudaSetDevice(srv->ctx->device);
    delete srv;
}

extern "C" crt_status crt_server_add_scene(crt_server *srv, crt_scene *scene, int32_t *scene_id) {
    return guard([&] {
        CRT_CHECK(srv && scene && scene_id && scene->renderable, CRT_ERR_INVALID,
                  "crt_server_add_scene: not a loaded scene");
        CRT_CHECK(scene->ctx->device == srv->ctx->device, CRT_ERR_INVALID,
                  "crt_server_add_scene: scene on another device");
        CRT_CHECK((int)srv->scenes.size() < kMaxScenes, CRT_ERR_CAPACITY, "crt_server_add_scene: too many scenes");
        const size_t b = scene_device_bytes(*scene);
        CRT_CHECK(srv->bytes_scenes + srv->bytes_wavefront + srv->bytes_requests + b <=
                      (size_t)srv->cfg.hbm_budget_bytes,
                  CRT_ERR_CAPACITY, "crt_server_add_scene: scene does not fit the HBM budget");
        CRT_CUDA(cudaSetDevice(srv->ctx->device));
        SceneView v = make_view(scene->bvh, scene->rd);
        const int id = (int)srv->scenes.size();
        CRT_CUDA(cudaMemcpy(srv->d_scenes + id, &v, sizeof(v), cudaMemcpyHostToDevice));
        srv->scenes.push_back(scene);
        srv->bytes_scenes += b;
        *scene_id = id;
    });
}

extern "C" crt_status crt_server_submit(crt_server *srv, const crt_request *req, int64_t *request_id) {
    return guard([&] {
        CRT_CHECK(srv && req && request_id, CRT_ERR_INVALID, "crt_server_submit: null argument");
        CRT_CHECK(req->scene >= 0 && req->scene < (int)srv->scenes.size(), CRT_ERR_INVALID,
                  "crt_server_submit: unknown scene id");
        CRT_CHECK(req->width > 0 && req->height > 0 && (int64_t)req->width * req->height <= (int64_t)kPixelMask,
                  CRT_ERR_INVALID, "crt_server_submit: bad resolution");
        CRT_CHECK(req->spp >= 0 && req->max_bounces >= 0, CRT_ERR_INVALID, "crt_server_submit: negative count");
        const int64_t px = (int64_t)req->width * req->height;
        auto r = std::make_unique<crt_server::Request>();
        r->bytes = (size_t)px * 2 * sizeof(float4);
        CRT_CHECK(srv->bytes_scenes + srv->bytes_wavefront + r->bytes <= (size_t)srv->cfg.hbm_budget_bytes,
                  CRT_ERR_CAPACITY, "crt_server_submit: request does not fit the HBM budget");
        const crt_scene *sc = srv->scenes[req->scene];
        CameraState c = sc->cam;
        for (int k = 0; k < 3; ++k) c.target[k] = req->camera.target[k];
        c.distance = req->camera.distance;
        c.theta = req->camera.theta_deg;
        c.phi = req->camera.phi_deg;
        c.fovy = req->camera.fovy_deg;
        c.width = req->width;
        c.height = req->height;
        compute_camera(c);
        ReqDesc &d = r->desc;
        for (int k = 0; k < 3; ++k) {
            d.cam.pos[k] = c.position[k];
            d.cam.ld[k] = c.left_down[k];
            d.cam.du[k] = c.du[k];
            d.cam.dv[k] = c.dv[k];
        }
        d.cam.w = req->width;
        d.cam.h = req->height;
        d.seed = req->seed;
        d.pixels = (int)px;
        d.max_bounces = req->max_bounces;
        d.rr = req->rr;
        d.rr_start = req->rr_start_bounce;
        r->scene = req->scene;
        r->total = req->max_bounces > 0 ? px * req->spp : 0;
        const int64_t id = srv->next_id++;
        r->id = id;
        srv->reqs.reserve(srv->reqs.size() + 1);
        srv->queued.push_back(r.get());
        srv->reqs[id] = r.release();
        *request_id = id;
    });
}

extern "C" crt_status crt_server_step(crt_server *srv, int32_t wait, int32_t *n_done) {
    return guard([&] {
        CRT_CHECK(srv, CRT_ERR_INVALID, "crt_server_step: null server");
        CRT_CUDA(cudaSetDevice(srv->ctx->device));
        int d = srv->step(wait != 0);
        if (n_done) *n_done = d;
    });
}

extern "C" crt_status crt_server_poll(crt_server *srv, int64_t request_id, int32_t *state) {
    return guard([&] {
        CRT_CHECK(srv && state, CRT_ERR_INVALID, "crt_server_poll: null argument");
        *state = srv->find(request_id)->state;
    });
}

extern "C" crt_status crt_server_result_device(crt_server *srv, int64_t request_id, const float **d_direct,
                                               const float **d_indirect) {
    return guard([&] {
        CRT_CHECK(srv && d_direct && d_indirect, CRT_ERR_INVALID, "crt_server_result_device: null argument");
        crt_server::Request *r = srv->find(request_id);
        CRT_CHECK(r->state == CRT_REQ_DONE, CRT_ERR_INVALID, "crt_server_result_device: request not finished");
        *d_direct = (const float *)r->desc.direct;
        *d_indirect = (const float *)r->desc.indirect;
    });
}

extern "C" crt_status crt_server_result(crt_server *srv, int64_t request_id, float *direct, float *indirect) {
    return guard([&] {
        CRT_CHECK(srv && direct && indirect, CRT_ERR_INVALID, "crt_server_result: null argument");
        crt_server::Request *r = srv->find(request_id);
        CRT_CHECK(r->state == CRT_REQ_DONE, CRT_ERR_INVALID, "crt_server_result: request not finished");
        CRT_CUDA(cudaSetDevice(srv->ctx->device));
        const size_t bytes = (size_t)r->desc.pixels * sizeof(float4);
        if (r->total == 0) CRT_CUDA(cudaStreamSynchronize(srv->stream));  // its clear was the last work
        CRT_CUDA(cudaMemcpyAsync(direct, r->desc.direct, bytes, cudaMemcpyDeviceToHost, srv->copy_stream));
        CRT_CUDA(cudaMemcpyAsync(indirect, r->desc.indirect, bytes, cudaMemcpyDeviceToHost, srv->copy_stream));
        CRT_CUDA(cudaStreamSynchronize(srv->copy_stream));
    });
}

extern "C" crt_status crt_server_release(crt_server *srv, int64_t request_id) {
    return guard([&] {
        CRT_CHECK(srv, CRT_ERR_INVALID, "crt_server_release: null server");
        crt_server::Request *r = srv->find(request_id);
        CRT_CHECK(r->state != CRT_REQ_RUNNING, CRT_ERR_INVALID, "crt_server_release: request still running");
        if (r->state == CRT_REQ_QUEUED) {
            srv->queued.erase(std::find(srv->queued.begin(), srv->queued.end(), r));
        } else {
            if (r->total == 0) CRT_CUDA(cudaStreamSynchronize(srv->stream));
            srv->pool.emplace(r->bytes, r->buf);
            srv->bytes_pool += r->bytes;
            srv->bytes_requests -= r->bytes;
            srv->free_slots.push_back(r->slot);
            --srv->n_done;
        }
        srv->reqs.erase(request_id);
        delete r;
    });
}

extern "C" crt_status crt_server_get_stats(crt_server *srv, crt_server_stats *st) {
    return guard([&] {
        CRT_CHECK(srv && st, CRT_ERR_INVALID, "crt_server_get_stats: null argument");
        st->queued = (int64_t)srv->queued.size();
        st->running = srv->n_running;
        st->done = srv->n_done;
        st->passes = srv->pass_seq;
        st->paths = srv->paths_done;
        st->bytes_budget = srv->cfg.hbm_budget_bytes;
        st->bytes_scenes = (int64_t)srv->bytes_scenes;
        st->bytes_wavefront = (int64_t)srv->bytes_wavefront;
        st->bytes_requests = (int64_t)srv->bytes_requests;
        st->bytes_pool = (int64_t)srv->bytes_pool;
        st->num_scenes = (int32_t)srv->scenes.size();
        st->passes_in_flight = (int32_t)srv->inflight.size();
    });
}
