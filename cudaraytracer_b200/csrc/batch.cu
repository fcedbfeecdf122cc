// Batched multi-view rendering: many camera views of one resident scene in
// shared wavefronts, one CUDA graph per wavefront pass.
//
// The reference renders one view, one sample per pixel per frame, with a
// host-synchronised launch sequence per bounce (Src/Core/renderer.cuh:
// 1144-1193: cudaDeviceSynchronize after every kernel, two blocking copies
// in every StreamCompaction). Here the flattened index space
// (view, sample, pixel) is cut into passes of `paths_per_pass` paths (view
// outermost, so a pass adds into the accumulators of a few views, which stay
// in L2, rather than of every view). One
// pass - view-aware raygen, max_bounces x (extend, shade, shadow), and a
// one-thread kernel that advances the device-side pass base - is captured
// once as a CUDA graph and replayed; queue lengths and the pass base live in
// device memory, so consecutive passes need no host involvement.
//
// Accumulators are view-major: view v's pixel p lives at v * W * H + p, and
// that index also selects the path's PCG32 stream.
#include "api_internal.h"
#include "render_kernels.cuh"
#include <algorithm>

namespace crt {
namespace {

// Per-pass state in device memory: [0] = first flattened path index of the
// pass, [1] = total paths of the request.
__global__ void k_raygen_views(const CamView *cams, int n_views, StepParams sp, int64_t *pass, int chunk,
                               QueueView q, int *counters) {
    const int64_t base = pass[0], total = pass[1];
    const int64_t left = total - base;
    const int n = (int)(left < chunk ? (left > 0 ? left : 0) : chunk);
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) {
        counters[0] = n;
        counters[kHitCounter] = 0;
        counters[kMissCounter] = 0;
        counters[kSssCounter] = 0;
    }
    if (i >= n) return;
    const int64_t g = base + i;
    const int64_t per_view = total / n_views;  // spp * pixels
    const int view = (int)(g / per_view);
    const int64_t rest = g % per_view;
    const uint32_t sample = (uint32_t)(sp.first_sample + rest / sp.pixels);
    const int pix = (int)(rest % sp.pixels);
    const CamView &cam = cams[view];
    const uint32_t pixel = (uint32_t)(view * sp.pixels + pix);  // accumulator index
    const int px = pix % cam.w, py = pix / cam.w;
    Pcg32 rng = pcg32_seed(sp.seed, pixel, sample);
    float u0 = pcg32_uniform(rng), u1 = pcg32_uniform(rng);
    V3 ld = ld3(cam.ld), du = ld3(cam.du), dv = ld3(cam.dv), pos = ld3(cam.pos);
    V3 pp = (ld + (px + u0) * du) + (py + u1) * dv;
    V3 d = normalized(pp - pos);
    const uint32_t meta = pixel | kFirst;
    q.p[0][i] = make_float4(pos.x, pos.y, pos.z, 0.f);
    q.p[1][i] = make_float4(d.x, d.y, d.z, __uint_as_float(meta));
    q.p[2][i] = make_float4(1.f, 1.f, 1.f, 0.f);
    q.p[3][i] = make_float4(0.f, 0.f, 0.f, 0.f);
    q.p[4][i] = make_float4(0.f, __uint_as_float((uint32_t)rng.state), __uint_as_float((uint32_t)(rng.state >> 32)),
                            0.f);
}

__global__ void k_advance_pass(int64_t *pass, int chunk) { pass[0] += chunk; }

}  // namespace

// Renders samples [first_sample, first_sample + spp) of every view into
// view-major accumulators. Returns the number of graph launches (passes).
int render_views(Scene &sc, const std::vector<CameraState> &cams, int first_sample, int spp, const Accum &acc,
                 bool use_graph, cudaStream_t stream) {
    const int W = sc.rp.width, H = sc.rp.height, P = W * H;
    const int V = (int)cams.size();
    CRT_CHECK(V > 0 && P > 0, CRT_ERR_INVALID, "render_views: no views");
    CRT_CHECK((int64_t)V * P <= (int64_t)kPixelMask, CRT_ERR_CAPACITY, "render_views: more than 2^30 pixels");
    const int64_t total = (int64_t)V * P * spp;
    int chunk = sc.rp.paths_per_pass > 0 ? sc.rp.paths_per_pass : (8 << 20);
    chunk = (int)std::min<int64_t>(chunk, std::max<int64_t>(total, 1));
    if ((size_t)chunk > sc.wf.cap) CRT_CUDA(cudaStreamSynchronize(stream));  // buffers are reallocated
    sc.wf.reserve((size_t)chunk);
    // view cameras + pass state on the device (scene-owned scratch)
    size_t cam_bytes = ((sizeof(CamView) * V + 255) / 256) * 256;
    sc.batch_scratch.reserve(cam_bytes + 256);
    CamView *d_cams = (CamView *)sc.batch_scratch.p;
    int64_t *d_pass = (int64_t *)((char *)sc.batch_scratch.p + cam_bytes);
    std::vector<CamView> hv(V);
    for (int v = 0; v < V; ++v) {
        for (int k = 0; k < 3; ++k) {
            hv[v].pos[k] = cams[v].position[k];
            hv[v].ld[k] = cams[v].left_down[k];
            hv[v].du[k] = cams[v].du[k];
            hv[v].dv[k] = cams[v].dv[k];
        }
        hv[v].w = W;
        hv[v].h = H;
    }
    int64_t pass_init[2] = {0, total};
    CRT_CUDA(cudaMemcpyAsync(d_cams, hv.data(), sizeof(CamView) * V, cudaMemcpyHostToDevice, stream));
    CRT_CUDA(cudaMemcpyAsync(d_pass, pass_init, sizeof(pass_init), cudaMemcpyHostToDevice, stream));
    CRT_CUDA(cudaStreamSynchronize(stream));  // pass_init is a host stack buffer

    const SceneView view = make_view(sc.bvh, sc.rd);
    AccumView av{acc.direct, acc.indirect, acc.sumsq};
    QueueView q[2];
    for (int j = 0; j < 2; ++j)
        for (int k = 0; k < 5; ++k) q[j].p[k] = sc.wf.q[j][k];
    ShadowView sh{{sc.wf.shadow[0], sc.wf.shadow[1], sc.wf.shadow[2], sc.wf.shadow[3]}};
    const ShadeOrder ord{sc.wf.order, (int)sc.wf.cap, sc.rd.slot_class};
    const int blk = sc.rp.block();
    const int smem = sc.rp.traversal(sc.bvh.num_tris);
    const int g_sh = persistent_grid((const void *)k_shade, blk);
    const int g_sm = persistent_grid((const void *)k_shade_miss, blk);
    StepParams sp;
    sp.bounce = 0;
    sp.rr = sc.rp.rr;
    sp.rr_start = sc.rp.rr_start_bounce;
    sp.seed = sc.rp.seed;
    sp.first_sample = first_sample;
    sp.pixels = P;
    const int passes = (int)((total + chunk - 1) / chunk);
    auto enqueue_pass = [&](cudaStream_t s) {
        k_raygen_views<<<(chunk + 255) / 256, 256, 0, s>>>(d_cams, V, sp, d_pass, chunk, q[0], sc.wf.counters);
        for (int b = 0; b < sc.rp.max_bounces; ++b) {
            const int in = b & 1, out = 1 - in;
            StepParams bp = sp;
            bp.bounce = b;
            launch_extend_stage(view.bvh, q[in], sc.wf.counters + in, sc.wf.hits, sc.wf.counters, out, smem, b,
                                ord, blk, s);
            k_shade<<<g_sh, blk, 0, s>>>(view, bp, q[in], sc.wf.hits, sc.wf.counters + in, q[out], sc.wf.counters,
                                         out, sh, sc.wf.term[0], sc.wf.term[1], av, ord);
            k_shade_miss<<<g_sm, blk, 0, s>>>(view, bp, q[in], sc.wf.hits, sc.wf.counters + in, q[out],
                                              sc.wf.counters, out, sh, sc.wf.term[0], sc.wf.term[1], av, ord);
            launch_shadow_stage(view.bvh, sh, sc.wf.counters, q[out], sc.wf.term[0], sc.wf.term[1], av, smem,
                                blk, s);
        }
        k_advance_pass<<<1, 1, 0, s>>>(d_pass, chunk);
    };
    if (!use_graph || passes == 1) {
        for (int p = 0; p < passes; ++p) enqueue_pass(stream);
        CRT_CUDA(cudaGetLastError());
        return passes;
    }
    // Capture on the context's second (non-blocking) stream, ordered after
    // and before the caller's stream with events, so any caller stream works
    // (the legacy default stream cannot be captured).
    cudaStream_t gs = sc.ctx->streams[1];
    cudaEvent_t ev_in, ev_out;
    CRT_CUDA(cudaEventCreateWithFlags(&ev_in, cudaEventDisableTiming));
    CRT_CUDA(cudaEventCreateWithFlags(&ev_out, cudaEventDisableTiming));
    CRT_CUDA(cudaEventRecord(ev_in, stream));
    CRT_CUDA(cudaStreamWaitEvent(gs, ev_in, 0));
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    CRT_CUDA(cudaStreamBeginCapture(gs, cudaStreamCaptureModeThreadLocal));
    enqueue_pass(gs);
    cudaError_t ce = cudaStreamEndCapture(gs, &graph);
    CRT_CHECK(ce == cudaSuccess, CRT_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
    CRT_CUDA(cudaGraphInstantiate(&exec, graph, 0));
    for (int p = 0; p < passes; ++p) CRT_CUDA(cudaGraphLaunch(exec, gs));
    CRT_CUDA(cudaEventRecord(ev_out, gs));
    CRT_CUDA(cudaStreamWaitEvent(stream, ev_out, 0));
    cudaGraphExecDestroy(exec);  // released once the launches finish
    cudaGraphDestroy(graph);
    cudaEventDestroy(ev_in);
    cudaEventDestroy(ev_out);
    return passes;
}

}  // namespace crt

using namespace crt;

extern "C" crt_status crt_render_views(crt_scene *scene, int32_t n_views, const crt_camera *cams,
                                       int32_t first_sample, int32_t spp, float *d_direct, float *d_indirect,
                                       float *d_sumsq, int32_t use_graph, void *stream) {
    return guard([&] {
        CRT_CHECK(scene && scene->renderable && cams && n_views > 0 && d_direct && d_indirect && spp >= 0 &&
                      first_sample >= 0,
                  CRT_ERR_INVALID, "crt_render_views: bad argument");
        CRT_CUDA(cudaSetDevice(scene->ctx->device));
        cudaStream_t s = stream ? (cudaStream_t)stream : scene->ctx->stream;
        std::vector<CameraState> cs(n_views);
        for (int v = 0; v < n_views; ++v) {
            CameraState c = scene->cam;
            for (int k = 0; k < 3; ++k) c.target[k] = cams[v].target[k];
            c.distance = cams[v].distance;
            c.theta = cams[v].theta_deg;
            c.phi = cams[v].phi_deg;
            c.fovy = cams[v].fovy_deg;
            c.width = scene->rp.width;
            c.height = scene->rp.height;
            compute_camera(c);
            cs[v] = c;
        }
        Accum acc;
        acc.direct = (float4 *)d_direct;
        acc.indirect = (float4 *)d_indirect;
        acc.sumsq = (float4 *)d_sumsq;
        acc.pixels = (size_t)n_views * scene->rp.width * scene->rp.height;
        scene->acquire_scratch(s);
        if (spp > 0) render_views(*scene, cs, first_sample, spp, acc, use_graph != 0, s);
        scene->release_scratch(s);
    });
}
