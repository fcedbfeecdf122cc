// crt_render_device_noalloc: the wavefront render pass without any device
// allocation.
//
// Who needs it: a host application that embeds the tracer in its own frame
// loop and owns the GPU memory pool (a game engine, a DCC viewport plugin, a
// real-time preview service). Such hosts forbid foreign cudaMalloc/cudaFree
// while a frame is in flight: those calls synchronise the device, can fail
// with out-of-memory in the middle of a frame, and fragment a pool the host
// budgets itself. crt_render_device allocates its path queues on first use
// (and grows them when the image or the samples per pass grow); this entry
// point instead runs the same stage kernels over a fixed scratch area that
// is part of the library's device image.
//
// The scratch is a file-scope __device__ array of kNoAllocBytes (18.4 MB)
// holding the path queues, hit records, shadow records, terminated-path
// records, the shade order and counters for at most kNoAllocMaxPaths = 65,536 paths per
// wavefront (pixels x samples per pass). Every GPU that loads the library
// holds this array until the process exits. Images with more than 65,536
// pixels are rejected with CRT_ERR_CAPACITY. The caller still provides the
// scene (already resident) and the accumulation buffers.
//
// The array's device address is looked up with cudaGetSymbolAddress the
// first time the entry point runs on a device (with that device current),
// so that first call must come before any stream capture on that device.
// All calls share the one array and it keeps the previous call's contents.
// Nothing stale is read: the stage kernels set every queue counter before
// it is used (k_raygen the input count and the shade-order counts, k_extend
// the next bounce's output, shadow and terminal counts, k_shadow the next
// bounce's shade-order counts), and the counter block is also zeroed at the
// start of every call as a defensive measure. Calls whose GPU work overlaps
// (two streams, two host threads, two scenes) race on the array, so they
// must be ordered by the caller.
//
// Block size and samples per wavefront follow the scene's render params as
// crt_render_device does (stage_block; spp_per_pass, capped at
// 65,536 / pixels so one wavefront fits the scratch).
#include "api_internal.h"
#include "render_kernels.cuh"
#include <algorithm>
#include <mutex>

namespace crt {
namespace {

constexpr size_t kNoAllocMaxPaths = 65536;
// per path: 2 queues x 5 float4 + hit + 4 shadow + 2 terminal float4 = 272 B,
// and 8 B of shade order
constexpr size_t kPlane = kNoAllocMaxPaths * sizeof(float4);
constexpr size_t kCounterBytes = 256;
constexpr size_t kOrderBytes = 2 * kNoAllocMaxPaths * sizeof(int);
constexpr size_t kNoAllocBytes = 17 * kPlane + kCounterBytes + kOrderBytes;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void *g_scratch[kMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device (looked up once
// per device; the host-side symbol itself is not a device address).
unsigned char *scratch_on_current_device() {
    int dev = 0;
    CRT_CUDA(cudaGetDevice(&dev));
    CRT_CHECK(dev >= 0 && dev < kMaxDevices, CRT_ERR_INVALID, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch[dev]) {
        void *ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        CRT_CHECK(e == cudaSuccess && ptr != nullptr, CRT_ERR_CUDA,
                  std::string("cudaGetSymbolAddress(no-alloc scratch): ") + cudaGetErrorString(e));
        g_scratch[dev] = ptr;
    }
    return static_cast<unsigned char *>(g_scratch[dev]);
}

}  // namespace
}  // namespace crt

using namespace crt;

extern "C" crt_status crt_render_device_noalloc(crt_scene *scene, int32_t first_sample, int32_t spp, float *d_direct,
                                                float *d_indirect, float *d_sumsq, void *stream) {
    return guard([&] {
        CRT_CHECK(scene && scene->renderable, CRT_ERR_INVALID, "crt_render_device_noalloc: not a loaded scene");
        CRT_CHECK(d_direct && d_indirect && spp >= 0 && first_sample >= 0, CRT_ERR_INVALID,
                  "crt_render_device_noalloc: bad argument");
        const int w = scene->rp.width, h = scene->rp.height;
        const size_t pixels = (size_t)w * h;
        CRT_CHECK(pixels <= kNoAllocMaxPaths, CRT_ERR_CAPACITY,
                  "crt_render_device_noalloc: " + std::to_string(w) + "x" + std::to_string(h) +
                      " exceeds the fixed scratch of 65536 paths per wavefront; use crt_render_device");
        CRT_CUDA(cudaSetDevice(scene->ctx->device));
        cudaStream_t s = stream ? (cudaStream_t)stream : scene->ctx->stream;
        unsigned char *base = scratch_on_current_device();
        float4 *plane[17];
        for (int k = 0; k < 17; ++k) plane[k] = reinterpret_cast<float4 *>(base + k * kPlane);
        int *counters = reinterpret_cast<int *>(base + 17 * kPlane);
        const ShadeOrder ord{reinterpret_cast<int *>(base + 17 * kPlane + kCounterBytes), (int)kNoAllocMaxPaths,
                             scene->rd.slot_class};
        QueueView q[2];
        for (int k = 0; k < 5; ++k) {
            q[0].p[k] = plane[k];
            q[1].p[k] = plane[5 + k];
        }
        float4 *hits = plane[10];
        ShadowView sh{{plane[11], plane[12], plane[13], plane[14]}};
        float4 *term0 = plane[15], *term1 = plane[16];
        CRT_CUDA(cudaMemsetAsync(counters, 0, kCounterBytes, s));  // defensive; see the header comment
        if (spp == 0) return;

        const SceneView view = make_view(scene->bvh, scene->rd);
        const CameraState &cam = scene->cam;
        const RenderParams &rp = scene->rp;
        CamView cv;
        for (int k = 0; k < 3; ++k) {
            cv.pos[k] = cam.position[k];
            cv.ld[k] = cam.left_down[k];
            cv.du[k] = cam.du[k];
            cv.dv[k] = cam.dv[k];
        }
        cv.w = w;
        cv.h = h;
        AccumView av{(float4 *)d_direct, (float4 *)d_indirect, (float4 *)d_sumsq};
        const int fit = (int)(kNoAllocMaxPaths / pixels);
        const int per_pass = std::max(1, std::min(spp, rp.spp_per_pass > 0 ? std::min(rp.spp_per_pass, fit) : fit));
        const int blk = rp.block();
        const int smem = rp.traversal(scene->bvh.num_tris);
        const int g_sh = persistent_grid((const void *)k_shade, blk);
        const int g_sm = persistent_grid((const void *)k_shade_miss, blk);
        for (int done = 0; done < spp; done += per_pass) {
            const int n = (int)pixels * std::min(per_pass, spp - done);
            StepParams sp;
            sp.bounce = 0;
            sp.rr = rp.rr;
            sp.rr_start = rp.rr_start_bounce;
            sp.seed = rp.seed;
            sp.first_sample = first_sample + done;
            sp.pixels = (int)pixels;
            k_raygen<<<(n + 255) / 256, 256, 0, s>>>(cv, sp, n, q[0], counters);
            for (int b = 0; b < rp.max_bounces; ++b) {
                const int in = b & 1, out = 1 - in;
                sp.bounce = b;
                launch_extend_stage(view.bvh, q[in], counters + in, hits, counters, out, smem, b, ord, blk, s);
                k_shade<<<g_sh, blk, 0, s>>>(view, sp, q[in], hits, counters + in, q[out], counters, out, sh, term0,
                                            term1, av, ord);
                k_shade_miss<<<g_sm, blk, 0, s>>>(view, sp, q[in], hits, counters + in, q[out], counters, out, sh,
                                                 term0, term1, av, ord);
                launch_shadow_stage(view.bvh, sh, counters, q[out], term0, term1, av, smem, blk, s);
            }
            CRT_CUDA(cudaGetLastError());
        }
    });
}
