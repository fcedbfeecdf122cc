// Internal definitions behind the opaque handles of include/crt.h.
#pragma once
#include "common.cuh"
#include <cuda_bf16.h>
#include "bvh_build.h"
#include "trace.cuh"
#include "render.h"
#include "scene_data.h"
#include "svgf.h"
#include <memory>
#include <vector>
#include <new>
#include <exception>

namespace crt {

// Device buffer that only grows.
struct DeviceScratch {
    void *p = nullptr;
    size_t cap = 0;
    void reserve(size_t bytes);
    ~DeviceScratch();
};

// Runs f and maps exceptions to a crt_status + last-error message.
template <class F>
crt_status guard(F &&f) {
    try {
        f();
        set_last_error("");
        return CRT_OK;
    } catch (const Error &e) {
        set_last_error(e.what());
        return e.status;
    } catch (const std::bad_alloc &) {
        set_last_error("host allocation failed");
        return CRT_ERR_OOM;
    } catch (const std::exception &e) {
        set_last_error(e.what());
        return CRT_ERR_INVALID;
    }
}

struct Scene;

}  // namespace crt

struct crt_ctx {
    int device = 0;
    cudaStream_t streams[2] = {nullptr, nullptr};
    cudaStream_t stream = nullptr;
    crt::DeviceScratch stage[2];
    // Device word set by tensor-core kernels whose bounded waits ran out
    // (read and cleared by crt_check_device_errors).
    int *d_err = nullptr;
};

namespace crt {
// Tensor-core 3x3 convolutions (conv.cu).
void conv3x3_launch(const __nv_bfloat16 *in, const __nv_bfloat16 *wgt, const float *bias, const __nv_bfloat16 *mask,
                    __nv_bfloat16 *out, float *out_f32, int *err, int nimg, int h, int w, int C, int N, bool flip,
                    bool relu, cudaStream_t s);
void conv3x3_wgrad_launch(const __nv_bfloat16 *in, const __nv_bfloat16 *g, float *dw, int *err, int nimg, int h, int w,
                          int C, int N, cudaStream_t s);
}  // namespace crt

namespace crt {
struct Scene {
    crt_ctx *ctx = nullptr;
    float *d_verts = nullptr;
    BvhBuffers bvh;
    // render path (scenes loaded from JSON)
    bool renderable = false;
    HostScene host;
    RenderData rd;
    CameraState cam;
    RenderParams rp;
    Wavefront wf;
    DeviceScratch accum;  // host-API render accumulators
    DeviceScratch batch_scratch;  // multi-view cameras + pass state
    // Every call that uses the wavefront/accumulator scratch waits for the
    // previous such call's work (whatever stream it ran on) and records its
    // own completion here, so calls on different streams cannot overlap on
    // the shared buffers.
    cudaEvent_t scratch_done = nullptr;
    void acquire_scratch(cudaStream_t s);
    void release_scratch(cudaStream_t s);
    ~Scene();
    void fill_info(crt_scene_info_t &info) const;
};
}  // namespace crt

struct crt_scene : crt::Scene {};

namespace crt {
int render_views(Scene &sc, const std::vector<CameraState> &cams, int first_sample, int spp, const Accum &acc,
                 bool use_graph, cudaStream_t stream);
}

struct crt_svgf {
    crt_ctx *ctx = nullptr;
    crt::SvgfState st;
    // owned buffers for crt_render_svgf_frame: two G-buffers, noisy planes
    crt::GBufferPlanes gb[2];
    float4 *noisy_d = nullptr, *noisy_i = nullptr;
    int gi = 0;               // G-buffer of the current frame
    bool have_prev_cam = false;
    crt::CameraState prev_cam;
    ~crt_svgf();
};
