// SVGF denoiser and primary-hit G-buffer (svgf.cu).
#pragma once
#include "render.h"

namespace crt {

// Device G-buffer planes, width*height each (encodings in svgf.cu).
struct GBufferPlanes {
    float4 *pos_tri = nullptr;
    ushort4 *normal_mat = nullptr;
    ushort4 *bary_mesh = nullptr;
    float4 *motion_depth = nullptr;
};

// DenoiseParam (Src/Utils/ui.h:14-25) defaults.
struct DenoiseParams {
    int max_history_length = 24;
    float sigma_light = 8.f;
    float sigma_normal = 256.f;
    float sigma_depth = 1.f;
    float reprojection_depth_factor = 0.1f;
    int atrous_iterations = 5;
};

// Temporal history, moments and history lengths (two of each, swapped every
// frame) plus the ping-pong filter buffers.
struct SvgfState {
    int W = 0, H = 0;
    float4 *buf_d[2] = {}, *buf_i[2] = {};
    float4 *hist_d[2] = {}, *hist_i[2] = {};
    float2 *mom_d[2] = {}, *mom_i[2] = {};
    int *hlen[2] = {};
    float4 *edge = nullptr;  // per-pixel decoded normal + depth of the current frame
    int2 *tag = nullptr;     // per-pixel material | mesh << 16, history length
    int t = 0;
    bool first = true;
    void allocate(int w, int h);
    void reset_sync();
    void release();
    ~SvgfState() { release(); }
};

void gbuffer_from_primary(const SceneView &view, const CameraState &cur, const CameraState &prev, const float bmin[3],
                          const float bmax[3], const GBufferPlanes &g, cudaStream_t stream);
// One SVGF frame: temporal reprojection of the noisy 1-spp buffers against
// the history, variance estimate, a-trous passes. Returns launches issued.
int svgf_frame(SvgfState &st, const DenoiseParams &p, const GBufferPlanes &cur, const GBufferPlanes &last,
               const float4 *noisy_d, const float4 *noisy_i, float4 *out_d, float4 *out_i, cudaStream_t s);

}  // namespace crt
