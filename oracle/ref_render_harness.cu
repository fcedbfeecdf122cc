// Headless CUDA build of the reference's renderer (DarrenChen-CN/
// CudaRayTracer): Scene::Scene(path) (Src/Core/scene.cpp:50) loads the scene
// with the reference's own loader, and the frame body of
// Renderer::RenderLoop without denoising (Src/Core/renderer.cuh:1144-1193:
// GenerateRayKernel, then per bounce IntersectionKernel, StreamCompaction,
// ShadingKernel, StreamCompaction) runs on the GPU for `spp` frames into the
// reference's float accumulators. The buffers CudaInit would allocate
// (renderer.cuh:1309-1340) are allocated here; no window, GL context or UI
// exists (the GL entry points the loader touches are no-op stubs,
// ref_gl_stubs.cpp). Per-pixel
// sums of squared per-frame sample values are formed from the accumulator
// increments of each frame, for z-tests. Test/bench infrastructure only.
// thrust algorithms renderer.cuh uses but does not include itself
#include <thrust/scan.h>
#include <thrust/scatter.h>
#include <thrust/sequence.h>
#include <thrust/sort.h>
#include "renderer.cuh"
#include <cstdio>

extern "C" void refr_install_gl_stubs(void);  // ref_gl_stubs.cpp

namespace {

__global__ void k_frame_moments(const float4 *d, const float4 *i, float4 *prev, float4 *sumsq, int n) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    float4 a = d[k], b = i[k], p = prev[k];
    float r = a.x + b.x, g = a.y + b.y, bl = a.z + b.z;
    float dr = r - p.x, dg = g - p.y, db = bl - p.z;
    float4 s = sumsq[k];
    sumsq[k] = make_float4(s.x + dr * dr, s.y + dg * dg, s.z + db * db, s.w + 1.f);
    prev[k] = make_float4(r, g, bl, 0.f);
}
}  // namespace

extern "C" {

void *refr_load(const char *path) {
    refr_install_gl_stubs();
    try {
        Scene *s = new Scene(std::string(path));
        fflush(stdout);
        return s;
    } catch (const std::exception &e) {
        fprintf(stderr, "reference scene load failed: %s\n", e.what());
        return nullptr;
    }
}

void refr_info(int *w, int *h, int *max_bounces, float *rr, float *cam) {
    *w = renderParam.width;
    *h = renderParam.height;
    *max_bounces = renderParam.maxBounces;
    *rr = renderParam.rr;
    for (int k = 0; k < 3; ++k) {
        cam[k] = cameraParam.position(k);
        cam[3 + k] = cameraParam.leftDownPosition(k);
        cam[6 + k] = cameraParam.du(k);
        cam[9 + k] = cameraParam.dv(k);
    }
}

// Renders spp frames (1 sample per pixel each) from cleared accumulators.
// Outputs w*h*4 floats each (direct, indirect sums; sumsq rgb + count),
// rows bottom-up. Returns 0 on success; *ms = GPU time of the frame loop.
int refr_render(void *h, int spp, int max_bounces, float *out_direct, float *out_indirect, float *out_sumsq,
                float *ms) {
    if (!h) return 1;
    if (max_bounces > 0) renderParam.maxBounces = max_bounces;
    const int width = renderParam.width, height = renderParam.height, n = width * height;
    cudaMalloc(&renderSegments, sizeof(RenderSegment) * n);
    cudaMalloc(&renderSegmentsBuffer, sizeof(RenderSegment) * n);
    cudaMalloc(&intersections, sizeof(IntersectionInfo) * n);
    cudaMalloc(&intersectionsBuffer, sizeof(IntersectionInfo) * n);
    cudaMalloc(&segmentValidFlags, sizeof(int) * n);
    cudaMalloc(&segmentPos, sizeof(int) * n);
    cudaMalloc(&materialIDs, sizeof(int) * n);
    cudaMemset(segmentValidFlags, 0, sizeof(int) * n);
    cudaMemset(segmentPos, 0, sizeof(int) * n);
    cudaMemset(renderSegmentsBuffer, 0, sizeof(RenderSegment) * n);
    RenderBuffer rb;
    cudaMalloc(&rb.directLightingBuffer, sizeof(float) * 4 * n);
    cudaMalloc(&rb.indirectLightingBuffer, sizeof(float) * 4 * n);
    cudaMemset(rb.directLightingBuffer, 0, sizeof(float) * 4 * n);
    cudaMemset(rb.indirectLightingBuffer, 0, sizeof(float) * 4 * n);
    float4 *prev = nullptr, *sumsq = nullptr;
    if (out_sumsq) {
        cudaMalloc(&prev, sizeof(float4) * n);
        cudaMalloc(&sumsq, sizeof(float4) * n);
        cudaMemset(prev, 0, sizeof(float4) * n);
        cudaMemset(sumsq, 0, sizeof(float4) * n);
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0);
    for (int f = 0; f < spp; ++f) {
        int numSegments = n;
        dim3 gr((width + generateRayBlockSize.x - 1) / generateRayBlockSize.x,
                (height + generateRayBlockSize.y - 1) / generateRayBlockSize.y);
        GenerateRayKernel<<<gr, generateRayBlockSize>>>(renderSegments, renderParam, cameraParam);
        cudaDeviceSynchronize();
        for (int i = 0; i < renderParam.maxBounces; i++) {
            if (numSegments <= 0) break;
            cudaMemset(intersections, 0, sizeof(IntersectionInfo) * numSegments);
            cudaMemset(intersectionsBuffer, 0, sizeof(IntersectionInfo) * numSegments);
            cudaMemset(materialIDs, 0, sizeof(int) * numSegments);
            dim3 rg((numSegments + renderBlockSize.x - 1) / renderBlockSize.x);
            IntersectionKernel<<<rg, renderBlockSize>>>(renderSegments, renderParam, intersections, numSegments,
                                                       segmentValidFlags, rb);
            cudaDeviceSynchronize();
            numSegments = StreamCompaction(segmentValidFlags, segmentPos, numSegments);
            if (numSegments <= 0) break;
            rg = dim3((numSegments + renderBlockSize.x - 1) / renderBlockSize.x);
            ShadingKernel<<<rg, renderBlockSize>>>(renderSegments, renderParam, intersections, numSegments, rb,
                                                  segmentValidFlags);
            cudaDeviceSynchronize();
            numSegments = StreamCompaction(segmentValidFlags, segmentPos, numSegments);
        }
        if (sumsq)
            k_frame_moments<<<(n + 255) / 256, 256>>>((float4 *)rb.directLightingBuffer,
                                                       (float4 *)rb.indirectLightingBuffer, prev, sumsq, n);
    }
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(ms, e0, e1);
    int err = (int)cudaGetLastError();
    cudaMemcpy(out_direct, rb.directLightingBuffer, sizeof(float) * 4 * n, cudaMemcpyDeviceToHost);
    cudaMemcpy(out_indirect, rb.indirectLightingBuffer, sizeof(float) * 4 * n, cudaMemcpyDeviceToHost);
    if (sumsq) cudaMemcpy(out_sumsq, sumsq, sizeof(float4) * n, cudaMemcpyDeviceToHost);
    cudaFree(renderSegments);
    cudaFree(renderSegmentsBuffer);
    cudaFree(intersections);
    cudaFree(intersectionsBuffer);
    cudaFree(segmentValidFlags);
    cudaFree(segmentPos);
    cudaFree(materialIDs);
    cudaFree(rb.directLightingBuffer);
    cudaFree(rb.indirectLightingBuffer);
    if (prev) cudaFree(prev);
    if (sumsq) cudaFree(sumsq);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return err;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// The reference's SVGF kernels on caller-provided inputs: the denoise block of
// RenderLoop (renderer.cuh:1207-1258, with the index flips of :1299-1304) for
// `frames` consecutive frames. Inputs per frame (host, w*h*4 each): noisy
// direct/indirect (rgb), G-buffer planes with the raster encodings. Outputs
// per frame: the final direct/indirect buffers (rgb + variance).
// ---------------------------------------------------------------------------
namespace {
cudaArray_t make_array(cudaChannelFormatDesc d, int w, int h) {
    cudaArray_t a;
    cudaMallocArray(&a, &d, w, h);
    return a;
}
}  // namespace

extern "C" int refr_svgf(int w, int h, int frames, const float *noisy_d, const float *noisy_i, const float *gb_pos,
                         const unsigned short *gb_nm, const unsigned short *gb_bm, const float *gb_md,
                         int max_history, float sigma_light, float sigma_normal, float sigma_depth, float reproj,
                         int atrous, float *out_d, float *out_i, float *ms_frames) {
    // ms_frames (optional, `frames` floats): GPU time of each frame's
    // denoise block, temporal kernel through the last a-trous pass (CUDA
    // events; the harness's host uploads and downloads excluded)
    const int n = w * h;
    cudaEvent_t ev0, ev1;
    cudaEventCreate(&ev0);
    cudaEventCreate(&ev1);
    renderParam.width = w;
    renderParam.height = h;
    DenoiseParam dp;
    dp.maxHistoryLength = max_history;
    dp.sigmaLight = sigma_light;
    dp.sigmaNormal = sigma_normal;
    dp.sigmaDepth = sigma_depth;
    dp.reprojectionDepthFactor = reproj;
    dp.atrousIterations = atrous;
    dp.currentTemporalBufferIndex = 0;
    for (int i = 0; i < 2; i++) {
        cudaMalloc(&dp.directMoments[i], sizeof(float2) * n);
        cudaMalloc(&dp.indirectMoments[i], sizeof(float2) * n);
        cudaMalloc(&dp.historyLength[i], sizeof(int) * n);
        cudaMemset(dp.directMoments[i], 0, sizeof(float2) * n);
        cudaMemset(dp.indirectMoments[i], 0, sizeof(float2) * n);
        cudaMemset(dp.historyLength[i], 0, sizeof(int) * n);
    }
    RenderBuffer rbs[2], hist[2];
    for (int i = 0; i < 2; i++) {
        cudaMalloc(&rbs[i].directLightingBuffer, sizeof(float) * 4 * n);
        cudaMalloc(&rbs[i].indirectLightingBuffer, sizeof(float) * 4 * n);
        cudaMalloc(&hist[i].directLightingBuffer, sizeof(float) * 4 * n);
        cudaMalloc(&hist[i].indirectLightingBuffer, sizeof(float) * 4 * n);
        cudaMemset(hist[i].directLightingBuffer, 0, sizeof(float) * 4 * n);
        cudaMemset(hist[i].indirectLightingBuffer, 0, sizeof(float) * 4 * n);
    }
    GBuffer gbs[2];
    cudaArray_t arrs[2][4];
    for (int i = 0; i < 2; i++) {
        arrs[i][0] = make_array(cudaCreateChannelDesc<float4>(), w, h);
        arrs[i][1] = make_array(cudaCreateChannelDesc<ushort4>(), w, h);
        arrs[i][2] = make_array(cudaCreateChannelDesc<ushort4>(), w, h);
        arrs[i][3] = make_array(cudaCreateChannelDesc<float4>(), w, h);
        for (int k = 0; k < 4; k++) {
            cudaArray_t a = arrs[i][k];
            cudaTextureObject_t t = CreateTextureObject(a, cudaAddressModeClamp, cudaFilterModePoint,
                                                        cudaReadModeElementType);
            if (k == 0) gbs[i].cudaTexObjPositionTriID = t;
            if (k == 1) gbs[i].cudaTexObjNormalMatID = t;
            if (k == 2) gbs[i].cudaTexObjBaryMeshID = t;
            if (k == 3) gbs[i].cudaTexObjMotionDepth = t;
        }
        gbs[i].width = w;
        gbs[i].height = h;
    }
    int cur = 0, gi = 0;
    bool firstFrame = true;
    dim3 grid((w + denoiseBlockSize.x - 1) / denoiseBlockSize.x, (h + denoiseBlockSize.y - 1) / denoiseBlockSize.y);
    for (int f = 0; f < frames; ++f) {
        size_t off = (size_t)f * n * 4;
        cudaMemcpy2DToArray(arrs[gi][0], 0, 0, gb_pos + off, w * 16, w * 16, h, cudaMemcpyHostToDevice);
        cudaMemcpy2DToArray(arrs[gi][1], 0, 0, gb_nm + off, w * 8, w * 8, h, cudaMemcpyHostToDevice);
        cudaMemcpy2DToArray(arrs[gi][2], 0, 0, gb_bm + off, w * 8, w * 8, h, cudaMemcpyHostToDevice);
        cudaMemcpy2DToArray(arrs[gi][3], 0, 0, gb_md + off, w * 16, w * 16, h, cudaMemcpyHostToDevice);
        RenderBuffer renderBuffer = rbs[cur];
        cudaMemcpy(renderBuffer.directLightingBuffer, noisy_d + off, sizeof(float) * 4 * n, cudaMemcpyHostToDevice);
        cudaMemcpy(renderBuffer.indirectLightingBuffer, noisy_i + off, sizeof(float) * 4 * n, cudaMemcpyHostToDevice);
        int t = dp.currentTemporalBufferIndex;
        RenderBuffer histCur = hist[t], histLast = hist[1 - t];
        GBuffer gBuffer = gbs[gi], lastGBuffer = gbs[1 - gi];
        cudaEventRecord(ev0);
        TemporalDenoiseKernel<<<grid, denoiseBlockSize>>>(dp, cameraParam, renderParam, renderBuffer, histLast, gBuffer,
                                                          lastGBuffer, firstFrame);
        cudaDeviceSynchronize();
        cudaMemcpy(histCur.directLightingBuffer, renderBuffer.directLightingBuffer, sizeof(float) * 4 * n,
                   cudaMemcpyDeviceToDevice);
        cudaMemcpy(histCur.indirectLightingBuffer, renderBuffer.indirectLightingBuffer, sizeof(float) * 4 * n,
                   cudaMemcpyDeviceToDevice);
        ComputeVarianceKernel<<<grid, denoiseBlockSize>>>(dp, renderParam, rbs[cur], rbs[1 - cur], gBuffer, 7);
        cudaDeviceSynchronize();
        cur = 1 - cur;
        if (!firstFrame) {
            int passes = max(1, min(8, dp.atrousIterations));
            for (int i = 0; i < passes; i++) {
                AtrousKernel<<<grid, denoiseBlockSize>>>(dp, cameraParam, renderParam, rbs[cur], rbs[1 - cur], gBuffer,
                                                         1 << i);
                cudaDeviceSynchronize();
                cur = 1 - cur;
            }
        }
        cudaEventRecord(ev1);
        cudaEventSynchronize(ev1);
        if (ms_frames) cudaEventElapsedTime(&ms_frames[f], ev0, ev1);
        cudaMemcpy(out_d + off, rbs[cur].directLightingBuffer, sizeof(float) * 4 * n, cudaMemcpyDeviceToHost);
        cudaMemcpy(out_i + off, rbs[cur].indirectLightingBuffer, sizeof(float) * 4 * n, cudaMemcpyDeviceToHost);
        // end of frame (renderer.cuh:1299-1304)
        cur = 1 - cur;
        gi = 1 - gi;
        dp.currentTemporalBufferIndex = 1 - dp.currentTemporalBufferIndex;
        firstFrame = false;
    }
    int err = (int)cudaGetLastError();
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
    for (int i = 0; i < 2; i++) {
        cudaFree(dp.directMoments[i]);
        cudaFree(dp.indirectMoments[i]);
        cudaFree(dp.historyLength[i]);
        cudaFree(rbs[i].directLightingBuffer);
        cudaFree(rbs[i].indirectLightingBuffer);
        cudaFree(hist[i].directLightingBuffer);
        cudaFree(hist[i].indirectLightingBuffer);
        cudaDestroyTextureObject(gbs[i].cudaTexObjPositionTriID);
        cudaDestroyTextureObject(gbs[i].cudaTexObjNormalMatID);
        cudaDestroyTextureObject(gbs[i].cudaTexObjBaryMeshID);
        cudaDestroyTextureObject(gbs[i].cudaTexObjMotionDepth);
        for (int k = 0; k < 4; k++) cudaFreeArray(arrs[i][k]);
    }
    return err;
}
