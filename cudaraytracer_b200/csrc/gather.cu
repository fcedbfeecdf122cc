// Display resolve and debug views: GatherKernel (Src/Core/renderer.cuh:
// 956-1030) over the float accumulators and the primary-hit G-buffer, into
// uchar4 pixels laid out as the reference's display buffer.
//   mode 0 colour: (direct + indirect) / spp (or the denoised sum), gamma
//          1/2.2, written to the vertically flipped row;
//   mode 1 linear depth between the near plane 0.1 and far = scene diagonal
//          + |camera - scene centre|;
//   mode 2 the encoded shading normal; mode 3 a colour per mesh id;
//   mode 4 the hit position normalised by the scene bounds.
// Modes 1-4 read the G-buffer at the flipped row and write the unflipped
// one, as the reference does (its point-sampled tex2D at (i + 0.5, j + 0.5)
// with j already flipped).
#include "api_internal.h"

namespace crt {
namespace {

struct GatherArgs {
    uchar4 *pixels;
    const float4 *direct, *indirect;
    GBufferPlanes gb;
    int W, H, spp, denoised, mode;
    float bmin[3], bmax[3];
    float far_plane;
};

__device__ __forceinline__ unsigned char to_byte(float x) {
    return static_cast<unsigned char>(fminf(fmaxf(x * 255.0f, 0.0f), 255.0f));
}

__global__ void k_gather(GatherArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j0 = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= a.W || j0 >= a.H) return;
    const int idx = j0 * a.W + i;
    const int j = a.H - j0 - 1;
    const int seg = j * a.W + i;
    if (a.mode == 0) {
        const float4 d = a.direct[idx], id = a.indirect[idx];
        float c[3] = {d.x + id.x, d.y + id.y, d.z + id.z};
        if (!a.denoised)
            for (int k = 0; k < 3; ++k) c[k] = c[k] / a.spp;
        uchar4 o;
        o.x = static_cast<unsigned char>(fminf(fmaxf(powf(c[0], 1.0f / 2.2f) * 255.0f, 0.0f), 255.0f));
        o.y = static_cast<unsigned char>(fminf(fmaxf(powf(c[1], 1.0f / 2.2f) * 255.0f, 0.0f), 255.0f));
        o.z = static_cast<unsigned char>(fminf(fmaxf(powf(c[2], 1.0f / 2.2f) * 255.0f, 0.0f), 255.0f));
        o.w = 255;
        a.pixels[seg] = o;
    } else if (a.mode == 1) {
        const float4 md = a.gb.motion_depth[seg];
        const float nearp = 0.1f;
        const unsigned char v = to_byte((md.z - nearp) / (a.far_plane - nearp));
        a.pixels[idx] = make_uchar4(v, v, v, 255);
    } else if (a.mode == 2) {
        const ushort4 nm = a.gb.normal_mat[seg];
        a.pixels[idx] = make_uchar4(to_byte(nm.x / 65535.0f), to_byte(nm.y / 65535.0f), to_byte(nm.z / 65535.0f), 255);
    } else if (a.mode == 3) {
        const unsigned short id = a.gb.bary_mesh[seg].w;
        a.pixels[idx] = make_uchar4((unsigned char)((id * 37) % 256), (unsigned char)((id * 57) % 256),
                                    (unsigned char)((id * 97) % 256), 255);
    } else {
        const float4 pt = a.gb.pos_tri[seg];
        a.pixels[idx] = make_uchar4(to_byte((pt.x - a.bmin[0]) / (a.bmax[0] - a.bmin[0])),
                                    to_byte((pt.y - a.bmin[1]) / (a.bmax[1] - a.bmin[1])),
                                    to_byte((pt.z - a.bmin[2]) / (a.bmax[2] - a.bmin[2])), 255);
    }
}

}  // namespace
}  // namespace crt

using namespace crt;

extern "C" crt_status crt_gather(crt_scene *scene, int32_t mode, int32_t spp, int32_t denoised, const float *d_direct,
                                 const float *d_indirect, const crt_gbuffer *gb, void *d_pixels, void *stream) {
    return guard([&] {
        CRT_CHECK(scene && scene->renderable && d_pixels, CRT_ERR_INVALID, "crt_gather: bad argument");
        CRT_CHECK(mode >= 0 && mode <= 4, CRT_ERR_INVALID, "crt_gather: mode must be 0..4");
        CRT_CHECK(mode != 0 || (d_direct && d_indirect && (denoised || spp > 0)), CRT_ERR_INVALID,
                  "crt_gather: colour mode needs the accumulators and spp > 0");
        CRT_CHECK(mode == 0 || (gb && gb->pos_tri && gb->normal_mat && gb->bary_mesh && gb->motion_depth),
                  CRT_ERR_INVALID, "crt_gather: debug views need a G-buffer");
        CRT_CUDA(cudaSetDevice(scene->ctx->device));
        cudaStream_t s = stream ? (cudaStream_t)stream : scene->ctx->stream;
        GatherArgs a;
        a.pixels = (uchar4 *)d_pixels;
        a.direct = (const float4 *)d_direct;
        a.indirect = (const float4 *)d_indirect;
        if (gb) {
            a.gb.pos_tri = (float4 *)gb->pos_tri;
            a.gb.normal_mat = (ushort4 *)gb->normal_mat;
            a.gb.bary_mesh = (ushort4 *)gb->bary_mesh;
            a.gb.motion_depth = (float4 *)gb->motion_depth;
        }
        a.W = scene->rp.width;
        a.H = scene->rp.height;
        a.spp = spp;
        a.denoised = denoised;
        a.mode = mode;
        float d[3], c[3];
        for (int k = 0; k < 3; ++k) {
            a.bmin[k] = scene->bvh.bounds_min[k];
            a.bmax[k] = scene->bvh.bounds_max[k];
            d[k] = a.bmax[k] - a.bmin[k];
            c[k] = scene->cam.position[k] - (a.bmin[k] + a.bmax[k]) * 0.5f;
        }
        // Bounds3D::DiagonalLength + (position - Center()).norm() in float
        a.far_plane = std::sqrt(d[0] * d[0] + (d[1] * d[1] + d[2] * d[2])) +
                      std::sqrt(c[0] * c[0] + (c[1] * c[1] + c[2] * c[2]));
        dim3 b(16, 16), g((a.W + 15) / 16, (a.H + 15) / 16);
        k_gather<<<g, b, 0, s>>>(a);
        CRT_CUDA(cudaGetLastError());
    });
}
