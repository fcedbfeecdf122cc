// Device BVH build interface (see bvh_build.cu).
#pragma once
#include "bvh.cuh"
#include "bvh8.cuh"
#include "bvh16.cuh"

namespace crt {

struct BvhBuffers {
    float4 *nodes = nullptr;    // 4 float4 per interior node
    float4 *tris = nullptr;     // 3 float4 per triangle, leaf order
    int *slot_of_prim = nullptr;  // original primitive index -> leaf-order slot
    int64_t num_nodes = 0;
    int num_tris = 0;
    int depth = 0;
    float bounds_min[3] = {0, 0, 0};
    float bounds_max[3] = {0, 0, 0};
    float build_ms = 0.f;
    // 8-wide quantised tree collapsed from `nodes` (bvh8.cuh)
    float4 *wnodes = nullptr;
    int *wlinks = nullptr;
    int64_t num_wide_nodes = 0;
    int wide_depth = 0;
    float wide_build_ms = 0.f;
    int *err = nullptr;  // the owning context's device error word
    float4 *cnodes = nullptr;  // 16-bit quantised copy of `nodes` (bvh16.cuh)
    QuantGrid grid{};
    BvhView view() const {
        return BvhView{nodes, tris, num_tris, wnodes, wlinks, (int)num_nodes, err, cnodes, grid};
    }
};

// Builds the BVH of n triangles given as n x 9 floats (v0, v1, v2) on the
// device. Synchronises `stream` before returning.
void build_bvh(const float *d_verts, int n, cudaStream_t stream, BvhBuffers &out);
void free_bvh(BvhBuffers &b);

}  // namespace crt
