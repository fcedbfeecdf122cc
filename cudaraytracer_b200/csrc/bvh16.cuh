// Binary BVH nodes with 16-bit quantised child boxes: 32 B per node, one
// sector, half the bytes of the 64 B float node (bvh.cuh).
//
// Per node (one 32 B read-only load):
//   words 0-5: twelve 16-bit grid indices, child 0 lo x/y/z then hi x/y/z,
//              then child 1 (word k holds indices 2k (low half) and 2k+1)
//   words 6-7: the two child links, as in the float node
// One grid per scene and axis: a bound decodes as fmaf(2^23 + q, s, p'),
// one rounding (2^23 + q is a byte permute of q into the mantissa of 2^23,
// the product by the power of two s is exact). The compression kernel
// (bvh16.cu) picks every index with that same fmaf so the decoded box
// contains the child's float box; the slab test is monotone in the bounds,
// so every box the float traversal accepts is accepted here too and the
// hit records are those of the triangle test (the visit order, and so the
// choice between triangles at equal t, can differ where enlarged boxes
// reorder near and far children).
#pragma once
#include "bvh.cuh"

namespace crt {

// The device decode (load_node16) is in bvh.cuh, beside the float node load.


// Device: builds b.cnodes and b.grid from b.nodes and the scene bounds
// (bvh16.cu). Records kErrTraversalBounds in `err` (if not null) should a
// decoded box fail to contain its child, which the construction rules out.
struct BvhBuffers;
void build_bvh16(BvhBuffers &b, int *err, cudaStream_t stream);
// Host: the grid of a scene box (also used by the CPU test).
QuantGrid quant_grid(const float lo[3], const float hi[3]);

}  // namespace crt
