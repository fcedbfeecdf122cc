// Force-included (after cuda_runtime.h) when the reference's own sources are
// compiled as host C++ into oracle/_ref. Supplies what nvcc would otherwise
// provide in device code: unqualified min/max for floats, and tex2D<T> on
// texture objects with CUDA's documented fetch semantics (see
// ref_texture_host.cpp). Test infrastructure only.
#pragma once
#include <algorithm>
#include <cmath>
using std::max;
using std::min;

template <class T>
T tex2D(cudaTextureObject_t obj, float x, float y);
template <>
float4 tex2D<float4>(cudaTextureObject_t obj, float x, float y);
template <>
ushort4 tex2D<ushort4>(cudaTextureObject_t obj, float x, float y);
