// Shared helpers for the crt CUDA sources: error plumbing, float3 math with
// explicit rounding (no FMA contraction), and the last-error slot of the C ABI.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <string>
#include <stdexcept>
#include "../../include/crt.h"

namespace crt {

// Error raised inside the library and turned into a crt_status at the ABI.
struct Error : std::runtime_error {
    crt_status status;
    Error(crt_status s, const std::string &m) : std::runtime_error(m), status(s) {}
};

void set_last_error(const std::string &msg);

// Bits of a context's device error word (crt_check_device_errors).
constexpr int kErrWaitGaveUp = 1;       // a tensor-core kernel gave up a bounded mbarrier wait
constexpr int kErrTraversalBounds = 2;  // a BVH traversal met an out-of-range node, leaf or stack depth

#define CRT_CUDA(call)                                                          \
    do {                                                                        \
        cudaError_t e_ = (call);                                                \
        if (e_ != cudaSuccess) {                                                \
            throw ::crt::Error(e_ == cudaErrorMemoryAllocation ? CRT_ERR_OOM    \
                                                               : CRT_ERR_CUDA,  \
                               std::string(#call) + ": " +                      \
                                   cudaGetErrorString(e_) + " (" __FILE__ ")"); \
        }                                                                       \
    } while (0)

#define CRT_CHECK(cond, status, msg)                  \
    do {                                              \
        if (!(cond)) throw ::crt::Error(status, msg); \
    } while (0)

// ---------------------------------------------------------------------------
// IEEE single-precision arithmetic with every rounding explicit. The
// reference's triangle test and visibility predicate are reproduced with the
// operation order of its Eigen expressions (a.dot(b) = a0*b0 + (a1*b1 +
// a2*b2); a.cross(b) = (a1*b2 - a2*b1, a2*b0 - a0*b2, a0*b1 - a1*b0)), with
// no multiply-add contraction, so results equal the reference evaluated in
// plain IEEE float (its host build) bit for bit.
// ---------------------------------------------------------------------------
struct V3 {
    float x, y, z;
};

__host__ __device__ __forceinline__ V3 v3(float x, float y, float z) { return V3{x, y, z}; }

#ifdef __CUDACC__
__device__ __forceinline__ float rmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float radd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float rsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float rdiv(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ float rsqrt_(float a) { return __fsqrt_rn(a); }
__device__ __forceinline__ float rrcp(float a) { return __frcp_rn(a); }

__device__ __forceinline__ V3 vsub(V3 a, V3 b) { return V3{rsub(a.x, b.x), rsub(a.y, b.y), rsub(a.z, b.z)}; }
__device__ __forceinline__ V3 vadd(V3 a, V3 b) { return V3{radd(a.x, b.x), radd(a.y, b.y), radd(a.z, b.z)}; }
__device__ __forceinline__ V3 vscale(V3 a, float s) { return V3{rmul(a.x, s), rmul(a.y, s), rmul(a.z, s)}; }
__device__ __forceinline__ V3 vneg(V3 a) { return V3{-a.x, -a.y, -a.z}; }
__device__ __forceinline__ float vdot(V3 a, V3 b) {
    return radd(rmul(a.x, b.x), radd(rmul(a.y, b.y), rmul(a.z, b.z)));
}
__device__ __forceinline__ V3 vcross(V3 a, V3 b) {
    return V3{rsub(rmul(a.y, b.z), rmul(a.z, b.y)), rsub(rmul(a.z, b.x), rmul(a.x, b.z)),
              rsub(rmul(a.x, b.y), rmul(a.y, b.x))};
}
__device__ __forceinline__ float vsqnorm(V3 a) { return vdot(a, a); }
__device__ __forceinline__ float vnorm(V3 a) { return rsqrt_(vsqnorm(a)); }
// Eigen normalized(): divide each component by sqrt(squaredNorm) when > 0.
__device__ __forceinline__ V3 vnormalized(V3 a) {
    float z = vsqnorm(a);
    if (z > 0.f) {
        float s = rsqrt_(z);
        return V3{rdiv(a.x, s), rdiv(a.y, s), rdiv(a.z, s)};
    }
    return a;
}
#endif

}  // namespace crt
