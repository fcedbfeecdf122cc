// Per-path PCG32 (O'Neill, pcg32_random_r / pcg32_srandom_r). The stream of
// a path is selected by its pixel (inc = 2*pixel + 1) and the state is seeded
// from (seed, sample index), so a path's draws depend only on
// (seed, pixel, sample) and need 8 bytes of state. The reference instead
// keeps one curand XORWOW state per compacted segment slot
// (Src/Core/sampler.cu:17-36, Src/Core/renderer.cuh:244), so the two agree
// in distribution, not in individual draws.
#pragma once
#include <stdint.h>

namespace crt {

struct Pcg32 {
    uint64_t state;
    uint64_t inc;
};

__host__ __device__ __forceinline__ uint32_t pcg32_next(Pcg32 &r) {
    uint64_t old = r.state;
    r.state = old * 6364136223846793005ULL + r.inc;
    uint32_t xorshifted = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    uint32_t rot = (uint32_t)(old >> 59u);
    return (xorshifted >> rot) | (xorshifted << ((0u - rot) & 31u));
}

__host__ __device__ __forceinline__ Pcg32 pcg32_seed(uint64_t seed, uint32_t pixel, uint32_t sample) {
    Pcg32 r;
    r.state = 0u;
    r.inc = ((uint64_t)pixel << 1u) | 1u;
    pcg32_next(r);
    r.state += seed * 0x9E3779B97F4A7C15ULL + (uint64_t)sample * 0xD1B54A32D192ED03ULL;
    pcg32_next(r);
    return r;
}

// Uniform float on (0, 1], the range of curand_uniform that the reference's
// Sampler::Get1D returns (Src/Core/sampler.cu:17-20).
__host__ __device__ __forceinline__ float pcg32_uniform(Pcg32 &r) {
    return (float)((pcg32_next(r) >> 8) + 1u) * (1.0f / 16777216.0f);
}

}  // namespace crt
