// Counter-based random numbers for the path tracer.
//
// The reference draws from a per-thread Mersenne twister
// (randomsampler.cpp, standardmtrand.cpp); parity with it is statistical.
// Here every number is a pure function of (seed, sample index, dimension), so
// any path can be replayed exactly (the adjoint pass does that) and results
// do not depend on launch shape or wave size. The mixer is the SplitMix64
// finaliser (Steele, Lea, Flood, "Fast splittable pseudorandom number
// generators", OOPSLA 2014) applied to the key combined with the dimension.
#pragma once
#include <cstdint>

namespace lmgpu {

__host__ __device__ __forceinline__ uint64_t mix64(uint64_t x)
{
    x ^= x >> 30;
    x *= 0xBF58476D1CE4E5B9ull;
    x ^= x >> 27;
    x *= 0x94D049BB133111EBull;
    x ^= x >> 31;
    return x;
}

// Per-sample key: seed and sample index, decorrelated.
__host__ __device__ __forceinline__ uint64_t sample_key(uint64_t seed, uint64_t sample)
{
    return mix64(mix64(seed + 0x9E3779B97F4A7C15ull) ^ (sample * 0xD1B54A32D192ED03ull));
}

// Uniform in [0, 1) with 24 random bits.
__host__ __device__ __forceinline__ float rng_uniform(uint64_t key, uint32_t dim)
{
    const uint64_t x = mix64(key ^ (uint64_t(dim + 1) * 0x9E3779B97F4A7C15ull));
    return float(uint32_t(x >> 40)) * (1.0f / 16777216.0f);
}

// Dimension layout of one sample: raster (0, 1); then per path vertex k >= 1
// a block of 8: light selection/position (0, 1), Russian roulette (2),
// BSDF direction (3, 4), BSDF component (5).
constexpr uint32_t DIM_RASTER = 0;
__host__ __device__ __forceinline__ uint32_t dim_vertex(int k) { return 8u * uint32_t(k); }
constexpr uint32_t DIM_LIGHT = 0, DIM_RR = 2, DIM_BSDF = 3, DIM_COMP = 5;

}  // namespace lmgpu
