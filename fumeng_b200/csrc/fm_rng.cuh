// Counter-based random numbers: one PCG32 stream per camera sample.
//
// The reference draws from one mt19937_64 shared by all threads, seeded from the clock
// (core/sampler.h:11-41), so its sequences are neither reproducible nor independent
// between threads.  Here each sample (scene seed, pixel, sample index) owns a PCG32
// stream (M. O'Neill, "PCG: A Family of Simple Fast Space-Efficient Statistically Good
// Algorithms for Random Number Generation", 2014) whose state is derived with the
// SplitMix64 finaliser.  This changes the variance realisation, not the expectation.
#pragma once
#include "fm_common.cuh"

namespace fm {

FM_HD uint64_t splitmix64(uint64_t x)
{
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

struct Rng {
    uint64_t state;
};

FM_HD Rng rng_for(uint64_t seed, uint64_t pixel, uint64_t sample)
{
    Rng r;
    r.state = splitmix64(seed ^ splitmix64(pixel * 0x100000001B3ull + splitmix64(sample + 0x632BE59BD9B4E019ull)));
    return r;
}

FM_HD uint32_t rng_u32(Rng& r)
{
    const uint64_t old = r.state;
    r.state = old * 6364136223846793005ull + 1442695040888963407ull;
    const uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    const uint32_t rot = (uint32_t)(old >> 59u);
    return (xs >> rot) | (xs << ((32u - rot) & 31u));
}

// Uniform float in [0, 1) with 24 random bits.
FM_HD float rng_1d(Rng& r) { return (float)(rng_u32(r) >> 8) * (1.0f / 16777216.0f); }
FM_HD f3 rng_3d(Rng& r)
{
    const float a = rng_1d(r);
    const float b = rng_1d(r);
    const float c = rng_1d(r);
    return f3{a, b, c};
}

}  // namespace fm
