/*
 * ag_rng.h -- counter-based random numbers shared by the host generators and
 * device kernels.  Draw k of stream s is a pure function of (seed, s, k), so a
 * graph generated on the host and one generated on the GPU are identical and
 * any sub-range can be generated in parallel.
 *
 * The mixing function is the SplitMix64 finaliser (Steele, Lea, Flood,
 * "Fast splittable pseudorandom number generators", OOPSLA 2014): a Weyl
 * sequence with increment 0x9E3779B97F4A7C15 passed through two
 * xor-shift-multiply rounds.
 */
#ifndef AG_RNG_H
#define AG_RNG_H

#include <stdint.h>

#if defined(__CUDACC__)
#define AG_HD __host__ __device__ __forceinline__
#else
#define AG_HD static inline
#endif

#define AG_GOLDEN64 0x9E3779B97F4A7C15ull

AG_HD uint64_t ag_mix64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

/* 64-bit draw number k of stream s under seed. */
AG_HD uint64_t ag_draw64(uint64_t seed, uint64_t s, uint64_t k)
{
    uint64_t base = ag_mix64(seed + AG_GOLDEN64);
    return ag_mix64(base + (s * 64ull + k + 1ull) * AG_GOLDEN64);
}

/* uniform float in [0,1) with 24 random mantissa bits */
AG_HD float ag_u01(uint64_t bits)
{
    return (float)(uint32_t)(bits >> 40) * (1.0f / 16777216.0f);
}

#endif /* AG_RNG_H */
