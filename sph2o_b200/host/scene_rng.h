/*
 * Seeded, counter-based lattice jitter shared by the host scene builder and
 * the oracle harness, so both perturb the same lattice by the same amounts.
 *
 * A scene JSON may carry two keys beyond the SPH2O schema in its
 * "Configuration" object: "jitter" (amplitude as a fraction of the particle
 * radius, e.g. 0.01 for +-0.01 r) and "jitterSeed". Coordinate c of fluid
 * particle i (in lattice build order) then moves by
 *     (2u - 1) * jitter * particleRadius,   u = sph_uniform(seed, 3 i + c)
 * rounded once to float and added in float. SPH2O's own loader ignores both
 * keys, so the same JSON runs unmodified through the reference.
 */
#ifndef SPH2O_SCENE_RNG_H
#define SPH2O_SCENE_RNG_H

#include <stdint.h>

static inline uint64_t sph_splitmix64(uint64_t x)
{
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

/* Uniform double in [0, 1) from (seed, counter). */
static inline double sph_uniform(uint64_t seed, uint64_t counter)
{
    const uint64_t z = sph_splitmix64(sph_splitmix64(seed) ^ (counter * 0xD1B54A32D192ED03ull));
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

/* Offset for coordinate c (0..2) of particle i. */
static inline float sph_jitter_offset(uint64_t seed, uint64_t i, int c, float jitter, float radius)
{
    const double u = sph_uniform(seed, 3ull * i + (uint64_t)c);
    return (float)((2.0 * u - 1.0) * (double)jitter * (double)radius);
}

#endif
