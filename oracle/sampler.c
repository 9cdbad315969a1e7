/*
 * Oracle (test infrastructure): the Owen-scrambled Sobol sampler of
 * shaders/sampler.glsl:8-55, with the direction numbers of shaders/sobol_table.glsl
 * derived here from the (s, a, m) parameters tools/sobol_table.py uses (Joe and
 * Kuo's new-joe-kuo-6.21201, dimensions 1..3; dimension 0 is van der Corput).
 */
#include "oracle.h"

static uint32_t directions[128];
static int directions_ready = 0;

/* The direction-number recurrence of tools/sobol_table.py:12-23. */
static void make_directions(void) {
    static const int s_of[3] = {1, 2, 3};
    static const int a_of[3] = {0, 1, 1};
    static const uint32_t m_of[3][3] = {{1, 0, 0}, {1, 3, 0}, {1, 3, 1}};
    for (int bit = 0; bit < 32; bit++) directions[bit] = 1u << (31 - bit);
    for (int dim = 0; dim < 3; dim++) {
        int s = s_of[dim], a = a_of[dim];
        uint64_t v[33];
        for (int k = 1; k <= 32; k++) {
            if (k <= s) {
                v[k] = (uint64_t)m_of[dim][k - 1] << (32 - k);
            } else {
                uint64_t value = v[k - s] ^ (v[k - s] >> s);
                for (int i = 1; i < s; i++)
                    if ((a >> (s - 1 - i)) & 1) value ^= v[k - i];
                v[k] = value;
            }
        }
        for (int k = 1; k <= 32; k++) directions[(dim + 1) * 32 + (k - 1)] = (uint32_t)(v[k] & 0xffffffffu);
    }
    directions_ready = 1;
}

const uint32_t *or_sobol_directions(void) {
    if (!directions_ready) make_directions();
    return directions;
}

/* hash_u32 (sampler.glsl:8-13) */
uint32_t or_hash_u32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x21f0aaadu;
    x ^= x >> 15;
    x *= 0x735a2d97u;
    x ^= x >> 15;
    return x;
}

/* hash_combine (sampler.glsl:15-17) */
uint32_t or_hash_combine(uint32_t seed, uint32_t value) {
    return seed ^ (or_hash_u32(value) + 0x9e3779b9u + (seed << 6) + (seed >> 2));
}

/* laine_karras (sampler.glsl:19-26) */
static uint32_t laine_karras(uint32_t x, uint32_t seed) {
    x += seed;
    x ^= x * 0x6c50b47cu;
    x ^= x * 0xb82f1e52u;
    x ^= x * 0xc7afe638u;
    x ^= x * 0x8d22f6e6u;
    return x;
}

static uint32_t reverse_bits(uint32_t x) {
    x = ((x >> 1) & 0x55555555u) | ((x & 0x55555555u) << 1);
    x = ((x >> 2) & 0x33333333u) | ((x & 0x33333333u) << 2);
    x = ((x >> 4) & 0x0f0f0f0fu) | ((x & 0x0f0f0f0fu) << 4);
    x = ((x >> 8) & 0x00ff00ffu) | ((x & 0x00ff00ffu) << 8);
    return (x >> 16) | (x << 16);
}

/* nested_uniform_scramble (sampler.glsl:28-30) */
static uint32_t nested_uniform_scramble(uint32_t x, uint32_t seed) {
    return reverse_bits(laine_karras(reverse_bits(x), seed));
}

/* sobol (sampler.glsl:32-37) */
uint32_t or_sobol(uint32_t index, uint32_t dimension) {
    const uint32_t *dirs = or_sobol_directions();
    uint32_t x = 0;
    for (uint32_t bit = 0; index != 0; bit++, index >>= 1)
        if (index & 1u) x ^= dirs[dimension * 32 + bit];
    return x;
}

/* sample4 (sampler.glsl:47-55); `seed` is the render's (params.seed). */
void or_sample4_bits(uint32_t seed, uint32_t pixel, uint32_t index, uint32_t group, uint32_t out[4]) {
    uint32_t s = or_hash_combine(or_hash_combine(seed, pixel), group);
    uint32_t shuffled = nested_uniform_scramble(index, or_hash_u32(s));
    for (uint32_t d = 0; d < 4; d++)
        out[d] = nested_uniform_scramble(or_sobol(shuffled, d), or_hash_combine(s, d + 1u)) >> 8;
}

void or_sample4(uint32_t seed, uint32_t pixel, uint32_t index, uint32_t group, double out[4]) {
    uint32_t bits[4];
    or_sample4_bits(seed, pixel, index, group, bits);
    for (int d = 0; d < 4; d++) out[d] = (double)bits[d] * (1.0 / 16777216.0);
}
