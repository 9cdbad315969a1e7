// Direction numbers of the first four Sobol dimensions for the Owen-scrambled sampler
// (shaders/sampler.glsl, shaders/sobol_table.glsl): dimension 0 is van der Corput, 1..3
// follow the primitive-polynomial recurrence with Joe and Kuo's (s, a, m) parameters
// (1, 0, {1}), (2, 1, {1, 3}), (3, 1, {1, 3, 1}), 32 bits each.
#include "common.hpp"

namespace lr {

const uint32_t *sobol_table() {
    static uint32_t table[128];
    static bool ready = false;
    if (ready) return table;
    struct Param {
        int s, a;
        uint32_t m[3];
    };
    const Param params[3] = {{1, 0, {1, 0, 0}}, {2, 1, {1, 3, 0}}, {3, 1, {1, 3, 1}}};
    for (int bit = 0; bit < 32; bit++) table[bit] = 1u << (31 - bit);
    for (int d = 0; d < 3; d++) {
        const Param &p = params[d];
        uint64_t v[33] = {0};
        for (int k = 1; k <= 32; k++) {
            if (k <= p.s) {
                v[k] = (uint64_t)p.m[k - 1] << (32 - k);
            } else {
                uint64_t value = v[k - p.s] ^ (v[k - p.s] >> p.s);
                for (int i = 1; i < p.s; i++)
                    if ((p.a >> (p.s - 1 - i)) & 1) value ^= v[k - i];
                v[k] = value;
            }
            table[(d + 1) * 32 + k - 1] = (uint32_t)v[k];
        }
    }
    ready = true;
    return table;
}

}  // namespace lr
