// Quantized child boxes of the compressed 8-wide BVH (wide.cpp builds them on the host,
// refit.cu again on the device after points move): one function both compile, so a refit
// of unmoved points writes the nodes the upload wrote.
//
// A node's up to eight child boxes are stored relative to the node's own box: its low
// corner as three floats, and per axis a power-of-two step 2^e with every child plane an
// 8-bit multiple of it (Ylitie, Karras and Laine, HPG 2017, section 3.1). Low planes round
// down and high planes up, so a decoded box always contains the box it stands for: the
// traversal stays conservative and the watertight hits exact.
//
// Node: 6 x 16 bytes (96 bytes, 16-byte aligned)
//   [0]  origin x, y, z; w: biased exponents ex, ey, ez (bytes 0-2) and the occupied
//        slots (byte 3, bit s: slot s holds a child)
//   [1]  child links of slots 0-3, [2] of slots 4-7 (>= 0 a node, < 0 a leaf:
//        -1 - (first << 4 | count - 1))
//   [3]  low x planes of slots 0-7 (bytes), then their high x planes
//   [4]  the same for y, [5] for z
// Which child takes which slot is the builder's choice (wide.cpp orders them by direction
// octant); an unused slot has link 0 and an inverted box (low plane 255, high plane 0).
#pragma once

#include <stdint.h>

#ifdef __CUDACC__
#define LR_HD __host__ __device__
#else
#define LR_HD
#endif

namespace lr {

constexpr int kQNodeFloat4s = 6;

// 2^e as a float for a biased exponent byte (1..254: normal floats).
LR_HD inline float q_step(uint32_t biased) {
    union {
        uint32_t u;
        float f;
    } v;
    v.u = biased << 23;
    return v.f;
}

// The smallest biased exponent whose step covers `extent` in 255 steps (at least 1). The
// search starts ten below extent's own exponent, where 255 steps cover less than a quarter
// of it, so it finds the same exponent as a search from 1 in a few steps.
LR_HD inline uint32_t q_exponent(float extent) {
    union {
        float f;
        uint32_t u;
    } v;
    v.f = extent;
    if (!(extent > 0.0f)) return 1;  // zero, negative or NaN: the first step already serves
    const uint32_t own = (v.u >> 23) & 0xffu;
    uint32_t e = own > 11 ? own - 10 : 1;
    while (e < 254 && q_step(e) * 255.0f < extent) e++;
    return e;
}

LR_HD inline float q_floor(float v) { return (float)(int64_t)(v >= 0.0f ? v : v - 0.99999994f); }

// Writes one node (24 floats, as 6 float4s) from the child boxes lo/hi (3 floats each,
// already widened) and links of the slots set in `occupied` (at least one).
LR_HD inline void quantize_node(uint32_t occupied, const float (*lo)[3], const float (*hi)[3], const int *links,
                                float *out) {
    float origin[3] = {0.0f, 0.0f, 0.0f}, top[3] = {0.0f, 0.0f, 0.0f};
    bool any = false;
    for (int c = 0; c < 8; c++) {
        if (!((occupied >> c) & 1u)) continue;
        for (int k = 0; k < 3; k++) {
            origin[k] = !any || lo[c][k] < origin[k] ? lo[c][k] : origin[k];
            top[k] = !any || hi[c][k] > top[k] ? hi[c][k] : top[k];
        }
        any = true;
    }
    uint32_t exps[3];
    uint8_t planes[3][2][8];
    for (int k = 0; k < 3; k++) {
        // The step: top - origin rounds, so grow it until every high plane fits.
        uint32_t e = q_exponent(top[k] - origin[k]);
        for (;;) {
            const float s = q_step(e);
            bool fits = true;
            for (int c = 0; c < 8 && fits; c++) {
                if (!((occupied >> c) & 1u)) {
                    planes[k][0][c] = 255;
                    planes[k][1][c] = 0;
                    continue;
                }
                // Low plane: the largest multiple at or below lo; high: the smallest at or
                // above hi (the products are exact, the sums checked as rounded).
                int32_t ql = (int32_t)q_floor((lo[c][k] - origin[k]) / s);
                if (ql < 0) ql = 0;
                while (ql > 0 && origin[k] + (float)ql * s > lo[c][k]) ql--;
                int32_t qh = (int32_t)q_floor((hi[c][k] - origin[k]) / s);
                if (qh < 0) qh = 0;
                while (qh < 256 && origin[k] + (float)qh * s < hi[c][k]) qh++;
                if (qh > 255 || origin[k] + (float)ql * s > lo[c][k]) {
                    fits = false;
                    break;
                }
                planes[k][0][c] = (uint8_t)ql;
                planes[k][1][c] = (uint8_t)qh;
            }
            if (fits || e >= 254) break;
            e++;
        }
        exps[k] = e;
    }
    union {
        uint32_t u;
        float f;
    } w;
    for (int k = 0; k < 3; k++) out[k] = origin[k];
    w.u = exps[0] | exps[1] << 8 | exps[2] << 16 | (occupied & 0xffu) << 24;
    out[3] = w.f;
    for (int c = 0; c < 8; c++) {
        w.u = (uint32_t)(((occupied >> c) & 1u) ? links[c] : 0);
        out[4 + c] = w.f;
    }
    for (int k = 0; k < 3; k++) {
        uint8_t *bytes = (uint8_t *)(out + 12 + k * 4);
        for (int c = 0; c < 8; c++) {
            bytes[c] = planes[k][0][c];
            bytes[8 + c] = planes[k][1][c];
        }
    }
}

}  // namespace lr
