// The light tree as the integrator's kernels walk it. The host builds the reference's
// tree (src/render/light_tree.lucb:41-244: pbrt-v4 light bounds over placed lights and
// emissive triangles) and lays it out for the device (loading.cpp `device_tree`) as one
// TreePair per interior node: both children's bounds, already in the form the importance
// test takes -- centre and radius of the box, the emission cone's axis, cosine and sine,
// the cutoff cosine, the power -- and where each child leads. A step of a descent reads
// one 96-byte record (six float4 loads) and weighs the two children together.
//
// Three walks share the step: choosing an emitter for a light sample by importance at a
// point and normal (with its probability), the probability of a given emitter along its
// recorded trail of left/right turns (for MIS), and choosing by power alone (where light
// paths start). The importance is pbrt-v4's LightBounds::Importance, as the reference's
// shaders/lighttree.glsl:18-45 evaluates it, so the densities are the oracle's.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "shading.cuh"

namespace lr {

constexpr uint32_t kTreeLeaf = 0x80000000u;  // TreePair lead: an emitter, not a pair

struct alignas(16) TreePair {
    float4 centre[2];  // the child's box: centre | radius (half its diagonal)
    float4 axis[2];    // the child's emission cone axis | power (<= 0: it emits nothing)
    // cos theta_o | sin theta_o | cos theta_e | lead (bits): the child's pair, or
    // kTreeLeaf | emitter
    float4 cone[2];
};

struct TreeTable {
    const TreePair *pairs = nullptr;
    const uint4 *records = nullptr;        // per emitter: code, trail, depth, 0
    const uint32_t *triangle_map = nullptr;  // per triangle slot: its emitter, or kNone
    // The walk's start: pair 0, kTreeLeaf | emitter for a tree of one emitter, kNone for
    // an empty tree.
    uint32_t root = kNone;
};

__device__ __forceinline__ float root_or_zero(float x) { return sqrtf(fmaxf(0.0f, x)); }

// cos(max(0, a - b)) for angles a, b in [0, pi] given by cosine and sine.
__device__ __forceinline__ void angle_less(float cos_a, float sin_a, float cos_b, float sin_b, float &cos_out,
                                           float &sin_out) {
    if (cos_a > cos_b) {  // a < b: clamped to zero
        cos_out = 1.0f;
        sin_out = 0.0f;
    } else {
        cos_out = cos_a * cos_b + sin_a * sin_b;
        sin_out = sin_a * cos_b - cos_a * sin_b;
    }
}

// How much a child may light point p with normal n (either side): its power over the
// squared distance, reduced by how far p lies outside the emission cone and by how
// obliquely n faces the box, each angle first reduced by the angle the box subtends.
__device__ __forceinline__ float child_importance(float4 centre, float4 axis, float4 cone, float3 p, float3 n) {
    if (axis.w <= 0.0f) return 0.0f;
    const float3 offset = p - xyz(centre);
    const float r = centre.w;
    const float o2 = dot(offset, offset);
    const float3 w = o2 > 0.0f ? offset * rsqrtf(o2) : xyz(axis);
    // theta_w: p off the axis; theta_b: the half angle the box subtends from p.
    const float cos_w = dot(xyz(axis), w), sin_w = root_or_zero(1.0f - cos_w * cos_w);
    const float cos_b = o2 < r * r ? -1.0f : root_or_zero(1.0f - r * r / o2);
    const float sin_b = root_or_zero(1.0f - cos_b * cos_b);
    float cos_x, sin_x, cos_p, sin_p;
    angle_less(cos_w, sin_w, cone.x, cone.y, cos_x, sin_x);  // beyond the emission cone
    angle_less(cos_x, sin_x, cos_b, sin_b, cos_p, sin_p);    // less what the box subtends
    if (cos_p <= cone.z) return 0.0f;
    const float cos_i = fabsf(dot(w, n)), sin_i = root_or_zero(1.0f - cos_i * cos_i);
    float cos_f, sin_f;
    angle_less(cos_i, sin_i, cos_b, sin_b, cos_f, sin_f);  // the receiver's tilt, less the same
    return fmaxf(axis.w * cos_p / fmaxf(o2, r) * cos_f, 0.0f);
}

// Both children's weights at pair `k`: importance at (p, n), or power alone.
template <bool kByPower>
__device__ __forceinline__ void pair_weights(const TreePair &pair, float3 p, float3 n, float &w0, float &w1,
                                             uint32_t &lead0, uint32_t &lead1) {
    const float4 a0 = __ldg(&pair.axis[0]), a1 = __ldg(&pair.axis[1]);
    const float4 k0 = __ldg(&pair.cone[0]), k1 = __ldg(&pair.cone[1]);
    lead0 = __float_as_uint(k0.w);
    lead1 = __float_as_uint(k1.w);
    if (kByPower) {
        w0 = fmaxf(a0.w, 0.0f);
        w1 = fmaxf(a1.w, 0.0f);
    } else {
        w0 = child_importance(__ldg(&pair.centre[0]), a0, k0, p, n);
        w1 = child_importance(__ldg(&pair.centre[1]), a1, k1, p, n);
    }
}

// Descends from the root choosing each child in proportion to its weight, u reused for
// every level (rescaled into the chosen interval): the emitter reached and the product of
// the chances taken. False for an empty tree or a point no child can light.
template <bool kByPower>
__device__ __forceinline__ bool tree_choose(const TreeTable &T, float u, float3 p, float3 n, uint32_t &emitter,
                                            float &chance) {
    chance = 1.0f;
    emitter = 0u;
    uint32_t at = T.root;
    if (at == kNone) return false;
    for (uint32_t level = 0; level < 64u; level++) {
        if (at & kTreeLeaf) {
            emitter = at & ~kTreeLeaf;
            return chance > 0.0f;
        }
        float w0, w1;
        uint32_t lead0, lead1;
        pair_weights<kByPower>(T.pairs[at], p, n, w0, w1, lead0, lead1);
        const float sum = w0 + w1;
        if (!(sum > 0.0f)) return false;
        const float left = w0 / sum;
        if (u < left) {
            u = fminf(u / left, 0.99999994f);
            chance *= left;
            at = lead0;
        } else {
            u = fminf((u - left) / (1.0f - left), 0.99999994f);
            chance *= 1.0f - left;
            at = lead1;
        }
    }
    return false;
}

// The chance tree_choose reaches `emitter`, following its recorded trail (bit k: the
// turn at depth k) instead of a sample.
template <bool kByPower>
__device__ __forceinline__ float tree_chance_of(const TreeTable &T, uint32_t emitter, float3 p, float3 n) {
    const uint4 record = __ldg(&T.records[emitter]);
    uint32_t at = T.root;
    float chance = 1.0f;
    for (uint32_t level = 0; level < record.z; level++) {
        if (at & kTreeLeaf) return 0.0f;
        float w0, w1;
        uint32_t lead0, lead1;
        pair_weights<kByPower>(T.pairs[at], p, n, w0, w1, lead0, lead1);
        const float sum = w0 + w1;
        if (!(sum > 0.0f)) return 0.0f;
        const bool right = (record.y >> level) & 1u;
        chance *= (right ? w1 : w0) / sum;
        at = right ? lead1 : lead0;
    }
    return chance;
}

__device__ __forceinline__ uint32_t emitter_code(const TreeTable &T, uint32_t emitter) {
    return __ldg(&T.records[emitter]).x;
}

}  // namespace lr
