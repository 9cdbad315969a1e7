// Device math the integrator's kernels share: vectors, the stateless Owen-scrambled
// Sobol sampler (shaders/sampler.glsl:8-55), hero-wavelength spectra
// (spectrum.glsl:10-118), the constants a member's kernels read, and the path helpers of
// common.glsl:103-276 (concentric disk, power-heuristic weight, origin offset, octahedral
// normals, orthonormal basis, bounce counters). Lights are in emitters.cuh, the light tree
// in lighttree.cuh, surfaces in surface.cuh.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace lr {

constexpr float kPi = 3.14159265358979323846f;
constexpr float kInfinity = 3.0e38f;
constexpr uint32_t kNone = 0xffffffffu;
constexpr uint32_t kLightHit = 0x80000000u;
constexpr uint32_t kEmitterTriangle = 0x80000000u;
constexpr uint32_t kLeafNode = 0x80000000u;

// ---- vectors ---------------------------------------------------------------------------

__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator-(float3 a) { return make_float3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ float3 operator*(float3 a, float s) { return make_float3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float3 operator*(float s, float3 a) { return make_float3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float3 operator/(float3 a, float s) { return make_float3(a.x / s, a.y / s, a.z / s); }
__device__ __forceinline__ float2 operator*(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
__device__ __forceinline__ float4 operator+(float4 a, float4 b) { return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
__device__ __forceinline__ float4 operator*(float4 a, float4 b) { return make_float4(a.x * b.x, a.y * b.y, a.z * b.z, a.w * b.w); }
__device__ __forceinline__ float4 operator*(float4 a, float s) { return make_float4(a.x * s, a.y * s, a.z * s, a.w * s); }
__device__ __forceinline__ float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 cross(float3 a, float3 b) {
    return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float length(float3 a) { return sqrtf(dot(a, a)); }
__device__ __forceinline__ float3 normalize(float3 a) { return a * rsqrtf(dot(a, a)); }
__device__ __forceinline__ float3 xyz(float4 a) { return make_float3(a.x, a.y, a.z); }

// ---- sampler.glsl --------------------------------------------------------------------

// Sobol dimensions 1..3 by bytes of the index: g_sobol_bytes[(d - 1) * 1024 + b * 256 + v]
// is the XOR of the direction numbers of the set bits of byte value v at byte position b,
// so a 32-bit index costs four lookups (XOR is associative: the same value as the
// bit-by-bit sum of sampler.glsl:32-37). Dimension 0 is van der Corput, a bit reversal.
static __device__ uint32_t g_sobol_bytes[3 * 4 * 256];

__device__ __forceinline__ uint32_t hash_u32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x21f0aaadu;
    x ^= x >> 15;
    x *= 0x735a2d97u;
    x ^= x >> 15;
    return x;
}

__device__ __forceinline__ uint32_t hash_combine(uint32_t seed, uint32_t value) {
    return seed ^ (hash_u32(value) + 0x9e3779b9u + (seed << 6) + (seed >> 2));
}

__device__ __forceinline__ uint32_t nested_uniform_scramble(uint32_t x, uint32_t seed) {
    x = __brev(x);
    x += seed;
    x ^= x * 0x6c50b47cu;
    x ^= x * 0xb82f1e52u;
    x ^= x * 0xc7afe638u;
    x ^= x * 0x8d22f6e6u;
    return __brev(x);
}

__device__ __forceinline__ uint32_t sobol(uint32_t index, uint32_t dimension) {
    if (dimension == 0) return __brev(index);
    const uint32_t *t = g_sobol_bytes + (dimension - 1) * 1024;
    return __ldg(&t[index & 0xffu]) ^ __ldg(&t[256 + ((index >> 8) & 0xffu)]) ^ __ldg(&t[512 + ((index >> 16) & 0xffu)]) ^
           __ldg(&t[768 + (index >> 24)]);
}

// sample4 (sampler.glsl:47-55): the 4-D point of `group` for this pixel's sample.
__device__ __forceinline__ float4 sample4(uint32_t seed, uint32_t pixel, uint32_t index, uint32_t group) {
    const uint32_t s = hash_combine(hash_combine(seed, pixel), group);
    const uint32_t shuffled = nested_uniform_scramble(index, hash_u32(s));
    float v[4];
#pragma unroll
    for (uint32_t d = 0; d < 4; d++)
        v[d] = (float)(nested_uniform_scramble(sobol(shuffled, d), hash_combine(s, d + 1u)) >> 8) * (1.0f / 16777216.0f);
    return make_float4(v[0], v[1], v[2], v[3]);
}

constexpr uint32_t kGroupCamera = 0, kGroupWavelength = 1;
__device__ __forceinline__ uint32_t group_light(uint32_t b) { return 2u + 3u * b; }
__device__ __forceinline__ uint32_t group_bsdf(uint32_t b) { return 3u + 3u * b; }
__device__ __forceinline__ uint32_t group_opacity(uint32_t b) { return 4u + 3u * b; }

// ---- common.glsl ---------------------------------------------------------------------

__device__ __forceinline__ float2 concentric(float2 u) {
    const float ox = 2.0f * u.x - 1.0f, oy = 2.0f * u.y - 1.0f;
    if (ox == 0.0f && oy == 0.0f) return make_float2(0.0f, 0.0f);
    float r, theta;
    if (fabsf(ox) > fabsf(oy)) {
        r = ox;
        theta = (kPi / 4.0f) * (oy / ox);
    } else {
        r = oy;
        theta = (kPi / 2.0f) - (kPi / 4.0f) * (ox / oy);
    }
    float s, c;
    sincosf(theta, &s, &c);
    return make_float2(r * c, r * s);
}

__device__ __forceinline__ float mis_weight(float a, float b) {
    a = fminf(a, 1e18f);
    b = fminf(b, 1e18f);
    return 1.0f / (1.0f + a * a + b * b);
}

__device__ __forceinline__ float3 offset_origin(float3 p, float3 n) {
    const float scale = fmaxf(1.0f, fmaxf(fabsf(p.x), fmaxf(fabsf(p.y), fabsf(p.z))));
    return p + n * (1e-4f * scale);
}

__device__ __forceinline__ uint32_t octahedral_encode(float3 n) {
    const float inv = 1.0f / (fabsf(n.x) + fabsf(n.y) + fabsf(n.z));
    float px = n.x * inv, py = n.y * inv;
    if (n.z < 0.0f) {
        const float qx = (1.0f - fabsf(py)) * (px >= 0.0f ? 1.0f : -1.0f);
        const float qy = (1.0f - fabsf(px)) * (py >= 0.0f ? 1.0f : -1.0f);
        px = qx;
        py = qy;
    }
    // packSnorm2x16: round(clamp(v, -1, 1) * 32767)
    const int ix = __float2int_rn(fminf(fmaxf(px, -1.0f), 1.0f) * 32767.0f);
    const int iy = __float2int_rn(fminf(fmaxf(py, -1.0f), 1.0f) * 32767.0f);
    return ((uint32_t)ix & 0xffffu) | ((uint32_t)iy << 16);
}

__device__ __forceinline__ float3 octahedral_decode(uint32_t packed) {
    // unpackSnorm2x16: clamp(v / 32767, -1, 1)
    float x = fmaxf((float)(int16_t)(packed & 0xffffu) / 32767.0f, -1.0f);
    float y = fmaxf((float)(int16_t)(packed >> 16) / 32767.0f, -1.0f);
    float3 n = make_float3(x, y, 1.0f - fabsf(x) - fabsf(y));
    if (n.z < 0.0f) {
        const float nx = (1.0f - fabsf(y)) * (x >= 0.0f ? 1.0f : -1.0f);
        const float ny = (1.0f - fabsf(x)) * (y >= 0.0f ? 1.0f : -1.0f);
        n.x = nx;
        n.y = ny;
    }
    return normalize(n);
}

// An orthonormal basis around n (Duff et al. 2017; common.glsl:270-276).
__device__ __forceinline__ void basis(float3 n, float3 &t, float3 &b) {
    const float s = n.z >= 0.0f ? 1.0f : -1.0f;
    const float a = -1.0f / (s + n.z);
    const float c = n.x * n.y * a;
    t = make_float3(1.0f + s * n.x * n.x * a, s * c, -s * n.x);
    b = make_float3(c, s + n.y * n.y * a, -n.y);
}

// next_bounce (common.glsl:229-234): one more bounce of `lobe`, or kNone past a limit.
__device__ __forceinline__ uint32_t next_bounce(uint32_t bounces, uint32_t lobe, const float *limits) {
    const uint32_t shift = 8u * (lobe + 1u);
    const uint32_t kind = ((bounces >> shift) & 0xffu) + 1u;
    if ((float)kind > limits[lobe] || (bounces & 0xffu) >= 255u) return kNone;
    return (bounces & ~(0xffu << shift)) + (kind << shift) + 1u;
}

// ---- spectrum.glsl -------------------------------------------------------------------

__device__ __forceinline__ float4 sample_wavelengths(float u) {
    float l[4];
#pragma unroll
    for (int i = 0; i < 4; i++) {
        float v = u + (float)i * 0.25f;
        v = v - floorf(v);
        l[i] = 538.0f - 138.888889f * atanhf(0.85691062f - 1.82750197f * v);
    }
    return make_float4(l[0], l[1], l[2], l[3]);
}

__device__ __forceinline__ float wavelength_pdf(float lambda) {
    if (lambda < 360.0f || lambda > 830.0f) return 0.0f;
    const float c = coshf(0.0072f * (lambda - 538.0f));
    return 0.0039398042f / (c * c);
}

__device__ __forceinline__ float cmf_lobe(float x, float mean, float below, float above) {
    const float t = (x - mean) / (x < mean ? below : above);
    return expf(-0.5f * t * t);
}

__device__ __forceinline__ float3 cmf(float l) {
    return make_float3(1.056f * cmf_lobe(l, 599.8f, 37.9f, 31.0f) + 0.362f * cmf_lobe(l, 442.0f, 16.0f, 26.7f) -
                           0.065f * cmf_lobe(l, 501.1f, 20.4f, 26.2f),
                       0.821f * cmf_lobe(l, 568.8f, 46.9f, 40.5f) + 0.286f * cmf_lobe(l, 530.9f, 16.3f, 31.1f),
                       1.217f * cmf_lobe(l, 437.0f, 11.8f, 36.0f) + 0.681f * cmf_lobe(l, 459.0f, 26.0f, 13.8f));
}

template <bool kSpectral>
__device__ __forceinline__ float4 spec_of(float4 fit, float3 rgb, float4 lambda) {
    if (!kSpectral) return make_float4(rgb.x, rgb.y, rgb.z, 0.0f);
    float l[4] = {lambda.x, lambda.y, lambda.z, lambda.w}, o[4];
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const float x = (l[i] - 360.0f) / (830.0f - 360.0f);
        const float z = (fit.x * x + fit.y) * x + fit.z;
        o[i] = fit.w * (0.5f + z / (2.0f * sqrtf(1.0f + z * z)));
    }
    return make_float4(o[0], o[1], o[2], o[3]);
}

__device__ __forceinline__ float blackbody(float lambda, float kelvin) {
    const float peak = 2.8977721e6f / kelvin;
    const float x = 1.4387769e7f / (lambda * kelvin);
    const float r = peak / lambda;
    return r * r * r * r * r * (142.32492f / (expf(x) - 1.0f));
}

template <bool kSpectral>
__device__ __forceinline__ float spec_max(float4 s) {
    return kSpectral ? fmaxf(fmaxf(s.x, s.y), fmaxf(s.z, s.w)) : fmaxf(s.x, fmaxf(s.y, s.z));
}

// The constants the integrator kernels read (spectral film, bounce limits, light
// selection), after the K_* rows of common.glsl:79-86 and loading.lucb:253-272.
struct Constants {
    float film[9];          // XYZ under E -> ACEScg, by rows
    float cmf_integrals[3];
    float limits[3];        // the most diffuse, glossy, transmission bounces
    float clamp_indirect;   // 0: off
    float4 background_fit;
    float3 background_rgb;
    float p_distant;        // the chance a light sample takes a distant light
    uint32_t max_bounces;
    uint32_t light_count;
    uint32_t tree_nodes;
    uint32_t seed;
    // Light paths from afar (lights.glsl:287-288): their share of light paths, and the
    // disk they start on, facing the light (radius, centre).
    float emit_share, emit_radius;
    float3 emit_center;
    float noise_threshold;  // adaptive sampling's (0: off)
};

template <bool kSpectral>
__device__ __forceinline__ float3 spec_to_film(float4 radiance, float4 lambda, const Constants &k) {
    if (!kSpectral) return xyz(radiance);
    float3 sum = make_float3(0.0f, 0.0f, 0.0f);
    const float l[4] = {lambda.x, lambda.y, lambda.z, lambda.w}, r[4] = {radiance.x, radiance.y, radiance.z, radiance.w};
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const float pdf = wavelength_pdf(l[i]);
        if (pdf > 0.0f) sum = sum + cmf(l[i]) * (r[i] / pdf);
    }
    return make_float3(sum.x * 0.25f / k.cmf_integrals[0], sum.y * 0.25f / k.cmf_integrals[1],
                       sum.z * 0.25f / k.cmf_integrals[2]);
}

}  // namespace lr
