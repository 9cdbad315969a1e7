// Device math of the integrator's shading: the stateless Owen-scrambled Sobol sampler
// (shaders/sampler.glsl:8-55), hero-wavelength spectra (spectrum.glsl:10-118), UsdLux
// lights (lights.glsl:24-282), the light tree (lighttree.glsl:18-137), EON diffuse
// (openpbr.glsl:87-113) and the path helpers of common.glsl:103-276. The layered OpenPBR
// surface is in openpbr.cuh.
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

// ---- lights.glsl ---------------------------------------------------------------------

constexpr uint32_t kLightStride = 7;
constexpr uint32_t kLightRect = 0, kLightDisk = 1, kLightSphere = 2, kLightDistant = 3, kLightDome = 4;

struct LightSample {
    float3 direction;
    float distance;
    float pdf;
    float cos_light;
    bool delta;
};

__device__ __forceinline__ float4 light_at(const float4 *lights, uint32_t light, uint32_t row) {
    return __ldg(&lights[light * kLightStride + row]);
}
__device__ __forceinline__ uint32_t light_type(const float4 *lights, uint32_t l) { return (uint32_t)light_at(lights, l, 0).w; }
__device__ __forceinline__ bool light_visible(const float4 *lights, uint32_t l) {
    return ((uint32_t)light_at(lights, l, 5).w & 1u) != 0u;
}

template <bool kSpectral>
__device__ __forceinline__ float4 light_radiance(const float4 *lights, uint32_t light, float4 lambda) {
    const float4 rgb = light_at(lights, light, 5);
    float4 radiance = spec_of<kSpectral>(light_at(lights, light, 4), xyz(rgb), lambda);
    if (kSpectral && ((uint32_t)rgb.w & 2u) != 0u) {
        const float kelvin = light_at(lights, light, 6).x;
        radiance.x *= blackbody(lambda.x, kelvin);
        radiance.y *= blackbody(lambda.y, kelvin);
        radiance.z *= blackbody(lambda.z, kelvin);
        radiance.w *= blackbody(lambda.w, kelvin);
    }
    return radiance;
}

// ---- Dome lights (lights.glsl:89-174): a lat-long image around the scene, its centre
// down the dome's -Z, its top +Y; a dome with no image (or not the one image the records
// hold) shines its colour evenly.

// Where the records keep the textured dome's image (loading.cpp's pack_lights): its
// texels (colour or basis weights, and the sampling weight), cumulative weights (each
// row's, then the rows'), size and weights' sum.
struct DomeImage {
    const float4 *texels;
    const float *cdf;
    uint32_t width, height;
    float total;
};

__device__ __forceinline__ bool dome_image(const float4 *lights, uint32_t light, DomeImage &image) {
    const uint32_t base = __float_as_uint(light_at(lights, light, 1).w);
    if (base == 0u) return false;
    image.texels = lights + base;
    image.width = __float_as_uint(light_at(lights, light, 2).w);
    image.height = __float_as_uint(light_at(lights, light, 3).w);
    image.cdf = reinterpret_cast<const float *>(lights) + __float_as_uint(light_at(lights, light, 6).w);
    image.total = light_at(lights, light, 0).x;
    return true;
}

// dome_texel (lights.glsl:99-110): the texel world direction d falls in, and sin theta there.
__device__ __forceinline__ uint32_t dome_texel(const float4 *lights, uint32_t light, const DomeImage &image, float3 d,
                                               float &sin_theta) {
    const float3 l = make_float3(dot(d, xyz(light_at(lights, light, 1))), dot(d, xyz(light_at(lights, light, 2))),
                                 dot(d, xyz(light_at(lights, light, 3))));
    const float u = 0.5f + atan2f(l.x, -l.z) * (0.5f / kPi);
    const float v = acosf(fminf(fmaxf(l.y, -1.0f), 1.0f)) / kPi;
    sin_theta = sqrtf(fmaxf(0.0f, 1.0f - l.y * l.y));
    const uint32_t x = min((uint32_t)(u * (float)image.width), image.width - 1u);
    const uint32_t y = min((uint32_t)(v * (float)image.height), image.height - 1u);
    return y * image.width + x;
}

// spec_of_texel (spectrum.glsl:61-80): the spectral build's texel holds the weights of
// three smooth spectra that sum to the flat one (blue, green, red); the RGB build's its
// ACEScg as it is.
template <bool kSpectral>
__device__ __forceinline__ float4 spec_of_texel(float3 texel, float4 lambda) {
    if (!kSpectral) return make_float4(texel.x, texel.y, texel.z, 0.0f);
    const float l[4] = {lambda.x, lambda.y, lambda.z, lambda.w};
    float out[4];
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const float blue = 1.0f - 1.0f / (1.0f + expf(-(l[i] - 490.0f) / 12.0f));
        const float red = 1.0f / (1.0f + expf(-(l[i] - 595.0f) / 12.0f));
        out[i] = texel.x * blue + texel.y * (1.0f - blue - red) + texel.z * red;
    }
    return make_float4(out[0], out[1], out[2], out[3]);
}

// dome_radiance (lights.glsl:112-118): the dome's radiance toward -d (d toward the dome).
// The dome functions are out of line: only scenes with a dome call them, and inlined
// into every light loop they would crowd the shading kernels' instruction cache.
template <bool kSpectral>
__device__ __noinline__ float4 dome_radiance(const float4 *lights, uint32_t light, float3 d, float4 lambda) {
    const float4 radiance = light_radiance<kSpectral>(lights, light, lambda);
    DomeImage image;
    if (!dome_image(lights, light, image)) return radiance;
    float sin_theta;
    const float4 texel = __ldg(&image.texels[dome_texel(lights, light, image, d, sin_theta)]);
    return radiance * spec_of_texel<kSpectral>(xyz(texel), lambda);
}

// dome_pdf (lights.glsl:120-129): the solid-angle pdf of sampling direction d (the
// selection's chance not included): a texel's weight over the sum, spread over its solid
// angle.
static __device__ __noinline__ float dome_pdf(const float4 *lights, uint32_t light, float3 d) {
    DomeImage image;
    if (!dome_image(lights, light, image)) return 1.0f / (4.0f * kPi);
    float sin_theta;
    const uint32_t texel = dome_texel(lights, light, image, d, sin_theta);
    if (sin_theta <= 0.0f) return 0.0f;
    const float weight = __ldg(&image.texels[texel]).w;
    return weight / image.total * (float)image.width * (float)image.height / (2.0f * kPi * kPi * sin_theta);
}

// dome_search (lights.glsl:136-150): the first of `count` cumulative weights from `first`
// that passes u, and u's place within it (0..1).
__device__ __forceinline__ uint32_t dome_search(const float *cdf, uint32_t first, uint32_t count, float u, float &within) {
    uint32_t low = 0u, high = count - 1u;
    while (low < high) {
        const uint32_t middle = (low + high) / 2u;
        if (__ldg(&cdf[first + middle]) > u) high = middle;
        else low = middle + 1u;
    }
    const float below = low > 0u ? __ldg(&cdf[first + low - 1u]) : 0.0f;
    const float above = __ldg(&cdf[first + low]);
    within = above > below ? fminf(fmaxf((u - below) / (above - below), 0.0f), 0.99999994f) : 0.5f;
    return low;
}

__device__ __forceinline__ uint32_t pick_distant(const float4 *lights, uint32_t count, float u, float &pdf) {
    uint32_t chosen = kNone;
    for (uint32_t light = 0; light < count; light++) {
        if (light_type(lights, light) < kLightDistant) continue;
        chosen = light;
        if (u < light_at(lights, light, 6).z) break;
    }
    pdf = chosen == kNone ? 0.0f : light_at(lights, chosen, 6).y;
    return chosen;
}

__device__ __forceinline__ float3 sample_cone(float3 axis, float cos_max, float2 u) {
    const float c = 1.0f - u.x * (1.0f - cos_max);
    const float s = sqrtf(fmaxf(0.0f, 1.0f - c * c));
    const float phi = 2.0f * kPi * u.y;
    float3 t, b;
    basis(axis, t, b);
    float sp, cp;
    sincosf(phi, &sp, &cp);
    return normalize(t * (s * cp) + b * (s * sp) + axis * c);
}

__device__ __forceinline__ float sphere_hit(float3 center, float radius, float3 o, float3 d) {
    const float3 oc = o - center;
    const float b = dot(oc, d);
    const float c = dot(oc, oc) - radius * radius;
    float h = b * b - c;
    if (h < 0.0f) return kInfinity;
    h = sqrtf(h);
    float t = -b - h;
    if (t > 0.0f) return t;
    t = -b + h;
    return t > 0.0f ? t : kInfinity;
}

// sample_dome (lights.glsl:152-174): a direction by the image's weights (rows, then the
// chosen row's texels), or uniform over the sphere for a dome without an image.
static __device__ __noinline__ bool sample_dome(const float4 *lights, uint32_t light, float2 u, LightSample &s) {
    s.distance = kInfinity;
    s.delta = false;
    s.cos_light = 1.0f;
    float3 l;
    DomeImage image;
    if (!dome_image(lights, light, image)) {
        const float z = 1.0f - 2.0f * u.x;
        const float r = sqrtf(fmaxf(0.0f, 1.0f - z * z));
        l = make_float3(r * cosf(2.0f * kPi * u.y), z, r * sinf(2.0f * kPi * u.y));
    } else {
        float fy, fx;
        const uint32_t y = dome_search(image.cdf, image.width * image.height, image.height, u.y, fy);
        const uint32_t x = dome_search(image.cdf, y * image.width, image.width, u.x, fx);
        const float theta = kPi * ((float)y + fy) / (float)image.height;
        const float phi = 2.0f * kPi * (((float)x + fx) / (float)image.width - 0.5f);
        l = make_float3(sinf(theta) * sinf(phi), cosf(theta), -sinf(theta) * cosf(phi));
    }
    s.direction = normalize(xyz(light_at(lights, light, 1)) * l.x + xyz(light_at(lights, light, 2)) * l.y +
                            xyz(light_at(lights, light, 3)) * l.z);
    s.pdf = dome_pdf(lights, light, s.direction);
    return s.pdf > 0.0f;
}

__device__ __forceinline__ bool sample_light(const float4 *lights, uint32_t light, float3 p, float2 u, LightSample &s) {
    const float4 row0 = light_at(lights, light, 0), row1 = light_at(lights, light, 1), row2 = light_at(lights, light, 2),
                 row3 = light_at(lights, light, 3);
    const uint32_t type = (uint32_t)row0.w;
    if (type == kLightDome) return sample_dome(lights, light, u, s);
    s.delta = false;
    s.cos_light = 1.0f;
    if (type == kLightRect || type == kLightDisk) {
        const float2 a = type == kLightRect ? make_float2(2.0f * u.x - 1.0f, 2.0f * u.y - 1.0f) : concentric(u);
        const float3 q = xyz(row0) + a.x * xyz(row1) + a.y * xyz(row2);
        const float3 d = q - p;
        const float d2 = dot(d, d);
        s.distance = sqrtf(d2);
        s.direction = d * (1.0f / s.distance);
        const float cos_light = -dot(s.direction, xyz(row3));
        if (cos_light <= 0.0f || row3.w <= 0.0f) return false;
        s.pdf = d2 / (cos_light * row3.w);
        s.cos_light = cos_light;
        return true;
    }
    if (type == kLightSphere) {
        const float3 to_center = xyz(row0) - p;
        const float d2 = dot(to_center, to_center);
        const float r = row1.w;
        if (d2 <= r * r) return false;
        const float cos_max = sqrtf(fmaxf(0.0f, 1.0f - r * r / d2));
        s.direction = sample_cone(to_center * rsqrtf(d2), cos_max, u);
        s.distance = sphere_hit(xyz(row0), r, p, s.direction);
        if (s.distance >= kInfinity) return false;
        s.pdf = 1.0f / (2.0f * kPi * (1.0f - cos_max));
        s.cos_light = fmaxf(0.0f, -dot(s.direction, normalize(p + s.direction * s.distance - xyz(row0))));
        return true;
    }
    const float3 axis = -xyz(row3);
    const float cos_half = row2.w;
    s.distance = kInfinity;
    if (cos_half >= 1.0f - 1e-7f) {
        s.direction = axis;
        s.pdf = 1.0f;
        s.delta = true;
        return true;
    }
    s.direction = sample_cone(axis, cos_half, u);
    s.pdf = 1.0f / (2.0f * kPi * (1.0f - cos_half));
    return true;
}

// intersect_light (lights.glsl:239-259). `flow`: the ray follows light (a light path), so a
// flat light stops it only when crossed the way it shines.
__device__ __forceinline__ float intersect_light(const float4 *lights, uint32_t light, float3 o, float3 d, float t_max,
                                                 bool flow = false) {
    const float4 row0 = light_at(lights, light, 0);
    const uint32_t type = (uint32_t)row0.w;
    if (type == kLightSphere) {
        const float t = sphere_hit(xyz(row0), light_at(lights, light, 1).w, o, d);
        return t < t_max ? t : kInfinity;
    }
    if (type >= kLightDistant) return kInfinity;
    const float3 u = xyz(light_at(lights, light, 1)), v = xyz(light_at(lights, light, 2)),
                 n = xyz(light_at(lights, light, 3));
    const float facing = dot(d, n);
    if (flow ? facing <= 0.0f : facing >= 0.0f) return kInfinity;
    const float t = dot(xyz(row0) - o, n) / facing;
    if (t <= 0.0f || t >= t_max) return kInfinity;
    const float3 q = o + t * d - xyz(row0);
    const float a = dot(q, u) / dot(u, u);
    const float b = dot(q, v) / dot(v, v);
    const bool inside = type == kLightRect ? (fabsf(a) <= 1.0f && fabsf(b) <= 1.0f) : (a * a + b * b <= 1.0f);
    return inside ? t : kInfinity;
}

__device__ __forceinline__ float light_hit_pdf(const float4 *lights, uint32_t light, float3 o, float3 d, float t) {
    const float4 row0 = light_at(lights, light, 0);
    const uint32_t type = (uint32_t)row0.w;
    if (type == kLightSphere) {
        const float3 to_center = xyz(row0) - o;
        const float r = light_at(lights, light, 1).w;
        const float cos_max = sqrtf(fmaxf(0.0f, 1.0f - r * r / dot(to_center, to_center)));
        return 1.0f / (2.0f * kPi * fmaxf(1e-12f, 1.0f - cos_max));
    }
    if (type == kLightDistant) return 1.0f / (2.0f * kPi * fmaxf(1e-12f, 1.0f - light_at(lights, light, 2).w));
    if (type == kLightDome) return dome_pdf(lights, light, d);
    const float4 row3 = light_at(lights, light, 3);
    const float cos_light = fmaxf(1e-12f, -dot(d, xyz(row3)));
    return t * t / (cos_light * row3.w);
}

// ---- lighttree.glsl ------------------------------------------------------------------

struct TreeView {
    const float4 *nodes;     // 3 per node
    const uint2 *links;      // per node: first child or emitter, leaf flag
    const uint4 *records;    // per emitter: code, trail, depth, -
    const uint32_t *triangle_map;  // per triangle slot: emitter or kNone
    uint32_t node_count;
};

__device__ __forceinline__ float safe_sqrt(float x) { return sqrtf(fmaxf(0.0f, x)); }

__device__ __forceinline__ float tree_importance(const TreeView &t, uint32_t node, float3 p, float3 n) {
    const float4 a = __ldg(&t.nodes[node * 3]), b = __ldg(&t.nodes[node * 3 + 1]), c = __ldg(&t.nodes[node * 3 + 2]);
    if (a.w <= 0.0f) return 0.0f;
    const float3 center = 0.5f * (xyz(a) + xyz(b));
    const float3 offset = p - center;
    const float radius = 0.5f * length(xyz(b) - xyz(a));
    const float oo = dot(offset, offset);
    const float distance2 = fmaxf(oo, radius);
    const float3 wi = oo > 0.0f ? normalize(offset) : xyz(c);
    const float cos_w = dot(xyz(c), wi);
    const float sin_w = safe_sqrt(1.0f - cos_w * cos_w);
    const float cos_b = oo < radius * radius ? -1.0f : safe_sqrt(1.0f - radius * radius / oo);
    const float sin_b = safe_sqrt(1.0f - cos_b * cos_b);
    const float cos_o = b.w;
    const float sin_o = safe_sqrt(1.0f - cos_o * cos_o);
    const float cos_x = cos_w > cos_o ? 1.0f : cos_w * cos_o + sin_w * sin_o;
    const float sin_x = cos_w > cos_o ? 0.0f : sin_w * cos_o - cos_w * sin_o;
    const float cos_p = cos_x > cos_b ? 1.0f : cos_x * cos_b + sin_x * sin_b;
    if (cos_p <= c.w) return 0.0f;
    const float importance = a.w * cos_p / distance2;
    const float cos_i = fabsf(dot(wi, n));
    const float sin_i = safe_sqrt(1.0f - cos_i * cos_i);
    const float cos_pi = cos_i > cos_b ? 1.0f : cos_i * cos_b + sin_i * sin_b;
    return fmaxf(importance * cos_pi, 0.0f);
}

__device__ __forceinline__ bool tree_sample(const TreeView &t, float u, float3 p, float3 n, uint32_t &emitter, float &pdf) {
    pdf = 1.0f;
    emitter = 0;
    if (t.node_count < 1) return false;
    uint32_t node = 0;
    for (uint32_t depth = 0; depth < 64u; depth++) {
        const uint2 link = __ldg(&t.links[node]);
        if ((link.y & kLeafNode) != 0u) {
            emitter = link.x;
            return pdf > 0.0f;
        }
        const float left = tree_importance(t, link.x, p, n);
        const float right = tree_importance(t, link.x + 1u, p, n);
        if (left + right <= 0.0f) return false;
        const float chance = left / (left + right);
        if (u < chance) {
            u = fminf(u / chance, 0.99999994f);
            pdf *= chance;
            node = link.x;
        } else {
            u = fminf((u - chance) / (1.0f - chance), 0.99999994f);
            pdf *= 1.0f - chance;
            node = link.x + 1u;
        }
    }
    return false;
}

__device__ __forceinline__ float tree_pdf(const TreeView &t, uint32_t emitter, float3 p, float3 n) {
    const uint4 record = __ldg(&t.records[emitter]);
    const uint32_t trail = record.y, depth = record.z;
    uint32_t node = 0;
    float pdf = 1.0f;
    for (uint32_t level = 0; level < depth; level++) {
        const uint32_t link = __ldg(&t.links[node]).x;
        const float left = tree_importance(t, link, p, n);
        const float right = tree_importance(t, link + 1u, p, n);
        if (left + right <= 0.0f) return 0.0f;
        const uint32_t bit = (trail >> level) & 1u;
        pdf *= bit == 0u ? left / (left + right) : right / (left + right);
        node = link + bit;
    }
    return pdf;
}

// ---- EON diffuse (openpbr.glsl:87-113) -----------------------------------------------

constexpr float kFonC1 = 0.5f - 2.0f / (3.0f * kPi);
constexpr float kFonC2 = 2.0f / 3.0f - 28.0f / (15.0f * kPi);

__device__ __forceinline__ float fon_albedo(float mu, float r) {
    const float m = 1.0f - mu;
    const float g_over_pi = m * (0.0571085289f + m * (0.491881867f + m * (-0.332181442f + m * 0.0714429953f)));
    return (1.0f + r * g_over_pi) / (1.0f + kFonC1 * r);
}

__device__ __forceinline__ float4 eon(float4 rho, float r, float3 wi, float3 wo) {
    const float mu_i = wi.z, mu_o = wo.z;
    const float s = dot(wi, wo) - mu_i * mu_o;
    const float s_over_t = s > 0.0f ? s / fmaxf(mu_i, mu_o) : s;
    const float a = 1.0f / (1.0f + kFonC1 * r);
    const float4 single = rho * (a * (1.0f + r * s_over_t) / kPi);
    const float e_o = fon_albedo(mu_o, r), e_i = fon_albedo(mu_i, r);
    const float average = a * (1.0f + kFonC2 * r);
    const float k = fmaxf(1e-7f, 1.0f - e_o) * fmaxf(1e-7f, 1.0f - e_i) / (kPi * fmaxf(1e-7f, 1.0f - average));
    float4 multiple;
    multiple.x = rho.x * rho.x * average / (1.0f - rho.x * (1.0f - average)) * k;
    multiple.y = rho.y * rho.y * average / (1.0f - rho.y * (1.0f - average)) * k;
    multiple.z = rho.z * rho.z * average / (1.0f - rho.z * (1.0f - average)) * k;
    multiple.w = rho.w * rho.w * average / (1.0f - rho.w * (1.0f - average)) * k;
    return single + multiple;
}

}  // namespace lr
