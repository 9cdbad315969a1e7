// UsdLux lights as the integrator's kernels read them: one DeviceLight record (8 float4)
// per light, built on the host (loading.cpp `device_lights`) from the reference's light
// records (src/render/lights.lucb:29-131) with each shape's constants worked out once:
// a flat light's edges with their inverse squared lengths, a sphere's squared radius, a
// cone's solid-angle pdf. Two index lists split the lights by how they are met: the
// finite ones (rect, disk, sphere) that rays can hit -- the closest-hit and connection
// tests loop over these alone -- and the ones from afar (distant lights and domes), in
// light order, that misses and light selection read. A dome's image sits in a DomeView.
//
// The mathematics is the reference's estimator (shaders/lights.glsl:31-282): the same
// map from a 2-D sample to a point or direction per shape, the same solid-angle
// densities, the same choice among lights from afar by power. Those are what the f64
// oracle restates and what the parity tests hold the kernels to.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "shading.cuh"

namespace lr {

constexpr uint32_t kShapeRect = 0, kShapeDisk = 1, kShapeSphere = 2, kShapeDistant = 3, kShapeDome = 4;
constexpr uint32_t kLightSeen = 1u, kLightBlackbody = 2u;  // DeviceLight::look.w flag bits

struct alignas(16) DeviceLight {
    // centre (rect, disk, sphere); w: the shape
    float4 centre;
    // rect, disk: half edge u and 1 / |u|^2; dome: the frame's x axis
    float4 u;
    // rect, disk: half edge v and 1 / |v|^2; dome: the frame's y axis
    float4 v;
    // rect, disk: the unit direction the light shines along and the area; distant: the
    // direction its light travels; dome: the frame's z axis
    float4 n;
    // sphere: radius, radius^2; distant: cos of the half angle, the cone's solid-angle
    // pdf, 1 for a delta (no angle)
    float4 cone;
    float4 fit;   // the emitted colour's spectral fit (c0, c1, c2, scale)
    float4 look;  // the emitted ACEScg radiance; w: flag bits (kLightSeen, kLightBlackbody)
    // kelvin; share among lights from afar; cumulative share; the light tree's emitter
    float4 pick;
};

// The textured dome's image (environment.lucb:60-156): per texel its colour (the
// spectral build: its three basis spectra's weights) and its sampling weight; each row's
// cumulative weights, then the rows'.
struct DomeView {
    const float4 *texels = nullptr;
    const float *cdf = nullptr;
    uint32_t width = 0, height = 0;
    uint32_t light = kNone;  // the dome the image belongs to
    float weight_sum = 0.0f;
};

struct LightTable {
    const DeviceLight *light = nullptr;
    const uint32_t *finite = nullptr;  // rect, disk and sphere lights
    const uint32_t *afar = nullptr;    // distant lights and domes, in light order
    uint32_t count = 0, finite_count = 0, afar_count = 0;
    DomeView dome;
};

// A light sample seen from the shaded point: unit direction toward the light, distance
// (kInfinity from afar), solid-angle pdf (1 for a delta), cosine at the light toward the
// point (1 from afar).
struct LightSample {
    float3 direction;
    float distance;
    float pdf;
    float cos_light;
    bool delta;
};

__device__ __forceinline__ uint32_t shape_of(const DeviceLight &l) { return __float_as_uint(l.centre.w); }
__device__ __forceinline__ uint32_t light_flags(const DeviceLight &l) { return __float_as_uint(l.look.w); }

// ---- small geometry ---------------------------------------------------------------------

// The first positive crossing of a sphere by a ray with a unit direction, or kInfinity.
__device__ __forceinline__ float sphere_crossing(float3 centre, float r2, float3 o, float3 d) {
    const float3 to_o = o - centre;
    const float half_b = dot(to_o, d);
    const float disc = half_b * half_b - (dot(to_o, to_o) - r2);
    if (disc < 0.0f) return kInfinity;
    const float root = sqrtf(disc);
    const float near = -half_b - root;
    if (near > 0.0f) return near;
    const float far = -half_b + root;
    return far > 0.0f ? far : kInfinity;
}

// A uniform direction in the cone of half-angle acos(cos_max) about the unit `axis`.
__device__ __forceinline__ float3 cone_direction(float3 axis, float cos_max, float2 u) {
    const float c = 1.0f - u.x * (1.0f - cos_max);
    const float s = sqrtf(fmaxf(0.0f, 1.0f - c * c));
    float sin_phi, cos_phi;
    sincosf(2.0f * kPi * u.y, &sin_phi, &cos_phi);
    float3 t, b;
    basis(axis, t, b);
    return normalize(t * (s * cos_phi) + b * (s * sin_phi) + axis * c);
}

// ---- hits -------------------------------------------------------------------------------

// Where a ray (unit direction) first meets finite light `l` on the side it is seen from,
// inside (0, t_max), or kInfinity. A flat light is seen against the direction it shines;
// `flow` (a light path's ray) meets it only crossing the way it shines, so a visibility
// test reads the same from either end.
__device__ __forceinline__ float light_crossing(const DeviceLight &l, float3 o, float3 d, float t_max, bool flow) {
    const float4 c = __ldg(&l.centre);
    if (__float_as_uint(c.w) == kShapeSphere) {
        const float t = sphere_crossing(xyz(c), __ldg(&l.cone).y, o, d);
        return t < t_max ? t : kInfinity;
    }
    const float3 n = xyz(__ldg(&l.n));
    const float along = dot(d, n);
    if (flow ? !(along > 0.0f) : !(along < 0.0f)) return kInfinity;
    const float t = dot(xyz(c) - o, n) / along;
    if (!(t > 0.0f && t < t_max)) return kInfinity;
    const float4 u = __ldg(&l.u), v = __ldg(&l.v);
    const float3 q = o + d * t - xyz(c);
    const float a = dot(q, xyz(u)) * u.w, b = dot(q, xyz(v)) * v.w;
    const bool within = __float_as_uint(c.w) == kShapeRect ? (fabsf(a) <= 1.0f && fabsf(b) <= 1.0f) : a * a + b * b <= 1.0f;
    return within ? t : kInfinity;
}

// The nearest finite light before `t` along a ray: updates t and returns the light, or
// kNone. Camera rays (`camera`) pass lights hidden from the camera.
__device__ __forceinline__ uint32_t nearest_light(const LightTable &T, float3 o, float3 d, float &t, bool camera,
                                                  bool flow) {
    uint32_t found = kNone;
    for (uint32_t k = 0; k < T.finite_count; k++) {
        const uint32_t index = __ldg(&T.finite[k]);
        const DeviceLight &l = T.light[index];
        if (camera && !(light_flags(l) & kLightSeen)) continue;
        const float hit = light_crossing(l, o, d, t, flow);
        if (hit < t) {
            t = hit;
            found = index;
        }
    }
    return found;
}

// Whether a light the camera sees stands on the segment (o, o + d * reach), crossed the
// way light flows along it.
__device__ __forceinline__ bool seen_light_between(const LightTable &T, float3 o, float3 d, float reach) {
    for (uint32_t k = 0; k < T.finite_count; k++) {
        const DeviceLight &l = T.light[__ldg(&T.finite[k])];
        if ((light_flags(l) & kLightSeen) && light_crossing(l, o, d, reach, true) < reach) return true;
    }
    return false;
}

// ---- emission ---------------------------------------------------------------------------

// The light's emitted radiance at the path's wavelengths (spectral) or in ACEScg (RGB).
template <bool kSpectral>
__device__ __forceinline__ float4 light_emission(const DeviceLight &l, float4 lambda) {
    const float4 look = __ldg(&l.look);
    float4 e = spec_of<kSpectral>(__ldg(&l.fit), xyz(look), lambda);
    if (kSpectral && (__float_as_uint(look.w) & kLightBlackbody)) {
        const float kelvin = __ldg(&l.pick).x;
        e = make_float4(e.x * blackbody(lambda.x, kelvin), e.y * blackbody(lambda.y, kelvin),
                        e.z * blackbody(lambda.z, kelvin), e.w * blackbody(lambda.w, kelvin));
    }
    return e;
}

// The chance a light sample picks light `l` among lights from afar (share x p_distant is
// the caller's).
__device__ __forceinline__ float afar_share(const DeviceLight &l) { return __ldg(&l.pick).y; }

// A light from afar chosen by power: the first whose cumulative share passes u (the last
// one otherwise), and its share.
__device__ __forceinline__ uint32_t choose_afar(const LightTable &T, float u, float &share) {
    uint32_t chosen = kNone;
    for (uint32_t k = 0; k < T.afar_count; k++) {
        chosen = __ldg(&T.afar[k]);
        if (u < __ldg(&T.light[chosen].pick).z) break;
    }
    share = chosen == kNone ? 0.0f : afar_share(T.light[chosen]);
    return chosen;
}

// ---- domes (environment.lucb; lights.glsl:89-174) ---------------------------------------

__device__ __forceinline__ bool dome_textured(const LightTable &T, uint32_t l) { return T.dome.light == l; }

// The dome frame's coordinates of world direction d.
__device__ __forceinline__ float3 dome_local(const DeviceLight &l, float3 d) {
    return make_float3(dot(d, xyz(__ldg(&l.u))), dot(d, xyz(__ldg(&l.v))), dot(d, xyz(__ldg(&l.n))));
}

// The texel of the lat-long image along world direction d, and sin(theta) there.
__device__ __forceinline__ uint32_t dome_texel(const DomeView &img, const DeviceLight &l, float3 d, float &sin_theta) {
    const float3 q = dome_local(l, d);
    const float s = 0.5f + atan2f(q.x, -q.z) * (0.5f / kPi);
    const float t = acosf(fminf(fmaxf(q.y, -1.0f), 1.0f)) * (1.0f / kPi);
    sin_theta = sqrtf(fmaxf(0.0f, 1.0f - q.y * q.y));
    const uint32_t col = min((uint32_t)(s * (float)img.width), img.width - 1u);
    const uint32_t row = min((uint32_t)(t * (float)img.height), img.height - 1u);
    return row * img.width + col;
}

// A texel's colour at the path's wavelengths: in the spectral build the weights of three
// logistic basis spectra (blue, middle, red) that sum to a flat one.
template <bool kSpectral>
__device__ __forceinline__ float4 texel_colour(float3 w, float4 lambda) {
    if (!kSpectral) return make_float4(w.x, w.y, w.z, 0.0f);
    auto at = [&](float nm) {
        const float blue = 1.0f - 1.0f / (1.0f + expf(-(nm - 490.0f) / 12.0f));
        const float red = 1.0f / (1.0f + expf(-(nm - 595.0f) / 12.0f));
        return w.x * blue + w.y * (1.0f - blue - red) + w.z * red;
    };
    return make_float4(at(lambda.x), at(lambda.y), at(lambda.z), at(lambda.w));
}

// The dome's radiance arriving along -d (d toward the dome). Out of line: only scenes
// with a dome call the dome functions, which would otherwise crowd every light loop.
template <bool kSpectral>
__device__ __noinline__ float4 dome_emission(const LightTable &T, uint32_t light, float3 d, float4 lambda) {
    const DeviceLight &l = T.light[light];
    const float4 e = light_emission<kSpectral>(l, lambda);
    if (!dome_textured(T, light)) return e;
    float sin_theta;
    const float4 w = __ldg(&T.dome.texels[dome_texel(T.dome, l, d, sin_theta)]);
    return e * texel_colour<kSpectral>(xyz(w), lambda);
}

// The solid-angle pdf of the dome's sampling choosing direction d: uniform over the sphere
// without an image; with one, the texel's weight share spread over its solid angle.
static __device__ __noinline__ float dome_density(const LightTable &T, uint32_t light, float3 d) {
    if (!dome_textured(T, light)) return 1.0f / (4.0f * kPi);
    float sin_theta;
    const uint32_t texel = dome_texel(T.dome, T.light[light], d, sin_theta);
    if (sin_theta <= 0.0f) return 0.0f;
    const float share = __ldg(&T.dome.texels[texel]).w / T.dome.weight_sum;
    return share * (float)T.dome.width * (float)T.dome.height / (2.0f * kPi * kPi * sin_theta);
}

// Inverse-CDF step over `count` cumulative weights from `first`: the first entry above u,
// and where u falls inside it (0..1; the middle of an empty entry).
__device__ __forceinline__ uint32_t invert_cdf(const float *cdf, uint32_t first, uint32_t count, float u, float &frac) {
    uint32_t lo = 0u, hi = count - 1u;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (__ldg(&cdf[first + mid]) > u) hi = mid;
        else lo = mid + 1u;
    }
    const float below = lo > 0u ? __ldg(&cdf[first + lo - 1u]) : 0.0f;
    const float above = __ldg(&cdf[first + lo]);
    frac = above > below ? fminf(fmaxf((u - below) / (above - below), 0.0f), 0.99999994f) : 0.5f;
    return lo;
}

static __device__ __noinline__ bool dome_sample(const LightTable &T, uint32_t light, float2 u, LightSample &s) {
    const DeviceLight &l = T.light[light];
    float3 q;
    if (!dome_textured(T, light)) {
        const float z = 1.0f - 2.0f * u.x;
        const float r = sqrtf(fmaxf(0.0f, 1.0f - z * z));
        float sin_phi, cos_phi;
        sincosf(2.0f * kPi * u.y, &sin_phi, &cos_phi);
        q = make_float3(r * cos_phi, z, r * sin_phi);
    } else {
        const DomeView &img = T.dome;
        float fy, fx;
        const uint32_t row = invert_cdf(img.cdf, img.width * img.height, img.height, u.y, fy);
        const uint32_t col = invert_cdf(img.cdf, row * img.width, img.width, u.x, fx);
        const float theta = kPi * ((float)row + fy) / (float)img.height;
        const float phi = 2.0f * kPi * (((float)col + fx) / (float)img.width - 0.5f);
        float st, ct, sp, cp;
        sincosf(theta, &st, &ct);
        sincosf(phi, &sp, &cp);
        q = make_float3(st * sp, ct, -st * cp);
    }
    s.direction = normalize(xyz(__ldg(&l.u)) * q.x + xyz(__ldg(&l.v)) * q.y + xyz(__ldg(&l.n)) * q.z);
    s.distance = kInfinity;
    s.cos_light = 1.0f;
    s.delta = false;
    s.pdf = dome_density(T, light, s.direction);
    return s.pdf > 0.0f;
}

// ---- sampling and densities -------------------------------------------------------------

// One sample of light `light` seen from p: a point uniform by area on a flat light (the
// square [-1, 1]^2 of a rect's half edges, the concentric disk of a disk's), a direction
// uniform in the cone a sphere subtends, a direction in a distant light's cone (its axis
// when it has no angle), or the dome's. False when the light cannot light p.
__device__ __forceinline__ bool light_sample(const LightTable &T, uint32_t light, float3 p, float2 u, LightSample &s) {
    const DeviceLight &l = T.light[light];
    const float4 c = __ldg(&l.centre);
    const uint32_t shape = __float_as_uint(c.w);
    s.delta = false;
    s.cos_light = 1.0f;
    switch (shape) {
        case kShapeRect:
        case kShapeDisk: {
            const float2 a = shape == kShapeRect ? make_float2(2.0f * u.x - 1.0f, 2.0f * u.y - 1.0f) : concentric(u);
            const float4 n = __ldg(&l.n);
            const float3 to = xyz(c) + xyz(__ldg(&l.u)) * a.x + xyz(__ldg(&l.v)) * a.y - p;
            const float d2 = dot(to, to);
            s.distance = sqrtf(d2);
            s.direction = to * (1.0f / s.distance);
            const float facing = -dot(s.direction, xyz(n));
            if (!(facing > 0.0f) || !(n.w > 0.0f)) return false;
            s.cos_light = facing;
            s.pdf = d2 / (facing * n.w);
            return true;
        }
        case kShapeSphere: {
            const float4 cone = __ldg(&l.cone);
            const float3 to = xyz(c) - p;
            const float d2 = dot(to, to);
            if (d2 <= cone.y) return false;
            const float cos_max = sqrtf(fmaxf(0.0f, 1.0f - cone.y / d2));
            s.direction = cone_direction(to * rsqrtf(d2), cos_max, u);
            s.distance = sphere_crossing(xyz(c), cone.y, p, s.direction);
            if (!(s.distance < kInfinity)) return false;
            s.pdf = 1.0f / (2.0f * kPi * (1.0f - cos_max));
            s.cos_light = fmaxf(0.0f, -dot(s.direction, normalize(p + s.direction * s.distance - xyz(c))));
            return true;
        }
        case kShapeDistant: {
            const float4 cone = __ldg(&l.cone);
            const float3 toward = -xyz(__ldg(&l.n));
            s.distance = kInfinity;
            if (cone.z != 0.0f) {
                s.direction = toward;
                s.pdf = 1.0f;
                s.delta = true;
                return true;
            }
            s.direction = cone_direction(toward, cone.x, u);
            s.pdf = cone.y;
            return true;
        }
        default:
            return dome_sample(T, light, u, s);
    }
}

// The solid-angle density light_sample gives the direction d from o, the light met at
// distance t (kInfinity for lights from afar).
__device__ __forceinline__ float light_density(const LightTable &T, uint32_t light, float3 o, float3 d, float t) {
    const DeviceLight &l = T.light[light];
    const float4 c = __ldg(&l.centre);
    switch (__float_as_uint(c.w)) {
        case kShapeSphere: {
            const float3 to = xyz(c) - o;
            const float cos_max = sqrtf(fmaxf(0.0f, 1.0f - __ldg(&l.cone).y / dot(to, to)));
            return 1.0f / (2.0f * kPi * fmaxf(1e-12f, 1.0f - cos_max));
        }
        case kShapeDistant:
            return 1.0f / (2.0f * kPi * fmaxf(1e-12f, 1.0f - __ldg(&l.cone).x));
        case kShapeDome:
            return dome_density(T, light, d);
        default: {
            const float4 n = __ldg(&l.n);
            return t * t / (fmaxf(1e-12f, -dot(d, xyz(n))) * n.w);
        }
    }
}

// The cosine at finite light `light`, toward where a ray from o along d that met it at t
// came from.
__device__ __forceinline__ float light_cosine(const LightTable &T, uint32_t light, float3 o, float3 d, float t) {
    const DeviceLight &l = T.light[light];
    const float4 c = __ldg(&l.centre);
    if (__float_as_uint(c.w) == kShapeSphere) return fmaxf(0.0f, -dot(d, normalize(o + d * t - xyz(c))));
    return fmaxf(0.0f, -dot(d, xyz(__ldg(&l.n))));
}

// A distant light with an angle, or a dome: light paths may start from it (from afar).
__device__ __forceinline__ bool emits_from_afar(const LightTable &T, uint32_t light) {
    const DeviceLight &l = T.light[light];
    const uint32_t shape = shape_of(l);
    return shape == kShapeDome || (shape == kShapeDistant && __ldg(&l.cone).z == 0.0f);
}

// A finite light's surface area (the density light emission spreads a point by).
__device__ __forceinline__ float light_area(const DeviceLight &l) {
    if (shape_of(l) == kShapeSphere) {
        const float r = __ldg(&l.cone).x;
        return 4.0f * kPi * r * r;
    }
    return __ldg(&l.n).w;
}

// A distant light's radiance for a miss along d (d toward the sky): zero outside its cone,
// and for a delta light, which no ray can find.
__device__ __forceinline__ bool distant_covers(const DeviceLight &l, float3 d) {
    const float4 cone = __ldg(&l.cone);
    return cone.z == 0.0f && !(dot(d, -xyz(__ldg(&l.n))) < cone.x);
}

}  // namespace lr
