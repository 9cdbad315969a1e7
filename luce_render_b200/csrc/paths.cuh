// Path shading for the wavefront (integrator.cu's kernels call these): starting camera
// rays and light paths, and shading one queue entry of a camera path or of a light path.
//
// The estimator is the reference's (shaders/camera.comp, shade_surface.comp,
// shade_miss.comp, light_emit.comp, light_paths.glsl, connect.glsl): one light sample and
// one BSDF sample a vertex, MIS by the power heuristic over two techniques, or three when
// light paths are traced (their camera connections weigh against both, with the
// densities the light tracer would have had). This file's own design:
//   - a queue entry is read into a PathView (the pool's path state) and, at a triangle,
//     a HitPoint (position, geometric normal on the arriving side, material);
//   - one body shades a camera path's hit whatever its surface kind -- all-diffuse
//     members (DiffuseSurface) or layered OpenPBR ones (Layers) -- through a small
//     SurfaceOps adaptor per kind; likewise one body for light paths;
//   - light choice and the light-tracing MIS ratios read the emitter table, the light
//     tree's pair records and the per-material codes, whatever the host could work out
//     before the pass having been worked out there.
#pragma once

#include "emitters.cuh"
#include "lighttree.cuh"
#include "surface.cuh"
#include "wave.cuh"

namespace lr {

// ---- geometry of a member's triangles ---------------------------------------------------

__device__ __forceinline__ float3 point_of(const Member &m, uint32_t index) {
    const float *p = m.scene.positions + (size_t)index * 3u;
    return make_float3(__ldg(p), __ldg(p + 1), __ldg(p + 2));
}

// A triangle's corners by leaf slot.
__device__ __forceinline__ void corners(const Member &m, uint32_t slot, float3 &a, float3 &b, float3 &c) {
    const uint32_t *t = m.scene.indices + (size_t)slot * 3u;
    a = point_of(m, __ldg(t));
    b = point_of(m, __ldg(t + 1));
    c = point_of(m, __ldg(t + 2));
}

// Where a ray met a triangle: the point, the unit geometric normal turned toward the side
// the ray came from, whether that is the triangle's back face, the material.
struct HitPoint {
    float3 p, g;
    uint32_t slot, material;
    bool back;
    uint4 shading;  // three octahedral normals and the material
};

__device__ __forceinline__ HitPoint hit_point(const Member &m, uint32_t slot, float3 origin, float3 dir, float t) {
    HitPoint h;
    float3 a, b, c;
    corners(m, slot, a, b, c);
    h.g = normalize(cross(b - a, c - a));
    // Triangles wind counter-clockwise seen from outside: a ray along the normal leaves.
    h.back = dot(h.g, dir) > 0.0f;
    if (h.back) h.g = -h.g;
    h.p = origin + t * dir;
    h.slot = slot;
    h.shading = __ldg(&m.scene.shading[slot]);
    h.material = h.shading.w;
    return h;
}

// The interpolated shading normal at barycentrics (u, v), on the geometric normal's side.
__device__ __forceinline__ float3 shading_normal(const HitPoint &h, float u, float v) {
    float3 n = normalize(octahedral_decode(h.shading.x) * (1.0f - u - v) + octahedral_decode(h.shading.y) * u +
                         octahedral_decode(h.shading.z) * v);
    return dot(n, h.g) < 0.0f ? -n : n;
}

// Uniform by area on triangle `slot` seen from p: direction, distance, solid-angle pdf,
// the cosine there; the triangle's emission (two-sided).
template <bool kSpectral>
__device__ __forceinline__ bool triangle_sample(const Member &m, uint32_t slot, float3 p, float2 u, float4 lambda,
                                                LightSample &s, float4 &emitted) {
    float3 a, b, c;
    corners(m, slot, a, b, c);
    const float r = sqrtf(u.x);
    const float3 q = a * (1.0f - r) + b * (r * (1.0f - u.y)) + c * (r * u.y);
    const float3 twice = cross(b - a, c - a);
    const float area = 0.5f * length(twice);
    const float3 to = q - p;
    const float d2 = dot(to, to);
    if (area <= 0.0f || d2 <= 0.0f) return false;
    s.distance = sqrtf(d2);
    s.direction = to * (1.0f / s.distance);
    const float facing = fabsf(dot(s.direction, twice)) / (2.0f * area);
    if (facing <= 0.0f) return false;
    s.pdf = d2 / (facing * area);
    s.cos_light = facing;
    s.delta = false;
    const MaterialCode &code = m.materials[__ldg(&m.scene.shading[slot]).w];
    emitted = spec_of<kSpectral>(__ldg(&code.glow_fit), xyz(__ldg(&code.glow_rgb)), lambda);
    return true;
}

// The solid-angle density triangle_sample gives the triangle met at distance t along d.
__device__ __forceinline__ float triangle_density(const Member &m, uint32_t slot, float3 d, float t) {
    float3 a, b, c;
    corners(m, slot, a, b, c);
    const float3 twice = cross(b - a, c - a);
    const float area = 0.5f * length(twice);
    const float facing = fabsf(dot(d, twice)) / fmaxf(1e-20f, 2.0f * area);
    return t * t / fmaxf(1e-20f, facing * area);
}

__device__ __forceinline__ float triangle_area(const Member &m, uint32_t slot) {
    float3 a, b, c;
    corners(m, slot, a, b, c);
    return 0.5f * length(cross(b - a, c - a));
}

// ---- the camera, seen from the scene (light tracing) ------------------------------------

__device__ __forceinline__ float3 frame_vec(const Member &m, int at) {
    return make_float3(m.frame[at], m.frame[at + 1], m.frame[at + 2]);
}

// The camera's density of a ray along d, per unit of a pixel's area on the image plane at
// unit distance (zero behind it).
__device__ __forceinline__ float camera_density(const Member &m, float3 d) {
    const float c = dot(d, make_float3(m.forward[0], m.forward[1], m.forward[2]));
    return c > 0.0f ? m.pixel_area_inv / (c * c * c) : 0.0f;
}

// A point on the lens (the pinhole when it has none).
__device__ __forceinline__ float3 lens_sample(const Member &m, float2 u) {
    const float3 eye = frame_vec(m, 0);
    if (m.lens_radius <= 0.0f) return eye;
    const float2 d = concentric(u) * m.lens_radius;
    return eye + normalize(frame_vec(m, 8)) * d.x + normalize(frame_vec(m, 12)) * d.y;
}

// The pixel through which the camera, from lens point `lens`, sees p; the unit direction
// and distance from the lens to p. False behind the camera or off the image.
__device__ __forceinline__ bool project_to_film(const Member &m, float3 p, float3 lens, uint32_t &pixel, float3 &d,
                                                float &distance) {
    const float3 offset = p - lens;
    distance = length(offset);
    d = offset * (1.0f / fmaxf(distance, 1e-20f));
    const float c = dot(d, make_float3(m.forward[0], m.forward[1], m.forward[2]));
    if (c <= 1e-6f || distance <= 0.0f) return false;
    const float3 du = frame_vec(m, 8), dv = frame_vec(m, 12);
    const float3 on_plane = m.lens_radius > 0.0f ? (lens + d * (m.focus_distance / c) - frame_vec(m, 0)) / m.focus_distance
                                                 : d / c;
    const float3 film = on_plane - frame_vec(m, 4);
    const float x = dot(film, du) / dot(du, du), y = dot(film, dv) / dot(dv, dv);
    if (!(x >= 0.0f && y >= 0.0f && x < (float)m.width && y < (float)m.height)) return false;
    pixel = (uint32_t)y * m.width + (uint32_t)x;
    return true;
}

// ---- emitters as light paths start from them --------------------------------------------

// A light path's emitter code for one leaving a light from afar.
constexpr uint32_t kAfarEmitter = 0x40000000u;

__device__ __forceinline__ bool triangle_emitter(uint32_t code) { return (code & kEmitterTriangle) != 0u; }

// The area density light emission gives a point on tree emitter `e`, its choice by power
// (the share light paths from afar leave to the tree) included.
__device__ __forceinline__ float emitter_area_density(const Member &m, uint32_t e) {
    const uint32_t code = emitter_code(m.tree, e);
    const float area = triangle_emitter(code) ? triangle_area(m, code & ~kEmitterTriangle) : light_area(m.lights.light[code]);
    if (!(area > 0.0f)) return 0.0f;
    return (1.0f - m.k->emit_share) * tree_chance_of<true>(m.tree, e, make_float3(0, 0, 0), make_float3(0, 0, 0)) / area;
}

// The density of a light path leaving emitter `e` at cosine c (cosine-weighted; over both
// hemispheres for an emissive triangle).
__device__ __forceinline__ float emitter_direction_density(const Member &m, uint32_t e, float c) {
    return fabsf(c) / (triangle_emitter(emitter_code(m.tree, e)) ? 2.0f * kPi : kPi);
}

// The chance a light path leaves light `light` from afar along -w (w toward the light).
__device__ __forceinline__ float afar_leave_density(const Member &m, uint32_t light, float3 w) {
    return m.k->emit_share * afar_share(m.lights.light[light]) *
           light_density(m.lights, light, make_float3(0.0f, 0.0f, 0.0f), w, kInfinity);
}

// The area density of a path from afar's first surface p (|cosine| c to w): uniform over
// the disk it started on, zero outside the disk's shadow.
__device__ __forceinline__ float afar_arrival_density(const Constants &k, float3 p, float3 w, float c) {
    const float3 offset = p - k.emit_center;
    const float3 across = offset - w * dot(offset, w);
    if (dot(across, across) > k.emit_radius * k.emit_radius) return 0.0f;
    return c / (kPi * k.emit_radius * k.emit_radius);
}

// At a tree emitter a camera path's BSDF ray found: the light tracer's density of that
// path over the camera's.
__device__ __forceinline__ float tracer_over_camera(const Member &m, float4 mis, uint32_t e, float cos_light, float d,
                                                    float bsdf_pdf) {
    if (e == kNone || mis.y <= 0.0f || bsdf_pdf <= 0.0f) return 0.0f;
    const float d2 = d * d;
    const float at_vertex = emitter_direction_density(m, e, cos_light) * mis.z / d2 / mis.y;
    const float at_light = emitter_area_density(m, e) / (bsdf_pdf * fabsf(cos_light) / d2);
    return mis.x * at_vertex * at_light;
}

// ---- light choice for a light sample ----------------------------------------------------

struct LightPick {
    LightSample s;
    float4 emitted;
    float chance = 0.0f;       // of the choice (0: none was made)
    uint32_t emitter = kNone;  // the tree's emitter chosen
    uint32_t afar = kNone;     // or the light from afar
};

// One light sample from p (from: p lifted off the surface, where the tree weighs; n: the
// shading normal): a light from afar by power with chance p_distant, else a tree emitter
// by importance.
template <bool kSpectral>
__device__ __forceinline__ LightPick pick_light(const Member &m, float4 u, float3 p, float3 from, float3 n, float4 lambda) {
    LightPick out;
    const float p_distant = m.k->p_distant;
    const float2 uv = make_float2(u.y, u.z);
    if (u.x < p_distant) {
        float share;
        const uint32_t light = choose_afar(m.lights, u.x / p_distant, share);
        if (light == kNone || !(share > 0.0f) || !light_sample(m.lights, light, p, uv, out.s)) return out;
        out.afar = light;
        out.emitted = shape_of(m.lights.light[light]) == kShapeDome
                          ? dome_emission<kSpectral>(m.lights, light, out.s.direction, lambda)
                          : light_emission<kSpectral>(m.lights.light[light], lambda);
        out.chance = p_distant * share;
        return out;
    }
    uint32_t e;
    float tree_chance;
    if (!tree_choose<false>(m.tree, (u.x - p_distant) / fmaxf(1e-7f, 1.0f - p_distant), from, n, e, tree_chance)) return out;
    out.emitter = e;
    const uint32_t code = emitter_code(m.tree, e);
    bool ok;
    if (triangle_emitter(code)) {
        ok = triangle_sample<kSpectral>(m, code & ~kEmitterTriangle, p, uv, lambda, out.s, out.emitted);
    } else {
        ok = light_sample(m.lights, code, p, uv, out.s);
        if (ok) out.emitted = light_emission<kSpectral>(m.lights.light[code], lambda);
    }
    if (ok) out.chance = (1.0f - p_distant) * tree_chance;
    return out;
}

// ---- shading outputs --------------------------------------------------------------------

// What shading a queue entry hands back: the path's next ray and a shadow ray (or a
// camera connection), either or both.
struct ShadeOut {
    bool next = false, shadow = false;
    float4 o, d, so, sd, sc;
};

__device__ __forceinline__ void continue_ray(ShadeOut &out, float3 o, float3 d, float tag_bits) {
    out.next = true;
    out.o = make_float4(o.x, o.y, o.z, tag_bits);
    out.d = make_float4(d.x, d.y, d.z, kInfinity);
}

// Indirect light held to the clamp: its largest lane at most `limit`, its colour kept.
template <bool kSpectral>
__device__ __forceinline__ float4 held(float4 c, uint32_t total, float limit) {
    if (total == 0u || limit <= 0.0f) return c;
    const float top = spec_max<kSpectral>(c);
    return top > limit ? c * (limit / top) : c;
}

__device__ __forceinline__ float lift(float3 p) { return 4e-4f * fmaxf(1.0f, fmaxf(fabsf(p.x), fmaxf(fabsf(p.y), fabsf(p.z)))); }

// Cut-out opacity: the ray passes through at the same bounce with probability
// 1 - opacity (the bounce's opacity number u, decorrelated by the hit distance).
__device__ __forceinline__ bool cut_through(const MaterialCode *codes, uint32_t material, float t, float u) {
    const float opacity = clamp01(__ldg(&codes[material].extra).x);
    if (!(opacity < 1.0f)) return false;
    const float v = u + (float)hash_u32(__float_as_uint(t)) * (1.0f / 4294967296.0f);
    return v - floorf(v) >= opacity;
}

// The path state a queue entry's path holds in the pool.
struct PathView {
    uint32_t path, tag;
    uint4 words;  // pixel (light paths: emitter), bounces, previous normal, ray pdf bits
    float4 throughput, lambda, vertex, mis;
    __device__ __forceinline__ uint32_t bounces() const { return words.y; }
    __device__ __forceinline__ uint32_t total() const { return words.y & 0xffu; }
    __device__ __forceinline__ float ray_pdf() const { return __uint_as_float(words.w); }
};

// ---- surface adaptors: what differs between all-diffuse and layered members ------------

struct DiffuseOps {
    static constexpr bool kLayered = false;
    DiffuseSurface s;
    float3 g;

    template <bool kSpectral>
    __device__ __forceinline__ void open(const Member &m, const HitPoint &h, float3 n, float3 dir, float4 lambda,
                                         float3 &wo) {
        s = diffuse_at<kSpectral>(n, m.materials[h.material], lambda);
        g = h.g;
        wo = s.local(-dir);
    }
    // f and the BSDF density toward a light sample; false when the sample is rejected.
    __device__ __forceinline__ bool toward_light(float3 wi, float3 wo, float side, float4 &f, float &pdf) const {
        if (!(side > 0.0f && wi.z > 0.0f && wo.z > 0.0f)) return false;
        pdf = s.chance * wi.z / kPi;
        if (!(pdf > 0.0f)) return false;
        f = eon(s.albedo, s.roughness, wi, wo);
        return true;
    }
    __device__ __forceinline__ bool sample(float3 wo, float4 u, float3 &wi, float4 &weight, float &pdf, uint32_t &lobe) const {
        if (wo.z <= 0.0f || !(u.w < s.chance)) return false;
        const float2 d = concentric(make_float2(u.x, u.y));
        wi = make_float3(d.x, d.y, sqrtf(fmaxf(0.0f, 1.0f - (d.x * d.x + d.y * d.y))));
        if (wi.z == 0.0f) return false;
        pdf = s.chance * wi.z / kPi;
        if (!(pdf > 0.0f)) return false;
        weight = eon(s.albedo, s.roughness, wi, wo) * (fabsf(wi.z) / pdf);
        lobe = kLobeDiffuse;
        return true;
    }
    __device__ __forceinline__ float light_sampler_pdf(const Member &, float3 from, float3 to, float) const {
        return diffuse_light_pdf(s.chance, s.n, g, from, to);
    }
};

struct LayeredOps {
    static constexpr bool kLayered = true;
    Layers s;

    template <bool kSpectral>
    __device__ __forceinline__ void open(const Member &m, const HitPoint &h, float3 n, float3 dir, float4 lambda,
                                         float3 &wo) {
        s = layers_at<kSpectral>(n, h.g, h.material, h.back, m.materials, -dir, lambda, wo);
    }
    __device__ __forceinline__ bool toward_light(float3 wi, float3 wo, float side, float4 &f, float &pdf) const {
        if (!((side > 0.0f) == (wi.z > 0.0f) && (side > 0.0f || s.p_trans > 0.0f))) return false;
        f = layers_f(s, wi, wo, pdf);
        return pdf > 0.0f;
    }
    __device__ __forceinline__ bool sample(float3 wo, float4 u, float3 &wi, float4 &weight, float &pdf, uint32_t &lobe) const {
        if (!layers_sample(s, wo, make_float3(u.x, u.y, u.w), wi, pdf, lobe)) return false;
        float again;
        weight = layers_f(s, wi, wo, again) * (fabsf(wi.z) / pdf);
        return true;
    }
    __device__ __forceinline__ float light_sampler_pdf(const Member &m, float3 from, float3 to, float hero) const {
        return layers_light_pdf(s, from, to, m.materials, hero);
    }
};

// ---- a camera path's queue entry --------------------------------------------------------

// A miss: the background and every light from afar the ray sees, each weighed against
// the light sample that could have found it (and, for a layered member tracing light
// paths, against light paths from afar).
template <bool kSpectral, bool kAfarTraced>
__device__ __forceinline__ float4 sky_radiance(const Member &m, const PathView &v, float3 dir, bool tracing) {
    const Constants &k = *m.k;
    const uint32_t total = v.total();
    const float ray_pdf = v.ray_pdf();
    float4 sum = spec_of<kSpectral>(k.background_fit, k.background_rgb, v.lambda);
    const LightTable &T = m.lights;
    for (uint32_t a = 0; a < T.afar_count; a++) {
        const uint32_t light = __ldg(&T.afar[a]);
        const DeviceLight &l = T.light[light];
        const bool dome = shape_of(l) == kShapeDome;
        if (!dome && !distant_covers(l, dir)) continue;
        float weight = 1.0f;
        if (total == 0u) {
            if (!(light_flags(l) & kLightSeen)) continue;
        } else if (ray_pdf > 0.0f) {
            float traced = 0.0f;
            if (kAfarTraced && tracing && emits_from_afar(T, light) && v.mis.y > 0.0f)
                traced = v.mis.x * (afar_arrival_density(k, xyz(v.vertex), dir, v.mis.z) / v.mis.y) *
                         (afar_leave_density(m, light, dir) / ray_pdf);
            const float by_light = light_density(T, light, make_float3(0.0f, 0.0f, 0.0f), dir, kInfinity) *
                                   (k.p_distant * afar_share(l)) / ray_pdf;
            weight = mis_weight(by_light, traced);
        }
        sum = sum + (dome ? dome_emission<kSpectral>(T, light, dir, v.lambda) : light_emission<kSpectral>(l, v.lambda)) *
                        weight;
    }
    return held<kSpectral>(v.throughput * sum, total, k.clamp_indirect);
}

// A camera path's queue entry of member m: a miss, a finite light, or a surface -- its
// emission, one light sample (a shadow ray in `out`) and one BSDF sample (the next ray).
template <bool kSpectral, bool kTracing, class Ops>
__device__ __forceinline__ void shade_camera_path(const Wave &w, const Member &m, uint32_t sample, uint32_t round,
                                                  uint32_t i, float4 ro, ShadeOut &out) {
    const Constants &k = *m.k;
    const uint32_t q = round & 1u;
    const float4 rd = w.ray_d[q][i], hit = w.hits[q][i];
    PathView v;
    v.tag = __float_as_uint(ro.w);
    v.path = v.tag & kPathMask;
    v.words = w.path[v.path];
    const uint32_t pixel = v.words.x;
    if (pixel == kNone) return;  // a converged pixel's (adaptive sampling)
    const uint32_t total = v.total();
    const float ray_pdf = v.ray_pdf();
    const float3 origin = xyz(ro), dir = xyz(rd);
    v.throughput = w.throughput[v.path];
    v.lambda = kSpectral ? w.lambda[v.path] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    const bool tracing = kTracing && m.light_paths != 0u;
    v.mis = tracing ? w.mis[v.path] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    float4 radiance = w.radiance[v.path];
    const uint32_t what = __float_as_uint(hit.y);

    if (what == kNone) {
        if (Ops::kLayered) v.vertex = w.vertex[v.path];
        w.radiance[v.path] = radiance + sky_radiance<kSpectral, Ops::kLayered>(m, v, dir, tracing);
        return;
    }
    v.vertex = w.vertex[v.path];
    const float3 last = xyz(v.vertex);
    if (what & kLightHit) {
        // A finite light, weighed against the light sample the last vertex took.
        const uint32_t light = what & ~kLightHit;
        const DeviceLight &l = m.lights.light[light];
        float weight = 1.0f;
        if (total == 0u) {
            if (!(light_flags(l) & kLightSeen)) return;
        } else if (ray_pdf > 0.0f) {
            const uint32_t e = __float_as_uint(__ldg(&l.pick).w);
            const float reach = length(last - (origin + hit.x * dir));
            const float chance = (1.0f - k.p_distant) * tree_chance_of<false>(m.tree, e, last, octahedral_decode(v.words.z));
            const float traced = tracing ? tracer_over_camera(m, v.mis, e, light_cosine(m.lights, light, last, dir, reach),
                                                              reach, ray_pdf)
                                         : 0.0f;
            weight = mis_weight(light_density(m.lights, light, last, dir, reach) * chance / ray_pdf, traced);
        }
        w.radiance[v.path] = radiance + held<kSpectral>(v.throughput * light_emission<kSpectral>(l, v.lambda) * weight,
                                                        total, k.clamp_indirect);
        return;
    }

    const HitPoint h = hit_point(m, what, origin, dir, hit.x);
    const float reach = length(last - h.p);
    // The camera's area density of this vertex, and what turns the light sampler's pdf
    // here toward the last vertex into that vertex's area density.
    const float density = (total == 0u ? v.mis.w : ray_pdf) * fabsf(dot(dir, h.g)) / (reach * reach);
    const float back_reach = v.mis.z / (reach * reach);
    if (m.cutouts && cut_through(m.materials, h.material, hit.x, sample4(k.seed, pixel, sample, group_opacity(total)).x)) {
        continue_ray(out, offset_origin(h.p, -h.g), dir, ro.w);
        return;
    }
    const MaterialCode &code = m.materials[h.material];
    if (kSpectral && Ops::kLayered && __ldg(&code.extra).y != 0.0f && v.lambda.y >= 0.0f) {
        // A dispersive material: its directions depend on the wavelength, so the three
        // secondary wavelengths end and the hero carries the sample.
        v.throughput = make_float4(v.throughput.x * 4.0f, 0.0f, 0.0f, 0.0f);
        radiance = make_float4(radiance.x * 4.0f, 0.0f, 0.0f, 0.0f);
        v.lambda = make_float4(v.lambda.x, -v.lambda.y, -v.lambda.z, -v.lambda.w);
        w.lambda[v.path] = v.lambda;
    }
    const float hero = kSpectral && v.lambda.y < 0.0f ? v.lambda.x : 0.0f;

    const float4 glow = __ldg(&code.glow_rgb);
    if (glow.w > 0.0f) {
        // Emission, weighed against the light sample the last vertex took.
        float weight = 1.0f;
        const uint32_t e = m.tree.triangle_map ? __ldg(&m.tree.triangle_map[h.slot]) : kNone;
        if (total > 0u && ray_pdf > 0.0f && e != kNone) {
            const float chance = (1.0f - k.p_distant) * tree_chance_of<false>(m.tree, e, last, octahedral_decode(v.words.z));
            const float traced = tracing ? tracer_over_camera(m, v.mis, e, fabsf(dot(dir, h.g)), reach, ray_pdf) : 0.0f;
            weight = mis_weight(triangle_density(m, h.slot, dir, reach) * chance / ray_pdf, traced);
        }
        radiance = radiance + held<kSpectral>(v.throughput * spec_of<kSpectral>(__ldg(&code.glow_fit), xyz(glow), v.lambda) *
                                                  weight,
                                              total, k.clamp_indirect);
    }
    if (total >= k.max_bounces) {  // past the limit: the ray here still counted its lights
        w.radiance[v.path] = radiance;
        return;
    }
    const float3 n = shading_normal(h, hit.z, hit.w);
    Ops ops;
    float3 wo;
    ops.template open<kSpectral>(m, h, n, dir, v.lambda, wo);
    const float3 from = offset_origin(h.p, h.g);

    // One light sample.
    const LightPick pick =
        pick_light<kSpectral>(m, sample4(k.seed, pixel, sample, group_light(total)), h.p, from, n, v.lambda);
    if (pick.chance > 0.0f) {
        const LightSample &s = pick.s;
        const float side = dot(s.direction, h.g);
        const float3 wi = ops.s.local(s.direction);
        float4 f;
        float bsdf_pdf;
        if (ops.toward_light(wi, wo, side, f, bsdf_pdf)) {
            const float light_pdf = s.pdf * pick.chance;
            // The light tracer's density of this path over the camera path's BSDF ray to
            // the same light point (three-technique MIS).
            float traced = 0.0f;
            if (tracing && density > 0.0f) {
                const bool tree_point = !s.delta && pick.emitter != kNone;
                const bool afar_point = Ops::kLayered && pick.afar != kNone && emits_from_afar(m.lights, pick.afar);
                if (tree_point || afar_point) {
                    const float at_last = total == 0u ? 1.0f
                                                      : ops.light_sampler_pdf(m, s.direction, -dir, hero) * back_reach /
                                                            v.mis.y;
                    if (tree_point) {
                        const float d2 = s.distance * s.distance;
                        const float at_vertex =
                            emitter_direction_density(m, pick.emitter, s.cos_light) * fabsf(side) / d2 / density;
                        const float at_light = emitter_area_density(m, pick.emitter) / (bsdf_pdf * s.cos_light / d2);
                        traced = v.mis.x * at_last * at_vertex * at_light;
                    }
                    if (afar_point) {
                        const float at_vertex = afar_arrival_density(k, h.p, s.direction, fabsf(side)) / density;
                        const float at_light = afar_leave_density(m, pick.afar, s.direction) / bsdf_pdf;
                        traced = v.mis.x * at_last * at_vertex * at_light;
                    }
                }
            }
            const float weight = s.delta ? 1.0f : mis_weight(bsdf_pdf / light_pdf, traced * bsdf_pdf / light_pdf);
            const float4 c = held<kSpectral>(v.throughput * f * pick.emitted * (fabsf(wi.z) * (weight / light_pdf)), total,
                                             k.clamp_indirect);
            // Stop short of the light by the lift origins leave surfaces, so a shadow ray
            // to an emissive triangle does not find the triangle itself.
            const float shadow_reach =
                s.distance >= kInfinity ? kInfinity : fmaxf(0.0f, s.distance - lift(h.p + s.direction * s.distance));
            const float3 so = offset_origin(h.p, side > 0.0f ? h.g : -h.g);
            out.shadow = true;
            out.so = make_float4(so.x, so.y, so.z, ro.w);
            out.sd = make_float4(s.direction.x, s.direction.y, s.direction.z, shadow_reach);
            out.sc = c;
        }
    }
    w.radiance[v.path] = radiance;

    // One BSDF sample: the path goes on (u.xy the direction, u.w the lobe, u.z roulette).
    const float4 u = sample4(k.seed, pixel, sample, group_bsdf(total));
    float3 wi;
    float4 weight;
    float pdf;
    uint32_t lobe;
    if (!ops.sample(wo, u, wi, weight, pdf, lobe)) return;
    const float3 direction = ops.s.world(wi);
    // A shading normal can send a ray to the wrong side of the true surface.
    const float side = dot(direction, h.g);
    if ((side > 0.0f) != (wi.z > 0.0f)) return;
    const uint32_t next_bounces = next_bounce(v.bounces(), lobe, k.limits);
    if (next_bounces == kNone) return;
    float4 throughput = v.throughput * weight;
    const float scale = fminf(v.vertex.w, 1e6f);
    if (total + 1u >= 3u) {  // Russian roulette, relative to the path's start
        const float survive = fminf(0.95f, spec_max<kSpectral>(throughput) * scale);
        if (u.z >= survive) return;
        throughput = make_float4(throughput.x / survive, throughput.y / survive, throughput.z / survive,
                                 throughput.w / survive);
    }
    const float3 next = side > 0.0f ? from : offset_origin(h.p, -h.g);
    if (tracing) {
        const float at_last = total == 0u ? 1.0f : ops.light_sampler_pdf(m, direction, -dir, hero) * back_reach / v.mis.y;
        w.mis[v.path] = make_float4(v.mis.x * at_last, density, fabsf(side), 0.0f);
    }
    w.path[v.path] = make_uint4(pixel, next_bounces, octahedral_encode(n), __float_as_uint(pdf));
    w.throughput[v.path] = throughput;
    w.vertex[v.path] = make_float4(next.x, next.y, next.z, scale);
    continue_ray(out, next, direction, ro.w);
}

// ---- a light path's queue entry ---------------------------------------------------------

// The light sample a camera path at p (the surface seen from the camera's side: normal
// sn, geometric sg) would take toward the light path's first point x0 (or, for a path
// from afar, toward its light's direction `toward`), over its BSDF density toward it.
__device__ __forceinline__ float first_vertex_ratio(const Member &m, uint32_t e, float3 sn, float3 sg, float3 p, float3 x0,
                                                    float3 toward, float bsdf_pdf) {
    if (!(bsdf_pdf > 0.0f)) return 0.0f;
    const Constants &k = *m.k;
    if (e & kAfarEmitter) {
        const uint32_t light = e & ~kAfarEmitter;
        return k.p_distant * afar_share(m.lights.light[light]) *
               light_density(m.lights, light, offset_origin(p, sg), toward, kInfinity) / bsdf_pdf;
    }
    const float3 from = offset_origin(p, sg);
    const float3 offset = x0 - from;
    const float d = length(offset);
    const float3 dir = offset / d;
    const float chance = (1.0f - k.p_distant) * tree_chance_of<false>(m.tree, e, from, sn);
    const uint32_t code = emitter_code(m.tree, e);
    const float pdf = triangle_emitter(code) ? triangle_density(m, code & ~kEmitterTriangle, dir, d)
                                             : light_density(m.lights, code, from, dir, d);
    return chance * pdf / bsdf_pdf;
}

// The surface a light path meets, seen from either side: the diffuse kind.
struct DiffuseLightOps {
    static constexpr bool kLayered = false;
    float4 albedo;
    float roughness, chance;
    float3 n, g;

    template <bool kSpectral>
    __device__ __forceinline__ void open(const Member &m, const HitPoint &h, float3 shading, float4 lambda) {
        const DiffuseSurface d = diffuse_at<kSpectral>(shading, m.materials[h.material], lambda);
        albedo = d.albedo;
        roughness = d.roughness;
        chance = d.chance;
        n = shading;
        g = h.g;
    }
    // f and the camera's BSDF density at the surface seen from `out` (the camera side)
    // with light arriving from `in`; false when the camera's sampler rejects it.
    template <bool kSpectral>
    __device__ __forceinline__ bool camera_view(const Member &, float3 out, float3 in, float4, float4 &f, float &pdf,
                                                float3 &sn, float3 &sg, bool strict) const {
        const float side = dot(out, g);
        sn = side > 0.0f ? n : -n;
        sg = side > 0.0f ? g : -g;
        float3 t, b;
        basis(sn, t, b);
        const float3 wo = make_float3(dot(out, t), dot(out, b), dot(out, sn));
        const float3 wi = make_float3(dot(in, t), dot(in, b), dot(in, sn));
        if ((dot(in, sg) > 0.0f) != (wi.z > 0.0f)) return false;
        const bool lobe = wo.z > 0.0f && wi.z > 0.0f;
        if (strict && !lobe) return false;
        pdf = lobe ? chance * wi.z / kPi : 0.0f;
        f = lobe ? eon(albedo, roughness, wi, wo) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        return true;
    }
    __device__ __forceinline__ bool scatter(float3 toward_light, float4 u, float3 &direction, float &pdf, uint32_t &lobe) const {
        if (dot(toward_light, n) <= 0.0f || !(u.w < chance)) return false;
        const float2 d = concentric(make_float2(u.x, u.y));
        const float3 wl = make_float3(d.x, d.y, sqrtf(fmaxf(0.0f, 1.0f - (d.x * d.x + d.y * d.y))));
        if (wl.z == 0.0f) return false;
        pdf = chance * wl.z / kPi;
        if (!(pdf > 0.0f)) return false;
        float3 t, b;
        basis(n, t, b);
        direction = t * wl.x + b * wl.y + n * wl.z;
        lobe = kLobeDiffuse;
        return (dot(direction, g) > 0.0f) == (wl.z > 0.0f);
    }
};

// The layered kind: the surface opened once on the side light arrives from (`lit`);
// the camera's view evaluates it oriented toward the camera, or opened again on the other
// side.
struct LayeredLightOps {
    static constexpr bool kLayered = true;
    Layers lit;
    float hero;

    template <bool kSpectral>
    __device__ __forceinline__ void open(const Member &m, const HitPoint &h, float3 shading, float4 lambda) {
        lit.n = shading;
        basis(shading, lit.t, lit.b);
        lit.g = h.g;
        lit.material = h.material;
        lit.back = h.back;
        hero = kSpectral && lambda.y < 0.0f ? lambda.x : 0.0f;
        open_layers(lit, m.materials[h.material], hero);
        colour_layers<kSpectral>(lit, m.materials[h.material], lambda);
    }
    template <bool kSpectral>
    __device__ __forceinline__ bool camera_view(const Member &m, float3 out, float3 in, float4 lambda, float4 &f,
                                                float &pdf, float3 &sn, float3 &sg, bool strict) const {
        const bool same = dot(out, lit.g) > 0.0f;
        Layers seen = lit;
        if (!same) {
            seen.n = -lit.n;
            seen.g = -lit.g;
            basis(seen.n, seen.t, seen.b);
            seen.back = !lit.back;
            open_layers(seen, m.materials[lit.material], hero);
            colour_layers<kSpectral>(seen, m.materials[lit.material], lambda);
        }
        const float3 wo = seen.local(out), wi = seen.local(in);
        if ((dot(in, seen.g) > 0.0f) != (wi.z > 0.0f)) return false;
        if (strict && !(wo.z > 0.0f)) return false;
        view_layers(seen, wo);
        coat_filter(seen);
        f = layers_f(seen, wi, wo, pdf);
        sn = seen.n;
        sg = seen.g;
        return true;
    }
    __device__ __forceinline__ bool scatter(float3 toward_light, float4 u, float3 &direction, float &pdf, uint32_t &lobe) const {
        Layers choosing = lit;
        light_path_lobes(choosing);
        float3 wl;
        if (!layers_sample(choosing, lit.local(toward_light), make_float3(u.x, u.y, u.w), wl, pdf, lobe)) return false;
        direction = lit.world(wl);
        return (dot(direction, lit.g) > 0.0f) == (wl.z > 0.0f);
    }
};

// A light path's queue entry of member m: at a surface it connects to the camera -- a
// shadow ray carrying, MIS-weighted and in the film's terms, what the camera sees of it
// through the pixel it projects to -- and scatters on, weighed by the BSDF as a camera
// arriving along the new direction evaluates it (with light paths' shading-normal
// correction). Lights and misses end it.
template <bool kSpectral, class Ops>
__device__ __forceinline__ void shade_light_path(const Wave &w, const Member &m, uint32_t sample, uint32_t round,
                                                 uint32_t i, float4 ro, ShadeOut &out) {
    const Constants &k = *m.k;
    const uint32_t q = round & 1u;
    const float4 hit = w.hits[q][i];
    const uint32_t what = __float_as_uint(hit.y);
    if (what == kNone || (what & kLightHit)) return;
    const float4 rd = w.ray_d[q][i];
    PathView v;
    v.tag = __float_as_uint(ro.w);
    v.path = v.tag & kPathMask;
    v.words = w.path[v.path];
    const uint32_t e = v.words.x, total = v.total();
    const float ray_pdf = v.ray_pdf();
    const float3 origin = xyz(ro), dir = xyz(rd);
    v.throughput = w.throughput[v.path];
    v.lambda = kSpectral ? w.lambda[v.path] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    v.vertex = w.vertex[v.path];
    v.mis = w.mis[v.path];
    const uint32_t id = 0x80000000u | (m.light_band + tag_light_index(w, v.tag));

    const HitPoint h = hit_point(m, what, origin, dir, hit.x);
    if (m.cutouts && cut_through(m.materials, h.material, hit.x, sample4(k.seed, id, sample, group_opacity(total)).x)) {
        continue_ray(out, offset_origin(h.p, -h.g), dir, ro.w);
        return;
    }
    if (total >= k.max_bounces) return;
    if (kSpectral && Ops::kLayered && __ldg(&m.materials[h.material].extra).y != 0.0f && v.lambda.y >= 0.0f) {
        v.throughput = make_float4(v.throughput.x * 4.0f, 0.0f, 0.0f, 0.0f);
        v.lambda = make_float4(v.lambda.x, -v.lambda.y, -v.lambda.z, -v.lambda.w);
        w.lambda[v.path] = v.lambda;
    }
    const float3 n = shading_normal(h, hit.z, hit.w);
    const float4 u_lens = sample4(k.seed, id, sample, group_light(total));
    uint32_t pixel = 0;
    float3 to_point;
    float camera_distance;
    const bool on_film = project_to_film(m, h.p, lens_sample(m, make_float2(u_lens.x, u_lens.y)), pixel, to_point,
                                         camera_distance);
    Ops ops;
    ops.template open<kSpectral>(m, h, n, v.lambda);
    const float3 toward_light = -dir;
    const float3 x_last = xyz(v.vertex);
    const float reach = length(x_last - h.p);
    const float cos_in = fabsf(dot(dir, h.g));
    float density = ray_pdf * cos_in / (reach * reach);
    float back_reach = v.mis.z / (reach * reach);
    if (Ops::kLayered && total == 0u && (e & kAfarEmitter)) {
        // A path from afar's first surface: its density on the disk's shadow; the light's
        // "point" is a direction (no distance to convert).
        density = afar_arrival_density(k, h.p, -dir, cos_in);
        back_reach = 1.0f;
        if (!(density > 0.0f)) return;
    }
    const float cos_shading_in = dot(toward_light, n);
    if (cos_shading_in <= 0.0f || cos_in < 1e-6f) return;
    const float shading_in = cos_shading_in / cos_in;
    const float paths = (float)m.light_paths;

    if (on_film) {
        const float3 to_camera = -to_point;
        float4 f;
        float camera_pdf;
        float3 sn, sg;
        if (ops.template camera_view<kSpectral>(m, to_camera, toward_light, v.lambda, f, camera_pdf, sn, sg, true)) {
            const float film_density = camera_density(m, to_point) * fabsf(dot(to_camera, h.g)) /
                                       (camera_distance * camera_distance);
            const float4 c = v.throughput * f * (shading_in * film_density / paths);
            if (spec_max<kSpectral>(c) > 0.0f) {
                // The camera techniques' densities over this one's.
                const float last = v.mis.y > 0.0f ? camera_pdf * back_reach / v.mis.y : 0.0f;
                const float ratio = v.mis.x * last * film_density / density;
                const float sample_ratio = total == 0u ? first_vertex_ratio(m, e, sn, sg, h.p, x_last, toward_light, camera_pdf)
                                                       : fmaxf(v.mis.w, 0.0f);
                const float weight = mis_weight(ratio / paths, ratio * sample_ratio / paths);
                const float3 so = offset_origin(h.p, sg);
                const float3 value = spec_to_film<kSpectral>(c * weight, v.lambda, k);
                out.shadow = true;
                out.so = make_float4(so.x, so.y, so.z, ro.w);
                out.sd = make_float4(to_camera.x, to_camera.y, to_camera.z, fmaxf(0.0f, camera_distance - lift(h.p)));
                out.sc = make_float4(value.x, value.y, value.z, __uint_as_float(pixel));
            }
        }
    }

    // Scatter on, unless the next vertex would be past the bounce limit.
    if (total + 1u >= k.max_bounces) return;
    const float4 u = sample4(k.seed, id, sample, group_bsdf(total));
    float3 direction;
    float light_pdf;
    uint32_t lobe;
    if (!ops.scatter(toward_light, u, direction, light_pdf, lobe)) return;
    const float side = dot(direction, h.g);
    float4 f;
    float camera_pdf;
    float3 sn, sg;
    if (!ops.template camera_view<kSpectral>(m, direction, toward_light, v.lambda, f, camera_pdf, sn, sg, false)) return;
    const uint32_t next_bounces = next_bounce(v.bounces(), lobe, k.limits);
    if (next_bounces == kNone) return;
    float4 throughput = v.throughput * f * (shading_in * fabsf(side) / light_pdf);
    const float scale = v.vertex.w;
    if (total + 1u >= 3u) {
        const float survive = fminf(0.95f, spec_max<kSpectral>(throughput) * scale);
        if (u.z >= survive) return;
        throughput = make_float4(throughput.x / survive, throughput.y / survive, throughput.z / survive,
                                 throughput.w / survive);
    }
    if (!(spec_max<kSpectral>(throughput) > 0.0f)) return;
    const float last = v.mis.y > 0.0f ? camera_pdf * back_reach / v.mis.y : 0.0f;
    const float sample_ratio =
        total == 0u ? first_vertex_ratio(m, e, sn, sg, h.p, x_last, toward_light, camera_pdf) : v.mis.w;
    const float3 next = offset_origin(h.p, side > 0.0f ? h.g : -h.g);
    w.path[v.path] = make_uint4(e, next_bounces, 0u, __float_as_uint(light_pdf));
    w.throughput[v.path] = throughput;
    w.vertex[v.path] = make_float4(h.p.x, h.p.y, h.p.z, scale);
    w.mis[v.path] = make_float4(v.mis.x * last, density, fabsf(side), sample_ratio);
    continue_ray(out, next, direction, ro.w);
}

// ---- starting paths ---------------------------------------------------------------------

// Pool path `path` of camera segment `si` (slot: its ray's place in the queue): a
// jittered ray through its pixel (pinhole, orthographic or thin lens), its wavelengths,
// and the camera's density for light tracing's MIS. A converged pixel (adaptive
// sampling) starts none: its ray reaches nothing and its shading ends at once.
__device__ __forceinline__ void start_camera_path(const Wave &w, const Member &m, const Segment &sg, uint32_t si,
                                                  uint32_t path, uint32_t slot) {
    const uint32_t pixel = sg.first_pixel + (path - sg.path_base);
    const float tag = __uint_as_float(path | (si << kPathBits));
    if (m.half && m.half[pixel].w > 0.5f) {
        w.path[path] = make_uint4(kNone, 0u, 0u, 0u);
        w.ray_o[0][slot] = make_float4(0.0f, 0.0f, 0.0f, tag);
        w.ray_d[0][slot] = make_float4(0.0f, 0.0f, 1.0f, 0.0f);
        return;
    }
    const uint32_t seed = m.k->seed;
    const float3 eye = frame_vec(m, 0), du = frame_vec(m, 8), dv = frame_vec(m, 12);
    const bool ortho = m.frame[3] > 0.5f;
    const float4 u = sample4(seed, pixel, sg.sample, kGroupCamera);
    const float3 film = frame_vec(m, 4) + ((float)(pixel % m.width) + u.x) * du + ((float)(pixel / m.width) + u.y) * dv;
    float3 origin = ortho ? eye + film : eye;
    float3 direction = normalize(ortho ? cross(du, dv) : film);
    if (!ortho && m.lens_radius > 0.0f) {
        // Thin lens: through the point on the focal plane the pinhole ray meets.
        const float3 focus = eye + direction * (m.focus_distance /
                                                dot(direction, make_float3(m.forward[0], m.forward[1], m.forward[2])));
        const float2 d = concentric(make_float2(u.z, u.w));
        origin = eye + normalize(du) * (d.x * m.lens_radius) + normalize(dv) * (d.y * m.lens_radius);
        direction = normalize(focus - origin);
    }
    w.path[path] = make_uint4(pixel, 0u, 0u, 0u);
    w.throughput[path] = make_float4(1.0f, 1.0f, 1.0f, 1.0f);
    w.radiance[path] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    w.vertex[path] = make_float4(origin.x, origin.y, origin.z, 1.0f);
    if (m.spectral) w.lambda[path] = sample_wavelengths(sample4(seed, pixel, sg.sample, kGroupWavelength).x);
    if (m.light_paths) w.mis[path] = make_float4((float)m.light_paths, 0.0f, 0.0f, camera_density(m, direction));
    w.ray_o[0][slot] = make_float4(origin.x, origin.y, origin.z, tag);
    w.ray_d[0][slot] = make_float4(direction.x, direction.y, direction.z, kInfinity);
}

// Light path `path` of light segment `si`, numbered for the sampler 0x80000000 | (band +
// its index): from a light from afar (by its share of light paths) on a disk facing it
// about the casters' centre, or from a tree emitter chosen by power -- a point on it
// uniform by area and a cosine-weighted direction (either side of an emissive triangle).
// A path that cannot start gets a ray that reaches nothing.
template <bool kSpectral>
__device__ __forceinline__ void start_light_path(const Wave &w, const Member &m, const Segment &sg, uint32_t si,
                                                 uint32_t path, uint32_t slot) {
    const Constants &k = *m.k;
    const uint32_t id = 0x80000000u | (m.light_band + sg.first_pixel + (path - sg.path_base));
    const float4 u_point = sample4(k.seed, id, sg.sample, kGroupCamera);
    const float4 u_pick = sample4(k.seed, id, sg.sample, kGroupWavelength);
    const float4 lambda = kSpectral ? sample_wavelengths(u_pick.x) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    const float tag = __uint_as_float(path | (si << kPathBits));
    auto launch = [&](uint4 words, float4 throughput, float3 at, float scale, float4 mis, float3 o, float3 d) {
        w.path[path] = words;
        w.throughput[path] = throughput;
        if (kSpectral) w.lambda[path] = lambda;
        w.vertex[path] = make_float4(at.x, at.y, at.z, scale);
        w.mis[path] = mis;
        w.ray_o[0][slot] = make_float4(o.x, o.y, o.z, tag);
        w.ray_d[0][slot] = make_float4(d.x, d.y, d.z, kInfinity);
    };
    auto dead = [&] {
        w.path[path] = make_uint4(kNone, 0u, 0u, 0u);
        w.ray_o[0][slot] = make_float4(0.0f, 0.0f, 0.0f, tag);
        w.ray_d[0][slot] = make_float4(0.0f, 0.0f, 1.0f, 0.0f);
    };
    const float afar = k.emit_share;
    if (u_pick.y < afar) {
        float share;
        const uint32_t light = choose_afar(m.lights, u_pick.y / afar, share);
        LightSample s;
        if (light == kNone || !(share > 0.0f) || !emits_from_afar(m.lights, light) ||
            !light_sample(m.lights, light, make_float3(0.0f, 0.0f, 0.0f), make_float2(u_point.x, u_point.y), s))
            return dead();
        const float3 toward = s.direction;
        float3 t, b;
        basis(toward, t, b);
        const float2 d = concentric(make_float2(u_point.z, u_point.w)) * k.emit_radius;
        const float3 start = k.emit_center + toward * (2.0f * k.emit_radius) + t * d.x + b * d.y;
        const float chance = afar * share * s.pdf;
        const float4 emitted = shape_of(m.lights.light[light]) == kShapeDome
                                   ? dome_emission<kSpectral>(m.lights, light, toward, lambda)
                                   : light_emission<kSpectral>(m.lights.light[light], lambda);
        const float4 carried = emitted * (kPi * k.emit_radius * k.emit_radius / chance);
        const float most = spec_max<kSpectral>(carried);
        if (!(most > 0.0f)) return dead();
        // The light's "point" is a direction: its density is the chance, and the camera's
        // density of it is its BSDF pdf alone.
        return launch(make_uint4(kAfarEmitter | light, 0u, 0u, 0u), carried, start, 1.0f / most,
                      make_float4(1.0f, chance, 1.0f, -1.0f), start, -toward);
    }
    uint32_t e;
    float chance;
    if (!tree_choose<true>(m.tree, (u_pick.y - afar) / fmaxf(1e-7f, 1.0f - afar), make_float3(0, 0, 0),
                           make_float3(0, 0, 0), e, chance))
        return dead();
    chance *= 1.0f - afar;
    const uint32_t code = emitter_code(m.tree, e);
    float3 q, n;
    float4 radiance;
    float area;
    bool both_sides = false;
    if (triangle_emitter(code)) {
        const uint32_t slot_t = code & ~kEmitterTriangle;
        float3 a, b, c;
        corners(m, slot_t, a, b, c);
        const float r = sqrtf(u_point.x);
        q = a * (1.0f - r) + b * (r * (1.0f - u_point.y)) + c * (r * u_point.y);
        const float3 twice = cross(b - a, c - a);
        area = 0.5f * length(twice);
        n = twice / fmaxf(2.0f * area, 1e-30f);
        if (u_pick.z < 0.5f) n = -n;
        both_sides = true;
        const MaterialCode &mc = m.materials[__ldg(&m.scene.shading[slot_t]).w];
        radiance = spec_of<kSpectral>(__ldg(&mc.glow_fit), xyz(__ldg(&mc.glow_rgb)), lambda);
    } else {
        const DeviceLight &l = m.lights.light[code];
        const float4 c = __ldg(&l.centre);
        if (shape_of(l) == kShapeSphere) {
            const float r = __ldg(&l.cone).x;
            const float z = 1.0f - 2.0f * u_point.x;
            const float ring = sqrtf(fmaxf(0.0f, 1.0f - z * z));
            float sp, cp;
            sincosf(2.0f * kPi * u_point.y, &sp, &cp);
            n = make_float3(ring * cp, ring * sp, z);
            q = xyz(c) + r * n;
            area = 4.0f * kPi * r * r;
        } else {
            const float2 a = shape_of(l) == kShapeRect ? make_float2(2.0f * u_point.x - 1.0f, 2.0f * u_point.y - 1.0f)
                                                       : concentric(make_float2(u_point.x, u_point.y));
            q = xyz(c) + a.x * xyz(__ldg(&l.u)) + a.y * xyz(__ldg(&l.v));
            const float4 nl = __ldg(&l.n);
            n = xyz(nl);
            area = nl.w;
        }
        radiance = light_emission<kSpectral>(l, lambda);
    }
    if (area <= 0.0f) return dead();
    const float2 d = concentric(make_float2(u_point.z, u_point.w));
    const float cos_n = sqrtf(fmaxf(0.0f, 1.0f - (d.x * d.x + d.y * d.y)));
    if (cos_n <= 0.0f) return dead();
    float3 t, b;
    basis(n, t, b);
    const float3 direction = normalize(t * d.x + b * d.y + n * cos_n);
    const float point_pdf = chance / area;
    const float direction_pdf = cos_n / (both_sides ? 2.0f * kPi : kPi);
    const float4 throughput = radiance * (cos_n / (point_pdf * direction_pdf));
    const float largest = spec_max<kSpectral>(throughput);
    if (!(largest > 0.0f)) return dead();
    // Russian roulette weighs throughput relative to the start's.
    launch(make_uint4(e, 0u, 0u, __float_as_uint(direction_pdf)), throughput, q, 1.0f / largest,
           make_float4(1.0f, point_pdf, cos_n, -1.0f), offset_origin(q, n), direction);
}

}  // namespace lr
