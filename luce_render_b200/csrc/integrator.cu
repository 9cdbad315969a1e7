// The wavefront path tracer (src/render/integrator.lucb, shaders/camera.comp,
// intersect_closest.comp, shade_surface.comp, shade_miss.comp, intersect_shadow.comp,
// finish.comp, film_convert.comp) on sm_100a.
//
// A pass traces one sample for one band of at most `pool` pixels:
//   begin -> camera -> (closest -> shade -> shadow) x (max_bounces + 1) -> finish -> convert
// Rays live in two ping-pong queues of structure-of-arrays float4 records (origin + path
// id, direction + t_max) that the traversal kernel reads with coalesced 128-bit loads;
// hits are written at the ray's queue index. The shade kernel takes every queue entry
// -- surface hit, light hit or miss (shade_surface + shade_miss of the reference) --
// and pushes surviving paths' next rays and shadow rays into compact queues with one
// atomic per warp. Queue sizes never leave the device: every kernel is a persistent
// grid-stride loop over the count its producer left, so the whole pass is one CUDA
// graph whose begin kernel derives the band and sample from a device pass counter.
#include <algorithm>
#include <memory>
#include <vector>

#include "device.hpp"
#include "loading.hpp"
#include "shading.cuh"
#include "traverse.cuh"

namespace lr {
namespace {

constexpr int kTraceBlock = 128;
constexpr int kShadeBlock = 128;
constexpr uint32_t kMaterialStride = 16;  // vec4 rows per material (openpbr.glsl:28)
constexpr size_t kDefaultPool = 2097152;  // 2^21 paths (integrator.lucb:98)

struct PassState {
    uint32_t band_start, band_count, sample, convert;
};

// Everything a pass's kernels read: passed by value, fixed for the renderer's life.
struct View {
    DeviceScene scene;
    const float4 *lights;
    uint32_t light_count;
    TreeView tree;
    const float4 *materials;
    const Constants *k;
    float frame[16];
    float lens_radius, focus_distance;
    float forward[3];
    uint32_t width, height, pool, bands, rounds;
    uint64_t pixels;
    // path state, one slot per path of the band
    float4 *throughput, *radiance, *lambda, *vertex;  // vertex: last scattering point, w survival scale
    uint4 *path;                                      // pixel, bounces, previous normal, ray pdf bits
    // ray queues (ping-pong by round) and their hits
    float4 *ray_o[2], *ray_d[2], *hits[2];
    float4 *shadow_o, *shadow_d, *shadow_c;
    // counters[r]: rays of round r; counters[rounds + 1 + r]: shadow rays of round r
    uint32_t *counters;
    PassState *pass;
    unsigned long long *pass_counter;
    float4 *film, *image;
    unsigned long long *stats;  // closest rays, shadow rays, shaded, passes
    int *status;
};

__device__ __forceinline__ uint32_t warp_push(uint32_t *counter, bool want) {
    const unsigned mask = __ballot_sync(0xffffffffu, want);
    if (mask == 0u) return 0u;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(mask) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(counter, (uint32_t)__popc(mask));
    base = __shfl_sync(0xffffffffu, base, leader);
    return base + (uint32_t)__popc(mask & ((1u << lane) - 1u));
}

__global__ void begin_kernel(View v) {
    if (threadIdx.x == 0) {
        const unsigned long long p = *v.pass_counter;
        const uint32_t band = (uint32_t)(p % v.bands);
        PassState s;
        s.sample = (uint32_t)(p / v.bands);
        const uint64_t start = (uint64_t)band * v.pool;
        s.band_start = (uint32_t)start;
        s.band_count = (uint32_t)min((uint64_t)v.pool, v.pixels - start);
        s.convert = band + 1 == v.bands ? 1u : 0u;
        *v.pass = s;
        *v.pass_counter = p + 1;
    }
    for (uint32_t i = threadIdx.x; i < 4 * v.rounds + 2; i += blockDim.x) v.counters[i] = 0;
}

// camera.comp:14-50: a jittered primary ray per pixel of the band.
template <bool kSpectral>
__global__ void __launch_bounds__(kShadeBlock) camera_kernel(View v) {
    const PassState ps = *v.pass;
    const Constants *k = v.k;
    const uint32_t seed = k->seed;
    const float3 position = make_float3(v.frame[0], v.frame[1], v.frame[2]);
    const float3 corner = make_float3(v.frame[4], v.frame[5], v.frame[6]);
    const float3 du = make_float3(v.frame[8], v.frame[9], v.frame[10]);
    const float3 dv = make_float3(v.frame[12], v.frame[13], v.frame[14]);
    const bool ortho = v.frame[3] > 0.5f;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t path = blockIdx.x * blockDim.x + threadIdx.x; path < ps.band_count; path += stride) {
        const uint32_t pixel = ps.band_start + path;
        const float4 u = sample4(seed, pixel, ps.sample, kGroupCamera);
        const float fx = (float)(pixel % v.width) + u.x, fy = (float)(pixel / v.width) + u.y;
        const float3 film = corner + fx * du + fy * dv;
        float3 origin = ortho ? position + film : position;
        float3 direction = normalize(ortho ? cross(du, dv) : film);
        if (!ortho && v.lens_radius > 0.0f) {
            const float3 forward = make_float3(v.forward[0], v.forward[1], v.forward[2]);
            const float3 focused = position + direction * (v.focus_distance / dot(direction, forward));
            const float2 disk = concentric(make_float2(u.z, u.w));
            origin = position + normalize(du) * (disk.x * v.lens_radius) + normalize(dv) * (disk.y * v.lens_radius);
            direction = normalize(focused - origin);
        }
        v.path[path] = make_uint4(pixel, 0u, 0u, 0u);
        v.throughput[path] = make_float4(1.0f, 1.0f, 1.0f, 1.0f);
        v.radiance[path] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        v.vertex[path] = make_float4(origin.x, origin.y, origin.z, 1.0f);
        if (kSpectral) v.lambda[path] = sample_wavelengths(sample4(seed, pixel, ps.sample, kGroupWavelength).x);
        v.ray_o[0][path] = make_float4(origin.x, origin.y, origin.z, __uint_as_float(path));
        v.ray_d[0][path] = make_float4(direction.x, direction.y, direction.z, kInfinity);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) v.counters[0] = ps.band_count;
}

// intersect_closest.comp:45-76: the nearest triangle, then the analytic lights
// before it (camera rays skip lights invisible to the camera).
template <int W, int kStack, bool kCount>
__global__ void __launch_bounds__(kTraceBlock) closest_kernel(View v, uint32_t round) {
    __shared__ int stack[TracerOf<W, false, kStack, kCount>::kInts * kTraceBlock];
    const uint32_t q = round & 1u;
    const uint32_t count = v.counters[round];
    bool overflow = false;
    Visits visits;
    const float4 *ray_o = v.ray_o[q], *ray_d = v.ray_d[q];
    float4 *hits = v.hits[q];
    auto load = [&](uint32_t i) {
        const float4 o = ray_o[i], d = ray_d[i];
        return Ray{xyz(o), 0.0f, xyz(d), d.w};
    };
    auto store = [&](uint32_t i, const Hit &h, const Ray &r) {
        uint32_t what = h.slot >= 0 ? (uint32_t)h.slot : kNone;
        float t = h.t;
        for (uint32_t light = 0; light < v.light_count; light++) {
            if (round == 0 && !light_visible(v.lights, light)) continue;
            const float tl = intersect_light(v.lights, light, r.o, r.d, t);
            if (tl < t) {
                t = tl;
                what = kLightHit | light;
            }
        }
        hits[i] = make_float4(t, __uint_as_float(what), h.u, h.v);
    };
    trace_strided<W, false, kStack, kCount>(v.scene, count, stack + threadIdx.x, kTraceBlock, load, store, overflow,
                                         visits);
    if (overflow) atomicAdd(&v.status[0], 1);
    if (kCount) add_visits(&v.stats[4], visits);
}

// intersect_shadow.comp:51-92: unblocked light samples join their path's radiance.
template <int W, int kStack, bool kCount>
__global__ void __launch_bounds__(kTraceBlock) shadow_kernel(View v, uint32_t round) {
    __shared__ int stack[TracerOf<W, true, kStack, kCount>::kInts * kTraceBlock];
    const uint32_t count = v.counters[v.rounds + 1 + round];
    bool overflow = false;
    Visits visits;
    auto load = [&](uint32_t i) {
        const float4 o = v.shadow_o[i], d = v.shadow_d[i];
        return Ray{xyz(o), 0.0f, xyz(d), d.w};
    };
    auto store = [&](uint32_t i, const Hit &h, const Ray &) {
        if (h.id < 0) {
            const uint32_t path = __float_as_uint(v.shadow_o[i].w);
            v.radiance[path] = v.radiance[path] + v.shadow_c[i];
        }
    };
    trace_strided<W, true, kStack, kCount>(v.scene, count, stack + threadIdx.x, kTraceBlock, load, store, overflow,
                                        visits);
    if (overflow) atomicAdd(&v.status[0], 1);
    if (kCount) add_visits(&v.stats[6], visits);
}

template <bool kSpectral>
__device__ __forceinline__ float4 clamped(float4 c, uint32_t total, float clamp_value) {
    if (total == 0u || clamp_value <= 0.0f) return c;
    const float largest = spec_max<kSpectral>(c);
    return largest > clamp_value ? c * (clamp_value / largest) : c;
}

__device__ __forceinline__ float4 material_at(const View &v, uint32_t m, uint32_t row) {
    return __ldg(&v.materials[m * kMaterialStride + row]);
}

__device__ __forceinline__ float3 position_of(const View &v, uint32_t index) {
    return make_float3(__ldg(&v.scene.positions[index * 3]), __ldg(&v.scene.positions[index * 3 + 1]),
                       __ldg(&v.scene.positions[index * 3 + 2]));
}

// triangle_hit_pdf (lighttree.glsl:131-137)
__device__ __forceinline__ float triangle_hit_pdf(const View &v, uint32_t slot, float3 d, float t) {
    const float3 a = position_of(v, v.scene.indices[slot * 3]);
    const float3 cr = cross(position_of(v, v.scene.indices[slot * 3 + 1]) - a, position_of(v, v.scene.indices[slot * 3 + 2]) - a);
    const float area = 0.5f * length(cr);
    const float cos_light = fabsf(dot(d, cr)) / fmaxf(1e-20f, 2.0f * area);
    return t * t / fmaxf(1e-20f, cos_light * area);
}

// sample_triangle (lighttree.glsl:107-128)
template <bool kSpectral>
__device__ __forceinline__ bool sample_triangle(const View &v, uint32_t slot, float3 p, float2 u, float4 lambda,
                                                LightSample &s, float4 &radiance) {
    const float3 a = position_of(v, v.scene.indices[slot * 3]);
    const float3 b = position_of(v, v.scene.indices[slot * 3 + 1]);
    const float3 c = position_of(v, v.scene.indices[slot * 3 + 2]);
    const float r = sqrtf(u.x);
    const float3 q = a * (1.0f - r) + b * (r * (1.0f - u.y)) + c * (r * u.y);
    const float3 cr = cross(b - a, c - a);
    const float area = 0.5f * length(cr);
    const float3 d = q - p;
    const float d2 = dot(d, d);
    if (area <= 0.0f || d2 <= 0.0f) return false;
    s.distance = sqrtf(d2);
    s.direction = d * (1.0f / s.distance);
    const float cos_light = fabsf(dot(s.direction, cr)) / (2.0f * area);
    if (cos_light <= 0.0f) return false;
    s.pdf = d2 / (cos_light * area);
    s.cos_light = cos_light;
    s.delta = false;
    const uint32_t m = __ldg(&v.scene.shading[slot]).w;
    radiance = spec_of<kSpectral>(material_at(v, m, 6), xyz(material_at(v, m, 7)), lambda);
    return true;
}

struct ShadeOut {
    bool next = false, shadow = false;
    float4 o, d, so, sd, sc;
};

__device__ __forceinline__ float rgb_luminance(float3 c) {
    return c.x * 0.2722287168f + c.y * 0.6740817658f + c.z * 0.0536895174f;
}

// One queue entry: a miss (shade_miss.comp:12-51), a light hit or a surface hit
// (shade_surface.comp:48-312 at the Lambertian settings).
template <bool kSpectral>
__device__ __forceinline__ void shade_one(const View &v, const Constants &k, const PassState &ps, uint32_t round,
                                          uint32_t i, ShadeOut &out) {
    const uint32_t q = round & 1u;
    const float4 ro = v.ray_o[q][i], rd = v.ray_d[q][i], hit = v.hits[q][i];
    const uint32_t path = __float_as_uint(ro.w);
    uint4 pu = v.path[path];
    const uint32_t pixel = pu.x, bounces = pu.y, total = bounces & 0xffu;
    const float ray_pdf = __uint_as_float(pu.w);
    const float3 origin = xyz(ro), dir = xyz(rd);
    float4 throughput = v.throughput[path];
    const float4 lambda = kSpectral ? v.lambda[path] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    const uint32_t what = __float_as_uint(hit.y);
    const float t = hit.x;
    float4 radiance = v.radiance[path];

    if (what == kNone) {
        float4 r = spec_of<kSpectral>(k.background_fit, k.background_rgb, lambda);
        for (uint32_t light = 0; light < v.light_count; light++) {
            const uint32_t type = light_type(v.lights, light);
            if (type < kLightDistant) continue;
            const float cos_half = light_at(v.lights, light, 2).w;
            if (cos_half >= 1.0f - 1e-7f || dot(dir, -xyz(light_at(v.lights, light, 3))) < cos_half) continue;
            float weight = 1.0f;
            if (total == 0u) {
                if (!light_visible(v.lights, light)) continue;
            } else if (ray_pdf > 0.0f) {
                const float select = k.p_distant * light_at(v.lights, light, 6).y;
                weight = mis_weight(light_hit_pdf(v.lights, light, make_float3(0.0f, 0.0f, 0.0f), dir, kInfinity) *
                                        select / ray_pdf, 0.0f);
            }
            r = r + light_radiance<kSpectral>(v.lights, light, lambda) * weight;
        }
        float4 contribution = throughput * r;
        const float largest = spec_max<kSpectral>(contribution);
        if (total > 0u && k.clamp_indirect > 0.0f && largest > k.clamp_indirect)
            contribution = contribution * (k.clamp_indirect / largest);
        v.radiance[path] = radiance + contribution;
        return;
    }
    const float4 vertex_row = v.vertex[path];
    const float3 vertex = xyz(vertex_row);
    if (what & kLightHit) {
        const uint32_t light = what & ~kLightHit;
        float weight = 1.0f;
        if (total == 0u) {
            if (!light_visible(v.lights, light)) return;
        } else if (ray_pdf > 0.0f) {
            const uint32_t emitter = (uint32_t)light_at(v.lights, light, 6).w;
            const float reach = length(vertex - (origin + t * dir));
            const float chance = (1.0f - k.p_distant) * tree_pdf(v.tree, emitter, vertex, octahedral_decode(pu.z));
            weight = mis_weight(light_hit_pdf(v.lights, light, vertex, dir, reach) * chance / ray_pdf, 0.0f);
        }
        v.radiance[path] = radiance + clamped<kSpectral>(throughput * light_radiance<kSpectral>(v.lights, light, lambda) * weight,
                                                          total, k.clamp_indirect);
        return;
    }

    // A surface.
    const uint32_t slot = what;
    const float3 p0 = position_of(v, v.scene.indices[slot * 3]);
    float3 geometric = normalize(cross(position_of(v, v.scene.indices[slot * 3 + 1]) - p0,
                                       position_of(v, v.scene.indices[slot * 3 + 2]) - p0));
    if (dot(geometric, dir) > 0.0f) geometric = -geometric;
    const uint4 attributes = __ldg(&v.scene.shading[slot]);
    const uint32_t m = attributes.w;
    const float3 p = origin + t * dir;
    const float reach = length(vertex - p);

    const float4 emission_row = material_at(v, m, 7);
    if (emission_row.w > 0.0f) {
        float weight = 1.0f;
        const uint32_t emitter = v.tree.triangle_map ? __ldg(&v.tree.triangle_map[slot]) : kNone;
        if (total > 0u && ray_pdf > 0.0f && emitter != kNone) {
            const float chance = (1.0f - k.p_distant) * tree_pdf(v.tree, emitter, vertex, octahedral_decode(pu.z));
            weight = mis_weight(triangle_hit_pdf(v, slot, dir, reach) * chance / ray_pdf, 0.0f);
        }
        radiance = radiance + clamped<kSpectral>(throughput * spec_of<kSpectral>(material_at(v, m, 6), xyz(emission_row), lambda) * weight,
                                                 total, k.clamp_indirect);
    }
    if (total >= k.max_bounces) {
        v.radiance[path] = radiance;
        return;
    }
    const float hu = hit.z, hv = hit.w;
    float3 normal = normalize(octahedral_decode(attributes.x) * (1.0f - hu - hv) + octahedral_decode(attributes.y) * hu +
                              octahedral_decode(attributes.z) * hv);
    if (dot(normal, geometric) < 0.0f) normal = -normal;
    float3 tangent, bitangent;
    basis(normal, tangent, bitangent);
    const float3 wo = make_float3(-dot(dir, tangent), -dot(dir, bitangent), -dot(dir, normal));
    const float4 base_rgb = material_at(v, m, 1);
    const float4 base = spec_of<kSpectral>(material_at(v, m, 0), xyz(base_rgb), lambda) * base_rgb.w;
    const float roughness = material_at(v, m, 10).y;
    const float p_diffuse = fmaxf(rgb_luminance(xyz(base_rgb) * base_rgb.w), 0.0f) > 0.0f ? 1.0f : 0.0f;
    const float3 from = offset_origin(p, geometric);

    // One light sample: a distant light by power, or an emitter of the light tree.
    const float4 u_light = sample4(k.seed, pixel, ps.sample, group_light(total));
    LightSample s;
    float4 emitted = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    float chance = 0.0f;
    bool sampled = false;
    if (u_light.x < k.p_distant) {
        float share;
        const uint32_t light = pick_distant(v.lights, v.light_count, u_light.x / k.p_distant, share);
        if (light != kNone && share > 0.0f && sample_light(v.lights, light, p, make_float2(u_light.y, u_light.z), s)) {
            chance = k.p_distant * share;
            emitted = light_radiance<kSpectral>(v.lights, light, lambda);
            sampled = true;
        }
    } else {
        uint32_t emitter;
        float tree_chance;
        if (tree_sample(v.tree, (u_light.x - k.p_distant) / fmaxf(1e-7f, 1.0f - k.p_distant), from, normal, emitter, tree_chance)) {
            chance = (1.0f - k.p_distant) * tree_chance;
            const uint32_t code = __ldg(&v.tree.records[emitter]).x;
            if (code & kEmitterTriangle) {
                sampled = sample_triangle<kSpectral>(v, code & ~kEmitterTriangle, p, make_float2(u_light.y, u_light.z), lambda, s, emitted);
            } else if (sample_light(v.lights, code, p, make_float2(u_light.y, u_light.z), s)) {
                emitted = light_radiance<kSpectral>(v.lights, code, lambda);
                sampled = true;
            }
        }
    }
    if (sampled && chance > 0.0f) {
        const float side = dot(s.direction, geometric);
        const float3 wi = make_float3(dot(s.direction, tangent), dot(s.direction, bitangent), dot(s.direction, normal));
        if (side > 0.0f && wi.z > 0.0f && wo.z > 0.0f) {
            const float bsdf_pdf = p_diffuse * wi.z / kPi;
            if (bsdf_pdf > 0.0f) {
                const float4 f = eon(base, roughness, wi, wo);
                const float light_pdf = s.pdf * chance;
                const float weight = s.delta ? 1.0f : mis_weight(bsdf_pdf / light_pdf, 0.0f);
                const float4 contribution = clamped<kSpectral>(throughput * f * emitted * (fabsf(wi.z) * (weight / light_pdf)),
                                                               total, k.clamp_indirect);
                const float3 target = p + s.direction * s.distance;
                const float margin = 4e-4f * fmaxf(1.0f, fmaxf(fabsf(target.x), fmaxf(fabsf(target.y), fabsf(target.z))));
                const float shadow_reach = s.distance >= kInfinity ? kInfinity : fmaxf(0.0f, s.distance - margin);
                const float3 so = offset_origin(p, geometric);
                out.shadow = true;
                out.so = make_float4(so.x, so.y, so.z, __uint_as_float(path));
                out.sd = make_float4(s.direction.x, s.direction.y, s.direction.z, shadow_reach);
                out.sc = contribution;
            }
        }
    }
    v.radiance[path] = radiance;

    // One BSDF sample (sample_surface with u.xyw: the lobe pick is u.w).
    const float4 u = sample4(k.seed, pixel, ps.sample, group_bsdf(total));
    if (wo.z <= 0.0f || !(u.w < p_diffuse)) return;
    const float2 disk = concentric(make_float2(u.x, u.y));
    const float3 wi = make_float3(disk.x, disk.y, sqrtf(fmaxf(0.0f, 1.0f - (disk.x * disk.x + disk.y * disk.y))));
    if (wi.z == 0.0f) return;
    const float pdf = p_diffuse * wi.z / kPi;
    if (!(pdf > 0.0f)) return;
    const float4 weight = eon(base, roughness, wi, wo) * (fabsf(wi.z) / pdf);
    const float3 direction = tangent * wi.x + bitangent * wi.y + normal * wi.z;
    const float side = dot(direction, geometric);
    if ((side > 0.0f) != (wi.z > 0.0f)) return;
    const uint32_t next_bounces = next_bounce(bounces, 0u, k.limits);
    if (next_bounces == kNone) return;
    throughput = throughput * weight;
    const float survival_scale = fminf(vertex_row.w, 1e6f);
    if (total + 1u >= 3u) {
        const float survive = fminf(0.95f, spec_max<kSpectral>(throughput) * survival_scale);
        if (u.z >= survive) return;
        throughput = make_float4(throughput.x / survive, throughput.y / survive, throughput.z / survive, throughput.w / survive);
    }
    const float3 next = side > 0.0f ? from : offset_origin(p, -geometric);
    v.path[path] = make_uint4(pixel, next_bounces, octahedral_encode(normal), __float_as_uint(pdf));
    v.throughput[path] = throughput;
    v.vertex[path] = make_float4(next.x, next.y, next.z, survival_scale);
    out.next = true;
    out.o = make_float4(next.x, next.y, next.z, __uint_as_float(path));
    out.d = make_float4(direction.x, direction.y, direction.z, kInfinity);
}

template <bool kSpectral>
__global__ void __launch_bounds__(kShadeBlock) shade_kernel(View v, uint32_t round) {
    const uint32_t count = v.counters[round];
    const PassState ps = *v.pass;
    const Constants &k = *v.k;
    const uint32_t nq = (round & 1u) ^ 1u;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t stride = gridDim.x * blockDim.x;
    uint32_t *next_counter = &v.counters[round + 1];
    uint32_t *shadow_counter = &v.counters[v.rounds + 1 + round];
    for (uint32_t base = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < count; base += stride) {
        const uint32_t i = base + lane;
        ShadeOut out;
        if (i < count) shade_one<kSpectral>(v, k, ps, round, i, out);
        const uint32_t at = warp_push(next_counter, out.next);
        if (out.next) {
            v.ray_o[nq][at] = out.o;
            v.ray_d[nq][at] = out.d;
        }
        const uint32_t sat = warp_push(shadow_counter, out.shadow);
        if (out.shadow) {
            v.shadow_o[sat] = out.so;
            v.shadow_d[sat] = out.sd;
            v.shadow_c[sat] = out.sc;
        }
    }
}

// finish.comp:13-39: each path's radiance into its pixel (one sample per pixel per pass).
template <bool kSpectral>
__global__ void __launch_bounds__(kShadeBlock) finish_kernel(View v) {
    const PassState ps = *v.pass;
    const Constants &k = *v.k;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t path = blockIdx.x * blockDim.x + threadIdx.x; path < ps.band_count; path += stride) {
        const uint32_t pixel = v.path[path].x;
        float3 value = spec_to_film<kSpectral>(v.radiance[path], kSpectral ? v.lambda[path] : make_float4(0, 0, 0, 0), k);
        if (!isfinite(value.x) || !isfinite(value.y) || !isfinite(value.z)) value = make_float3(0.0f, 0.0f, 0.0f);
        const float4 f = v.film[pixel];
        v.film[pixel] = make_float4(f.x + value.x, f.y + value.y, f.z + value.z, f.w + 1.0f);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        unsigned long long closest = 0, shadow = 0;
        for (uint32_t r = 0; r < v.rounds; r++) {
            closest += v.counters[r];
            shadow += v.counters[v.rounds + 1 + r];
        }
        v.stats[0] += closest;
        v.stats[1] += shadow;
        v.stats[2] += ps.band_count;
        v.stats[3] += 1;
    }
}

// film_convert.comp:36-53: the film's average into the rgba32f ACEScg image.
template <bool kSpectral>
__global__ void __launch_bounds__(kShadeBlock) convert_kernel(View v) {
    if (!v.pass->convert) return;
    const Constants &k = *v.k;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t pixel = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; pixel < v.pixels; pixel += stride) {
        const float4 sum = v.film[pixel];
        const float w = fmaxf(sum.w, 1.0f);
        float3 value = make_float3(sum.x / w, sum.y / w, sum.z / w);
        if (kSpectral)
            value = make_float3(k.film[0] * value.x + k.film[1] * value.y + k.film[2] * value.z,
                                k.film[3] * value.x + k.film[4] * value.y + k.film[5] * value.z,
                                k.film[6] * value.x + k.film[7] * value.y + k.film[8] * value.z);
        v.image[pixel] = make_float4(value.x, value.y, value.z, 1.0f);
    }
}

// Kernel kinds for profiling (integrator.lucb:105-115).
enum Kind { kCamera = 0, kClosest = 1, kSurface = 2, kMiss = 3, kShadow = 4, kLightEmit = 5, kFinish = 6, kConvert = 7,
            kAdaptive = 8, kRest = 9 };

template <typename K>
int grid_of(K kernel, int block, int sm_count) {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, 0);
    return std::max(1, per_sm) * sm_count;
}

size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

}  // namespace
}  // namespace lr

using namespace lr;

struct lr_renderer {
    lr_context *ctx = nullptr;
    lr_settings settings{};
    lr_frame frame{};
    lr_gpu_scene *gs = nullptr;
    Loaded loaded;
    void *block = nullptr;  // one device allocation for everything below the scene
    View view{};
    int width = 2, stack = 32;  // the traversal variant (BVH width, stack entries)
    int grid_trace = 0, grid_shade = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    // passes: recorded, retired; in flight (oldest first) with their end events
    uint64_t recorded = 0, retired = 0;
    std::vector<cudaEvent_t> done_events;  // a ring of two
    std::vector<uint64_t> in_flight;       // pass numbers
    uint32_t bands = 1;
    // profiling: events after each kernel of the pass in flight, and ms per kind
    std::vector<std::vector<std::pair<cudaEvent_t, int>>> marks;
    cudaEvent_t mark_start[2] = {nullptr, nullptr};
    double kernel_ms[10] = {0};
};

namespace lr {
namespace {

// Records one pass on `stream`. With `marks`, an event follows each kernel (profiling);
// kCount instantiates the traversal kernels that count their work.
template <bool kSpectral, int W, int kStack, bool kCount>
void record_pass(lr_renderer *r, cudaStream_t stream, std::vector<std::pair<cudaEvent_t, int>> *marks) {
    View &v = r->view;
    auto mark = [&](int kind) {
        if (!marks) return;
        cudaEvent_t e;
        LR_CUDA(cudaEventCreate(&e));
        LR_CUDA(cudaEventRecord(e, stream));
        marks->push_back({e, kind});
    };
    begin_kernel<<<1, 256, 0, stream>>>(v);
    mark(kRest);
    camera_kernel<kSpectral><<<r->grid_shade, kShadeBlock, 0, stream>>>(v);
    mark(kCamera);
    for (uint32_t round = 0; round < v.rounds; round++) {
        closest_kernel<W, kStack, kCount><<<r->grid_trace, kTraceBlock, 0, stream>>>(v, round);
        mark(kClosest);
        shade_kernel<kSpectral><<<r->grid_shade, kShadeBlock, 0, stream>>>(v, round);
        mark(kSurface);
        shadow_kernel<W, kStack, kCount><<<r->grid_trace, kTraceBlock, 0, stream>>>(v, round);
        mark(kShadow);
    }
    finish_kernel<kSpectral><<<r->grid_shade, kShadeBlock, 0, stream>>>(v);
    mark(kFinish);
    convert_kernel<kSpectral><<<r->grid_shade, kShadeBlock, 0, stream>>>(v);
    mark(kConvert);
    LR_CUDA(cudaGetLastError());
}

// The traversal variants a renderer can take: (BVH width, stack entries).
#define LR_TRAVERSALS(X) X(8, 32) X(8, 48) X(4, 32) X(4, 48) X(2, 32) X(2, 64) X(2, 96)

template <bool kSpectral, bool kCount>
void record_any(lr_renderer *r, cudaStream_t stream, std::vector<std::pair<cudaEvent_t, int>> *marks) {
    switch (r->width * 1000 + r->stack) {
#define LR_CASE(w, k)                                                   \
    case w * 1000 + k:                                                  \
        record_pass<kSpectral, w, k, kCount>(r, stream, marks);         \
        break;
        LR_TRAVERSALS(LR_CASE)
#undef LR_CASE
        default: fail(LR_LIMIT, "no traversal variant for this scene");
    }
}

void record(lr_renderer *r, cudaStream_t stream, std::vector<std::pair<cudaEvent_t, int>> *marks) {
    const bool count = r->settings.profile == 2;
    if (r->settings.spectral) {
        if (count) record_any<true, true>(r, stream, marks);
        else record_any<true, false>(r, stream, marks);
    } else {
        if (count) record_any<false, true>(r, stream, marks);
        else record_any<false, false>(r, stream, marks);
    }
}

template <bool kSpectral>
void size_grids(lr_renderer *r) {
    const int sms = r->ctx->sm_count;
    switch (r->width * 1000 + r->stack) {
#define LR_CASE(w, k)                                                            \
    case w * 1000 + k:                                                           \
        r->grid_trace = grid_of(closest_kernel<w, k, false>, kTraceBlock, sms);  \
        break;
        LR_TRAVERSALS(LR_CASE)
#undef LR_CASE
        default: fail(LR_LIMIT, "no traversal variant for this scene");
    }
    r->grid_shade = grid_of(shade_kernel<kSpectral>, kShadeBlock, sms);
}

void settle(lr_renderer *r) {
    for (size_t i = 0; i < r->in_flight.size(); i++) LR_CUDA(cudaEventSynchronize(r->done_events[r->in_flight[i] & 1]));
}

// Retire the oldest pass in flight if it has finished (integrator.lucb:622-645).
bool retire_one(lr_renderer *r, bool wait) {
    if (r->in_flight.empty()) return false;
    const uint64_t pass = r->in_flight.front();
    cudaEvent_t e = r->done_events[pass & 1];
    if (wait) {
        LR_CUDA(cudaEventSynchronize(e));
    } else {
        cudaError_t q = cudaEventQuery(e);
        if (q == cudaErrorNotReady) return false;
        LR_CUDA(q);
    }
    if (r->settings.profile && !r->marks.empty()) {
        auto &ms = r->marks[pass & 1];
        cudaEvent_t prev = r->mark_start[pass & 1];
        for (auto &[ev, kind] : ms) {
            float t = 0.0f;
            LR_CUDA(cudaEventElapsedTime(&t, prev, ev));
            r->kernel_ms[kind] += t;
            prev = ev;
        }
        for (auto &[ev, kind] : ms) cudaEventDestroy(ev);
        ms.clear();
    }
    r->in_flight.erase(r->in_flight.begin());
    r->retired = pass + 1;
    return true;
}

void launch_pass(lr_renderer *r) {
    cudaStream_t stream = r->ctx->stream;
    const uint64_t pass = r->recorded;
    if (r->settings.profile) {
        LR_CUDA(cudaEventRecord(r->mark_start[pass & 1], stream));
        record(r, stream, &r->marks[pass & 1]);
    } else {
        LR_CUDA(cudaGraphLaunch(r->exec, stream));
    }
    LR_CUDA(cudaEventRecord(r->done_events[pass & 1], stream));
    r->in_flight.push_back(pass);
    r->recorded = pass + 1;
}

void validate(const lr_settings &s, const lr_frame &f) {
    if (f.width == 0 || f.height == 0 || f.width > 16384 || f.height > 16384)
        fail(LR_INVALID, "an image is 1 to 16384 pixels on a side");
    if (s.samples == 0 || s.max_bounces == 0 || s.max_bounces > 1024)
        fail(LR_INVALID, "a render needs samples and 1 to 1024 bounces");
    if (s.noise_threshold > 0.0) fail(LR_INVALID, "adaptive sampling is not part of this build (noise_threshold 0)");
    if (s.guiding) fail(LR_INVALID, "path guiding is not part of this build (guiding off)");
    if (s.max_bounces > 253) fail(LR_INVALID, "this build traces at most 253 bounces");
}

void create(lr_context *ctx, const lr_scene *scene, const lr_settings &settings, const lr_frame &frame, lr_renderer **out) {
    validate(settings, frame);
    auto r = std::make_unique<lr_renderer>();
    r->ctx = ctx;
    r->settings = settings;
    r->settings.width = frame.width;
    r->settings.height = frame.height;
    r->frame = frame;
    LR_CUDA(cudaSetDevice(ctx->device));
    r->loaded = load(*scene, settings);
    lr_gpu_scene *gs = nullptr;
    int status = lr_gpu_scene_upload(ctx, scene, &gs);
    if (status != LR_OK) fail(status, lr_last_error());
    r->gs = gs;

    const Loaded &L = r->loaded;
    const uint64_t pixels = (uint64_t)frame.width * frame.height;
    const uint64_t pool = std::min<uint64_t>(settings.pool ? settings.pool : kDefaultPool, pixels);
    r->bands = (uint32_t)((pixels + pool - 1) / pool);
    const uint32_t rounds = settings.max_bounces + 1;

    // Device layout: one allocation, arrays at 256-byte offsets.
    Constants k{};
    for (int i = 0; i < 9; i++) k.film[i] = (float)L.film.m[i];
    k.cmf_integrals[0] = (float)L.cmf_integrals.x;
    k.cmf_integrals[1] = (float)L.cmf_integrals.y;
    k.cmf_integrals[2] = (float)L.cmf_integrals.z;
    k.limits[0] = (float)settings.diffuse_bounces;
    k.limits[1] = (float)settings.glossy_bounces;
    k.limits[2] = (float)settings.transmission_bounces;
    k.clamp_indirect = (float)settings.clamp_indirect;
    k.background_fit = make_float4((float)L.background_fit[0], (float)L.background_fit[1], (float)L.background_fit[2],
                                   (float)L.background_fit[3]);
    k.background_rgb = make_float3((float)settings.background[0], (float)settings.background[1], (float)settings.background[2]);
    k.p_distant = (float)L.p_distant;
    k.max_bounces = settings.max_bounces;
    k.light_count = (uint32_t)L.lights.count;
    k.tree_nodes = (uint32_t)L.tree.node_count;
    k.seed = settings.seed;

    struct Part {
        const void *src;
        size_t bytes;
        size_t offset;
    };
    std::vector<Part> parts;
    auto add = [&](const void *src, size_t bytes) {
        parts.push_back({src, bytes, 0});
        return parts.size() - 1;
    };
    const size_t p_lights = add(L.lights.rows.data(), L.lights.rows.size() * 4);
    const size_t p_tree_nodes = add(L.tree.nodes.data(), L.tree.nodes.size() * 4);
    const size_t p_tree_links = add(L.tree.links.data(), L.tree.links.size() * 4);
    const size_t p_tree_records = add(L.tree.records.data(), L.tree.records.size() * 4);
    const size_t p_tree_map = add(L.tree.triangle_map.data(), L.tree.triangle_map.size() * 4);
    const size_t p_materials = add(L.materials.data(), L.materials.size() * 4);
    const size_t p_constants = add(&k, sizeof k);
    const size_t p_throughput = add(nullptr, pool * 16);
    const size_t p_radiance = add(nullptr, pool * 16);
    const size_t p_lambda = add(nullptr, settings.spectral ? pool * 16 : 16);
    const size_t p_vertex = add(nullptr, pool * 16);
    const size_t p_path = add(nullptr, pool * 16);
    size_t p_ray[2][3];
    for (int q = 0; q < 2; q++)
        for (int j = 0; j < 3; j++) p_ray[q][j] = add(nullptr, pool * 16);
    const size_t p_shadow_o = add(nullptr, pool * 16);
    const size_t p_shadow_d = add(nullptr, pool * 16);
    const size_t p_shadow_c = add(nullptr, pool * 16);
    const size_t p_counters = add(nullptr, (4 * rounds + 2) * 4);
    const size_t p_pass = add(nullptr, sizeof(PassState));
    const size_t p_pass_counter = add(nullptr, 8);
    const size_t p_film = add(nullptr, pixels * 16);
    const size_t p_image = add(nullptr, pixels * 16);
    const size_t p_stats = add(nullptr, 8 * 8);
    size_t total = 0;
    for (auto &p : parts) {
        p.offset = total;
        total += align256(std::max<size_t>(p.bytes, 64));
    }
    LR_CUDA(cudaMalloc(&r->block, total));
    char *base = (char *)r->block;
    LR_CUDA(cudaMemsetAsync(base, 0, total, ctx->stream));
    for (auto &p : parts)
        if (p.src && p.bytes) LR_CUDA(cudaMemcpyAsync(base + p.offset, p.src, p.bytes, cudaMemcpyHostToDevice, ctx->stream));
    static std::vector<uint32_t> sobol_bytes;
    if (sobol_bytes.empty()) {
        const uint32_t *dirs = sobol_table();
        sobol_bytes.assign(3 * 4 * 256, 0u);
        for (int d = 1; d < 4; d++)
            for (int b = 0; b < 4; b++)
                for (int value = 0; value < 256; value++) {
                    uint32_t x = 0;
                    for (int bit = 0; bit < 8; bit++)
                        if (value & (1 << bit)) x ^= dirs[d * 32 + b * 8 + bit];
                    sobol_bytes[(d - 1) * 1024 + b * 256 + value] = x;
                }
    }
    LR_CUDA(cudaMemcpyToSymbolAsync(g_sobol_bytes, sobol_bytes.data(), sobol_bytes.size() * sizeof(uint32_t), 0,
                                    cudaMemcpyHostToDevice, ctx->stream));
    LR_CUDA(cudaStreamSynchronize(ctx->stream));
    auto at = [&](size_t i) { return (void *)(base + parts[i].offset); };

    View &v = r->view;
    v.scene = gs->scene;
    v.lights = (const float4 *)at(p_lights);
    v.light_count = (uint32_t)L.lights.count;
    v.tree.nodes = (const float4 *)at(p_tree_nodes);
    v.tree.links = (const uint2 *)at(p_tree_links);
    v.tree.records = (const uint4 *)at(p_tree_records);
    v.tree.triangle_map = L.tree.triangle_map.empty() ? nullptr : (const uint32_t *)at(p_tree_map);
    v.tree.node_count = (uint32_t)L.tree.node_count;
    v.materials = (const float4 *)at(p_materials);
    v.k = (const Constants *)at(p_constants);
    pack_frame(frame, v.frame);
    v.lens_radius = (float)frame.lens_radius;
    v.focus_distance = (float)frame.focus_distance;
    for (int i = 0; i < 3; i++) v.forward[i] = (float)frame.forward[i];
    v.width = frame.width;
    v.height = frame.height;
    v.pool = (uint32_t)pool;
    v.bands = r->bands;
    v.rounds = rounds;
    v.pixels = pixels;
    v.throughput = (float4 *)at(p_throughput);
    v.radiance = (float4 *)at(p_radiance);
    v.lambda = (float4 *)at(p_lambda);
    v.vertex = (float4 *)at(p_vertex);
    v.path = (uint4 *)at(p_path);
    for (int q = 0; q < 2; q++) {
        v.ray_o[q] = (float4 *)at(p_ray[q][0]);
        v.ray_d[q] = (float4 *)at(p_ray[q][1]);
        v.hits[q] = (float4 *)at(p_ray[q][2]);
    }
    v.shadow_o = (float4 *)at(p_shadow_o);
    v.shadow_d = (float4 *)at(p_shadow_d);
    v.shadow_c = (float4 *)at(p_shadow_c);
    v.counters = (uint32_t *)at(p_counters);
    v.pass = (PassState *)at(p_pass);
    v.pass_counter = (unsigned long long *)at(p_pass_counter);
    v.film = (float4 *)at(p_film);
    v.image = (float4 *)at(p_image);
    v.stats = (unsigned long long *)at(p_stats);
    v.status = ctx->status;

    const TraversalChoice traversal = choose_traversal(gs->scene, 0);
    r->width = traversal.width;
    r->stack = traversal.stack;
    if (settings.spectral) size_grids<true>(r.get());
    else size_grids<false>(r.get());
    r->done_events.resize(2);
    for (auto &e : r->done_events) LR_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    if (settings.profile) {
        r->marks.resize(2);
        for (auto &e : r->mark_start) LR_CUDA(cudaEventCreate(&e));
    } else {
        // The pass as one graph, captured on a private stream.
        cudaStream_t capture;
        LR_CUDA(cudaStreamCreateWithFlags(&capture, cudaStreamNonBlocking));
        LR_CUDA(cudaStreamBeginCapture(capture, cudaStreamCaptureModeThreadLocal));
        record(r.get(), capture, nullptr);
        LR_CUDA(cudaStreamEndCapture(capture, &r->graph));
        LR_CUDA(cudaStreamDestroy(capture));
        LR_CUDA(cudaGraphInstantiate(&r->exec, r->graph, 0));
    }
    *out = r.release();
}

}  // namespace
}  // namespace lr

extern "C" {

void lr_settings_default(lr_settings *s, uint32_t width, uint32_t height, uint32_t samples) {
    if (!s) return;
    *s = lr_settings{};
    s->width = width;
    s->height = height;
    s->samples = samples;
    s->max_bounces = 12;
    s->spectral = 1;
    s->camera = -1;
    lr_openpbr_standard(&s->material);
    s->pool = 0;
    s->seed = 1;
    s->software_bvh = 0;
    s->diffuse_bounces = s->glossy_bounces = s->transmission_bounces = 1024;
    s->clamp_indirect = 0.0;
    s->noise_threshold = 0.0;
    s->adaptive_minimum = 16;
    s->profile = 0;
    s->guiding = 0;
    s->light_tracing = 0.5;
}

int lr_renderer_create(lr_context *ctx, const lr_scene *scene, const lr_settings *settings, lr_renderer **out) {
    return guarded([&] {
        if (!ctx || !scene || !settings || !out) fail(LR_INVALID, "a renderer needs a context, a scene and settings");
        *out = nullptr;
        if (settings->width == 0 || settings->height == 0 || settings->width > 16384 || settings->height > 16384)
            fail(LR_INVALID, "an image is 1 to 16384 pixels on a side");
        lr_camera cam;
        if (settings->camera >= 0) {
            if ((size_t)settings->camera >= scene->cameras.size()) fail(LR_INVALID, "the scene object is not a camera");
            cam = scene->cameras[(size_t)settings->camera];
        } else {
            if (scene->cameras.empty()) fail(LR_INVALID, "the scene has no camera");
            cam = scene->cameras[0];
        }
        lr_frame frame;
        camera_frame(cam, settings->width, settings->height, frame);
        create(ctx, scene, *settings, frame, out);
    });
}

int lr_renderer_create_viewed(lr_context *ctx, const lr_scene *scene, const lr_settings *settings, const lr_frame *frame,
                              lr_renderer **out) {
    return guarded([&] {
        if (!ctx || !scene || !settings || !frame || !out) fail(LR_INVALID, "a renderer needs a context, a scene and settings");
        *out = nullptr;
        create(ctx, scene, *settings, *frame, out);
    });
}

int lr_renderer_advance(lr_renderer *r, int32_t *more) {
    return guarded([&] {
        if (!r || !more) fail(LR_INVALID, "no renderer");
        while (retire_one(r, false)) {
        }
        // Two passes in flight (integrator.lucb:651-655); profiling keeps its events per
        // pass, so it may too.
        const size_t depth = 2;
        if (r->in_flight.size() >= depth) {
            *more = 1;
            return;
        }
        const uint64_t total_passes = (uint64_t)r->settings.samples * r->bands;
        if (r->recorded >= total_passes) {
            *more = r->in_flight.empty() ? 0 : 1;
            return;
        }
        launch_pass(r);
        *more = 1;
    });
}

int lr_renderer_finish(lr_renderer *r) {
    return guarded([&] {
        if (!r) fail(LR_INVALID, "no renderer");
        for (;;) {
            int32_t more = 0;
            int status = lr_renderer_advance(r, &more);
            if (status != LR_OK) fail(status, lr_last_error());
            if (!more) break;
            if (!r->in_flight.empty()) retire_one(r, true);
        }
        check_status(r->ctx);
    });
}

uint32_t lr_renderer_samples_done(const lr_renderer *r) { return r ? (uint32_t)(r->retired / r->bands) : 0u; }

int lr_renderer_passes(const lr_renderer *r, uint64_t *recorded, uint64_t *finished, uint32_t *bands) {
    return guarded([&] {
        if (!r) fail(LR_INVALID, "no renderer");
        if (recorded) *recorded = r->recorded;
        if (finished) *finished = r->retired;
        if (bands) *bands = r->bands;
    });
}

int lr_renderer_image(lr_renderer *r, void **device_rgba) {
    return guarded([&] {
        if (!r || !device_rgba) fail(LR_INVALID, "no renderer");
        *device_rgba = r->view.image;
    });
}

int lr_renderer_read(lr_renderer *r, float *rgba, uint64_t count) {
    return guarded([&] {
        if (!r || !rgba) fail(LR_INVALID, "no renderer");
        if (count != r->view.pixels * 4) fail(LR_INVALID, "reading the image needs four floats a pixel");
        LR_CUDA(cudaMemcpyAsync(rgba, r->view.image, count * 4, cudaMemcpyDeviceToHost, r->ctx->stream));
        LR_CUDA(cudaStreamSynchronize(r->ctx->stream));
    });
}

int lr_renderer_set_samples(lr_renderer *r, uint32_t samples) {
    return guarded([&] {
        if (!r) fail(LR_INVALID, "no renderer");
        if (samples == 0) fail(LR_INVALID, "a render needs samples");
        r->settings.samples = samples;
    });
}

int lr_renderer_kernel_times(lr_renderer *r, double out[10]) {
    return guarded([&] {
        if (!r || !out) fail(LR_INVALID, "kernel times need ten numbers");
        // Finished passes count: wait for those in flight and retire them.
        settle(r);
        while (retire_one(r, false)) {
        }
        for (int i = 0; i < 10; i++) out[i] = r->kernel_ms[i];
    });
}

int lr_renderer_stats(lr_renderer *r, lr_render_stats *out) {
    return guarded([&] {
        if (!r || !out) fail(LR_INVALID, "no renderer");
        settle(r);
        while (retire_one(r, false)) {
        }
        unsigned long long s[8];
        LR_CUDA(cudaMemcpyAsync(s, r->view.stats, sizeof s, cudaMemcpyDeviceToHost, r->ctx->stream));
        LR_CUDA(cudaStreamSynchronize(r->ctx->stream));
        out->closest_rays = s[0];
        out->shadow_rays = s[1];
        out->shaded = s[2];
        out->passes = s[3];
        out->closest_nodes = s[4];
        out->closest_tests = s[5];
        out->shadow_nodes = s[6];
        out->shadow_tests = s[7];
    });
}

void lr_renderer_destroy(lr_renderer *r) {
    if (!r) return;
    cudaSetDevice(r->ctx->device);
    cudaStreamSynchronize(r->ctx->stream);
    for (auto &ms : r->marks)
        for (auto &[e, k] : ms) cudaEventDestroy(e);
    for (auto e : r->mark_start)
        if (e) cudaEventDestroy(e);
    for (auto e : r->done_events) cudaEventDestroy(e);
    if (r->exec) cudaGraphExecDestroy(r->exec);
    if (r->graph) cudaGraphDestroy(r->graph);
    if (r->block) cudaFree(r->block);
    lr_gpu_scene_destroy(r->gs);
    delete r;
}

}  // extern "C"
