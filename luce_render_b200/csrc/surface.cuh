// Surface scattering for the integrator: OpenPBR Surface's layers (the model the
// reference shades in shaders/openpbr.glsl and microfacet.glsl) as this build evaluates
// them on sm_100a.
//
// Everything about a material that does not depend on the hit is worked out once on the
// host (loading.cpp `material_code`) into a MaterialCode record: clamped weights, the
// base's roughness and index with and without the coat above it, GGX widths, the
// hemispherical Fresnel averages, the colours' luminances and spectral fits. A hit then
// resolves its side (an object's inside has no coat), orients the layers to the view
// direction (albedo-table lookups, the lobe choice), fills the colours at the path's
// wavelengths, and evaluates, samples and weighs directions. Members whose materials are
// all diffuse take `DiffuseSurface`, the same model reduced to EON diffuse (the layered
// surface's diffuse lobe with every other layer at weight zero).
//
// Published pieces: the GGX (Trowbridge-Reitz) distribution with height-correlated Smith
// masking (Heitz 2014), visible-normal sampling by spherical caps (Dupuy and Benyoub
// 2023), Kulla and Conty's (2017) energy compensation 1 + F_avg (1 - E) / E from tabulated
// directional albedos, the F82-tint metal Fresnel (Kutz et al. 2021, as adopted by
// OpenPBR), and energy-preserving Oren-Nayar diffuse (EON: Portsmouth, Kutz and Hill
// 2025). The lobe weights and choice are OpenPBR's as the reference's estimator uses
// them, so the f64 oracle's densities are the kernels' (tested to f32 rounding).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "shading.cuh"

namespace lr {

// ---- small helpers ----------------------------------------------------------------------

__device__ __forceinline__ float lerpf(float a, float b, float t) { return a * (1.0f - t) + b * t; }
__device__ __forceinline__ float4 lerp4(float4 a, float4 b, float t) { return a * (1.0f - t) + b * t; }
__device__ __forceinline__ float4 fill4(float v) { return make_float4(v, v, v, v); }
__device__ __forceinline__ float4 one_minus(float4 v) { return make_float4(1.0f - v.x, 1.0f - v.y, 1.0f - v.z, 1.0f - v.w); }
__device__ __forceinline__ float4 saturate4(float4 v) {
    return make_float4(__saturatef(v.x), __saturatef(v.y), __saturatef(v.z), __saturatef(v.w));
}
__device__ __forceinline__ float clamp01(float v) { return fminf(fmaxf(v, 0.0f), 1.0f); }

// ---- GGX --------------------------------------------------------------------------------

struct Ggx {
    float ax, ay;
};

// OpenPBR's widths from roughness and anisotropy: alpha = r^2 stretched by
// sqrt(2 / (1 + (1 - a)^2)) along x and shrunk by (1 - a) along y, at least 1e-4.
__device__ __forceinline__ Ggx ggx_widths(float roughness, float anisotropy) {
    const float squeeze = 1.0f - anisotropy;
    const float t = roughness * roughness * sqrtf(2.0f / (1.0f + squeeze * squeeze));
    return Ggx{fmaxf(t, 1e-4f), fmaxf(squeeze * t, 1e-4f)};
}

__device__ __forceinline__ float ggx_d(const Ggx &g, float3 m) {
    if (m.z <= 0.0f) return 0.0f;
    const float x = m.x / g.ax, y = m.y / g.ay;
    const float k = x * x + y * y + m.z * m.z;
    return 1.0f / (kPi * g.ax * g.ay * k * k);
}

// Smith's Lambda for direction v (kInfinity at grazing).
__device__ __forceinline__ float ggx_lambda(const Ggx &g, float3 v) {
    const float z2 = v.z * v.z;
    if (z2 <= 0.0f) return kInfinity;
    const float slope2 = (g.ax * g.ax * v.x * v.x + g.ay * g.ay * v.y * v.y) / z2;
    return 0.5f * (sqrtf(1.0f + slope2) - 1.0f);
}

__device__ __forceinline__ float ggx_g1(const Ggx &g, float3 v) { return 1.0f / (1.0f + ggx_lambda(g, v)); }
__device__ __forceinline__ float ggx_g2(const Ggx &g, float3 a, float3 b) {
    return 1.0f / (1.0f + ggx_lambda(g, a) + ggx_lambda(g, b));
}

// A microfacet normal seen from wo (above), distributed as the visible normals.
__device__ __forceinline__ float3 ggx_visible(const Ggx &g, float3 wo, float2 u) {
    const float3 v = normalize(make_float3(wo.x * g.ax, wo.y * g.ay, wo.z));
    const float z = (1.0f - u.y) * (1.0f + v.z) - v.z;
    const float ring = sqrtf(clamp01(1.0f - z * z));
    float sp, cp;
    sincosf(2.0f * kPi * u.x, &sp, &cp);
    const float3 h = make_float3(ring * cp + v.x, ring * sp + v.y, z + v.z);
    return normalize(make_float3(h.x * g.ax, h.y * g.ay, fmaxf(h.z, 1e-6f)));
}

// The density of reflecting wo about a visible normal h, per solid angle of wi.
__device__ __forceinline__ float ggx_reflection_pdf(const Ggx &g, float3 wo, float3 h) {
    return ggx_g1(g, wo) * ggx_d(g, h) / (4.0f * wo.z);
}

// ---- Fresnel ----------------------------------------------------------------------------

// Unpolarised reflectance at a dielectric interface (eta: far side over near side).
__device__ __forceinline__ float fresnel(float cos_i, float eta) {
    const float c = fabsf(cos_i);
    const float g2 = eta * eta - 1.0f + c * c;
    if (g2 <= 0.0f) return 1.0f;  // total internal reflection
    const float g = sqrtf(g2);
    const float s = (g - c) / (g + c);
    const float p = (c * (g + c) - 1.0f) / (c * (g - c) + 1.0f);
    return 0.5f * s * s * (1.0f + p * p);
}

// Its hemispherical average for eta > 1, by the closed fit OpenPBR's reference code uses.
__device__ __forceinline__ float fresnel_mean(float eta) {
    return logf((10893.0f * eta - 1438.2f) / (-774.4f * eta * eta + 10212.0f * eta + 1.0f));
}

// F82-tint metal: Schlick's curve from F0, pulled down near grazing (82 degrees) toward
// the tint.
__device__ __forceinline__ float4 metal_fresnel(float4 f0, float4 tint, float mu) {
    constexpr float kBar = 1.0f / 7.0f;             // cos of the tint's angle
    const float b5 = 0.46266436f;                   // (1 - kBar)^5
    const float m = 1.0f - mu, m5 = m * m * m * m * m;
    const float4 schlick = f0 + one_minus(f0) * m5;
    const float4 at_bar = f0 + one_minus(f0) * b5;
    const float4 pull = at_bar * one_minus(tint) * (1.0f / (kBar * b5 * (1.0f - kBar)));
    return saturate4(schlick + pull * (-(mu * m5 * m)));
}

__device__ __forceinline__ float3 mirror(float3 i, float3 n) { return i - n * (2.0f * dot(n, i)); }

// Refraction of incident direction i through normal n at ratio eta (near over far); the
// zero vector on total internal reflection.
__device__ __forceinline__ float3 bend(float3 i, float3 n, float eta) {
    const float d = dot(n, i);
    const float k = 1.0f - eta * eta * (1.0f - d * d);
    if (k < 0.0f) return make_float3(0.0f, 0.0f, 0.0f);
    return i * eta - n * (eta * d + sqrtf(k));
}

// ---- directional albedo tables ----------------------------------------------------------
// E_ggx(mu, r): GGX reflection with F = 1; its average over mu; E_dielectric(mu, r, z):
// GGX reflection with a dielectric's Fresnel, the index through z = sqrt(|eta - 1| / (eta +
// 1)). 32 view cosines in [0.02, 1], 32 roughnesses in [0, 1], 16 z in [0, 0.8]; each node
// the mean of F G2 / G1 over a 32 x 32 stratified grid of visible normals (tables.comp's
// nodes, so the tables equal the oracle's within f32 rounding).

constexpr uint32_t kTableMu = 32, kTableRoughness = 32, kTableEta = 16;
constexpr float kTableZMax = 0.8f, kTableMuMin = 0.02f;
constexpr uint32_t kTablePlane = kTableMu * kTableRoughness;
constexpr uint32_t kTableAverage = kTablePlane;                           // after E_ggx
constexpr uint32_t kTableDielectric = kTablePlane + kTableRoughness;      // after the averages
constexpr uint32_t kTableSize = kTableDielectric + kTablePlane * kTableEta;

static __device__ float g_albedo_tables[kTableSize];

__device__ __forceinline__ float eta_at_z(float z) { return (1.0f + z * z) / (1.0f - z * z); }
__device__ __forceinline__ float z_at_eta(float eta) { return sqrtf(fabsf(eta - 1.0f) / (eta + 1.0f)); }
__device__ __forceinline__ float mu_node(uint32_t i) { return lerpf(kTableMuMin, 1.0f, (float)i / (float)(kTableMu - 1u)); }

// Bilinear lookup in the plane at `base` (rows of roughness, columns of mu).
__device__ __forceinline__ float plane_lookup(uint32_t base, float mu, float r) {
    const float fx = fminf(fmaxf((mu - kTableMuMin) / (1.0f - kTableMuMin) * (float)(kTableMu - 1u), 0.0f), (float)(kTableMu - 1u));
    const float fy = fminf(fmaxf(r * (float)(kTableRoughness - 1u), 0.0f), (float)(kTableRoughness - 1u));
    const uint32_t x0 = (uint32_t)fx, y0 = (uint32_t)fy;
    const uint32_t x1 = min(x0 + 1u, kTableMu - 1u), y1 = min(y0 + 1u, kTableRoughness - 1u);
    const float *t = g_albedo_tables + base;
    const float low = lerpf(__ldg(&t[y0 * kTableMu + x0]), __ldg(&t[y0 * kTableMu + x1]), fx - (float)x0);
    const float high = lerpf(__ldg(&t[y1 * kTableMu + x0]), __ldg(&t[y1 * kTableMu + x1]), fx - (float)x0);
    return lerpf(low, high, fy - (float)y0);
}

__device__ __forceinline__ float albedo_ggx(float mu, float r) { return plane_lookup(0u, mu, r); }

__device__ __forceinline__ float albedo_dielectric(float mu, float r, float eta) {
    const float fz = fminf(fmaxf(z_at_eta(eta) / kTableZMax * (float)(kTableEta - 1u), 0.0f), (float)(kTableEta - 1u));
    const uint32_t z0 = (uint32_t)fz, z1 = min(z0 + 1u, kTableEta - 1u);
    return lerpf(plane_lookup(kTableDielectric + z0 * kTablePlane, mu, r),
                 plane_lookup(kTableDielectric + z1 * kTablePlane, mu, r), fz - (float)z0);
}

// One node: the stratified mean of F G2 / G1 over reflected visible normals (eta <= 0:
// F = 1).
__device__ __forceinline__ float albedo_node(float mu, float roughness, float eta) {
    const float3 wo = make_float3(sqrtf(1.0f - mu * mu), 0.0f, mu);
    const Ggx g = ggx_widths(roughness, 0.0f);
    const float g1 = ggx_g1(g, wo);
    float sum = 0.0f;
    for (uint32_t i = 0; i < 32u; i++)
        for (uint32_t j = 0; j < 32u; j++) {
            const float3 h = ggx_visible(g, wo, make_float2(((float)i + 0.5f) / 32.0f, ((float)j + 0.5f) / 32.0f));
            const float3 wi = mirror(-wo, h);
            if (wi.z <= 0.0f) continue;
            sum += (eta > 0.0f ? fresnel(dot(wo, h), eta) : 1.0f) * ggx_g2(g, wi, wo) / g1;
        }
    return sum * (1.0f / 1024.0f);
}

// Pass 0: one thread a node of E_ggx and E_dielectric. Pass 1: one thread a roughness,
// E_ggx's cosine-weighted average over mu (2 * integral of E mu dmu by trapezoids).
static __global__ void albedo_table_kernel(uint32_t pass) {
    const uint32_t id = blockIdx.x * blockDim.x + threadIdx.x;
    if (pass == 0u) {
        if (id >= kTablePlane * (1u + kTableEta)) return;
        const uint32_t layer = id / kTablePlane, at = id % kTablePlane;
        const float mu = mu_node(at % kTableMu), r = (float)(at / kTableMu) / (float)(kTableRoughness - 1u);
        if (layer == 0u) {
            g_albedo_tables[at] = albedo_node(mu, r, -1.0f);
        } else {
            const float eta = eta_at_z(kTableZMax * (float)(layer - 1u) / (float)(kTableEta - 1u));
            g_albedo_tables[kTableDielectric + (layer - 1u) * kTablePlane + at] = albedo_node(mu, r, eta);
        }
        return;
    }
    if (id >= kTableRoughness) return;
    const float *row = g_albedo_tables + id * kTableMu;
    float sum = 0.0f;
    for (uint32_t k = 0; k + 1u < kTableMu; k++) {
        const float a = mu_node(k), b = mu_node(k + 1u);
        sum += 0.5f * (row[k] * a + row[k + 1u] * b) * (b - a);
    }
    g_albedo_tables[kTableAverage + id] = 2.0f * sum;
}

// ---- EON diffuse ------------------------------------------------------------------------

constexpr float kFonA = 0.5f - 2.0f / (3.0f * kPi);               // Fujii's A constant
constexpr float kFonMean = 2.0f / 3.0f - 28.0f / (15.0f * kPi);     // its cosine-weighted mean term

// The single-scattering albedo of Fujii's Oren-Nayar (FON) at cosine mu, roughness r.
__device__ __forceinline__ float fon_albedo(float mu, float r) {
    const float m = 1.0f - mu;
    const float g = m * (0.0571085289f + m * (0.491881867f + m * (-0.332181442f + m * 0.0714429953f)));
    return (1.0f + r * g) / (1.0f + kFonA * r);
}

// EON's f for albedo rho at roughness r (local directions, both above): FON single
// scattering plus the energy its multiple scattering restores.
__device__ __forceinline__ float4 eon(float4 rho, float r, float3 wi, float3 wo) {
    const float s = dot(wi, wo) - wi.z * wo.z;
    const float s_over_t = s > 0.0f ? s / fmaxf(wi.z, wo.z) : s;
    const float a = 1.0f / (1.0f + kFonA * r);
    const float4 single = rho * (a * (1.0f + r * s_over_t) / kPi);
    const float mean = a * (1.0f + kFonMean * r);
    const float k = fmaxf(1e-7f, 1.0f - fon_albedo(wo.z, r)) * fmaxf(1e-7f, 1.0f - fon_albedo(wi.z, r)) /
                    (kPi * fmaxf(1e-7f, 1.0f - mean));
    auto multiple = [&](float p) { return p * p * mean / (1.0f - p * (1.0f - mean)) * k; };
    return single + make_float4(multiple(rho.x), multiple(rho.y), multiple(rho.z), multiple(rho.w));
}

// ---- per-material records ---------------------------------------------------------------

constexpr uint32_t kLobeDiffuse = 0, kLobeGlossy = 1, kLobeTransmission = 2;

// A material as the kernels read it (built on the host once per member).
struct alignas(16) MaterialCode {
    float4 base_fit, base_rgb;    // base colour x base weight; rgb.w: luminance of that
    float4 tint_fit, tint_rgb;    // specular colour; rgb.w: its luminance
    float4 trans_fit, trans_rgb;  // transmission colour; rgb.w: its luminance, at least 0.05
    float4 coat_fit, coat_rgb;    // coat colour; rgb.w: its luminance
    float4 glow_fit, glow_rgb;    // emission colour x luminance; rgb.w: the luminance (> 0 emits)
    float4 weights;    // metalness, specular weight, transmission, coat (each clamped)
    float4 rough;      // diffuse roughness, specular roughness, coat roughness, coat darkening
    float4 coated;     // base under the coat: GGX widths x, y; index relative to the coat's; its mean Fresnel
    float4 bare;       // base with no coat above: the same four
    float4 coat_lobe;  // coat GGX widths x, y; coat index; its mean Fresnel
    float4 extra;      // cut-out opacity; Cauchy's dispersion coefficient; the base's index; specular anisotropy
};

// ---- a hit's layered surface ------------------------------------------------------------

struct Layers {
    float3 n, t, b, g;  // shading frame and geometric normal, facing the side seen from
    uint32_t material;
    bool back, inside;  // behind the triangle's front face; inside a transmissive object
    // the material on this side
    float metal, spec_w, trans, coat, dark, diffuse_r, spec_r, coat_r;
    Ggx base_lobe, coat_lobe;
    float ior, eta, coat_eta, mean_f, coat_mean_f;
    float lum_base, lum_spec, lum_trans, lum_coat;
    // for the view direction
    float comp_dielectric, missing, spec_albedo, comp_coat, coat_albedo, coat_k;
    float p_coat, p_metal, p_spec, p_trans, p_diffuse;
    // at the path's wavelengths
    float4 base, tint, spec_tint, trans_tint, coat_tint, substrate;

    __device__ __forceinline__ float3 local(float3 v) const { return make_float3(dot(v, t), dot(v, b), dot(v, n)); }
    __device__ __forceinline__ float3 world(float3 v) const { return t * v.x + b * v.y + n * v.z; }
};

__device__ __forceinline__ float luma(float3 c) { return c.x * 0.2722287168f + c.y * 0.6740817658f + c.z * 0.0536895174f; }

// Cauchy's index at `nm` through `ior` at 587.6 nm.
__device__ __forceinline__ float cauchy_ior(float ior, float b, float nm) {
    return ior + b * (1.0f / (nm * nm) - 1.0f / (587.6f * 587.6f));
}

// The material's values on the side the surface is seen from. `hero`: the path's hero
// wavelength once a dispersive material has ended the others (0 before), at which a
// dispersive base's index is taken.
__device__ __forceinline__ void open_layers(Layers &s, const MaterialCode &c, float hero) {
    const float4 w = __ldg(&c.weights), r = __ldg(&c.rough);
    s.metal = w.x;
    s.spec_w = w.y;
    s.trans = w.z;
    s.inside = s.back && s.trans > 0.0f;      // only a transmissive object has an inside
    s.coat = s.inside ? 0.0f : w.w;           // whose layers face the outside
    s.diffuse_r = r.x;
    s.coat_r = r.z;
    s.dark = r.w;
    const float4 lobe = __ldg(s.coat > 0.0f ? &c.coated : &c.bare);
    const float4 cl = __ldg(&c.coat_lobe);
    s.base_lobe = Ggx{lobe.x, lobe.y};
    s.coat_lobe = s.coat > 0.0f ? Ggx{cl.x, cl.y} : Ggx{1.0f, 1.0f};
    s.coat_eta = cl.z;
    s.coat_mean_f = cl.w;
    s.ior = lobe.z;
    s.mean_f = lobe.w;
    // The base's roughness under the coat (its lobe widths above are the same mix).
    const float r4 = r.y * r.y * r.y * r.y, c4 = r.z * r.z * r.z * r.z;
    s.spec_r = s.coat > 0.0f ? lerpf(r.y, fminf(1.0f, sqrtf(sqrtf(r4 + 2.0f * c4))), s.coat) : r.y;
    const float4 extra = __ldg(&c.extra);
    if (extra.y != 0.0f && hero > 0.0f) {
        const float eta = fmaxf(cauchy_ior(extra.z, extra.y, hero), 1.0001f);
        float relative = eta / s.coat_eta;
        if (relative < 1.0f) relative = 1.0f / relative;
        s.ior = fmaxf(lerpf(eta, relative, s.coat), 1.0001f);
        s.mean_f = fresnel_mean(s.ior);
    }
    s.eta = s.inside ? 1.0f / s.ior : s.ior;
    s.lum_base = __ldg(&c.base_rgb).w;
    s.lum_spec = __ldg(&c.tint_rgb).w;
    s.lum_trans = __ldg(&c.trans_rgb).w;
    s.lum_coat = __ldg(&c.coat_rgb).w;
}

// The lobe choice from what reaches under the coat (`under`, a luminance) and the
// specular and coat albedos: each lobe's share of the light it may return.
__device__ __forceinline__ void weigh_lobes(Layers &s, float under, float spec_albedo, float coat_albedo) {
    const float dielectric = 1.0f - s.metal;
    float w_coat = s.coat * coat_albedo;
    float w_metal = under * s.metal;
    float w_spec = under * dielectric * spec_albedo * s.lum_spec;
    float w_trans = under * dielectric * s.trans * (1.0f - spec_albedo) * s.lum_trans;
    float w_diffuse = under * dielectric * (1.0f - s.trans) * (1.0f - spec_albedo) * s.lum_base;
    if (s.inside) {  // from within: the interface alone
        w_metal = w_diffuse = 0.0f;
        w_spec = fmaxf(w_spec, 0.05f);
        w_trans = fmaxf(w_trans, s.trans > 0.0f ? 0.05f : 0.0f);
    }
    const float total = w_coat + w_metal + w_spec + w_trans + w_diffuse;
    const float inv = total > 0.0f ? 1.0f / total : 0.0f;
    s.p_coat = w_coat * inv;
    s.p_metal = w_metal * inv;
    s.p_spec = w_spec * inv;
    s.p_trans = w_trans * inv;
    s.p_diffuse = w_diffuse * inv;
}

// The layers as seen along wo (local): the albedos f needs and the lobe choice.
__device__ __forceinline__ void view_layers(Layers &s, float3 wo) {
    const float mu = clamp01(wo.z);
    s.comp_coat = 1.0f;
    s.coat_albedo = 0.0f;
    if (s.coat > 0.0f) {
        const float e = fmaxf(albedo_ggx(mu, s.coat_r), 1e-4f);
        s.comp_coat = 1.0f + s.coat_mean_f * (1.0f - e) / e;
        s.coat_albedo = clamp01(s.comp_coat * albedo_dielectric(mu, s.coat_r, s.coat_eta));
    }
    const float e = fmaxf(albedo_ggx(mu, s.spec_r), 1e-4f);
    s.missing = (1.0f - e) / e;
    s.comp_dielectric = 1.0f + s.mean_f * s.missing;
    s.spec_albedo = clamp01(s.spec_w * s.comp_dielectric * albedo_dielectric(mu, s.spec_r, s.ior));
    float under = 1.0f;
    s.coat_k = 0.0f;
    if (s.coat > 0.0f) {
        // What the coat sends back down: Fresnel at the view for a smooth base, the
        // hemispherical internal average for a rough one.
        const float smooth = fresnel(mu, s.coat_eta);
        const float rough = 1.0f - (1.0f - s.coat_mean_f) / (s.coat_eta * s.coat_eta);
        s.coat_k = lerpf(smooth, rough, lerpf(1.0f, s.spec_r, s.metal));
        const float darker = (1.0f - s.coat_k) / fmaxf(1e-4f, 1.0f - s.lum_base * s.coat_k);
        under = lerpf(1.0f, s.lum_coat * (1.0f - s.coat_albedo) * lerpf(1.0f, darker, s.dark), s.coat);
    }
    weigh_lobes(s, under, s.spec_albedo, s.coat_albedo);
}

// What reaches the layers under the coat, at the path's wavelengths.
__device__ __forceinline__ void coat_filter(Layers &s) {
    s.substrate = fill4(1.0f);
    if (s.coat > 0.0f) {
        const float4 k = fill4(s.coat_k);
        const float4 darker = make_float4((1.0f - k.x) / (1.0f - s.base.x * k.x), (1.0f - k.y) / (1.0f - s.base.y * k.y),
                                          (1.0f - k.z) / (1.0f - s.base.z * k.z), (1.0f - k.w) / (1.0f - s.base.w * k.w));
        const float4 under = s.coat_tint * (1.0f - s.coat_albedo) * lerp4(fill4(1.0f), darker, s.dark);
        s.substrate = lerp4(fill4(1.0f), under, s.coat);
    }
}

template <bool kSpectral>
__device__ __forceinline__ void colour_layers(Layers &s, const MaterialCode &c, float4 lambda) {
    s.base = spec_of<kSpectral>(__ldg(&c.base_fit), xyz(__ldg(&c.base_rgb)), lambda);
    s.tint = spec_of<kSpectral>(__ldg(&c.tint_fit), xyz(__ldg(&c.tint_rgb)), lambda);
    s.spec_tint = s.tint * s.spec_w;
    s.trans_tint = spec_of<kSpectral>(__ldg(&c.trans_fit), xyz(__ldg(&c.trans_rgb)), lambda);
    s.coat_tint = s.coat > 0.0f ? spec_of<kSpectral>(__ldg(&c.coat_fit), xyz(__ldg(&c.coat_rgb)), lambda) : fill4(1.0f);
}

// The surface at a hit: shading normal n and geometric g facing the side it is seen
// from (`back`: behind the triangle's front face), opened, viewed along wo and coloured.
template <bool kSpectral>
__device__ __forceinline__ Layers layers_at(float3 n, float3 g, uint32_t material, bool back, const MaterialCode *codes,
                                            float3 wo_world, float4 lambda, float3 &wo) {
    Layers s;
    s.n = n;
    basis(n, s.t, s.b);
    s.g = g;
    s.material = material;
    s.back = back;
    const float hero = kSpectral && lambda.y < 0.0f ? lambda.x : 0.0f;
    open_layers(s, codes[material], hero);
    wo = s.local(wo_world);
    view_layers(s, wo);
    colour_layers<kSpectral>(s, codes[material], lambda);
    coat_filter(s);
    return s;
}

// The choice light paths sample with (Fresnel at normal incidence, so it holds for every
// direction).
__device__ __forceinline__ void light_path_lobes(Layers &s) {
    const float f0 = (s.ior - 1.0f) / (s.ior + 1.0f);
    const float spec_albedo = clamp01(s.spec_w * f0 * f0);
    float coat_albedo = 0.0f;
    if (s.coat > 0.0f) {
        const float c0 = (s.coat_eta - 1.0f) / (s.coat_eta + 1.0f);
        coat_albedo = c0 * c0;
    }
    weigh_lobes(s, lerpf(1.0f, s.lum_coat * (1.0f - coat_albedo), s.coat), spec_albedo, coat_albedo);
}

// The half vector of a refraction of wo into wi (opposite sides, ratio eta), turned to
// +z; false when it does not separate them.
__device__ __forceinline__ bool refraction_half(float3 wi, float3 wo, float eta, float3 &h) {
    h = normalize(wo + wi * eta);
    if (h.z < 0.0f) h = -h;
    return dot(wo, h) > 0.0f && dot(wi, h) < 0.0f;
}

// The density of sampling wi for wo over all lobes.
__device__ __forceinline__ float layers_pdf(const Layers &s, float3 wi, float3 wo) {
    if (wo.z <= 0.0f || wi.z == 0.0f) return 0.0f;
    if (wi.z < 0.0f) {
        if (s.p_trans <= 0.0f) return 0.0f;
        float3 h;
        if (!refraction_half(wi, wo, s.eta, h)) return 0.0f;
        const float oh = dot(wo, h), ih = dot(wi, h);
        const float den = oh + s.eta * ih;
        return s.p_trans * ggx_g1(s.base_lobe, wo) * ggx_d(s.base_lobe, h) * oh / wo.z *
               (s.eta * s.eta * fabsf(ih) / (den * den));
    }
    const float3 h = normalize(wi + wo);
    float pdf = (s.p_spec + s.p_metal) * ggx_reflection_pdf(s.base_lobe, wo, h);
    if (s.p_coat > 0.0f) pdf += s.p_coat * ggx_reflection_pdf(s.coat_lobe, wo, h);
    if (!s.inside) pdf += s.p_diffuse * wi.z / kPi;
    return pdf;
}

// f (no cosine) for wi, wo, and the density of sampling wi.
__device__ __forceinline__ float4 layers_f(const Layers &s, float3 wi, float3 wo, float &pdf) {
    pdf = 0.0f;
    if (wo.z <= 0.0f || wi.z == 0.0f) return fill4(0.0f);
    pdf = layers_pdf(s, wi, wo);
    const float dielectric = 1.0f - s.metal;
    if (wi.z < 0.0f) {  // through the interface
        if (s.p_trans <= 0.0f) return fill4(0.0f);
        float3 h;
        if (!refraction_half(wi, wo, s.eta, h)) return fill4(0.0f);
        const float oh = dot(wo, h), ih = dot(wi, h);
        const float den = oh + s.eta * ih;
        const float f = (1.0f - fresnel(oh, s.eta)) * ggx_d(s.base_lobe, h) * ggx_g2(s.base_lobe, -wi, wo) * fabsf(ih) *
                        oh / (fabsf(wi.z) * wo.z * den * den);
        return s.substrate * s.trans_tint * (dielectric * s.trans * f);
    }
    const float3 h = normalize(wi + wo);
    const float oh = dot(wo, h);
    float4 top = fill4(0.0f);
    if (s.p_coat > 0.0f) {
        const float spike = ggx_d(s.coat_lobe, h) * ggx_g2(s.coat_lobe, wi, wo) / (4.0f * wi.z * wo.z);
        top = fill4(s.coat * fresnel(oh, s.coat_eta) * s.comp_coat * spike);
    }
    const float spike = ggx_d(s.base_lobe, h) * ggx_g2(s.base_lobe, wi, wo) / (4.0f * wi.z * wo.z);
    float4 under = fill4(0.0f);
    if (!s.inside) under = eon(s.base, s.diffuse_r, wi, wo) * (dielectric * (1.0f - s.trans) * (1.0f - s.spec_albedo));
    if (dielectric > 0.0f) under = under + s.spec_tint * (dielectric * fresnel(oh, s.eta) * s.comp_dielectric * spike);
    if (s.metal > 0.0f && !s.inside) {
        // Kulla-Conty for a coloured conductor: 1 + F_avg (1 - E) / E with F_avg from F0
        // (the closed form (20 F0 + 1) / 21 for Schlick's curve).
        const float4 mean = (s.base * 20.0f + fill4(1.0f)) * (1.0f / 21.0f);
        const float4 boost = fill4(1.0f) + mean * s.missing;
        const float4 fm = metal_fresnel(s.base, s.tint, oh) * s.spec_w;
        under = under + make_float4(fminf(1.0f, fm.x), fminf(1.0f, fm.y), fminf(1.0f, fm.z), fminf(1.0f, fm.w)) * boost *
                            (s.metal * spike);
    }
    return top + s.substrate * under;
}

// A direction for wo from u.xy, the lobe picked by u.z (cumulative: diffuse, coat,
// specular and metal, transmission); its density over all lobes and the lobe kind.
__device__ __forceinline__ bool layers_sample(const Layers &s, float3 wo, float3 u, float3 &wi, float &pdf,
                                              uint32_t &lobe) {
    pdf = 0.0f;
    if (wo.z <= 0.0f) return false;
    const float2 uv = make_float2(u.x, u.y);
    float pick = u.z;
    if (pick < s.p_diffuse) {
        const float2 d = concentric(uv);
        wi = make_float3(d.x, d.y, sqrtf(fmaxf(0.0f, 1.0f - (d.x * d.x + d.y * d.y))));
        lobe = kLobeDiffuse;
    } else if ((pick -= s.p_diffuse) < s.p_coat) {
        wi = mirror(-wo, ggx_visible(s.coat_lobe, wo, uv));
        lobe = kLobeGlossy;
    } else if ((pick -= s.p_coat) < s.p_spec + s.p_metal) {
        wi = mirror(-wo, ggx_visible(s.base_lobe, wo, uv));
        lobe = kLobeGlossy;
    } else if (s.p_trans > 0.0f) {
        wi = bend(-wo, ggx_visible(s.base_lobe, wo, uv), 1.0f / s.eta);
        if (dot(wi, wi) == 0.0f) return false;
        lobe = kLobeTransmission;
    } else {
        return false;
    }
    if (wi.z == 0.0f) return false;
    pdf = layers_pdf(s, wi, wo);
    return pdf > 0.0f;
}

// The density the light sampler at this point gives `to` when a light path arrived from
// `from` (world, unit, both leaving the point): the surface seen from `from`'s side
// (opened again when that is the other side), with the light paths' lobe choice; zero
// where the sampler would reject `to`.
__device__ __forceinline__ float layers_light_pdf(const Layers &s, float3 from, float3 to, const MaterialCode *codes,
                                                  float hero) {
    Layers v = s;
    if (dot(from, s.g) < 0.0f) {
        v.n = -s.n;
        v.g = -s.g;
        basis(v.n, v.t, v.b);
        v.back = !s.back;
        open_layers(v, codes[s.material], hero);
    }
    const float3 wo = v.local(from), wi = v.local(to);
    if ((dot(to, v.g) > 0.0f) != (wi.z > 0.0f)) return 0.0f;
    light_path_lobes(v);
    return layers_pdf(v, wi, wo);
}

// ---- all-diffuse members ----------------------------------------------------------------

// EON diffuse alone (the layered surface with no specular, metal, coat or transmission
// weight): chosen with probability 1 when its albedo's luminance is positive, else never.
struct DiffuseSurface {
    float3 n, t, b;
    float4 albedo;
    float roughness, chance;

    __device__ __forceinline__ float3 local(float3 v) const { return make_float3(dot(v, t), dot(v, b), dot(v, n)); }
    __device__ __forceinline__ float3 world(float3 v) const { return t * v.x + b * v.y + n * v.z; }
};

template <bool kSpectral>
__device__ __forceinline__ DiffuseSurface diffuse_at(float3 n, const MaterialCode &c, float4 lambda) {
    DiffuseSurface s;
    s.n = n;
    basis(n, s.t, s.b);
    const float4 rgb = __ldg(&c.base_rgb);
    s.albedo = spec_of<kSpectral>(__ldg(&c.base_fit), xyz(rgb), lambda);
    s.roughness = __ldg(&c.rough).x;
    s.chance = rgb.w > 0.0f ? 1.0f : 0.0f;
    return s;
}

// The density the light sampler gives `to` at an all-diffuse point (normal n, geometric
// g) when a light path arrived from `from`.
__device__ __forceinline__ float diffuse_light_pdf(float chance, float3 n, float3 g, float3 from, float3 to) {
    const bool front = dot(from, g) >= 0.0f;
    const float3 nv = front ? n : -n, gv = front ? g : -g;
    const float out_z = dot(from, nv), in_z = dot(to, nv);
    if ((dot(to, gv) > 0.0f) != (in_z > 0.0f)) return 0.0f;
    if (out_z <= 0.0f || in_z <= 0.0f) return 0.0f;
    return chance * in_z / kPi;
}

}  // namespace lr
