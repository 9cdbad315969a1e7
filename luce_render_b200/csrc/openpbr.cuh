// OpenPBR Surface's layered lobes on the device (shaders/openpbr.glsl:196-556,
// microfacet.glsl:1-120): an F82-tint metal and a GGX dielectric specular over EON diffuse,
// rough refraction into transmissive objects, a GGX coat with darkening, each microfacet
// lobe compensated for multiple scattering by albedo tables made on the device
// (albedo_table_kernel). Spectra are float4 lanes (hero wavelengths or RGB). Material records
// are 16 float4s as the reference packs them (loading.cpp `pack_material`).
#pragma once

#include "shading.cuh"

namespace lr {

// ---- GGX (microfacet.glsl) -----------------------------------------------------------

__device__ __forceinline__ float2 ggx_alpha(float roughness, float anisotropy) {
    const float r2 = roughness * roughness;
    const float t = r2 * sqrtf(2.0f / (1.0f + (1.0f - anisotropy) * (1.0f - anisotropy)));
    return make_float2(fmaxf(t, 1e-4f), fmaxf((1.0f - anisotropy) * t, 1e-4f));
}

__device__ __forceinline__ float ggx_d(float3 m, float2 alpha) {
    if (m.z <= 0.0f) return 0.0f;
    const float3 s = make_float3(m.x / alpha.x, m.y / alpha.y, m.z);
    const float k = dot(s, s);
    return 1.0f / (kPi * alpha.x * alpha.y * k * k);
}

__device__ __forceinline__ float ggx_lambda(float3 v, float2 alpha) {
    const float z2 = v.z * v.z;
    if (z2 <= 0.0f) return kInfinity;
    const float a2 = (alpha.x * alpha.x * v.x * v.x + alpha.y * alpha.y * v.y * v.y) / z2;
    return 0.5f * (-1.0f + sqrtf(1.0f + a2));
}

__device__ __forceinline__ float ggx_g1(float3 v, float2 alpha) { return 1.0f / (1.0f + ggx_lambda(v, alpha)); }
__device__ __forceinline__ float ggx_g2(float3 wi, float3 wo, float2 alpha) {
    return 1.0f / (1.0f + ggx_lambda(wi, alpha) + ggx_lambda(wo, alpha));
}

// A visible normal for wo (above the surface) by spherical caps (Dupuy and Benyoub 2023).
__device__ __forceinline__ float3 ggx_sample(float3 wo, float2 alpha, float2 u) {
    const float3 v = normalize(make_float3(wo.x * alpha.x, wo.y * alpha.y, wo.z));
    const float phi = 2.0f * kPi * u.x;
    const float z = (1.0f - u.y) * (1.0f + v.z) - v.z;
    const float s = sqrtf(fminf(fmaxf(1.0f - z * z, 0.0f), 1.0f));
    float sp, cp;
    sincosf(phi, &sp, &cp);
    const float3 h = make_float3(s * cp, s * sp, z) + v;
    return normalize(make_float3(h.x * alpha.x, h.y * alpha.y, fmaxf(h.z, 1e-6f)));
}

__device__ __forceinline__ float ggx_reflection_pdf(float3 wo, float3 h, float2 alpha) {
    return ggx_g1(wo, alpha) * ggx_d(h, alpha) / (4.0f * wo.z);
}

// Unpolarized Fresnel reflectance of a dielectric interface (eta: transmitted over incident).
__device__ __forceinline__ float fresnel_dielectric(float cos_i, float eta) {
    const float c = fabsf(cos_i);
    const float g2 = eta * eta - 1.0f + c * c;
    if (g2 <= 0.0f) return 1.0f;
    const float g = sqrtf(g2);
    const float a = (g - c) / (g + c);
    const float b = (c * (g + c) - 1.0f) / (c * (g - c) + 1.0f);
    return 0.5f * a * a * (1.0f + b * b);
}

// Its hemispherical average, by the closed fit OpenPBR's reference uses (eta > 1).
__device__ __forceinline__ float fresnel_dielectric_average(float eta) {
    return logf((10893.0f * eta - 1438.2f) / (-774.4f * eta * eta + 10212.0f * eta + 1.0f));
}

__device__ __forceinline__ float3 reflect_about(float3 i, float3 n) { return i - n * (2.0f * dot(n, i)); }

// GLSL's refract: the zero vector on total internal reflection.
__device__ __forceinline__ float3 refract_through(float3 i, float3 n, float eta) {
    const float d = dot(n, i);
    const float k = 1.0f - eta * eta * (1.0f - d * d);
    if (k < 0.0f) return make_float3(0.0f, 0.0f, 0.0f);
    return i * eta - n * (eta * d + sqrtf(k));
}

__device__ __forceinline__ float mixf(float a, float b, float t) { return a * (1.0f - t) + b * t; }
__device__ __forceinline__ float4 mix4(float4 a, float4 b, float t) { return a * (1.0f - t) + b * t; }
__device__ __forceinline__ float4 splat4(float v) { return make_float4(v, v, v, v); }
__device__ __forceinline__ float4 clamp01(float4 v) {
    return make_float4(fminf(fmaxf(v.x, 0.0f), 1.0f), fminf(fmaxf(v.y, 0.0f), 1.0f), fminf(fmaxf(v.z, 0.0f), 1.0f),
                       fminf(fmaxf(v.w, 0.0f), 1.0f));
}
__device__ __forceinline__ float4 min4(float4 a, float4 b) {
    return make_float4(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z), fminf(a.w, b.w));
}
__device__ __forceinline__ float4 div4(float4 a, float4 b) { return make_float4(a.x / b.x, a.y / b.y, a.z / b.z, a.w / b.w); }
__device__ __forceinline__ float4 sub4(float a, float4 b) { return make_float4(a - b.x, a - b.y, a - b.z, a - b.w); }

// ---- Albedo tables (microfacet.glsl:96-120, openpbr.glsl:126-150) ---------------------

constexpr uint32_t kTableMu = 32, kTableRoughness = 32, kTableEta = 16;
constexpr float kTableZMax = 0.8f, kTableMuMin = 0.02f;
constexpr uint32_t kTableGgx = 0;                                          // E(mu, r): GGX, F = 1
constexpr uint32_t kTableGgxAverage = kTableMu * kTableRoughness;          // Eavg(r)
constexpr uint32_t kTableDielectric = kTableGgxAverage + kTableRoughness;  // E(mu, r, z): GGX x Fresnel
constexpr uint32_t kTableSize = kTableDielectric + kTableMu * kTableRoughness * kTableEta;

__device__ __forceinline__ float eta_of_z(float z) { return (1.0f + z * z) / (1.0f - z * z); }
__device__ __forceinline__ float z_of_eta(float eta) { return sqrtf(fabsf(eta - 1.0f) / (eta + 1.0f)); }
__device__ __forceinline__ float table_mu(uint32_t i) {
    return mixf(kTableMuMin, 1.0f, (float)i / (float)(kTableMu - 1u));
}
__device__ __forceinline__ float table_roughness(uint32_t i) { return (float)i / (float)(kTableRoughness - 1u); }
__device__ __forceinline__ float table_z(uint32_t i) { return kTableZMax * (float)i / (float)(kTableEta - 1u); }

__device__ __forceinline__ float table_row(const float *t, uint32_t base, float r, float mu) {
    const float x = fminf(fmaxf((mu - kTableMuMin) / (1.0f - kTableMuMin) * (float)(kTableMu - 1u), 0.0f), (float)(kTableMu - 1u));
    const float y = fminf(fmaxf(r * (float)(kTableRoughness - 1u), 0.0f), (float)(kTableRoughness - 1u));
    const uint32_t x0 = (uint32_t)x, y0 = (uint32_t)y;
    const uint32_t x1 = min(x0 + 1u, kTableMu - 1u), y1 = min(y0 + 1u, kTableRoughness - 1u);
    const float fx = x - (float)x0, fy = y - (float)y0;
    const float a = mixf(__ldg(&t[base + y0 * kTableMu + x0]), __ldg(&t[base + y0 * kTableMu + x1]), fx);
    const float b = mixf(__ldg(&t[base + y1 * kTableMu + x0]), __ldg(&t[base + y1 * kTableMu + x1]), fx);
    return mixf(a, b, fy);
}

__device__ __forceinline__ float table_ggx(const float *t, float mu, float r) { return table_row(t, kTableGgx, r, mu); }

__device__ __forceinline__ float table_dielectric(const float *t, float mu, float r, float eta) {
    const float z = fminf(fmaxf(z_of_eta(eta) / kTableZMax * (float)(kTableEta - 1u), 0.0f), (float)(kTableEta - 1u));
    const uint32_t z0 = (uint32_t)z, z1 = min((uint32_t)z + 1u, kTableEta - 1u);
    const uint32_t plane = kTableMu * kTableRoughness;
    return mixf(table_row(t, kTableDielectric + z0 * plane, r, mu), table_row(t, kTableDielectric + z1 * plane, r, mu),
                z - (float)z0);
}

// What one table node holds: the mean of F G2 / G1 over a 32 x 32 stratified grid of
// visible normals (tables.comp:20-35); eta <= 0 for F = 1.
__device__ __forceinline__ float table_albedo(float mu, float roughness, float eta) {
    const float3 wo = make_float3(sqrtf(1.0f - mu * mu), 0.0f, mu);
    const float2 alpha = ggx_alpha(roughness, 0.0f);
    float sum = 0.0f;
    for (uint32_t i = 0; i < 32u; i++)
        for (uint32_t j = 0; j < 32u; j++) {
            const float2 u = make_float2(((float)i + 0.5f) / 32.0f, ((float)j + 0.5f) / 32.0f);
            const float3 h = ggx_sample(wo, alpha, u);
            const float3 wi = reflect_about(-wo, h);
            if (wi.z <= 0.0f) continue;
            const float f = eta > 0.0f ? fresnel_dielectric(dot(wo, h), eta) : 1.0f;
            sum += f * ggx_g2(wi, wo, alpha) / ggx_g1(wo, alpha);
        }
    return sum / 1024.0f;
}

// The tables, one copy a device, made once by albedo_table_kernel.
__device__ float g_albedo_tables[kTableSize];

// tables.comp:38-61: phase 0, one thread a node of E_ggx and E_dielectric; phase 1, one a
// roughness of E_ggx's average over mu (2 * integral of E mu dmu, trapezoids on the nodes).
__global__ void albedo_table_kernel(uint32_t phase) {
    const uint32_t cell = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t plane = kTableMu * kTableRoughness;
    if (phase == 0u) {
        if (cell >= plane * (1u + kTableEta)) return;
        const uint32_t layer = cell / plane, at = cell % plane;
        const float mu = table_mu(at % kTableMu), roughness = table_roughness(at / kTableMu);
        if (layer == 0u) g_albedo_tables[kTableGgx + at] = table_albedo(mu, roughness, -1.0f);
        else g_albedo_tables[kTableDielectric + (layer - 1u) * plane + at] = table_albedo(mu, roughness, eta_of_z(table_z(layer - 1u)));
        return;
    }
    if (cell >= kTableRoughness) return;
    float sum = 0.0f;
    for (uint32_t m = 0; m + 1u < kTableMu; m++) {
        const float a = table_mu(m), b = table_mu(m + 1u);
        sum += 0.5f * (g_albedo_tables[kTableGgx + cell * kTableMu + m] * a + g_albedo_tables[kTableGgx + cell * kTableMu + m + 1u] * b) * (b - a);
    }
    g_albedo_tables[kTableGgxAverage + cell] = 2.0f * sum;
}

// ---- F82-tint metal Fresnel (openpbr.glsl:152-161) ------------------------------------

__device__ __forceinline__ float4 fresnel_f82(float4 f0, float4 tint, float mu) {
    const float bar = 1.0f / 7.0f;
    const float m = 1.0f - mu;
    const float m5 = m * m * m * m * m;
    const float b5 = powf(1.0f - bar, 5.0f);
    const float4 schlick = f0 + sub4(1.0f, f0) * m5;
    const float4 schlick_bar = f0 + sub4(1.0f, f0) * b5;
    const float4 a = schlick_bar * sub4(1.0f, tint) * (1.0f / (bar * b5 * (1.0f - bar)));
    return clamp01(schlick + a * (-(mu * m5 * m)));
}

// ---- The surface at a hit (openpbr.glsl:196-420) --------------------------------------

constexpr uint32_t kLobeDiffuse = 0, kLobeGlossy = 1, kLobeTransmission = 2;

struct Surface {
    float3 normal, tangent, bitangent, geometric;  // facing the side it is seen from
    uint32_t material;
    bool back, inside;
    float diffuse_roughness, metalness, specular_weight, transmission, roughness, coat_roughness, ior, darkening;
    float lum_base, lum_specular, lum_transmission, lum_coat;
    float2 alpha;
    float eta, coat;
    float2 coat_alpha;
    float coat_eta;
    float dielectric_compensation, metal_missing, specular_albedo, coat_compensation, coat_albedo, coat_k;
    float p_coat, p_metal, p_specular, p_transmission, p_diffuse;
    float4 base, metal_tint, specular_tint, transmission_tint, coat_tint, substrate;
};

__device__ __forceinline__ float3 to_local(const Surface &s, float3 v) {
    return make_float3(dot(v, s.tangent), dot(v, s.bitangent), dot(v, s.normal));
}
__device__ __forceinline__ float3 to_world(const Surface &s, float3 v) {
    return s.tangent * v.x + s.bitangent * v.y + s.normal * v.z;
}

__device__ __forceinline__ Surface surface_at(float3 normal, float3 geometric, uint32_t material, bool back) {
    Surface s;
    s.normal = normal;
    basis(normal, s.tangent, s.bitangent);
    s.geometric = geometric;
    s.material = material;
    s.back = back;
    return s;
}

// The same point seen from its other side (a refracted direction's viewer); read again.
__device__ __forceinline__ Surface turned(const Surface &s) {
    return surface_at(-s.normal, -s.geometric, s.material, !s.back);
}

__device__ __forceinline__ float rgb_luma(float3 c) {
    return c.x * 0.2722287168f + c.y * 0.6740817658f + c.z * 0.0536895174f;
}

// Cauchy's index at `lambda` nm through `ior` at 587.6 nm (openpbr.glsl:177-180).
__device__ __forceinline__ float dispersed_ior(float ior, float b, float lambda) {
    return ior + b * (1.0f / (lambda * lambda) - 1.0f / (587.6f * 587.6f));
}

// read_material (openpbr.glsl:264-320) without node graphs. `hero`: the path's hero
// wavelength once a dispersive hit has ended the others (0 before), at which a
// dispersive material's index is taken.
__device__ __forceinline__ void read_material(Surface &s, const float4 *materials, float hero = 0.0f) {
    const float4 *row = materials + (size_t)s.material * 16u;
    const float4 base_rgb = __ldg(&row[1]), specular_rgb = __ldg(&row[3]), coat_rgb = __ldg(&row[5]);
    const float4 transmission_rgb = __ldg(&row[9]), scalars = __ldg(&row[10]), indices = __ldg(&row[11]);
    const float4 geometry = __ldg(&row[12]);
    s.diffuse_roughness = scalars.y;
    s.metalness = fminf(fmaxf(scalars.x, 0.0f), 1.0f);
    s.specular_weight = fmaxf(specular_rgb.w, 0.0f);
    s.transmission = fminf(fmaxf(transmission_rgb.w, 0.0f), 1.0f);
    s.inside = s.back && s.transmission > 0.0f;
    s.coat = !s.inside ? fminf(fmaxf(coat_rgb.w, 0.0f), 1.0f) : 0.0f;
    s.coat_roughness = fminf(fmaxf(indices.y, 0.0f), 1.0f);
    s.coat_eta = fmaxf(indices.z, 1.0001f);
    s.coat_alpha = make_float2(1.0f, 1.0f);
    if (s.coat > 0.0f) s.coat_alpha = ggx_alpha(s.coat_roughness, fminf(fmaxf(geometry.z, 0.0f), 1.0f));
    s.darkening = fminf(fmaxf(indices.w, 0.0f), 1.0f);
    const float roughness = fminf(fmaxf(scalars.z, 0.0f), 1.0f);
    const float r4 = roughness * roughness * roughness * roughness;
    const float c4 = s.coat_roughness * s.coat_roughness * s.coat_roughness * s.coat_roughness;
    s.roughness = mixf(roughness, fminf(1.0f, powf(r4 + 2.0f * c4, 0.25f)), s.coat);
    s.alpha = ggx_alpha(s.roughness, fminf(fmaxf(scalars.w, 0.0f), 1.0f));
    float eta = fmaxf(indices.x, 1.0001f);
    if (geometry.w != 0.0f && hero > 0.0f) eta = fmaxf(dispersed_ior(eta, geometry.w, hero), 1.0001f);
    float relative = eta / s.coat_eta;
    if (relative < 1.0f) relative = 1.0f / relative;
    s.ior = fmaxf(mixf(eta, relative, s.coat), 1.0001f);
    s.eta = s.inside ? 1.0f / s.ior : s.ior;
    s.lum_base = fmaxf(rgb_luma(xyz(base_rgb) * base_rgb.w), 0.0f);
    s.lum_specular = fmaxf(rgb_luma(xyz(specular_rgb)), 0.0f);
    s.lum_transmission = fmaxf(rgb_luma(xyz(transmission_rgb)), 0.05f);
    s.lum_coat = rgb_luma(xyz(coat_rgb));
}

// The lobe choice shared by orient_lobes and light_lobes (openpbr.glsl:352-370, 433-449).
__device__ __forceinline__ void choose_lobes(Surface &s, float substrate_rgb, float specular_albedo, float coat_albedo) {
    const float dielectric = 1.0f - s.metalness;
    const float w_coat = s.coat * coat_albedo;
    float w_metal = substrate_rgb * s.metalness;
    float w_specular = substrate_rgb * dielectric * specular_albedo * s.lum_specular;
    float w_transmission = substrate_rgb * dielectric * s.transmission * (1.0f - specular_albedo) * s.lum_transmission;
    float w_diffuse = substrate_rgb * dielectric * (1.0f - s.transmission) * (1.0f - specular_albedo) * s.lum_base;
    if (s.inside) {
        w_metal = 0.0f;
        w_diffuse = 0.0f;
        w_specular = fmaxf(w_specular, 0.05f);
        w_transmission = fmaxf(w_transmission, s.transmission > 0.0f ? 0.05f : 0.0f);
    }
    const float total = w_coat + w_metal + w_specular + w_transmission + w_diffuse;
    const float scale = total > 0.0f ? 1.0f / total : 0.0f;
    s.p_coat = w_coat * scale;
    s.p_metal = w_metal * scale;
    s.p_specular = w_specular * scale;
    s.p_transmission = w_transmission * scale;
    s.p_diffuse = w_diffuse * scale;
}

// orient_lobes (openpbr.glsl:323-370): the albedos f needs and the lobe choice for wo.
__device__ __forceinline__ void orient_lobes(Surface &s, float3 wo) {
    const float *tables = g_albedo_tables;
    const float mu = fminf(fmaxf(wo.z, 0.0f), 1.0f);
    s.coat_compensation = 1.0f;
    s.coat_albedo = 0.0f;
    if (s.coat > 0.0f) {
        const float e_coat_ggx = fmaxf(table_ggx(tables, mu, s.coat_roughness), 1e-4f);
        s.coat_compensation = 1.0f + fresnel_dielectric_average(s.coat_eta) * (1.0f - e_coat_ggx) / e_coat_ggx;
        s.coat_albedo = fminf(fmaxf(s.coat_compensation * table_dielectric(tables, mu, s.coat_roughness, s.coat_eta), 0.0f), 1.0f);
    }
    const float e_ggx = fmaxf(table_ggx(tables, mu, s.roughness), 1e-4f);
    const float missing = (1.0f - e_ggx) / e_ggx;
    s.metal_missing = missing;
    s.dielectric_compensation = 1.0f + fresnel_dielectric_average(s.ior) * missing;
    s.specular_albedo = fminf(fmaxf(s.specular_weight * s.dielectric_compensation * table_dielectric(tables, mu, s.roughness, s.ior),
                                    0.0f), 1.0f);
    float substrate_rgb = 1.0f;
    s.coat_k = 0.0f;
    if (s.coat > 0.0f) {
        const float k_smooth = fresnel_dielectric(mu, s.coat_eta);
        const float k_rough = 1.0f - (1.0f - fresnel_dielectric_average(s.coat_eta)) / (s.coat_eta * s.coat_eta);
        const float base_roughness = mixf(1.0f, s.roughness, s.metalness);
        s.coat_k = mixf(k_smooth, k_rough, base_roughness);
        const float delta_rgb = (1.0f - s.coat_k) / fmaxf(1e-4f, 1.0f - s.lum_base * s.coat_k);
        substrate_rgb = mixf(1.0f, s.lum_coat * (1.0f - s.coat_albedo) * mixf(1.0f, delta_rgb, s.darkening), s.coat);
    }
    choose_lobes(s, substrate_rgb, s.specular_albedo, s.coat_albedo);
}

// update_substrate (openpbr.glsl:380-388).
__device__ __forceinline__ void update_substrate(Surface &s) {
    s.substrate = splat4(1.0f);
    if (s.coat > 0.0f) {
        const float4 delta = div4(splat4(1.0f - s.coat_k), sub4(1.0f, s.base * s.coat_k));
        const float4 under = s.coat_tint * (1.0f - s.coat_albedo) * mix4(splat4(1.0f), delta, s.darkening);
        s.substrate = mix4(splat4(1.0f), under, s.coat);
    }
}

// read_colors (openpbr.glsl:391-402) without node graphs.
template <bool kSpectral>
__device__ __forceinline__ void read_colors(Surface &s, const float4 *materials, float4 lambda) {
    const float4 *row = materials + (size_t)s.material * 16u;
    auto color = [&](uint32_t r) { return spec_of<kSpectral>(__ldg(&row[r]), xyz(__ldg(&row[r + 1])), lambda); };
    s.base = color(0) * __ldg(&row[1]).w;
    s.metal_tint = color(2);
    s.specular_tint = s.metal_tint * s.specular_weight;
    s.transmission_tint = color(8);
    s.coat_tint = s.coat > 0.0f ? color(4) : splat4(1.0f);
}

template <bool kSpectral>
__device__ __forceinline__ void prepare_surface(Surface &s, float3 wo, float4 lambda, const float4 *materials) {
    read_material(s, materials, kSpectral && lambda.y < 0.0f ? lambda.x : 0.0f);
    orient_lobes(s, wo);
    read_colors<kSpectral>(s, materials, lambda);
    update_substrate(s);
}

__device__ __forceinline__ void orient_surface(Surface &s, float3 wo) {
    orient_lobes(s, wo);
    update_substrate(s);
}

// light_lobes (openpbr.glsl:420-450): the choice light paths sample with, by Fresnel at
// normal incidence, so it holds for every direction.
__device__ __forceinline__ void light_lobes(Surface &s) {
    const float f0 = (s.ior - 1.0f) / (s.ior + 1.0f);
    const float specular_albedo = fminf(fmaxf(s.specular_weight * f0 * f0, 0.0f), 1.0f);
    float coat_albedo = 0.0f;
    if (s.coat > 0.0f) {
        const float c0 = (s.coat_eta - 1.0f) / (s.coat_eta + 1.0f);
        coat_albedo = c0 * c0;
    }
    const float substrate_rgb = mixf(1.0f, s.lum_coat * (1.0f - coat_albedo), s.coat);
    choose_lobes(s, substrate_rgb, specular_albedo, coat_albedo);
}

// The refraction half-vector for wo, wi on opposite sides at ratio eta, facing +z.
__device__ __forceinline__ bool refraction_half(float3 wi, float3 wo, float eta, float3 &h) {
    h = normalize(wo + wi * eta);
    if (h.z < 0.0f) h = -h;
    return dot(wo, h) > 0.0f && dot(wi, h) < 0.0f;
}

// surface_pdf (openpbr.glsl:460-479).
__device__ __forceinline__ float surface_pdf(const Surface &s, float3 wi, float3 wo) {
    if (wo.z <= 0.0f || wi.z == 0.0f) return 0.0f;
    if (wi.z < 0.0f) {
        if (s.p_transmission <= 0.0f) return 0.0f;
        float3 h;
        if (!refraction_half(wi, wo, s.eta, h)) return 0.0f;
        const float o_h = dot(wo, h), i_h = dot(wi, h);
        const float denominator = o_h + s.eta * i_h;
        const float jacobian = s.eta * s.eta * fabsf(i_h) / (denominator * denominator);
        return s.p_transmission * ggx_g1(wo, s.alpha) * ggx_d(h, s.alpha) * o_h / wo.z * jacobian;
    }
    const float3 h = normalize(wi + wo);
    float pdf = 0.0f;
    if (s.p_coat > 0.0f) pdf += s.p_coat * ggx_reflection_pdf(wo, h, s.coat_alpha);
    if (!s.inside) pdf += s.p_diffuse * wi.z / kPi;
    pdf += (s.p_specular + s.p_metal) * ggx_reflection_pdf(wo, h, s.alpha);
    return pdf;
}

// evaluate_surface (openpbr.glsl:481-520): f (cosine not included) and the pdf of wi.
__device__ __forceinline__ float4 evaluate_surface(const Surface &s, float3 wi, float3 wo, float &pdf) {
    pdf = 0.0f;
    const float4 zero = splat4(0.0f);
    if (wo.z <= 0.0f || wi.z == 0.0f) return zero;
    pdf = surface_pdf(s, wi, wo);
    const float dielectric = 1.0f - s.metalness;
    if (wi.z < 0.0f) {
        if (s.p_transmission <= 0.0f) return zero;
        float3 h;
        if (!refraction_half(wi, wo, s.eta, h)) return zero;
        const float o_h = dot(wo, h), i_h = dot(wi, h);
        const float denominator = o_h + s.eta * i_h;
        const float d = ggx_d(h, s.alpha);
        const float f = (1.0f - fresnel_dielectric(o_h, s.eta)) * d * ggx_g2(-wi, wo, s.alpha) * fabsf(i_h) * o_h /
                        (fabsf(wi.z) * wo.z * denominator * denominator);
        return s.substrate * s.transmission_tint * (dielectric * s.transmission * f);
    }
    const float3 h = normalize(wi + wo);
    const float cos_h = dot(wo, h);
    float4 f = zero;
    if (s.p_coat > 0.0f) {
        const float coat = ggx_d(h, s.coat_alpha) * ggx_g2(wi, wo, s.coat_alpha) / (4.0f * wi.z * wo.z);
        f = f + splat4(s.coat * fresnel_dielectric(cos_h, s.coat_eta) * s.coat_compensation * coat);
    }
    float4 below = zero;
    if (!s.inside)
        below = below + eon(s.base, s.diffuse_roughness, wi, wo) *
                            (dielectric * (1.0f - s.transmission) * (1.0f - s.specular_albedo));
    const float microfacet = ggx_d(h, s.alpha) * ggx_g2(wi, wo, s.alpha) / (4.0f * wi.z * wo.z);
    if (dielectric > 0.0f)
        below = below + s.specular_tint * (dielectric * fresnel_dielectric(cos_h, s.eta) * s.dielectric_compensation * microfacet);
    if (s.metalness > 0.0f && !s.inside) {
        const float4 average = (s.base * 20.0f + splat4(1.0f)) * (1.0f / 21.0f);
        const float4 compensation = splat4(1.0f) + average * s.metal_missing;
        below = below + min4(splat4(1.0f), fresnel_f82(s.base, s.metal_tint, cos_h) * s.specular_weight) * compensation *
                            (s.metalness * microfacet);
    }
    return f + s.substrate * below;
}

// sample_direction (openpbr.glsl:522-548): wi for wo from u.xy (direction) and u.z
// (lobe), its pdf over all lobes, and the lobe (for the bounce limits).
__device__ __forceinline__ bool sample_direction(const Surface &s, float3 wo, float3 u, float3 &wi, float &pdf,
                                                 uint32_t &lobe) {
    pdf = 0.0f;
    if (wo.z <= 0.0f) return false;
    float pick = u.z;
    const float2 uv = make_float2(u.x, u.y);
    if (pick < s.p_diffuse) {
        const float2 disk = concentric(uv);
        wi = make_float3(disk.x, disk.y, sqrtf(fmaxf(0.0f, 1.0f - (disk.x * disk.x + disk.y * disk.y))));
        lobe = kLobeDiffuse;
    } else if ((pick -= s.p_diffuse) < s.p_coat) {
        wi = reflect_about(-wo, ggx_sample(wo, s.coat_alpha, uv));
        lobe = kLobeGlossy;
    } else if ((pick -= s.p_coat) < s.p_specular + s.p_metal) {
        wi = reflect_about(-wo, ggx_sample(wo, s.alpha, uv));
        lobe = kLobeGlossy;
    } else if (s.p_transmission > 0.0f) {
        const float3 h = ggx_sample(wo, s.alpha, uv);
        wi = refract_through(-wo, h, 1.0f / s.eta);
        if (dot(wi, wi) == 0.0f) return false;
        lobe = kLobeTransmission;
    } else {
        return false;
    }
    if (wi.z == 0.0f) return false;
    pdf = surface_pdf(s, wi, wo);
    return pdf > 0.0f;
}

// light_sampler_pdf (connect.glsl:51-60): the pdf the light sampler at this point gives `to`
// when the light path arrived from `from` (world, unit, both leaving the point): the
// surface (read) seen from `from`'s side, choosing lobes by light_lobes; zero where the
// sampler would reject `to`.
__device__ __forceinline__ float light_sampler_pdf(const Surface &s, float3 from, float3 to, const float4 *materials,
                                                  float hero) {
    const bool same = dot(from, s.geometric) >= 0.0f;
    Surface v = same ? s : turned(s);
    const float3 wo = to_local(v, from), wi = to_local(v, to);
    if ((dot(to, v.geometric) > 0.0f) != (wi.z > 0.0f)) return 0.0f;
    if (!same) read_material(v, materials, hero);
    light_lobes(v);
    return surface_pdf(v, wi, wo);
}

}  // namespace lr
