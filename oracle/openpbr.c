/*
 * Oracle (test infrastructure): OpenPBR Surface restated in f64 -- GGX microfacets
 * (microfacet.glsl:9-63), the albedo tables (tables.comp:21-61, microfacet.glsl:67-84,
 * openpbr.glsl:126-150), F82-tint metal (openpbr.glsl:154-163), EON diffuse
 * (openpbr.glsl:87-113) and the layered surface (openpbr.glsl:196-556).
 */
#include <pthread.h>
#include <string.h>

#include "oracle_openpbr.h"

#define INFINITY_F 3.0e38

/* ---- GGX (microfacet.glsl:9-63) ----------------------------------------------------- */

static void ggx_alpha(double roughness, double anisotropy, double alpha[2]) {
    double r2 = roughness * roughness;
    double t = r2 * sqrt(2.0 / (1.0 + (1.0 - anisotropy) * (1.0 - anisotropy)));
    alpha[0] = fmax(t, 1e-4);
    alpha[1] = fmax((1.0 - anisotropy) * t, 1e-4);
}

static double ggx_d(d3 m, const double a[2]) {
    if (m.z <= 0.0) return 0.0;
    d3 s = v3(m.x / a[0], m.y / a[1], m.z);
    double k = dot(s, s);
    return 1.0 / (PI * a[0] * a[1] * k * k);
}

static double ggx_lambda(d3 v, const double a[2]) {
    double z2 = v.z * v.z;
    if (z2 <= 0.0) return INFINITY_F;
    double a2 = (a[0] * a[0] * v.x * v.x + a[1] * a[1] * v.y * v.y) / z2;
    return 0.5 * (-1.0 + sqrt(1.0 + a2));
}

static double ggx_g1(d3 v, const double a[2]) { return 1.0 / (1.0 + ggx_lambda(v, a)); }
static double ggx_g2(d3 wi, d3 wo, const double a[2]) { return 1.0 / (1.0 + ggx_lambda(wi, a) + ggx_lambda(wo, a)); }

/* A visible normal by spherical caps (Dupuy and Benyoub 2023). */
static d3 ggx_sample(d3 wo, const double a[2], double u0, double u1) {
    d3 v = norm(v3(wo.x * a[0], wo.y * a[1], wo.z));
    double phi = 2.0 * PI * u0;
    double z = (1.0 - u1) * (1.0 + v.z) - v.z;
    double s = sqrt(fmin(fmax(1.0 - z * z, 0.0), 1.0));
    d3 h = add(v3(s * cos(phi), s * sin(phi), z), v);
    return norm(v3(h.x * a[0], h.y * a[1], fmax(h.z, 1e-6)));
}

static double ggx_reflection_pdf(d3 wo, d3 h, const double a[2]) { return ggx_g1(wo, a) * ggx_d(h, a) / (4.0 * wo.z); }

static double fresnel_dielectric(double cos_i, double eta) {
    double c = fabs(cos_i);
    double g2 = eta * eta - 1.0 + c * c;
    if (g2 <= 0.0) return 1.0;
    double g = sqrt(g2);
    double a = (g - c) / (g + c);
    double b = (c * (g + c) - 1.0) / (c * (g - c) + 1.0);
    return 0.5 * a * a * (1.0 + b * b);
}

static double fresnel_dielectric_average(double eta) {
    return log((10893.0 * eta - 1438.2) / (-774.4 * eta * eta + 10212.0 * eta + 1.0));
}

static d3 reflect_about(d3 i, d3 n) { return sub(i, mul(n, 2.0 * dot(n, i))); }

static d3 refract_through(d3 i, d3 n, double eta) {
    double d = dot(n, i);
    double k = 1.0 - eta * eta * (1.0 - d * d);
    if (k < 0.0) return v3(0, 0, 0);
    return sub(mul(i, eta), mul(n, eta * d + sqrt(k)));
}

static double mixd(double a, double b, double t) { return a * (1.0 - t) + b * t; }
static double clampd(double x, double lo, double hi) { return fmin(fmax(x, lo), hi); }

/* ---- Albedo tables ------------------------------------------------------------------ */

#define TABLE_MU 32u
#define TABLE_ROUGHNESS 32u
#define TABLE_ETA 16u
#define TABLE_Z_MAX 0.8
#define TABLE_MU_MIN 0.02
#define TABLE_GGX 0u
#define TABLE_GGX_AVERAGE (TABLE_MU * TABLE_ROUGHNESS)
#define TABLE_DIELECTRIC (TABLE_GGX_AVERAGE + TABLE_ROUGHNESS)
#define TABLE_SIZE (TABLE_DIELECTRIC + TABLE_MU * TABLE_ROUGHNESS * TABLE_ETA)

static double eta_of_z(double z) { return (1.0 + z * z) / (1.0 - z * z); }
static double z_of_eta(double eta) { return sqrt(fabs(eta - 1.0) / (eta + 1.0)); }
static double table_mu(uint32_t i) { return mixd(TABLE_MU_MIN, 1.0, (double)i / (double)(TABLE_MU - 1u)); }
static double table_roughness(uint32_t i) { return (double)i / (double)(TABLE_ROUGHNESS - 1u); }
static double table_z(uint32_t i) { return TABLE_Z_MAX * (double)i / (double)(TABLE_ETA - 1u); }

/* The mean of F G2 / G1 over a 32 x 32 stratified grid of visible normals (eta <= 0: F = 1). */
double or_table_albedo(double mu, double roughness, double eta) {
    d3 wo = v3(sqrt(1.0 - mu * mu), 0.0, mu);
    double a[2];
    ggx_alpha(roughness, 0.0, a);
    double sum = 0.0;
    for (uint32_t i = 0; i < 32u; i++)
        for (uint32_t j = 0; j < 32u; j++) {
            d3 h = ggx_sample(wo, a, ((double)i + 0.5) / 32.0, ((double)j + 0.5) / 32.0);
            d3 wi = reflect_about(neg(wo), h);
            if (wi.z <= 0.0) continue;
            double f = eta > 0.0 ? fresnel_dielectric(dot(wo, h), eta) : 1.0;
            sum += f * ggx_g2(wi, wo, a) / ggx_g1(wo, a);
        }
    return sum / 1024.0;
}

static double g_tables[TABLE_SIZE];
static pthread_once_t g_tables_once = PTHREAD_ONCE_INIT;

static void make_tables(void) {
    const uint32_t plane = TABLE_MU * TABLE_ROUGHNESS;
    for (uint32_t cell = 0; cell < plane * (1u + TABLE_ETA); cell++) {
        uint32_t layer = cell / plane, at = cell % plane;
        double mu = table_mu(at % TABLE_MU), roughness = table_roughness(at / TABLE_MU);
        if (layer == 0u) g_tables[TABLE_GGX + at] = or_table_albedo(mu, roughness, -1.0);
        else g_tables[TABLE_DIELECTRIC + (layer - 1u) * plane + at] = or_table_albedo(mu, roughness, eta_of_z(table_z(layer - 1u)));
    }
    /* 2 * integral of E(mu) mu dmu by the trapezoid rule over the mu nodes. */
    for (uint32_t r = 0; r < TABLE_ROUGHNESS; r++) {
        double sum = 0.0;
        for (uint32_t m = 0; m + 1u < TABLE_MU; m++) {
            double a = table_mu(m), b = table_mu(m + 1u);
            sum += 0.5 * (g_tables[TABLE_GGX + r * TABLE_MU + m] * a + g_tables[TABLE_GGX + r * TABLE_MU + m + 1u] * b) * (b - a);
        }
        g_tables[TABLE_GGX_AVERAGE + r] = 2.0 * sum;
    }
}

const double *or_albedo_tables(void) {
    pthread_once(&g_tables_once, make_tables);
    return g_tables;
}

static double table_row(uint32_t base, double r, double mu) {
    const double *t = or_albedo_tables();
    double x = clampd((mu - TABLE_MU_MIN) / (1.0 - TABLE_MU_MIN) * (double)(TABLE_MU - 1u), 0.0, (double)(TABLE_MU - 1u));
    double y = clampd(r * (double)(TABLE_ROUGHNESS - 1u), 0.0, (double)(TABLE_ROUGHNESS - 1u));
    uint32_t x0 = (uint32_t)x, y0 = (uint32_t)y;
    uint32_t x1 = x0 + 1u < TABLE_MU ? x0 + 1u : TABLE_MU - 1u, y1 = y0 + 1u < TABLE_ROUGHNESS ? y0 + 1u : TABLE_ROUGHNESS - 1u;
    double fx = x - (double)x0, fy = y - (double)y0;
    double a = mixd(t[base + y0 * TABLE_MU + x0], t[base + y0 * TABLE_MU + x1], fx);
    double b = mixd(t[base + y1 * TABLE_MU + x0], t[base + y1 * TABLE_MU + x1], fx);
    return mixd(a, b, fy);
}

static double table_ggx(double mu, double r) { return table_row(TABLE_GGX, r, mu); }

static double table_dielectric(double mu, double r, double eta) {
    double z = clampd(z_of_eta(eta) / TABLE_Z_MAX * (double)(TABLE_ETA - 1u), 0.0, (double)(TABLE_ETA - 1u));
    uint32_t z0 = (uint32_t)z, z1 = z0 + 1u < TABLE_ETA ? z0 + 1u : TABLE_ETA - 1u;
    const uint32_t plane = TABLE_MU * TABLE_ROUGHNESS;
    return mixd(table_row(TABLE_DIELECTRIC + z0 * plane, r, mu), table_row(TABLE_DIELECTRIC + z1 * plane, r, mu), z - (double)z0);
}

/* ---- EON diffuse (openpbr.glsl:87-113) ----------------------------------------------- */

static double fon_albedo(double mu, double rr) {
    double m = 1.0 - mu;
    double g = m * (0.0571085289 + m * (0.491881867 + m * (-0.332181442 + m * 0.0714429953)));
    return (1.0 + rr * g) / (1.0 + (0.5 - 2.0 / (3.0 * PI)) * rr);
}

static spec eon(spec rho, double rr, d3 wi, d3 wo) {
    const double c1 = 0.5 - 2.0 / (3.0 * PI), c2 = 2.0 / 3.0 - 28.0 / (15.0 * PI);
    double s = dot(wi, wo) - wi.z * wo.z;
    double st = s > 0.0 ? s / fmax(wi.z, wo.z) : s;
    double a = 1.0 / (1.0 + c1 * rr);
    double eo = fon_albedo(wo.z, rr), ei = fon_albedo(wi.z, rr);
    double avg = a * (1.0 + c2 * rr);
    double k = fmax(1e-7, 1.0 - eo) * fmax(1e-7, 1.0 - ei) / (PI * fmax(1e-7, 1.0 - avg));
    spec out;
    for (int i = 0; i < 4; i++) {
        double single = rho.s[i] * (a * (1.0 + rr * st) / PI);
        double ms = rho.s[i] * rho.s[i] * avg / (1.0 - rho.s[i] * (1.0 - avg));
        out.s[i] = single + ms * k;
    }
    return out;
}

/* ---- F82-tint metal (openpbr.glsl:154-163) -------------------------------------------- */

static spec fresnel_f82(spec f0, spec tint, double mu) {
    const double bar = 1.0 / 7.0;
    double m = 1.0 - mu, m5 = m * m * m * m * m, b5 = pow(1.0 - bar, 5.0);
    spec out;
    for (int i = 0; i < 4; i++) {
        double schlick = f0.s[i] + (1.0 - f0.s[i]) * m5;
        double schlick_bar = f0.s[i] + (1.0 - f0.s[i]) * b5;
        double a = schlick_bar * (1.0 - tint.s[i]) / (bar * b5 * (1.0 - bar));
        out.s[i] = clampd(schlick - a * (mu * m5 * m), 0.0, 1.0);
    }
    return out;
}

/* ---- The surface (openpbr.glsl:243-556) ------------------------------------------------ */

static const float *mrow(const float *materials, uint32_t m, int k) { return &materials[m * 64 + k * 4]; }

static double rgb_luma(const float *rgb, double scale) {
    return (rgb[0] * 0.2722287168 + rgb[1] * 0.6740817658 + rgb[2] * 0.0536895174) * scale;
}

d3 or_to_local(const or_surface *s, d3 v) { return v3(dot(v, s->tangent), dot(v, s->bitangent), dot(v, s->normal)); }
d3 or_to_world(const or_surface *s, d3 v) {
    return add(add(mul(s->tangent, v.x), mul(s->bitangent, v.y)), mul(s->normal, v.z));
}

or_surface or_surface_at(d3 normal, d3 geometric, uint32_t material, int back) {
    or_surface s;
    memset(&s, 0, sizeof s);
    s.normal = normal;
    onb(normal, &s.tangent, &s.bitangent);
    s.geometric = geometric;
    s.material = material;
    s.back = back;
    return s;
}

or_surface or_turned(const or_surface *s) { return or_surface_at(neg(s->normal), neg(s->geometric), s->material, !s->back); }

void or_read_material(or_surface *s, const float *materials, double hero) {
    const float *base_rgb = mrow(materials, s->material, 1), *specular_rgb = mrow(materials, s->material, 3);
    const float *coat_rgb = mrow(materials, s->material, 5), *transmission_rgb = mrow(materials, s->material, 9);
    const float *scalars = mrow(materials, s->material, 10), *indices = mrow(materials, s->material, 11);
    const float *geometry = mrow(materials, s->material, 12);
    s->diffuse_roughness = scalars[1];
    s->metalness = clampd(scalars[0], 0.0, 1.0);
    s->specular_weight = fmax(specular_rgb[3], 0.0);
    s->transmission = clampd(transmission_rgb[3], 0.0, 1.0);
    s->inside = s->back && s->transmission > 0.0;
    s->coat = !s->inside ? clampd(coat_rgb[3], 0.0, 1.0) : 0.0;
    s->coat_roughness = clampd(indices[1], 0.0, 1.0);
    s->coat_eta = fmax(indices[2], 1.0001);
    s->coat_alpha[0] = s->coat_alpha[1] = 1.0;
    if (s->coat > 0.0) ggx_alpha(s->coat_roughness, clampd(geometry[2], 0.0, 1.0), s->coat_alpha);
    s->darkening = clampd(indices[3], 0.0, 1.0);
    double roughness = clampd(scalars[2], 0.0, 1.0);
    double r4 = roughness * roughness * roughness * roughness;
    double c4 = s->coat_roughness * s->coat_roughness * s->coat_roughness * s->coat_roughness;
    s->roughness = mixd(roughness, fmin(1.0, pow(r4 + 2.0 * c4, 0.25)), s->coat);
    ggx_alpha(s->roughness, clampd(scalars[3], 0.0, 1.0), s->alpha);
    double eta = fmax(indices[0], 1.0001);
    /* Cauchy's index at the hero wavelength once dispersion split the path (openpbr.glsl:177-180, 309). */
    if (geometry[3] != 0.0f && hero > 0.0)
        eta = fmax(eta + geometry[3] * (1.0 / (hero * hero) - 1.0 / (587.6 * 587.6)), 1.0001);
    double relative = eta / s->coat_eta;
    if (relative < 1.0) relative = 1.0 / relative;
    s->ior = fmax(mixd(eta, relative, s->coat), 1.0001);
    s->eta = s->inside ? 1.0 / s->ior : s->ior;
    s->lum_base = fmax(rgb_luma(base_rgb, base_rgb[3]), 0.0);
    s->lum_specular = fmax(rgb_luma(specular_rgb, 1.0), 0.0);
    s->lum_transmission = fmax(rgb_luma(transmission_rgb, 1.0), 0.05);
    s->lum_coat = rgb_luma(coat_rgb, 1.0);
}

static void choose_lobes(or_surface *s, double substrate_rgb, double specular_albedo, double coat_albedo) {
    double dielectric = 1.0 - s->metalness;
    double w_coat = s->coat * coat_albedo;
    double w_metal = substrate_rgb * s->metalness;
    double w_specular = substrate_rgb * dielectric * specular_albedo * s->lum_specular;
    double w_transmission = substrate_rgb * dielectric * s->transmission * (1.0 - specular_albedo) * s->lum_transmission;
    double w_diffuse = substrate_rgb * dielectric * (1.0 - s->transmission) * (1.0 - specular_albedo) * s->lum_base;
    if (s->inside) {
        w_metal = 0.0;
        w_diffuse = 0.0;
        w_specular = fmax(w_specular, 0.05);
        w_transmission = fmax(w_transmission, s->transmission > 0.0 ? 0.05 : 0.0);
    }
    double total = w_coat + w_metal + w_specular + w_transmission + w_diffuse;
    double scale = total > 0.0 ? 1.0 / total : 0.0;
    s->p_coat = w_coat * scale;
    s->p_metal = w_metal * scale;
    s->p_specular = w_specular * scale;
    s->p_transmission = w_transmission * scale;
    s->p_diffuse = w_diffuse * scale;
}

void or_orient_lobes(or_surface *s, d3 wo) {
    double mu = clampd(wo.z, 0.0, 1.0);
    s->coat_compensation = 1.0;
    s->coat_albedo = 0.0;
    if (s->coat > 0.0) {
        double e_coat = fmax(table_ggx(mu, s->coat_roughness), 1e-4);
        s->coat_compensation = 1.0 + fresnel_dielectric_average(s->coat_eta) * (1.0 - e_coat) / e_coat;
        s->coat_albedo = clampd(s->coat_compensation * table_dielectric(mu, s->coat_roughness, s->coat_eta), 0.0, 1.0);
    }
    double e_ggx = fmax(table_ggx(mu, s->roughness), 1e-4);
    double missing = (1.0 - e_ggx) / e_ggx;
    s->metal_missing = missing;
    s->dielectric_compensation = 1.0 + fresnel_dielectric_average(s->ior) * missing;
    s->specular_albedo =
        clampd(s->specular_weight * s->dielectric_compensation * table_dielectric(mu, s->roughness, s->ior), 0.0, 1.0);
    double substrate_rgb = 1.0;
    s->coat_k = 0.0;
    if (s->coat > 0.0) {
        double k_smooth = fresnel_dielectric(mu, s->coat_eta);
        double k_rough = 1.0 - (1.0 - fresnel_dielectric_average(s->coat_eta)) / (s->coat_eta * s->coat_eta);
        s->coat_k = mixd(k_smooth, k_rough, mixd(1.0, s->roughness, s->metalness));
        double delta_rgb = (1.0 - s->coat_k) / fmax(1e-4, 1.0 - s->lum_base * s->coat_k);
        substrate_rgb = mixd(1.0, s->lum_coat * (1.0 - s->coat_albedo) * mixd(1.0, delta_rgb, s->darkening), s->coat);
    }
    choose_lobes(s, substrate_rgb, s->specular_albedo, s->coat_albedo);
}

void or_update_substrate(or_surface *s) {
    s->substrate = spec_all(1.0);
    if (s->coat > 0.0)
        for (int i = 0; i < 4; i++) {
            double delta = (1.0 - s->coat_k) / (1.0 - s->base.s[i] * s->coat_k);
            double under = s->coat_tint.s[i] * (1.0 - s->coat_albedo) * mixd(1.0, delta, s->darkening);
            s->substrate.s[i] = mixd(1.0, under, s->coat);
        }
}

void or_read_colors(or_surface *s, const float *materials, int spectral, const double lambda[4]) {
    uint32_t m = s->material;
#define COLOR(r) spec_fit(spectral, mrow(materials, m, r), mrow(materials, m, (r) + 1), lambda)
    s->base = spec_scale(COLOR(0), mrow(materials, m, 1)[3]);
    s->metal_tint = COLOR(2);
    s->specular_tint = spec_scale(s->metal_tint, s->specular_weight);
    s->transmission_tint = COLOR(8);
    s->coat_tint = s->coat > 0.0 ? COLOR(4) : spec_all(1.0);
#undef COLOR
}

void or_prepare_surface(or_surface *s, d3 wo, const float *materials, int spectral, const double lambda[4]) {
    or_read_material(s, materials, spectral && lambda[1] < 0.0 ? lambda[0] : 0.0);
    or_orient_lobes(s, wo);
    or_read_colors(s, materials, spectral, lambda);
    or_update_substrate(s);
}

void or_orient_surface(or_surface *s, d3 wo) {
    or_orient_lobes(s, wo);
    or_update_substrate(s);
}

void or_light_lobes(or_surface *s) {
    double f0 = (s->ior - 1.0) / (s->ior + 1.0);
    double specular_albedo = clampd(s->specular_weight * f0 * f0, 0.0, 1.0);
    double coat_albedo = 0.0;
    if (s->coat > 0.0) {
        double c0 = (s->coat_eta - 1.0) / (s->coat_eta + 1.0);
        coat_albedo = c0 * c0;
    }
    choose_lobes(s, mixd(1.0, s->lum_coat * (1.0 - coat_albedo), s->coat), specular_albedo, coat_albedo);
}

static int refraction_half(d3 wi, d3 wo, double eta, d3 *h) {
    *h = norm(add(wo, mul(wi, eta)));
    if (h->z < 0.0) *h = neg(*h);
    return dot(wo, *h) > 0.0 && dot(wi, *h) < 0.0;
}

double or_surface_pdf(const or_surface *s, d3 wi, d3 wo) {
    if (wo.z <= 0.0 || wi.z == 0.0) return 0.0;
    if (wi.z < 0.0) {
        if (s->p_transmission <= 0.0) return 0.0;
        d3 h;
        if (!refraction_half(wi, wo, s->eta, &h)) return 0.0;
        double o_h = dot(wo, h), i_h = dot(wi, h);
        double denominator = o_h + s->eta * i_h;
        double jacobian = s->eta * s->eta * fabs(i_h) / (denominator * denominator);
        return s->p_transmission * ggx_g1(wo, s->alpha) * ggx_d(h, s->alpha) * o_h / wo.z * jacobian;
    }
    d3 h = norm(add(wi, wo));
    double pdf = 0.0;
    if (s->p_coat > 0.0) pdf += s->p_coat * ggx_reflection_pdf(wo, h, s->coat_alpha);
    if (!s->inside) pdf += s->p_diffuse * wi.z / PI;
    pdf += (s->p_specular + s->p_metal) * ggx_reflection_pdf(wo, h, s->alpha);
    return pdf;
}

spec or_evaluate_surface(const or_surface *s, d3 wi, d3 wo, double *pdf) {
    *pdf = 0.0;
    if (wo.z <= 0.0 || wi.z == 0.0) return spec_zero();
    *pdf = or_surface_pdf(s, wi, wo);
    double dielectric = 1.0 - s->metalness;
    if (wi.z < 0.0) {
        if (s->p_transmission <= 0.0) return spec_zero();
        d3 h;
        if (!refraction_half(wi, wo, s->eta, &h)) return spec_zero();
        double o_h = dot(wo, h), i_h = dot(wi, h);
        double denominator = o_h + s->eta * i_h;
        double f = (1.0 - fresnel_dielectric(o_h, s->eta)) * ggx_d(h, s->alpha) * ggx_g2(neg(wi), wo, s->alpha) * fabs(i_h) *
                   o_h / (fabs(wi.z) * wo.z * denominator * denominator);
        return spec_scale(spec_mul(s->substrate, s->transmission_tint), dielectric * s->transmission * f);
    }
    d3 h = norm(add(wi, wo));
    double cos_h = dot(wo, h);
    spec f = spec_zero();
    if (s->p_coat > 0.0) {
        double coat = ggx_d(h, s->coat_alpha) * ggx_g2(wi, wo, s->coat_alpha) / (4.0 * wi.z * wo.z);
        f = spec_all(s->coat * fresnel_dielectric(cos_h, s->coat_eta) * s->coat_compensation * coat);
    }
    spec below = spec_zero();
    if (!s->inside)
        below = spec_scale(eon(s->base, s->diffuse_roughness, wi, wo),
                           dielectric * (1.0 - s->transmission) * (1.0 - s->specular_albedo));
    double microfacet = ggx_d(h, s->alpha) * ggx_g2(wi, wo, s->alpha) / (4.0 * wi.z * wo.z);
    if (dielectric > 0.0)
        below = spec_add(below, spec_scale(s->specular_tint, dielectric * fresnel_dielectric(cos_h, s->eta) *
                                                                 s->dielectric_compensation * microfacet));
    if (s->metalness > 0.0 && !s->inside) {
        spec fm = fresnel_f82(s->base, s->metal_tint, cos_h);
        for (int i = 0; i < 4; i++) {
            double average = (20.0 * s->base.s[i] + 1.0) / 21.0;
            double compensation = 1.0 + average * s->metal_missing;
            below.s[i] += fmin(1.0, s->specular_weight * fm.s[i]) * compensation * (s->metalness * microfacet);
        }
    }
    return spec_add(f, spec_mul(s->substrate, below));
}

int or_sample_direction(const or_surface *s, d3 wo, double u0, double u1, double pick, d3 *wi, double *pdf,
                        uint32_t *lobe) {
    *pdf = 0.0;
    if (wo.z <= 0.0) return 0;
    if (pick < s->p_diffuse) {
        double dx, dy;
        concentric(u0, u1, &dx, &dy);
        *wi = v3(dx, dy, sqrt(fmax(0.0, 1.0 - (dx * dx + dy * dy))));
        *lobe = OR_LOBE_DIFFUSE;
    } else if ((pick -= s->p_diffuse) < s->p_coat) {
        *wi = reflect_about(neg(wo), ggx_sample(wo, s->coat_alpha, u0, u1));
        *lobe = OR_LOBE_GLOSSY;
    } else if ((pick -= s->p_coat) < s->p_specular + s->p_metal) {
        *wi = reflect_about(neg(wo), ggx_sample(wo, s->alpha, u0, u1));
        *lobe = OR_LOBE_GLOSSY;
    } else if (s->p_transmission > 0.0) {
        d3 h = ggx_sample(wo, s->alpha, u0, u1);
        *wi = refract_through(neg(wo), h, 1.0 / s->eta);
        if (dot(*wi, *wi) == 0.0) return 0;
        *lobe = OR_LOBE_TRANSMISSION;
    } else {
        return 0;
    }
    if (wi->z == 0.0) return 0;
    *pdf = or_surface_pdf(s, *wi, wo);
    return *pdf > 0.0;
}

double or_light_sampler_pdf(const or_surface *s, const float *materials, d3 from, d3 to, double hero) {
    int same = dot(from, s->geometric) >= 0.0;
    or_surface v = same ? *s : or_turned(s);
    d3 wo = or_to_local(&v, from), wi = or_to_local(&v, to);
    if ((dot(to, v.geometric) > 0.0) != (wi.z > 0.0)) return 0.0;
    if (!same) or_read_material(&v, materials, hero);
    or_light_lobes(&v);
    return or_surface_pdf(&v, wi, wo);
}
