/*
 * Oracle (test infrastructure): OpenPBR Surface's lobes restated in f64 (openpbr.c),
 * after shaders/openpbr.glsl:196-556 and microfacet.glsl:1-84, with the albedo tables of
 * tables.comp:19-62 computed here in f64 on the same nodes and sample grid.
 */
#ifndef LUCE_ORACLE_OPENPBR_H
#define LUCE_ORACLE_OPENPBR_H

#include <stdint.h>

#include "oracle_vec.h"

#define OR_LOBE_DIFFUSE 0u
#define OR_LOBE_GLOSSY 1u
#define OR_LOBE_TRANSMISSION 2u

/* The surface at a hit, as openpbr.glsl's Surface: the frame (facing the side it is seen
 * from), the material as read, the lobes for a view direction, the colors at the path's
 * wavelengths. */
typedef struct {
    d3 normal, tangent, bitangent, geometric;
    uint32_t material;
    int back, inside;
    double diffuse_roughness, metalness, specular_weight, transmission, roughness, coat_roughness, ior, darkening;
    double lum_base, lum_specular, lum_transmission, lum_coat;
    double alpha[2], eta, coat, coat_alpha[2], coat_eta;
    double dielectric_compensation, metal_missing, specular_albedo, coat_compensation, coat_albedo, coat_k;
    double p_coat, p_metal, p_specular, p_transmission, p_diffuse;
    spec base, metal_tint, specular_tint, transmission_tint, coat_tint, substrate;
} or_surface;

/* The albedo tables (E_ggx, its average over mu, E_dielectric), computed on first use. */
const double *or_albedo_tables(void);
double or_table_albedo(double mu, double roughness, double eta);

or_surface or_surface_at(d3 normal, d3 geometric, uint32_t material, int back);
or_surface or_turned(const or_surface *s);
d3 or_to_local(const or_surface *s, d3 v);
d3 or_to_world(const or_surface *s, d3 v);
void or_read_material(or_surface *s, const float *materials, double hero);
void or_orient_lobes(or_surface *s, d3 wo);
void or_update_substrate(or_surface *s);
void or_read_colors(or_surface *s, const float *materials, int spectral, const double lambda[4]);
void or_prepare_surface(or_surface *s, d3 wo, const float *materials, int spectral, const double lambda[4]);
void or_orient_surface(or_surface *s, d3 wo);
void or_light_lobes(or_surface *s);
double or_surface_pdf(const or_surface *s, d3 wi, d3 wo);
spec or_evaluate_surface(const or_surface *s, d3 wi, d3 wo, double *pdf);
int or_sample_direction(const or_surface *s, d3 wo, double u0, double u1, double pick, d3 *wi, double *pdf,
                        uint32_t *lobe);
/* connect.glsl:51-60: the pdf the light sampler gives `to` when light arrived from `from`;
 * `hero`: the path's hero wavelength after a dispersive hit (0 before). */
double or_light_sampler_pdf(const or_surface *s, const float *materials, d3 from, d3 to, double hero);

#endif
