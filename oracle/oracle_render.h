/*
 * Oracle (test infrastructure): the f64 restatement of the integrator's estimator
 * (oracle/integrator.c). The caller passes the compiled scene (leaf order), the loaded
 * records (light rows, light tree, material records as the reference packs them) and the
 * view; the oracle returns per pixel the mean and variance of the samples' ACEScg values.
 */
#ifndef LUCE_ORACLE_RENDER_H
#define LUCE_ORACLE_RENDER_H

#include <stddef.h>
#include <stdint.h>

#include "oracle.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    const float *positions;
    const uint32_t *indices;
    const uint32_t *shading;
    size_t triangle_count;
    const or_node *nodes;
    const float *light_rows; /* 28 floats per light */
    uint32_t light_count;
    const float *tree_nodes; /* 12 floats per node */
    const uint32_t *tree_links;
    const uint32_t *tree_records; /* 4 per emitter, then the triangle map */
    uint32_t tree_node_count, emitter_count;
    const float *materials; /* 64 floats per material */
    double p_distant;
    float background_fit[4], background_rgb[3];
    double film[9], cmf_integrals[3];
    float frame[16];
    double lens_radius, focus_distance, forward[3];
    uint32_t width, height, max_bounces, spectral, seed;
    double limits[3], clamp; /* the most diffuse, glossy and transmission bounces */
    /* Light tracing (connect.glsl): light paths a sample (0: none), the band they follow
     * (their sampler numbers are 0x80000000 | (band + i)), 1 / a pixel's area at unit
     * distance. */
    uint32_t light_paths, light_band;
    double pixel_area_inv;
    /* Light paths from afar (lights.glsl:283-308): their share of light paths and the disk
     * they start on, facing the light (radius, centre); share 0 for none. */
    double emit_share, emit_radius, emit_center[3];
    /* Rounds beyond the bounces for rays passing through cut-outs (8 when a material the
     * triangles use has geometry_opacity below 1, else 0). */
    uint32_t through;
} or_render_desc;

void or_render(const or_render_desc *r, uint32_t samples, double *mean, double *var, int threads);
/* The same over pixels [first, first + count) and samples [sample_first, sample_first +
 * samples); `rays` (may be NULL) counts the closest and shadow rays traced. */
void or_render_region(const or_render_desc *r, uint32_t samples, uint32_t sample_first, size_t first, size_t count,
                      double *mean, double *var, uint64_t rays[2], int threads);

/* With light tracing: per sample, every pixel's camera value plus the splats its light
 * paths leave there; the mean and variance over samples [sample_first, + samples) of
 * those images (ACEScg, 3 per pixel, all pixels). */
void or_render_traced(const or_render_desc *r, uint32_t samples, uint32_t sample_first, double *mean, double *var,
                      uint64_t rays[2], int threads);

#ifdef __cplusplus
}
#endif
#endif
