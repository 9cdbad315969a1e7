/*
 * CPU oracle for the luce-render hot path: TEST INFRASTRUCTURE, never product code.
 *
 * A plain-C restatement of the reference's algorithms (luce-render, Luce + GLSL), used
 * only by tests/, the smoke check and the CPU-baseline leg of bench.py to check the
 * CUDA path. Each function names the reference file:line it follows. Arithmetic is
 * IEEE single precision without contraction (built with -ffp-contract=off) wherever
 * the reference computes in f32, and double where it computes in f64.
 *
 * Parity status: the reference cannot be built or run in this environment (it needs
 * the `luc` compiler, luce-gpu, luce-geocore and a Vulkan/Metal device), so this
 * restatement is pinned against the reference's own known-answer tests
 * (src/render/tests.lucb, the closed forms in tests/gpu/integrator.lucb) and against golden vectors
 * generated by the one piece of the reference that runs here, tools/sobol_table.py.
 */
#ifndef LUCE_ORACLE_H
#define LUCE_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OR_NONE 0xffffffffu

/* The reference's BVH node: src/render/bvh.lucb:23-27 (std430 vec3 lo, uint first,
 * vec3 hi, uint count; 32 bytes). */
typedef struct {
    float lo[3];
    uint32_t first;
    float hi[3];
    uint32_t count;
} or_node;

/* ---- BVH build (src/render/bvh.lucb) ---------------------------------------- */

/* build_bvh (bvh.lucb:66-82) + build_tree (85-129): binned SAH over the triangles'
 * boxes. `nodes` must hold 2*max(count,1) entries, `order` count entries. Returns
 * the node count. Triangles are NOT reordered here (see or_reorder). */
size_t or_build_bvh(const float *positions, const uint32_t *indices, size_t triangle_count,
                    or_node *nodes, uint32_t *order);

/* reorder (bvh.lucb:198-217): permute per-triangle arrays into leaf order. Any of
 * the arrays may be NULL. */
void or_reorder(const uint32_t *order, size_t count, uint32_t *indices, uint32_t *faces,
                uint32_t *shading, float *uvs);

/* The deepest leaf's depth (root = 0). */
uint32_t or_bvh_depth(const or_node *nodes, size_t node_count);

/* ---- Scene compile (src/render/scene.lucb) ---------------------------------- */

/* A mesh as the boundary takes it: points, triangles, a polygon per triangle (NULL: its
 * own), per-point or per-corner normals (NULL: the triangle's own), a material per
 * polygon (library index + 1; NULL or unknown: 0) and a 12-double placement (columns x,
 * y, z, translation; all zero: identity). */
typedef struct {
    const float *positions;
    uint64_t point_count;
    const uint32_t *indices;
    uint64_t triangle_count;
    const uint32_t *faces;
    uint32_t face_count;
    const float *normals;
    int normals_per_corner;
    const uint32_t *face_materials;
    double transform[12];
} or_mesh;

/* compile_scene (scene.lucb:111-129, add_mesh 253-294, shading_normals 364-398) and
 * build_bvh + reorder: world-space points (3 floats each), then indices (3), shading
 * (3 octahedral normals + material) and polygons per triangle in leaf order, the BVH
 * (2 * max(T, 1) nodes) and the leaf order. Returns 0, or -1 for a triangle naming a
 * point or polygon its mesh lacks. */
int or_compile_meshes(const or_mesh *meshes, size_t mesh_count, size_t library, float *positions, uint32_t *indices,
                      uint32_t *shading, uint32_t *faces, or_node *nodes, uint32_t *order, size_t *node_count);

/* ---- Traversal (shaders/bvh.glsl) ------------------------------------------- */

typedef struct {
    float t;
    uint32_t triangle; /* leaf-order slot, OR_NONE on a miss */
    float u, v;
} or_hit;

typedef struct {
    uint64_t interior; /* interior nodes visited (each reads both children: 64 B) */
    uint64_t triangles; /* triangle tests (48 B each) */
    uint64_t dropped; /* stack pushes past the reference's 32 entries */
} or_counts;

/* trace_closest (bvh.glsl:51-90) with triangle_hit (27-47) and box_entry (17-25).
 * `stack_limit` 32 reproduces the reference's silently dropped pushes; 0 means
 * an unbounded stack. `counts` may be NULL. */
or_hit or_trace_closest(const or_node *nodes, const float *positions, const uint32_t *indices,
                        const float o[3], const float d[3], float t_max, int stack_limit,
                        or_counts *counts);

/* trace_any (bvh.glsl:93-122). */
int or_trace_any(const or_node *nodes, const float *positions, const uint32_t *indices,
                 const float o[3], const float d[3], float t_max, int stack_limit,
                 or_counts *counts);

/* Batch forms over n rays (rays: 8 floats each: o.xyz, tmin, d.xyz, tmax; tmin is
 * ignored, the reference tests t > 0). `threads` 0 = all host cores. */
void or_trace_closest_batch(const or_node *nodes, const float *positions, const uint32_t *indices,
                            const float *rays, size_t n, int stack_limit, or_hit *out,
                            or_counts *counts, int threads);
void or_trace_any_batch(const or_node *nodes, const float *positions, const uint32_t *indices,
                        const float *rays, size_t n, int stack_limit, uint8_t *out,
                        or_counts *counts, int threads);

/* ---- Brute force --------------------------------------------------------------- */

/* tests/gpu/main.lucb:82-119: f64 Moller-Trumbore over every triangle; per ray the
 * nearest polygon (faces[slot], -1 none), its distance and the relative margin to
 * the next different polygon. Threaded over rays. */
void or_nearest_f64(const float *positions, const uint32_t *indices, const uint32_t *faces,
                    size_t triangle_count, const float *rays, size_t n, int64_t *face,
                    double *distance, double *margin, int threads);

/* The watertight FP32 test the CUDA kernels run (Woop, Benthin and Wald, JCGT 2013),
 * over every triangle: per ray the nearest hit with ties broken toward the smaller
 * triangle id (ids: `ids[slot]`, or the slot when ids is NULL). Accepts t with
 * tmin < t < tmax. any_hit: stop at the first hit (then prim is any hitting id and
 * t its distance). */
void or_brute_watertight(const float *positions, const uint32_t *indices, const uint32_t *ids,
                         size_t triangle_count, const float *rays, size_t n, int any_hit,
                         int32_t *prim, float *t, float *u, float *v, int threads);

/* The watertight test of one triangle; 1 on a hit in (tmin, tmax). */
int or_watertight(const float o[3], const float d[3], float tmin, float tmax, const float a[3],
                  const float b[3], const float c[3], float *t, float *u, float *v);

/* ---- Camera (src/render/camera.lucb) -------------------------------------------- */

typedef struct {
    double position[3], corner[3], du[3], dv[3], forward[3];
    int orthographic;
    uint32_t width, height;
    double lens_radius, focus_distance;
} or_frame;

/* ray_frame (camera.lucb:57-76). matrix: 12 doubles, columns x, y, z, translation.
 * projection 0 perspective, 1 orthographic. Returns 0 or 400. */
int or_ray_frame(const double matrix[12], int projection, double focal_length,
                 double horizontal_aperture, double f_stop, double focus_distance, uint32_t width,
                 uint32_t height, or_frame *out);
/* look_frame (camera.lucb:84-95). Returns 0 or 400. */
int or_look_frame(const double position[3], const double forward[3], const double up[3],
                  double tan_half_height, uint32_t width, uint32_t height, int orthographic,
                  or_frame *out);
/* RayFrame.pack (camera.lucb:41-47). */
void or_frame_pack(const or_frame *f, float out[16]);
/* RayFrame.ray (camera.lucb:51-54), in f64. */
void or_frame_ray(const or_frame *f, double x, double y, double origin[3], double direction[3]);
/* The probe's pixel-centre rays as the kernel makes them from the packed block
 * (probe.comp:21-34), f32: 8 floats per ray (o, 0, d, 3e38). */
void or_probe_rays(const float block[16], float *rays);

/* ---- Sampler (shaders/sampler.glsl, shaders/sobol_table.glsl) ------------------- */

uint32_t or_hash_u32(uint32_t x);
uint32_t or_hash_combine(uint32_t seed, uint32_t value);
uint32_t or_sobol(uint32_t index, uint32_t dimension);
const uint32_t *or_sobol_directions(void); /* 128 words */
/* sample4 (sampler.glsl:47-55): four 24-bit values (bits >> 8) of the point. */
void or_sample4_bits(uint32_t seed, uint32_t pixel, uint32_t index, uint32_t group, uint32_t out[4]);
void or_sample4(uint32_t seed, uint32_t pixel, uint32_t index, uint32_t group, double out[4]);

/* ---- Spectrum (src/render/spectrum.lucb, shaders/spectrum.glsl) ----------------- */

void or_cmf(double lambda, double out[3]);
void or_cmf_integrals(double out[3]);
void or_film_matrix(double out[9]);
void or_acescg_to_xyz_e(double out[9]);
/* fit_spectrum (spectrum.lucb:136-168): c0, c1, c2, scale. */
void or_fit_spectrum(const double rgb[3], double out[4]);
double or_blackbody(double lambda, double kelvin);
void or_blackbody_xyz(double kelvin, double out[3]);
void or_sample_wavelengths(double u, double out[4]);
double or_wavelength_pdf(double lambda);

/* ---- Octahedral normals (src/render/scene.lucb:400-412, common.glsl:256-267) ---- */
uint32_t or_octahedral(const double n[3]);
void or_octahedral_decode(uint32_t packed, double out[3]);

/* ---- Lights, materials, light tree (lights.lucb, materials.lucb, light_tree.lucb) */

typedef struct {
    double matrix[12]; /* columns x, y, z, translation */
    int shape;         /* 0 rect, 1 disk, 2 sphere, 3 distant, 4 dome */
    double color[3];
    double intensity, exposure, temperature;
    double width, height, radius, angle;
    int normalize, visible;
    const float *image; /* a dome's linear Rec.709 RGB, 3 floats a pixel, rows from the top */
    uint32_t image_width, image_height;
} or_light;

typedef struct {
    double base_weight, base_color[3], base_metalness, base_diffuse_roughness;
    double specular_weight, specular_color[3], specular_roughness, specular_roughness_anisotropy,
        specular_ior;
    double transmission_weight, transmission_color[3];
    double coat_weight, coat_color[3], coat_roughness, coat_roughness_anisotropy, coat_ior,
        coat_darkening;
    double emission_luminance, emission_color[3];
    double geometry_opacity;
    int geometry_thin_walled;
    double transmission_dispersion_scale, transmission_dispersion_abbe_number;
} or_material;

void or_material_standard(or_material *m);
/* pack_material (materials.lucb:105-119): 64 floats. */
void or_pack_material(const or_material *m, float program, float out[64]);
/* pack_lights (lights.lucb:29-131): 28 floats per light into `out`, then the textured
 * dome's image as environment_of (environment.lucb:118-156) makes it: its texels (ACEScg
 * and weight, 4 floats each) and cumulative weights (each row's, then the rows'), padded
 * to a multiple of 4 floats; the dome's record holds where (row 0 x the weights' sum;
 * rows 1, 2, 3 w the texels' first float4, the width, the height; row 6 w the cumulative
 * weights' first float; the integers as their bits). `out` holds or_pack_lights_size
 * floats. Returns the light count; *distant_power the distant lights' and domes' power. */
size_t or_pack_lights_size(const or_light *lights, size_t count);
size_t or_pack_lights(const or_light *lights, size_t count, double radius, float *out,
                      double *distant_power);
void or_basis_spectra(double lambda, double out[3]);
void or_basis_weights(double out[9]);

typedef struct {
    float *nodes;      /* 12 floats per node */
    uint32_t *links;   /* 2 per node */
    uint32_t *records; /* 4 per emitter, then one per triangle */
    size_t node_count, emitter_count, triangle_count;
    double energy;
} or_light_tree;

/* build_light_tree (light_tree.lucb:91-199). Frees with or_light_tree_free. */
int or_build_light_tree(const float *positions, const uint32_t *indices, const uint32_t *shading,
                        size_t triangle_count, const float *light_rows, size_t light_count,
                        const or_material *library, size_t library_count, or_light_tree *out);
void or_light_tree_free(or_light_tree *t);

#ifdef __cplusplus
}
#endif
#endif
