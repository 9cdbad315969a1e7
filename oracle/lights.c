/*
 * Oracle (test infrastructure): light records (src/render/lights.lucb:29-131),
 * OpenPBR material records (src/render/materials.lucb:46-119) and the light tree
 * (src/render/light_tree.lucb:41-244), restated.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

#define PI 3.14159265358979323846

static double luminance(const double rgb[3]) {
    return 0.2722287168 * rgb[0] + 0.6740817658 * rgb[1] + 0.0536895174 * rgb[2];
}

static double vlen(const double v[3]) { return sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]); }

static void vcross(const double a[3], const double b[3], double out[3]) {
    double r[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
    memcpy(out, r, sizeof r);
}

/* OpenPbr.standard (materials.lucb:46-53) */
void or_material_standard(or_material *m) {
    memset(m, 0, sizeof *m);
    m->base_weight = 1.0;
    for (int k = 0; k < 3; k++) {
        m->base_color[k] = 0.8;
        m->specular_color[k] = 1.0;
        m->transmission_color[k] = 1.0;
        m->coat_color[k] = 1.0;
        m->emission_color[k] = 1.0;
    }
    m->specular_weight = 1.0;
    m->specular_roughness = 0.3;
    m->specular_ior = 1.5;
    m->coat_ior = 1.6;
    m->coat_darkening = 1.0;
    m->geometry_opacity = 1.0;
    m->transmission_dispersion_abbe_number = 20.0;
}

/* cauchy_b (materials.lucb:90-101) */
static double cauchy_b(const or_material *m) {
    double scale = m->transmission_dispersion_scale, abbe = m->transmission_dispersion_abbe_number;
    if (scale <= 0.0 || abbe <= 0.0 || m->transmission_weight <= 0.0) return 0.0;
    double f = 486.1, c = 656.3;
    return (m->specular_ior - 1.0) * scale / (abbe * (1.0 / (f * f) - 1.0 / (c * c)));
}

/* pack_material (materials.lucb:105-119) */
void or_pack_material(const or_material *m, float program, float out[64]) {
    double colors[5][3];
    memcpy(colors[0], m->base_color, sizeof colors[0]);
    memcpy(colors[1], m->specular_color, sizeof colors[1]);
    memcpy(colors[2], m->coat_color, sizeof colors[2]);
    for (int k = 0; k < 3; k++) colors[3][k] = m->emission_color[k] * m->emission_luminance;
    memcpy(colors[4], m->transmission_color, sizeof colors[4]);
    double weights[5] = {m->base_weight, m->specular_weight, m->coat_weight, m->emission_luminance,
                         m->transmission_weight};
    int at = 0;
    for (int i = 0; i < 5; i++) {
        double clipped[3] = {fmax(colors[i][0], 0.0), fmax(colors[i][1], 0.0), fmax(colors[i][2], 0.0)};
        double fit[4];
        or_fit_spectrum(clipped, fit);
        double values[8] = {fit[0], fit[1], fit[2], fit[3], colors[i][0], colors[i][1], colors[i][2], weights[i]};
        for (int k = 0; k < 8; k++) out[at++] = (float)values[k];
    }
    double rest[24] = {m->base_metalness, m->base_diffuse_roughness, m->specular_roughness,
                       m->specular_roughness_anisotropy, m->specular_ior, m->coat_roughness, m->coat_ior,
                       m->coat_darkening, m->geometry_opacity, m->geometry_thin_walled ? 1.0 : 0.0,
                       m->coat_roughness_anisotropy, cauchy_b(m), (double)program, 0, 0, 0,
                       0, 0, 0, 0, 0, 0, 0, 0};
    for (int k = 0; k < 24; k++) out[at++] = (float)rest[k];
}

/* The first dome with an image (loading.lucb:55-61), or -1. */
static long textured_dome(const or_light *lights, size_t count) {
    for (size_t i = 0; i < count; i++)
        if (lights[i].shape == 4 && lights[i].image && lights[i].image_width > 0 && lights[i].image_height > 0)
            return (long)i;
    return -1;
}

size_t or_pack_lights_size(const or_light *lights, size_t count) {
    size_t floats = count * 28;
    long dome = textured_dome(lights, count);
    if (dome >= 0) {
        size_t texels = (size_t)lights[dome].image_width * lights[dome].image_height;
        floats += texels * 4 + texels + lights[dome].image_height + 3;
    }
    return floats;
}

static float float_bits(size_t v) {
    uint32_t u = (uint32_t)v;
    float f;
    memcpy(&f, &u, 4);
    return f;
}

/* environment_of (environment.lucb:118-156) into `texels` (4 floats each) and `cdf`
 * (width*height + height floats); *total the weights' sum, *average the mean luminance. */
static void environment_of(const or_light *light, float *texels, float *cdf, double *total, double *average) {
    static const double to_acescg[9] = {0.613097, 0.339523, 0.047379, 0.070194, 0.916354, 0.013452,
                                        0.020616, 0.109570, 0.869815};
    const uint32_t width = light->image_width, height = light->image_height;
    double *rows = malloc(sizeof(double) * height);
    double luminance_sum = 0.0, solid_angle = 0.0;
    size_t at_cdf = 0, at_texel = 0;
    for (uint32_t y = 0; y < height; y++) {
        double sin_theta = sin(PI * ((double)y + 0.5) / (double)height);
        double row = 0.0;
        size_t start = at_cdf;
        for (uint32_t x = 0; x < width; x++) {
            const float *p = &light->image[((size_t)y * width + x) * 3];
            double source[3] = {p[0], p[1], p[2]}, rgb[3];
            for (int i = 0; i < 3; i++)
                rgb[i] = fmax(0.0, to_acescg[i * 3] * source[0] + to_acescg[i * 3 + 1] * source[1] +
                                       to_acescg[i * 3 + 2] * source[2]);
            double lum = luminance(rgb), weight = lum * sin_theta;
            texels[at_texel++] = (float)rgb[0];
            texels[at_texel++] = (float)rgb[1];
            texels[at_texel++] = (float)rgb[2];
            texels[at_texel++] = (float)weight;
            row += weight;
            cdf[at_cdf++] = (float)row;
            luminance_sum += lum * sin_theta;
            solid_angle += sin_theta;
        }
        for (uint32_t x = 0; x < width; x++)
            cdf[start + x] = (float)(row > 0.0 ? (double)cdf[start + x] / row : (double)(x + 1) / (double)width);
        rows[y] = row;
    }
    double sum = 0.0, running = 0.0;
    for (uint32_t y = 0; y < height; y++) sum += rows[y];
    for (uint32_t y = 0; y < height; y++) {
        running += rows[y];
        cdf[at_cdf++] = (float)(sum > 0.0 ? running / sum : (double)(y + 1) / (double)height);
    }
    free(rows);
    *total = sum;
    *average = solid_angle > 0.0 ? luminance_sum / solid_angle : 0.0;
}

/* pack_lights (lights.lucb:29-131). */
size_t or_pack_lights(const or_light *lights, size_t count, double radius, float *out,
                      double *distant_power) {
    double film[9];
    or_film_matrix(film);
    double *powers = malloc(sizeof(double) * (count + 1));
    size_t n = 0;
    long dome = textured_dome(lights, count);
    long dome_record = -1;
    double dome_total = 0.0, dome_average = 0.0;
    float *texels = NULL, *cdf = NULL;
    if (dome >= 0) {
        size_t pixels = (size_t)lights[dome].image_width * lights[dome].image_height;
        texels = malloc(sizeof(float) * pixels * 4);
        cdf = malloc(sizeof(float) * (pixels + lights[dome].image_height));
        environment_of(&lights[dome], texels, cdf, &dome_total, &dome_average);
    }
    for (size_t index = 0; index < count; index++) {
        const or_light *light = &lights[index];
        const double *m = light->matrix;
        double position[3] = {m[9], m[10], m[11]};
        double minus_z[3] = {-m[6], -m[7], -m[8]};
        double l = vlen(minus_z);
        if (!(l > 0.0)) continue;
        double emits[3] = {minus_z[0] / l, minus_z[1] / l, minus_z[2] / l};
        double u[3] = {0, 0, 0}, v[3] = {0, 0, 0}, uv[3];
        double size = 0.0, area = 0.0, cos_half = 1.0, kind = 0.0;
        if (light->shape == 0) {
            for (int k = 0; k < 3; k++) {
                u[k] = m[k] * (0.5 * light->width);
                v[k] = m[3 + k] * (0.5 * light->height);
            }
            vcross(u, v, uv);
            area = 4.0 * vlen(uv);
        } else if (light->shape == 1) {
            kind = 1.0;
            for (int k = 0; k < 3; k++) {
                u[k] = m[k] * light->radius;
                v[k] = m[3 + k] * light->radius;
            }
            vcross(u, v, uv);
            area = PI * vlen(uv);
        } else if (light->shape == 2) {
            kind = 2.0;
            double det = m[0] * (m[4] * m[8] - m[5] * m[7]) - m[3] * (m[1] * m[8] - m[2] * m[7]) +
                         m[6] * (m[1] * m[5] - m[2] * m[4]);
            size = light->radius * cbrt(fabs(det));
            area = 4.0 * PI * size * size;
        } else if (light->shape == 4) {
            /* Rows 1-3 are the dome's axes (X, Y, Z): world to its frame. */
            kind = 4.0;
            double lx = vlen(&m[0]), ly = vlen(&m[3]), lz = vlen(&m[6]);
            for (int k = 0; k < 3; k++) {
                u[k] = m[k] / lx;
                v[k] = m[3 + k] / ly;
                emits[k] = m[6 + k] / lz;
            }
        } else {
            kind = 3.0;
            cos_half = cos(0.5 * light->angle * PI / 180.0);
        }
        double scale = light->intensity * exp2(light->exposure);
        if (kind < 3.0 && light->normalize) {
            if (area <= 0.0) continue;
            scale = scale / area;
        }
        if (kind == 3.0 && cos_half < 1.0 - 1e-7) scale = scale / (2.0 * PI * (1.0 - cos_half));
        double rgb[3] = {light->color[0] * scale, light->color[1] * scale, light->color[2] * scale};
        double fit[4];
        or_fit_spectrum(light->color, fit);
        fit[3] = fit[3] * scale;
        double flags = light->visible ? 1.0 : 0.0;
        if (light->temperature > 0.0) {
            double tint[3], unit[3], tinted[3];
            or_blackbody_xyz(light->temperature, tint);
            fit[3] = fit[3] / tint[1];
            for (int k = 0; k < 3; k++) unit[k] = tint[k] * (1.0 / tint[1]);
            for (int i = 0; i < 3; i++) tinted[i] = film[i * 3] * unit[0] + film[i * 3 + 1] * unit[1] + film[i * 3 + 2] * unit[2];
            for (int k = 0; k < 3; k++) rgb[k] = rgb[k] * tinted[k];
            flags += 2.0;
        }
        double power = -1.0;
        if (kind == 3.0)
            power = fmax(0.0, luminance(rgb)) * (cos_half < 1.0 - 1e-7 ? 2.0 * PI * (1.0 - cos_half) : 1.0) *
                    PI * radius * radius;
        if (kind == 4.0) {
            /* What a sphere of its mean radiance pours into the scene's disk. */
            double mean = 1.0;
            if ((long)index == dome) {
                mean = dome_average;
                dome_record = (long)n;
            }
            power = fmax(0.0, luminance(rgb)) * mean * PI * PI * radius * radius;
        }
        powers[n] = power;
        double rows[28] = {position[0], position[1], position[2], kind, u[0], u[1], u[2], size,
                           v[0], v[1], v[2], cos_half, emits[0], emits[1], emits[2], area,
                           fit[0], fit[1], fit[2], fit[3], rgb[0], rgb[1], rgb[2], flags,
                           light->temperature, 0.0, 0.0, 0.0};
        for (int k = 0; k < 28; k++) out[n * 28 + k] = (float)rows[k];
        n++;
    }
    double total = 0.0;
    size_t distant = 0;
    for (size_t i = 0; i < n; i++)
        if (powers[i] >= 0.0) {
            total += powers[i];
            distant++;
        }
    double running = 0.0;
    size_t emitter = 0;
    for (size_t i = 0; i < n; i++) {
        float *row6 = &out[i * 28 + 24];
        if (powers[i] < 0.0) {
            row6[3] = (float)emitter;
            emitter++;
            continue;
        }
        double share = total > 0.0 ? powers[i] / total : 1.0 / (double)distant;
        running += share;
        row6[1] = (float)share;
        row6[2] = (float)running;
    }
    free(powers);
    if (dome_record >= 0) {
        const uint32_t width = lights[dome].image_width, height = lights[dome].image_height;
        const size_t pixels = (size_t)width * height;
        size_t at = n * 28;
        const size_t texel_base = at / 4;
        memcpy(&out[at], texels, sizeof(float) * pixels * 4);
        at += pixels * 4;
        const size_t cdf_base = at;
        memcpy(&out[at], cdf, sizeof(float) * (pixels + height));
        at += pixels + height;
        while (at % 4 != 0) out[at++] = 0.0f;
        float *record = &out[dome_record * 28];
        record[0] = (float)dome_total;
        record[1] = record[2] = 0.0f;
        record[7] = float_bits(texel_base);
        record[11] = float_bits(width);
        record[15] = float_bits(height);
        record[27] = float_bits(cdf_base);
    }
    free(texels);
    free(cdf);
    if (distant_power) *distant_power = total;
    return n;
}

/* ---- the light tree (light_tree.lucb) ------------------------------------------- */

#define EMITTER_TRIANGLE 0x80000000u
#define LEAF_NODE 0x80000000u

typedef struct {
    double lo[3], hi[3], axis[3];
    double theta_o, theta_e, energy;
    uint32_t code;
} emitter_t;

/* cone_union (light_tree.lucb:41-56) */
static void cone_union(const double a[3], double a_theta, const double b[3], double b_theta,
                       double out_axis[3], double *out_theta) {
    double dot = a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
    double theta_d = acos(fmin(fmax(dot, -1.0), 1.0));
    if (fmin(theta_d + b_theta, PI) <= a_theta) {
        memcpy(out_axis, a, sizeof(double) * 3), *out_theta = a_theta;
        return;
    }
    if (fmin(theta_d + a_theta, PI) <= b_theta) {
        memcpy(out_axis, b, sizeof(double) * 3), *out_theta = b_theta;
        return;
    }
    double theta_o = 0.5 * (a_theta + theta_d + b_theta);
    if (theta_o >= PI) {
        memcpy(out_axis, a, sizeof(double) * 3), *out_theta = PI;
        return;
    }
    double rotate = theta_o - a_theta;
    double w[3];
    vcross(a, b, w);
    double wl = vlen(w);
    if (wl < 1e-12) {
        memcpy(out_axis, a, sizeof(double) * 3), *out_theta = PI;
        return;
    }
    double k[3] = {w[0] * (1.0 / wl), w[1] * (1.0 / wl), w[2] * (1.0 / wl)}, ka[3];
    vcross(k, a, ka);
    double kdota = k[0] * a[0] + k[1] * a[1] + k[2] * a[2];
    double c = cos(rotate), s = sin(rotate);
    double turned[3];
    for (int i = 0; i < 3; i++) turned[i] = a[i] * c + ka[i] * s + k[i] * (kdota * (1.0 - c));
    double tl = vlen(turned);
    if (tl > 0.0 && isfinite(tl))
        for (int i = 0; i < 3; i++) out_axis[i] = turned[i] / tl;
    else
        memcpy(out_axis, a, sizeof(double) * 3);
    *out_theta = theta_o;
}

static double key_of(const emitter_t *e, uint32_t index, int axis) {
    return (e[index].lo[axis] + e[index].hi[axis]) * 0.5;
}

static void swap_u(uint32_t *o, size_t a, size_t b) {
    uint32_t h = o[a];
    o[a] = o[b];
    o[b] = h;
}

/* select (light_tree.lucb:217-239) */
static void select_k(const emitter_t *e, uint32_t *order, size_t length, size_t k, int axis) {
    size_t low = 0, high = length;
    while (high - low > 1) {
        double pivot = key_of(e, order[(low + high) / 2], axis);
        size_t less = low, at = low, more = high;
        while (at < more) {
            double key = key_of(e, order[at], axis);
            if (key < pivot) {
                swap_u(order, at, less);
                less++;
                at++;
            } else if (key > pivot) {
                more--;
                swap_u(order, at, more);
            } else {
                at++;
            }
        }
        if (k < less)
            high = less;
        else if (k >= more)
            low = more;
        else
            return;
    }
}

typedef struct {
    size_t node, first, count;
    uint32_t trail, depth;
} tree_job;

/* build_light_tree (light_tree.lucb:91-199) */
int or_build_light_tree(const float *positions, const uint32_t *indices, const uint32_t *shading,
                        size_t triangle_count, const float *rows, size_t light_count,
                        const or_material *library, size_t library_count, or_light_tree *tree) {
    memset(tree, 0, sizeof *tree);
    tree->triangle_count = triangle_count;
    emitter_t *emitters = malloc(sizeof(emitter_t) * (light_count + triangle_count + 1));
    size_t count = 0;
    for (size_t index = 0; index < light_count; index++) {
        const float *row = &rows[index * 28];
        double kind = row[3];
        if (kind >= 3.0) continue;
        double position[3] = {row[0], row[1], row[2]};
        double u[3] = {row[4], row[5], row[6]}, v[3] = {row[8], row[9], row[10]};
        double normal[3] = {row[12], row[13], row[14]};
        double area = row[15];
        double rgb[3] = {row[20], row[21], row[22]};
        double extent[3] = {fabs(u[0]) + fabs(v[0]), fabs(u[1]) + fabs(v[1]), fabs(u[2]) + fabs(v[2])};
        double theta_o = 0.0;
        if (kind == 2.0) {
            double radius = row[7];
            extent[0] = extent[1] = extent[2] = radius;
            theta_o = PI;
        }
        emitter_t *e = &emitters[count++];
        for (int k = 0; k < 3; k++) {
            e->lo[k] = position[k] - extent[k];
            e->hi[k] = position[k] + extent[k];
            e->axis[k] = normal[k];
        }
        e->theta_o = theta_o;
        e->theta_e = 0.5 * PI;
        e->energy = fmax(0.0, luminance(rgb)) * area * PI;
        e->code = (uint32_t)index;
    }
    int emissive = 0;
    for (size_t i = 0; i < library_count; i++) emissive = emissive || library[i].emission_luminance > 0.0;
    for (size_t t = 0; emissive && t < triangle_count; t++) {
        uint32_t material = shading[t * 4 + 3];
        if ((size_t)material >= library_count) continue;
        const or_material *m = &library[material];
        if (m->emission_luminance <= 0.0) continue;
        double p[3][3];
        for (int c = 0; c < 3; c++)
            for (int k = 0; k < 3; k++) p[c][k] = positions[(size_t)indices[t * 3 + c] * 3 + k];
        double e1[3], e2[3], cr[3];
        for (int k = 0; k < 3; k++) {
            e1[k] = p[1][k] - p[0][k];
            e2[k] = p[2][k] - p[0][k];
        }
        vcross(e1, e2, cr);
        double area = 0.5 * vlen(cr);
        if (area <= 0.0) continue;
        emitter_t *e = &emitters[count++];
        for (int k = 0; k < 3; k++) {
            e->lo[k] = fmin(p[0][k], fmin(p[1][k], p[2][k]));
            e->hi[k] = fmax(p[0][k], fmax(p[1][k], p[2][k]));
            e->axis[k] = cr[k] * (0.5 / area);
        }
        double emission[3] = {m->emission_color[0] * m->emission_luminance,
                              m->emission_color[1] * m->emission_luminance,
                              m->emission_color[2] * m->emission_luminance};
        e->theta_o = PI;
        e->theta_e = 0.5 * PI;
        e->energy = fmax(0.0, luminance(emission)) * area * 2.0 * PI;
        e->code = EMITTER_TRIANGLE | (uint32_t)t;
    }
    tree->emitter_count = count;
    tree->records = calloc(count * 4 + triangle_count + 1, sizeof(uint32_t));
    for (size_t t = 0; t < triangle_count; t++) tree->records[count * 4 + t] = OR_NONE;
    for (size_t i = 0; i < count; i++) {
        uint32_t code = emitters[i].code;
        tree->records[i * 4] = code;
        if (code & EMITTER_TRIANGLE) tree->records[count * 4 + (code & ~EMITTER_TRIANGLE)] = (uint32_t)i;
    }
    tree->nodes = calloc((2 * count + 1) * 12, sizeof(float));
    tree->links = calloc((2 * count + 1) * 2, sizeof(uint32_t));
    if (count == 0) {
        free(emitters);
        return 0;
    }
    uint32_t *order = malloc(sizeof(uint32_t) * count);
    for (size_t i = 0; i < count; i++) order[i] = (uint32_t)i;
    tree->node_count = 1;
    tree_job *stack = malloc(sizeof(tree_job) * (2 * count + 2));
    size_t depth = 0;
    stack[depth++] = (tree_job){0, 0, count, 0, 0};
    while (depth > 0) {
        tree_job job = stack[--depth];
        uint32_t *range = order + job.first;
        const emitter_t *first = &emitters[range[0]];
        double lo[3], hi[3], axis[3];
        memcpy(lo, first->lo, sizeof lo);
        memcpy(hi, first->hi, sizeof hi);
        memcpy(axis, first->axis, sizeof axis);
        double theta_o = first->theta_o, theta_e = first->theta_e, energy = 0.0;
        for (size_t i = 0; i < job.count; i++) {
            const emitter_t *e = &emitters[range[i]];
            for (int k = 0; k < 3; k++) {
                lo[k] = fmin(lo[k], e->lo[k]);
                hi[k] = fmax(hi[k], e->hi[k]);
            }
            double merged[3], mt;
            cone_union(axis, theta_o, e->axis, e->theta_o, merged, &mt);
            memcpy(axis, merged, sizeof axis);
            theta_o = mt;
            theta_e = fmax(theta_e, e->theta_e);
            energy += e->energy;
        }
        double values[12] = {lo[0], lo[1], lo[2], energy, hi[0], hi[1], hi[2], cos(theta_o),
                             axis[0], axis[1], axis[2], cos(theta_e)};
        for (int k = 0; k < 12; k++) tree->nodes[job.node * 12 + k] = (float)values[k];
        if (job.node == 0) tree->energy = energy;
        if (job.count == 1) {
            uint32_t emitter = range[0];
            tree->links[job.node * 2] = emitter;
            tree->links[job.node * 2 + 1] = LEAF_NODE;
            tree->records[emitter * 4 + 1] = job.trail;
            tree->records[emitter * 4 + 2] = job.depth;
            continue;
        }
        int axis_index = 0;
        double size[3] = {hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]};
        if (size[1] > size[0] && size[1] >= size[2])
            axis_index = 1;
        else if (size[2] > size[0] && size[2] > size[1])
            axis_index = 2;
        size_t half = job.count / 2;
        select_k(emitters, range, job.count, half, axis_index);
        size_t child = tree->node_count;
        tree->node_count += 2;
        tree->links[job.node * 2] = (uint32_t)child;
        tree->links[job.node * 2 + 1] = 0;
        stack[depth++] = (tree_job){child + 1, job.first + half, job.count - half,
                                    job.trail | (1u << job.depth), job.depth + 1};
        stack[depth++] = (tree_job){child, job.first, half, job.trail, job.depth + 1};
    }
    free(stack);
    free(order);
    free(emitters);
    return 0;
}

void or_light_tree_free(or_light_tree *t) {
    free(t->nodes);
    free(t->links);
    free(t->records);
    memset(t, 0, sizeof *t);
}
