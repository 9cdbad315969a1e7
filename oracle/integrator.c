/*
 * Oracle (test infrastructure): the reference's path-tracing estimator restated in f64,
 * one path at a time over the same Owen-scrambled Sobol samples the kernels draw:
 * camera.comp:14-50, intersect_closest.comp:45-76, shade_surface.comp:48-312 with the
 * OpenPBR surface of openpbr.c, shade_miss.comp:12-51, intersect_shadow.comp:51-92 (opaque),
 * finish.comp:13-39 and film_convert.comp:36-53, with the helpers of common.glsl,
 * spectrum.glsl, lights.glsl, lighttree.glsl and openpbr.glsl (EON, 87-113).
 * Traversal walks the same BVH nodes in f64 (box tests and Moller-Trumbore in f64).
 * Per pixel it returns the mean and the variance of the per-sample ACEScg values.
 */
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include "oracle.h"
#include "oracle_render.h"
#include "oracle_vec.h"
#include "oracle_openpbr.h"

#define INF 3.0e38
#define NONE 0xffffffffu
#define LIGHT_HIT 0x80000000u

/* ---- scene access ----------------------------------------------------------------- */

static d3 point(const or_render_desc *r, uint32_t i) {
    const float *p = &r->positions[(size_t)i * 3];
    return v3(p[0], p[1], p[2]);
}

static double box_entry64(const or_node *n, d3 o, d3 inv, double tmax) {
    double lo[3] = {n->lo[0], n->lo[1], n->lo[2]}, hi[3] = {n->hi[0], n->hi[1], n->hi[2]};
    double oo[3] = {o.x, o.y, o.z}, iv[3] = {inv.x, inv.y, inv.z};
    double enter = 0.0, leave = tmax;
    for (int k = 0; k < 3; k++) {
        double a = (lo[k] - oo[k]) * iv[k], b = (hi[k] - oo[k]) * iv[k];
        double n0 = a < b ? a : b, f0 = a < b ? b : a;
        if (n0 > enter) enter = n0;
        if (f0 < leave) leave = f0;
    }
    /* A little slack for f64 rounding at box faces. */
    return enter <= leave * (1.0 + 1e-12) + 1e-12 ? enter : -1.0;
}

static double tri_hit64(const or_render_desc *r, uint32_t slot, d3 o, d3 d, double tmax, double *u_out, double *v_out) {
    d3 a = point(r, r->indices[slot * 3]);
    d3 e1 = sub(point(r, r->indices[slot * 3 + 1]), a), e2 = sub(point(r, r->indices[slot * 3 + 2]), a);
    d3 q = cross(d, e2);
    double det = dot(e1, q);
    if (fabs(det) < 1e-30) return -1.0;
    d3 s = sub(o, a);
    double u = dot(s, q) / det;
    if (u < 0.0 || u > 1.0) return -1.0;
    d3 rr = cross(s, e1);
    double v = dot(d, rr) / det;
    if (v < 0.0 || u + v > 1.0) return -1.0;
    double t = dot(e2, rr) / det;
    if (!(t > 0.0 && t < tmax)) return -1.0;
    *u_out = u;
    *v_out = v;
    return t;
}

/* trace_closest / trace_any over the BVH, in f64. Returns the slot or NONE. */
static uint32_t trace64(const or_render_desc *r, d3 o, d3 d, double tmax, int any, double *t_out, double *u_out,
                        double *v_out) {
    const or_node *nodes = r->nodes;
    *t_out = tmax;
    if (r->triangle_count == 0) return NONE;
    d3 inv;
    double dd[3] = {d.x, d.y, d.z}, iv[3];
    for (int k = 0; k < 3; k++) {
        double x = dd[k];
        if (fabs(x) < 1e-20) x = x > 0 ? 1e-20 : (x < 0 ? -1e-20 : 1e-20);
        iv[k] = 1.0 / x;
    }
    inv = v3(iv[0], iv[1], iv[2]);
    if (box_entry64(&nodes[0], o, inv, tmax) < 0.0) return NONE;
    uint32_t stack[128];
    int depth = 0;
    uint32_t node = 0, best = NONE;
    double best_t = tmax;
    for (;;) {
        const or_node *n = &nodes[node];
        if (n->count > 0) {
            for (uint32_t i = 0; i < n->count; i++) {
                double u, v;
                double t = tri_hit64(r, n->first + i, o, d, best_t, &u, &v);
                if (t > 0.0) {
                    best_t = t;
                    best = n->first + i;
                    *u_out = u;
                    *v_out = v;
                    if (any) {
                        *t_out = best_t;
                        return best;
                    }
                }
            }
        } else {
            double a = box_entry64(&nodes[n->first], o, inv, best_t);
            double b = box_entry64(&nodes[n->first + 1], o, inv, best_t);
            if (a >= 0.0 && b >= 0.0) {
                uint32_t near_ = a <= b ? n->first : n->first + 1;
                stack[depth++] = near_ == n->first ? n->first + 1 : n->first;
                node = near_;
                continue;
            }
            if (a >= 0.0) { node = n->first; continue; }
            if (b >= 0.0) { node = n->first + 1; continue; }
        }
        if (depth == 0) break;
        node = stack[--depth];
    }
    *t_out = best_t;
    return best;
}

/* ---- spectra and lights ---------------------------------------------------------------- */

static spec spec_of(const or_render_desc *r, const float fit[4], const float rgb[3], const double lambda[4]) {
    return spec_fit(r->spectral, fit, rgb, lambda);
}

static double spec_max(const or_render_desc *r, spec s) {
    double m = fmax(s.s[0], fmax(s.s[1], s.s[2]));
    return r->spectral ? fmax(m, s.s[3]) : m;
}

static double blackbody_f(double lambda, double kelvin) {
    double peak = 2.8977721e6 / kelvin, x = 1.4387769e7 / (lambda * kelvin), q = peak / lambda;
    return q * q * q * q * q * (142.32492 / (exp(x) - 1.0));
}

static const float *row(const or_render_desc *r, uint32_t light, int k) { return &r->light_rows[light * 28 + k * 4]; }
static uint32_t light_type(const or_render_desc *r, uint32_t l) { return (uint32_t)row(r, l, 0)[3]; }
static int light_visible(const or_render_desc *r, uint32_t l) { return ((uint32_t)row(r, l, 5)[3] & 1u) != 0; }
static d3 rv(const float *x) { return v3(x[0], x[1], x[2]); }

static spec light_radiance(const or_render_desc *r, uint32_t light, const double lambda[4]) {
    const float *rgb = row(r, light, 5);
    spec s = spec_of(r, row(r, light, 4), rgb, lambda);
    if (r->spectral && ((uint32_t)rgb[3] & 2u))
        for (int i = 0; i < 4; i++) s.s[i] *= blackbody_f(lambda[i], row(r, light, 6)[0]);
    return s;
}

typedef struct {
    d3 direction;
    double distance, pdf, cos_light;
    int delta;
} lsample;

/* ---- dome lights (lights.glsl:89-174, environment.lucb) --------------------------------- */

typedef struct {
    const float *texels, *cdf;
    uint32_t width, height;
    double total;
} dome_img;

static uint32_t bits_of(float f) {
    uint32_t u;
    memcpy(&u, &f, 4);
    return u;
}

/* The textured dome's image, where its record says the light rows hold it. */
static int dome_image(const or_render_desc *r, uint32_t light, dome_img *img) {
    uint32_t base = bits_of(row(r, light, 1)[3]);
    if (base == 0) return 0;
    img->texels = &r->light_rows[(size_t)base * 4];
    img->width = bits_of(row(r, light, 2)[3]);
    img->height = bits_of(row(r, light, 3)[3]);
    img->cdf = &r->light_rows[bits_of(row(r, light, 6)[3])];
    img->total = row(r, light, 0)[0];
    return 1;
}

/* dome_texel (lights.glsl:99-110). */
static uint32_t dome_texel(const or_render_desc *r, uint32_t light, const dome_img *img, d3 d, double *sin_theta) {
    d3 l = v3(dot(d, rv(row(r, light, 1))), dot(d, rv(row(r, light, 2))), dot(d, rv(row(r, light, 3))));
    double u = 0.5 + atan2(l.x, -l.z) * (0.5 / PI);
    double v = acos(fmin(fmax(l.y, -1.0), 1.0)) / PI;
    *sin_theta = sqrt(fmax(0.0, 1.0 - l.y * l.y));
    uint32_t x = (uint32_t)(u * (double)img->width), y = (uint32_t)(v * (double)img->height);
    if (x > img->width - 1) x = img->width - 1;
    if (y > img->height - 1) y = img->height - 1;
    return y * img->width + x;
}

static double basis_matrix[9];
static pthread_once_t basis_once = PTHREAD_ONCE_INIT;
static void basis_init(void) { or_basis_weights(basis_matrix); }

/* spec_of_texel (spectrum.glsl:61-80): ACEScg through the basis spectra, or as it is. */
static spec spec_of_texel(const or_render_desc *r, const float *texel, const double lambda[4]) {
    spec s = spec_zero();
    if (!r->spectral) {
        for (int i = 0; i < 3; i++) s.s[i] = texel[i];
        return s;
    }
    pthread_once(&basis_once, basis_init);
    double w[3];
    for (int i = 0; i < 3; i++)
        w[i] = basis_matrix[i * 3] * texel[0] + basis_matrix[i * 3 + 1] * texel[1] + basis_matrix[i * 3 + 2] * texel[2];
    for (int i = 0; i < 4; i++) {
        double b[3];
        or_basis_spectra(lambda[i], b);
        s.s[i] = w[0] * b[0] + w[1] * b[1] + w[2] * b[2];
    }
    return s;
}

/* dome_radiance (lights.glsl:112-118): toward -d, d toward the dome. */
static spec dome_radiance(const or_render_desc *r, uint32_t light, d3 d, const double lambda[4]) {
    spec radiance = light_radiance(r, light, lambda);
    dome_img img;
    if (!dome_image(r, light, &img)) return radiance;
    double sin_theta;
    uint32_t texel = dome_texel(r, light, &img, d, &sin_theta);
    return spec_mul(radiance, spec_of_texel(r, &img.texels[(size_t)texel * 4], lambda));
}

/* dome_pdf (lights.glsl:120-129). */
static double dome_pdf(const or_render_desc *r, uint32_t light, d3 d) {
    dome_img img;
    if (!dome_image(r, light, &img)) return 1.0 / (4.0 * PI);
    double sin_theta;
    uint32_t texel = dome_texel(r, light, &img, d, &sin_theta);
    if (sin_theta <= 0.0) return 0.0;
    double weight = img.texels[(size_t)texel * 4 + 3];
    return weight / img.total * (double)img.width * (double)img.height / (2.0 * PI * PI * sin_theta);
}

/* dome_search (lights.glsl:136-150). */
static uint32_t dome_search(const float *cdf, uint32_t first, uint32_t count, double u, double *within) {
    uint32_t low = 0, high = count - 1;
    while (low < high) {
        uint32_t middle = (low + high) / 2;
        if (cdf[first + middle] > u) high = middle;
        else low = middle + 1;
    }
    double below = low > 0 ? cdf[first + low - 1] : 0.0, above = cdf[first + low];
    *within = above > below ? fmin(fmax((u - below) / (above - below), 0.0), 0.99999994) : 0.5;
    return low;
}

/* sample_dome (lights.glsl:152-174). */
static int sample_dome(const or_render_desc *r, uint32_t light, double u0, double u1, lsample *s) {
    s->distance = INF;
    s->delta = 0;
    s->cos_light = 1.0;
    d3 l;
    dome_img img;
    if (!dome_image(r, light, &img)) {
        double z = 1.0 - 2.0 * u0, rr = sqrt(fmax(0.0, 1.0 - z * z));
        l = v3(rr * cos(2.0 * PI * u1), z, rr * sin(2.0 * PI * u1));
    } else {
        double fy, fx;
        uint32_t y = dome_search(img.cdf, img.width * img.height, img.height, u1, &fy);
        uint32_t x = dome_search(img.cdf, y * img.width, img.width, u0, &fx);
        double theta = PI * ((double)y + fy) / (double)img.height;
        double phi = 2.0 * PI * (((double)x + fx) / (double)img.width - 0.5);
        l = v3(sin(theta) * sin(phi), cos(theta), -sin(theta) * cos(phi));
    }
    s->direction = norm(add(add(mul(rv(row(r, light, 1)), l.x), mul(rv(row(r, light, 2)), l.y)), mul(rv(row(r, light, 3)), l.z)));
    s->pdf = dome_pdf(r, light, s->direction);
    return s->pdf > 0.0;
}

/* The radiance a dome or distant light sends toward -d. */
static spec far_radiance(const or_render_desc *r, uint32_t light, d3 d, const double lambda[4]) {
    return light_type(r, light) == 4 ? dome_radiance(r, light, d, lambda) : light_radiance(r, light, lambda);
}

static d3 sample_cone(d3 axis, double cos_max, double u0, double u1) {
    double c = 1.0 - u0 * (1.0 - cos_max), s = sqrt(fmax(0.0, 1.0 - c * c)), phi = 2.0 * PI * u1;
    d3 t, b;
    onb(axis, &t, &b);
    return norm(add(add(mul(t, s * cos(phi)), mul(b, s * sin(phi))), mul(axis, c)));
}

static double sphere_hit(d3 c, double radius, d3 o, d3 d) {
    d3 oc = sub(o, c);
    double b = dot(oc, d), cc = dot(oc, oc) - radius * radius, h = b * b - cc;
    if (h < 0.0) return INF;
    h = sqrt(h);
    double t = -b - h;
    if (t > 0.0) return t;
    t = -b + h;
    return t > 0.0 ? t : INF;
}

static int sample_light(const or_render_desc *r, uint32_t light, d3 p, double u0, double u1, lsample *s) {
    const float *r0 = row(r, light, 0), *r1 = row(r, light, 1), *r2 = row(r, light, 2), *r3 = row(r, light, 3);
    uint32_t type = (uint32_t)r0[3];
    if (type == 4) return sample_dome(r, light, u0, u1, s);
    s->delta = 0;
    s->cos_light = 1.0;
    if (type == 0 || type == 1) {
        double ax, ay;
        if (type == 0) ax = 2.0 * u0 - 1.0, ay = 2.0 * u1 - 1.0;
        else concentric(u0, u1, &ax, &ay);
        d3 q = add(add(rv(r0), mul(rv(r1), ax)), mul(rv(r2), ay));
        d3 d = sub(q, p);
        double d2 = dot(d, d);
        s->distance = sqrt(d2);
        s->direction = mul(d, 1.0 / s->distance);
        double cl = -dot(s->direction, rv(r3));
        if (cl <= 0.0 || r3[3] <= 0.0) return 0;
        s->pdf = d2 / (cl * r3[3]);
        s->cos_light = cl;
        return 1;
    }
    if (type == 2) {
        d3 tc = sub(rv(r0), p);
        double d2 = dot(tc, tc), rad = r1[3];
        if (d2 <= rad * rad) return 0;
        double cos_max = sqrt(fmax(0.0, 1.0 - rad * rad / d2));
        s->direction = sample_cone(mul(tc, 1.0 / sqrt(d2)), cos_max, u0, u1);
        s->distance = sphere_hit(rv(r0), rad, p, s->direction);
        if (s->distance >= INF) return 0;
        s->pdf = 1.0 / (2.0 * PI * (1.0 - cos_max));
        s->cos_light = fmax(0.0, -dot(s->direction, norm(sub(add(p, mul(s->direction, s->distance)), rv(r0)))));
        return 1;
    }
    d3 axis = neg(rv(r3));
    double cos_half = r2[3];
    s->distance = INF;
    if (cos_half >= 1.0 - 1e-7) {
        s->direction = axis;
        s->pdf = 1.0;
        s->delta = 1;
        return 1;
    }
    s->direction = sample_cone(axis, cos_half, u0, u1);
    s->pdf = 1.0 / (2.0 * PI * (1.0 - cos_half));
    return 1;
}

/* intersect_light (lights.glsl:239-259); `flow`: the ray follows light (a light path), so
 * a flat light stops it only when crossed the way it shines. */
static double intersect_light(const or_render_desc *r, uint32_t light, d3 o, d3 d, double t_max, int flow) {
    const float *r0 = row(r, light, 0);
    uint32_t type = (uint32_t)r0[3];
    if (type == 2) {
        double t = sphere_hit(rv(r0), row(r, light, 1)[3], o, d);
        return t < t_max ? t : INF;
    }
    if (type >= 3) return INF;
    d3 u = rv(row(r, light, 1)), v = rv(row(r, light, 2)), n = rv(row(r, light, 3));
    double facing = dot(d, n);
    if (flow ? facing <= 0.0 : facing >= 0.0) return INF;
    double t = dot(sub(rv(r0), o), n) / facing;
    if (t <= 0.0 || t >= t_max) return INF;
    d3 q = sub(add(o, mul(d, t)), rv(r0));
    double a = dot(q, u) / dot(u, u), b = dot(q, v) / dot(v, v);
    int inside = type == 0 ? (fabs(a) <= 1.0 && fabs(b) <= 1.0) : (a * a + b * b <= 1.0);
    return inside ? t : INF;
}

static double light_hit_pdf(const or_render_desc *r, uint32_t light, d3 o, d3 d, double t) {
    const float *r0 = row(r, light, 0);
    uint32_t type = (uint32_t)r0[3];
    if (type == 2) {
        d3 tc = sub(rv(r0), o);
        double rad = row(r, light, 1)[3];
        double cos_max = sqrt(fmax(0.0, 1.0 - rad * rad / dot(tc, tc)));
        return 1.0 / (2.0 * PI * fmax(1e-12, 1.0 - cos_max));
    }
    if (type == 3) return 1.0 / (2.0 * PI * fmax(1e-12, 1.0 - row(r, light, 2)[3]));
    if (type == 4) return dome_pdf(r, light, d);
    const float *r3 = row(r, light, 3);
    double cl = fmax(1e-12, -dot(d, rv(r3)));
    return t * t / (cl * r3[3]);
}

static uint32_t pick_distant(const or_render_desc *r, double u, double *pdf) {
    uint32_t chosen = NONE;
    for (uint32_t l = 0; l < r->light_count; l++) {
        if (light_type(r, l) < 3) continue;
        chosen = l;
        if (u < row(r, l, 6)[2]) break;
    }
    *pdf = chosen == NONE ? 0.0 : row(r, chosen, 6)[1];
    return chosen;
}

static double ssqrt(double x) { return sqrt(fmax(0.0, x)); }

static double tree_importance(const or_render_desc *r, uint32_t node, d3 p, d3 n) {
    const float *a = &r->tree_nodes[node * 12], *b = a + 4, *c = a + 8;
    if (a[3] <= 0.0f) return 0.0;
    d3 center = mul(add(rv(a), rv(b)), 0.5);
    d3 offset = sub(p, center);
    double radius = 0.5 * len(sub(rv(b), rv(a)));
    double oo = dot(offset, offset);
    double distance2 = fmax(oo, radius);
    d3 wi = oo > 0.0 ? norm(offset) : rv(c);
    double cos_w = dot(rv(c), wi), sin_w = ssqrt(1.0 - cos_w * cos_w);
    double cos_b = oo < radius * radius ? -1.0 : ssqrt(1.0 - radius * radius / oo);
    double sin_b = ssqrt(1.0 - cos_b * cos_b);
    double cos_o = b[3], sin_o = ssqrt(1.0 - cos_o * cos_o);
    double cos_x = cos_w > cos_o ? 1.0 : cos_w * cos_o + sin_w * sin_o;
    double sin_x = cos_w > cos_o ? 0.0 : sin_w * cos_o - cos_w * sin_o;
    double cos_p = cos_x > cos_b ? 1.0 : cos_x * cos_b + sin_x * sin_b;
    if (cos_p <= c[3]) return 0.0;
    double importance = a[3] * cos_p / distance2;
    double cos_i = fabs(dot(wi, n)), sin_i = ssqrt(1.0 - cos_i * cos_i);
    double cos_pi = cos_i > cos_b ? 1.0 : cos_i * cos_b + sin_i * sin_b;
    return fmax(importance * cos_pi, 0.0);
}

static int tree_sample(const or_render_desc *r, double u, d3 p, d3 n, uint32_t *emitter, double *pdf) {
    *pdf = 1.0;
    *emitter = 0;
    if (r->tree_node_count < 1) return 0;
    uint32_t node = 0;
    for (int depth = 0; depth < 64; depth++) {
        uint32_t link = r->tree_links[node * 2];
        if (r->tree_links[node * 2 + 1] & 0x80000000u) {
            *emitter = link;
            return *pdf > 0.0;
        }
        double left = tree_importance(r, link, p, n), right = tree_importance(r, link + 1, p, n);
        if (left + right <= 0.0) return 0;
        double chance = left / (left + right);
        if (u < chance) {
            u = fmin(u / chance, 0.99999994);
            *pdf *= chance;
            node = link;
        } else {
            u = fmin((u - chance) / (1.0 - chance), 0.99999994);
            *pdf *= 1.0 - chance;
            node = link + 1;
        }
    }
    return 0;
}

static double tree_pdf(const or_render_desc *r, uint32_t emitter, d3 p, d3 n) {
    uint32_t trail = r->tree_records[emitter * 4 + 1], depth = r->tree_records[emitter * 4 + 2];
    uint32_t node = 0;
    double pdf = 1.0;
    for (uint32_t level = 0; level < depth; level++) {
        uint32_t link = r->tree_links[node * 2];
        double left = tree_importance(r, link, p, n), right = tree_importance(r, link + 1, p, n);
        if (left + right <= 0.0) return 0.0;
        uint32_t bit = (trail >> level) & 1u;
        pdf *= bit == 0 ? left / (left + right) : right / (left + right);
        node = link + bit;
    }
    return pdf;
}

static const float *material(const or_render_desc *r, uint32_t m, int k) { return &r->materials[m * 64 + k * 4]; }

/* ---- Light tracing (shaders/connect.glsl, common.glsl:112-140) ----------------------- */

/* camera_pdf (common.glsl:132-135): per unit of a pixel's area at unit distance. */
static double camera_pdf(const or_render_desc *r, d3 d) {
    double c = dot(d, v3(r->forward[0], r->forward[1], r->forward[2]));
    return c > 0.0 ? r->pixel_area_inv / (c * c * c) : 0.0;
}

/* lens_point (common.glsl:125-130). */
static d3 lens_point(const or_render_desc *r, double u0, double u1) {
    const float *f = r->frame;
    d3 position = v3(f[0], f[1], f[2]);
    if (r->lens_radius <= 0.0) return position;
    double dx, dy;
    concentric(u0, u1, &dx, &dy);
    dx *= r->lens_radius;
    dy *= r->lens_radius;
    return add(add(position, mul(norm(v3(f[8], f[9], f[10])), dx)), mul(norm(v3(f[12], f[13], f[14])), dy));
}

/* camera_pixel (connect.glsl:30-45). */
static int camera_pixel(const or_render_desc *r, d3 p, d3 lens, uint32_t *pixel, d3 *d_out, double *distance) {
    const float *f = r->frame;
    d3 offset = sub(p, lens);
    *distance = len(offset);
    d3 d = mul(offset, 1.0 / fmax(*distance, 1e-20));
    *d_out = d;
    double c = dot(d, v3(r->forward[0], r->forward[1], r->forward[2]));
    if (c <= 1e-6 || *distance <= 0.0) return 0;
    d3 position = v3(f[0], f[1], f[2]), corner = v3(f[4], f[5], f[6]), du = v3(f[8], f[9], f[10]), dv = v3(f[12], f[13], f[14]);
    double focus = r->focus_distance;
    d3 film = sub(r->lens_radius > 0.0 ? mul(sub(add(lens, mul(d, focus / c)), position), 1.0 / focus) : mul(d, 1.0 / c), corner);
    double x = dot(film, du) / dot(du, du), y = dot(film, dv) / dot(dv, dv);
    if (!(x >= 0.0 && y >= 0.0 && x < (double)r->width && y < (double)r->height)) return 0;
    *pixel = (uint32_t)y * r->width + (uint32_t)x;
    return 1;
}

static double node_energy(const or_render_desc *r, uint32_t node) { return fmax(r->tree_nodes[node * 12 + 3], 0.0); }

/* emitter_power_pdf (connect.glsl:68-83). */
static double emitter_power_pdf(const or_render_desc *r, uint32_t emitter) {
    uint32_t trail = r->tree_records[emitter * 4 + 1], depth = r->tree_records[emitter * 4 + 2];
    uint32_t node = 0;
    double pdf = 1.0;
    for (uint32_t level = 0; level < depth; level++) {
        uint32_t link = r->tree_links[node * 2];
        double left = node_energy(r, link), right = node_energy(r, link + 1);
        if (left + right <= 0.0) return 0.0;
        uint32_t bit = (trail >> level) & 1u;
        pdf *= (bit == 0 ? left : right) / (left + right);
        node = link + bit;
    }
    return pdf;
}

/* emitter_by_power (connect.glsl:86-110). */
static int emitter_by_power(const or_render_desc *r, double u, uint32_t *emitter, double *pdf) {
    *pdf = 1.0;
    *emitter = 0;
    if (r->tree_node_count < 1) return 0;
    uint32_t node = 0;
    for (int depth = 0; depth < 64; depth++) {
        uint32_t link = r->tree_links[node * 2];
        if (r->tree_links[node * 2 + 1] & 0x80000000u) {
            *emitter = link;
            return *pdf > 0.0;
        }
        double left = node_energy(r, link), right = node_energy(r, link + 1);
        if (left + right <= 0.0) return 0;
        double chance = left / (left + right);
        if (u < chance) {
            u = fmin(u / chance, 0.99999994);
            *pdf *= chance;
            node = link;
        } else {
            u = fmin((u - chance) / (1.0 - chance), 0.99999994);
            *pdf *= 1.0 - chance;
            node = link + 1;
        }
    }
    return 0;
}

static int emitter_is_triangle(const or_render_desc *r, uint32_t emitter) {
    return (r->tree_records[emitter * 4] & 0x80000000u) != 0;
}

/* emitter_area_pdf (connect.glsl:116-132); no light paths start from afar here. */
static double emitter_area_pdf(const or_render_desc *r, uint32_t emitter) {
    uint32_t code = r->tree_records[emitter * 4];
    double area;
    if (code & 0x80000000u) {
        uint32_t t = code & 0x7fffffffu;
        d3 a = point(r, r->indices[t * 3]);
        area = 0.5 * len(cross(sub(point(r, r->indices[t * 3 + 1]), a), sub(point(r, r->indices[t * 3 + 2]), a)));
    } else if (light_type(r, code) == 2) {
        double rad = row(r, code, 1)[3];
        area = 4.0 * PI * rad * rad;
    } else {
        area = row(r, code, 3)[3];
    }
    /* Emitters of the tree share light paths with lights from afar. */
    return area > 0.0 ? (1.0 - r->emit_share) * emitter_power_pdf(r, emitter) / area : 0.0;
}

/* ---- light paths from afar (lights.glsl:283-308) --------------------------------------- */

#define AFAR_EMITTER 0x40000000u

static int emits_from_afar(const or_render_desc *r, uint32_t light) {
    uint32_t type = light_type(r, light);
    return type == 4 || (type == 3 && row(r, light, 2)[3] < 1.0f - 1e-7f);
}

static double afar_emission_pdf(const or_render_desc *r, uint32_t light, d3 w) {
    return r->emit_share * row(r, light, 6)[1] * light_hit_pdf(r, light, v3(0, 0, 0), w, INF);
}

static double afar_first_density(const or_render_desc *r, d3 p, d3 w, double c) {
    d3 offset = sub(p, v3(r->emit_center[0], r->emit_center[1], r->emit_center[2]));
    d3 across = sub(offset, mul(w, dot(offset, w)));
    if (dot(across, across) > r->emit_radius * r->emit_radius) return 0.0;
    return c / (PI * r->emit_radius * r->emit_radius);
}

static double emission_direction_pdf(const or_render_desc *r, uint32_t emitter, double c) {
    return fabs(c) / (emitter_is_triangle(r, emitter) ? 2.0 * PI : PI);
}

/* camera_hit_ratio (connect.glsl:141-149). */
static double camera_hit_ratio(const or_render_desc *r, const double mis[4], uint32_t emitter, double cos_light,
                               double distance, double bsdf_pdf) {
    if (emitter == NONE || mis[1] <= 0.0 || bsdf_pdf <= 0.0) return 0.0;
    double d2 = distance * distance;
    double at_vertex = emission_direction_pdf(r, emitter, cos_light) * mis[2] / d2 / mis[1];
    double at_light = emitter_area_pdf(r, emitter) / (bsdf_pdf * fabs(cos_light) / d2);
    return mis[0] * at_vertex * at_light;
}

/* light_cos (lights.glsl:228-232). */
static double light_cos(const or_render_desc *r, uint32_t light, d3 o, d3 d, double t) {
    const float *r0 = row(r, light, 0);
    if ((uint32_t)r0[3] == 2) return fmax(0.0, -dot(d, norm(sub(add(o, mul(d, t)), rv(r0)))));
    return fmax(0.0, -dot(d, rv(row(r, light, 3))));
}

static double mis_weight(double a, double b) {
    a = fmin(a, 1e18);
    b = fmin(b, 1e18);
    return 1.0 / (1.0 + a * a + b * b);
}

static d3 offset_origin(d3 p, d3 n) {
    double s = fmax(1.0, fmax(fabs(p.x), fmax(fabs(p.y), fabs(p.z))));
    return add(p, mul(n, 1e-4 * s));
}

static spec clamped(const or_render_desc *r, spec c, uint32_t total) {
    if (total == 0 || r->clamp <= 0.0) return c;
    double m = spec_max(r, c);
    return m > r->clamp ? spec_scale(c, r->clamp / m) : c;
}

static d3 oct_decode(uint32_t packed) {
    double n[3];
    /* The kernels decode in f32; f64 here. */
    double x = fmax((double)(int16_t)(packed & 0xffff) / 32767.0, -1.0);
    double y = fmax((double)(int16_t)(packed >> 16) / 32767.0, -1.0);
    n[0] = x, n[1] = y, n[2] = 1.0 - fabs(x) - fabs(y);
    if (n[2] < 0.0) {
        double nx = (1.0 - fabs(y)) * (x >= 0.0 ? 1.0 : -1.0), ny = (1.0 - fabs(x)) * (y >= 0.0 ? 1.0 : -1.0);
        n[0] = nx, n[1] = ny;
    }
    return norm(v3(n[0], n[1], n[2]));
}

static double tri_hit_pdf(const or_render_desc *r, uint32_t slot, d3 d, double t) {
    d3 a = point(r, r->indices[slot * 3]);
    d3 cr = cross(sub(point(r, r->indices[slot * 3 + 1]), a), sub(point(r, r->indices[slot * 3 + 2]), a));
    double area = 0.5 * len(cr);
    double cl = fabs(dot(d, cr)) / fmax(1e-20, 2.0 * area);
    return t * t / fmax(1e-20, cl * area);
}

static void spec_to_film(const or_render_desc *r, spec rad, const double lambda[4], double out[3]) {
    if (!r->spectral) {
        out[0] = rad.s[0], out[1] = rad.s[1], out[2] = rad.s[2];
        return;
    }
    double sum[3] = {0, 0, 0};
    for (int i = 0; i < 4; i++) {
        double pdf = or_wavelength_pdf(lambda[i]);
        if (pdf > 0.0) {
            double c[3];
            or_cmf(lambda[i], c);
            for (int k = 0; k < 3; k++) sum[k] += c[k] * (rad.s[i] / pdf);
        }
    }
    for (int k = 0; k < 3; k++) out[k] = sum[k] * 0.25 / r->cmf_integrals[k];
}

/* Cut-out opacity (shade_surface.comp:95-104): whether a ray passes through material `m`
 * at a hit at distance t (f32, as the kernels hold it), with the path's opacity number u. */
static int passes_through(const or_render_desc *r, uint32_t m, float t, double u) {
    double opacity = fmin(fmax(material(r, m, 12)[0], 0.0), 1.0);
    if (!(opacity < 1.0)) return 0;
    uint32_t bits;
    memcpy(&bits, &t, 4);
    double v = u + (double)or_hash_u32(bits) * (1.0 / 4294967296.0);
    return v - floor(v) >= opacity;
}

/* intersect_shadow.comp:58-91: what of a shadow ray's light arrives: 1 unblocked, 0 when
 * something opaque stands in it; through cut-outs (scenes with any), (1 - opacity) of it
 * at each, walked with closest hits. */
static double shadow_kept(const or_render_desc *r, d3 o, d3 d, double reach) {
    double tt, uu, vv;
    if (!r->through) return trace64(r, o, d, reach, 1, &tt, &uu, &vv) == NONE ? 1.0 : 0.0;
    d3 from = o;
    double remaining = reach, kept = 1.0;
    for (int hop = 0; hop < 16; hop++) {
        uint32_t slot = trace64(r, from, d, remaining, 0, &tt, &uu, &vv);
        if (slot == NONE) return kept;
        kept *= 1.0 - fmin(fmax(material(r, r->shading[slot * 4 + 3], 12)[0], 0.0), 1.0);
        if (kept < 1e-4) return 0.0;
        d3 p = add(from, mul(d, tt));
        double margin = 1e-4 * fmax(1.0, fmax(fabs(p.x), fmax(fabs(p.y), fabs(p.z))));
        from = add(p, mul(d, margin));
        remaining -= tt + margin;
        if (remaining <= 0.0) return kept;
    }
    return 0.0;
}

/* One sample of one pixel: its ACEScg value. */
static void render_sample(const or_render_desc *r, uint32_t pixel, uint32_t sample, double out[3], uint64_t rays[2]) {
    const float *f = r->frame;
    double u4[4];
    or_sample4(r->seed, pixel, sample, 0, u4);
    double fx = (double)(pixel % r->width) + u4[0], fy = (double)(pixel / r->width) + u4[1];
    d3 position = v3(f[0], f[1], f[2]), corner = v3(f[4], f[5], f[6]), du = v3(f[8], f[9], f[10]),
       dv = v3(f[12], f[13], f[14]);
    d3 film = add(add(corner, mul(du, fx)), mul(dv, fy));
    int ortho = f[3] > 0.5f;
    d3 origin = ortho ? add(position, film) : position;
    d3 dir = norm(ortho ? cross(du, dv) : film);
    if (!ortho && r->lens_radius > 0.0) {
        d3 fw = v3(r->forward[0], r->forward[1], r->forward[2]);
        d3 focused = add(position, mul(dir, r->focus_distance / dot(dir, fw)));
        double dx, dy;
        concentric(u4[2], u4[3], &dx, &dy);
        origin = add(add(position, mul(norm(du), dx * r->lens_radius)), mul(norm(dv), dy * r->lens_radius));
        dir = norm(sub(focused, origin));
    }
    double lambda[4] = {0, 0, 0, 0};
    if (r->spectral) {
        double w[4];
        or_sample4(r->seed, pixel, sample, 1, w);
        or_sample_wavelengths(w[0], lambda);
    }
    spec throughput = {{1, 1, 1, 1}}, radiance = spec_zero();
    uint32_t bounces = 0;
    d3 vertex = origin, prev_normal = v3(0, 0, 1);
    double survival = 1.0, ray_pdf = 0.0;
    /* Light tracing's MIS state (common.glsl:136-143, camera.comp:42). */
    const int tracing = r->light_paths > 0;
    double mis[4] = {0, 0, 0, 0};
    if (tracing) mis[0] = (double)r->light_paths, mis[3] = camera_pdf(r, dir);
    for (uint32_t round = 0; round < r->max_bounces + 1 + r->through; round++) {
        uint32_t total = bounces & 0xffu;
        double t, hu = 0, hv = 0;
        uint32_t what = trace64(r, origin, dir, INF, 0, &t, &hu, &hv);
        rays[0]++;
        for (uint32_t l = 0; l < r->light_count; l++) {
            if (round == 0 && !light_visible(r, l)) continue;
            double tl = intersect_light(r, l, origin, dir, t, 0);
            if (tl < t) {
                t = tl;
                what = LIGHT_HIT | l;
            }
        }
        if (what == NONE) {
            spec bg = spec_of(r, r->background_fit, r->background_rgb, lambda);
            for (uint32_t l = 0; l < r->light_count; l++) {
                if (light_type(r, l) < 3) continue;
                if (light_type(r, l) == 3) {
                    double cos_half = row(r, l, 2)[3];
                    if (cos_half >= 1.0 - 1e-7 || dot(dir, neg(rv(row(r, l, 3)))) < cos_half) continue;
                }
                double weight = 1.0;
                if (total == 0) {
                    if (!light_visible(r, l)) continue;
                } else if (ray_pdf > 0.0) {
                    /* With light tracing, paths from this light's disk weigh in too. */
                    double traced = 0.0;
                    if (tracing && emits_from_afar(r, l) && mis[1] > 0.0)
                        traced = mis[0] * (afar_first_density(r, vertex, dir, mis[2]) / mis[1]) * (afar_emission_pdf(r, l, dir) / ray_pdf);
                    weight = mis_weight(light_hit_pdf(r, l, v3(0, 0, 0), dir, INF) * (r->p_distant * row(r, l, 6)[1]) / ray_pdf, traced);
                }
                bg = spec_add(bg, spec_scale(far_radiance(r, l, dir, lambda), weight));
            }
            spec c = spec_mul(throughput, bg);
            double m = spec_max(r, c);
            if (total > 0 && r->clamp > 0.0 && m > r->clamp) c = spec_scale(c, r->clamp / m);
            radiance = spec_add(radiance, c);
            break;
        }
        if (what & LIGHT_HIT) {
            uint32_t l = what & ~LIGHT_HIT;
            double weight = 1.0;
            if (total == 0) {
                if (!light_visible(r, l)) break;
            } else if (ray_pdf > 0.0) {
                uint32_t emitter = (uint32_t)row(r, l, 6)[3];
                double reach = len(sub(vertex, add(origin, mul(dir, t))));
                double chance = (1.0 - r->p_distant) * tree_pdf(r, emitter, vertex, prev_normal);
                double traced = tracing ? camera_hit_ratio(r, mis, emitter, light_cos(r, l, vertex, dir, reach), reach, ray_pdf) : 0.0;
                weight = mis_weight(light_hit_pdf(r, l, vertex, dir, reach) * chance / ray_pdf, traced);
            }
            radiance = spec_add(radiance, clamped(r, spec_scale(spec_mul(throughput, light_radiance(r, l, lambda)), weight), total));
            break;
        }
        uint32_t slot = what;
        d3 p0 = point(r, r->indices[slot * 3]);
        d3 geometric = norm(cross(sub(point(r, r->indices[slot * 3 + 1]), p0), sub(point(r, r->indices[slot * 3 + 2]), p0)));
        /* Faces wind counter-clockwise seen from outside: a ray along the normal leaves. */
        int inside = dot(geometric, dir) > 0.0;
        if (inside) geometric = neg(geometric);
        const uint32_t *attr = &r->shading[slot * 4];
        uint32_t m = attr[3];
        d3 p = add(origin, mul(dir, t));
        double reach = len(sub(vertex, p));
        /* The camera's density of this vertex, and what turns the light sampler's pdf here
         * toward the last vertex into that vertex's density (shade_surface.comp:91-94). */
        double density = (total == 0 ? mis[3] : ray_pdf) * fabs(dot(dir, geometric)) / (reach * reach);
        double back_reach = mis[2] / (reach * reach);
        if (r->through) {
            /* A cut-out: pass straight through at the same bounce. */
            double uo[4];
            or_sample4(r->seed, pixel, sample, 4 + 3 * total, uo);
            if (passes_through(r, m, (float)t, uo[0])) {
                origin = offset_origin(p, neg(geometric));
                continue;
            }
        }
        /* A dispersive material ends the secondary wavelengths; the hero carries the sample
         * (openpbr.glsl:182-194). */
        if (r->spectral && material(r, m, 12)[3] != 0.0f && lambda[1] >= 0.0) {
            throughput.s[0] *= 4.0, throughput.s[1] = throughput.s[2] = throughput.s[3] = 0.0;
            radiance.s[0] *= 4.0, radiance.s[1] = radiance.s[2] = radiance.s[3] = 0.0;
            lambda[1] = -lambda[1], lambda[2] = -lambda[2], lambda[3] = -lambda[3];
        }
        const double hero = r->spectral && lambda[1] < 0.0 ? lambda[0] : 0.0;
        const float *em = material(r, m, 7);
        if (em[3] > 0.0f) {
            double weight = 1.0;
            uint32_t emitter = r->tree_records && slot < r->triangle_count ? r->tree_records[r->emitter_count * 4 + slot] : NONE;
            if (total > 0 && ray_pdf > 0.0 && emitter != NONE) {
                double chance = (1.0 - r->p_distant) * tree_pdf(r, emitter, vertex, prev_normal);
                double traced = tracing ? camera_hit_ratio(r, mis, emitter, fabs(dot(dir, geometric)), reach, ray_pdf) : 0.0;
                weight = mis_weight(tri_hit_pdf(r, slot, dir, reach) * chance / ray_pdf, traced);
            }
            radiance = spec_add(radiance, clamped(r, spec_scale(spec_mul(throughput, spec_of(r, material(r, m, 6), em, lambda)), weight), total));
        }
        if (total >= r->max_bounces) break;
        d3 normal = norm(add(add(mul(oct_decode(attr[0]), 1.0 - hu - hv), mul(oct_decode(attr[1]), hu)), mul(oct_decode(attr[2]), hv)));
        if (dot(normal, geometric) < 0.0) normal = neg(normal);
        or_surface surface = or_surface_at(normal, geometric, m, inside);
        d3 wo = or_to_local(&surface, neg(dir));
        or_prepare_surface(&surface, wo, r->materials, (int)r->spectral, lambda);
        d3 from = offset_origin(p, geometric);
        double ul[4];
        or_sample4(r->seed, pixel, sample, 2 + 3 * total, ul);
        lsample s;
        spec emitted = spec_zero();
        double chance = 0.0;
        int sampled = 0;
        uint32_t nee_emitter = NONE, afar = NONE;
        if (ul[0] < r->p_distant) {
            double share;
            uint32_t l = pick_distant(r, ul[0] / r->p_distant, &share);
            if (l != NONE && share > 0.0 && sample_light(r, l, p, ul[1], ul[2], &s)) {
                afar = l;
                chance = r->p_distant * share;
                emitted = far_radiance(r, l, s.direction, lambda);
                sampled = 1;
            }
        } else {
            uint32_t emitter;
            double tc;
            if (tree_sample(r, (ul[0] - r->p_distant) / fmax(1e-7, 1.0 - r->p_distant), from, normal, &emitter, &tc)) {
                chance = (1.0 - r->p_distant) * tc;
                nee_emitter = emitter;
                uint32_t code = r->tree_records[emitter * 4];
                if (code & 0x80000000u) {
                    uint32_t ts = code & 0x7fffffffu;
                    d3 a = point(r, r->indices[ts * 3]), b = point(r, r->indices[ts * 3 + 1]), c = point(r, r->indices[ts * 3 + 2]);
                    double rr = sqrt(ul[1]);
                    d3 q = add(add(mul(a, 1.0 - rr), mul(b, rr * (1.0 - ul[2]))), mul(c, rr * ul[2]));
                    d3 cr = cross(sub(b, a), sub(c, a));
                    double area = 0.5 * len(cr);
                    d3 d = sub(q, p);
                    double d2 = dot(d, d);
                    if (area > 0.0 && d2 > 0.0) {
                        s.distance = sqrt(d2);
                        s.direction = mul(d, 1.0 / s.distance);
                        double cl = fabs(dot(s.direction, cr)) / (2.0 * area);
                        if (cl > 0.0) {
                            s.pdf = d2 / (cl * area);
                            s.cos_light = cl;
                            s.delta = 0;
                            uint32_t tm = r->shading[ts * 4 + 3];
                            emitted = spec_of(r, material(r, tm, 6), material(r, tm, 7), lambda);
                            sampled = 1;
                        }
                    }
                } else if (sample_light(r, code, p, ul[1], ul[2], &s)) {
                    emitted = light_radiance(r, code, lambda);
                    sampled = 1;
                }
            }
        }
        if (sampled && chance > 0.0) {
            double side = dot(s.direction, geometric);
            d3 wi = or_to_local(&surface, s.direction);
            if ((side > 0.0) == (wi.z > 0.0) && (side > 0.0 || surface.p_transmission > 0.0)) {
                double bsdf_pdf;
                spec fv = or_evaluate_surface(&surface, wi, wo, &bsdf_pdf);
                if (bsdf_pdf > 0.0) {
                    double light_pdf = s.pdf * chance;
                    /* The light tracer's density of this path over the camera's BSDF ray
                     * reaching the same light point (shade_surface.comp:210-224). */
                    double traced = 0.0;
                    if (tracing && !s.delta && nee_emitter != NONE && density > 0.0) {
                        double d2 = s.distance * s.distance;
                        double at_last = total == 0 ? 1.0
                                                    : or_light_sampler_pdf(&surface, r->materials, s.direction, neg(dir), hero) *
                                                          back_reach / mis[1];
                        double at_vertex = emission_direction_pdf(r, nee_emitter, s.cos_light) * fabs(side) / d2 / density;
                        double at_light = emitter_area_pdf(r, nee_emitter) / (bsdf_pdf * s.cos_light / d2);
                        traced = mis[0] * at_last * at_vertex * at_light;
                    }
                    if (tracing && afar != NONE && emits_from_afar(r, afar) && density > 0.0) {
                        double at_last = total == 0 ? 1.0
                                                    : or_light_sampler_pdf(&surface, r->materials, s.direction, neg(dir), hero) *
                                                          back_reach / mis[1];
                        double at_vertex = afar_first_density(r, p, s.direction, fabs(side)) / density;
                        double at_light = afar_emission_pdf(r, afar, s.direction) / bsdf_pdf;
                        traced = mis[0] * at_last * at_vertex * at_light;
                    }
                    double weight = s.delta ? 1.0 : mis_weight(bsdf_pdf / light_pdf, traced * bsdf_pdf / light_pdf);
                    spec c = clamped(r, spec_scale(spec_mul(spec_mul(throughput, fv), emitted), fabs(wi.z) * (weight / light_pdf)), total);
                    d3 target = add(p, mul(s.direction, s.distance));
                    double margin = 4e-4 * fmax(1.0, fmax(fabs(target.x), fmax(fabs(target.y), fabs(target.z))));
                    double sreach = s.distance >= INF ? INF : fmax(0.0, s.distance - margin);
                    rays[1]++;
                    double kept = shadow_kept(r, offset_origin(p, side > 0.0 ? geometric : neg(geometric)), s.direction, sreach);
                    if (kept > 0.0) radiance = spec_add(radiance, spec_scale(c, kept));
                }
            }
        }
        double u[4];
        or_sample4(r->seed, pixel, sample, 3 + 3 * total, u);
        d3 wi;
        double pdf, pdf_again;
        uint32_t lobe;
        if (!or_sample_direction(&surface, wo, u[0], u[1], u[3], &wi, &pdf, &lobe)) break;
        spec weight = spec_scale(or_evaluate_surface(&surface, wi, wo, &pdf_again), fabs(wi.z) / pdf);
        d3 direction = or_to_world(&surface, wi);
        /* A shading normal can send a ray to the wrong side of the true surface. */
        double side = dot(direction, geometric);
        if ((side > 0.0) != (wi.z > 0.0)) break;
        uint32_t kind = ((bounces >> (8u * (lobe + 1u))) & 0xffu) + 1u;
        if ((double)kind > r->limits[lobe] || (bounces & 0xffu) >= 255u) break;
        bounces = (bounces & ~(0xffu << (8u * (lobe + 1u)))) + (kind << (8u * (lobe + 1u))) + 1u;
        throughput = spec_mul(throughput, weight);
        double scale = fmin(survival, 1e6);
        if (total + 1 >= 3) {
            double survive = fmin(0.95, spec_max(r, throughput) * scale);
            if (u[2] >= survive) break;
            throughput = spec_scale(throughput, 1.0 / survive);
        }
        d3 next = side > 0.0 ? from : offset_origin(p, neg(geometric));
        if (tracing) {
            /* This vertex's factor of the light tracer's density, settled now that the light
             * sampler's direction here is known (shade_surface.comp:304-307). */
            double at_last = total == 0 ? 1.0
                                        : or_light_sampler_pdf(&surface, r->materials, direction, neg(dir), hero) * back_reach / mis[1];
            mis[0] *= at_last;
            mis[1] = density;
            mis[2] = fabs(side);
            mis[3] = 0.0;
        }
        prev_normal = normal;
        origin = next;
        vertex = next;
        survival = scale;
        dir = direction;
        ray_pdf = pdf;
    }
    double value[3];
    spec_to_film(r, radiance, lambda, value);
    if (!isfinite(value[0]) || !isfinite(value[1]) || !isfinite(value[2])) value[0] = value[1] = value[2] = 0.0;
    if (r->spectral) {
        for (int i = 0; i < 3; i++) out[i] = r->film[i * 3] * value[0] + r->film[i * 3 + 1] * value[1] + r->film[i * 3 + 2] * value[2];
    } else {
        out[0] = value[0], out[1] = value[1], out[2] = value[2];
    }
}

/* light_sample_ratio (light_paths.glsl:15-29): the light sample a camera path at p (the
 * surface `s` faces its side) would take toward the light path's first point x0, over its
 * BSDF pdf toward it. */
static double light_sample_ratio(const or_render_desc *r, uint32_t emitter, const or_surface *s, d3 p, d3 x0,
                                 d3 toward, double bsdf_pdf) {
    if (!(bsdf_pdf > 0.0)) return 0.0;
    d3 from = offset_origin(p, s->geometric);
    if (emitter & AFAR_EMITTER) {
        uint32_t l = emitter & ~AFAR_EMITTER;
        return r->p_distant * row(r, l, 6)[1] * light_hit_pdf(r, l, from, toward, INF) / bsdf_pdf;
    }
    d3 offset = sub(x0, from);
    double reach = len(offset);
    d3 d = mul(offset, 1.0 / reach);
    double chance = (1.0 - r->p_distant) * tree_pdf(r, emitter, from, s->normal);
    uint32_t code = r->tree_records[emitter * 4];
    double pdf = (code & 0x80000000u) ? tri_hit_pdf(r, code & 0x7fffffffu, d, reach) : light_hit_pdf(r, code, from, d, reach);
    return chance * pdf / bsdf_pdf;
}

/* light_emit.comp:21-130 and light_paths.glsl:31-189: light path `index` of sample
 * `sample`, from a distant light with a size (by its share) on a disk facing it, or from
 * an emitter of the light tree chosen by power; each surface it reaches connected to the
 * camera -- what gets through is added, in the film's terms, to `splat` (3 per pixel) --
 * and scattered on by light_lobes' choice. */
static void trace_light_path(const or_render_desc *r, uint32_t sample, uint32_t index, double *splat,
                             uint64_t rays[2]) {
    const uint32_t id = 0x80000000u | (r->light_band + index);
    const double L = (double)r->light_paths;
    double u_point[4], u_pick[4];
    or_sample4(r->seed, id, sample, 0, u_point);
    or_sample4(r->seed, id, sample, 1, u_pick);
    double lambda[4] = {0, 0, 0, 0};
    if (r->spectral) or_sample_wavelengths(u_pick[0], lambda);
    d3 origin, vertex, dir;
    spec throughput;
    double survival, ray_pdf, mis[4];
    uint32_t emitter, code = 0;
    double afar = r->emit_share;
    if (u_pick[1] < afar) {
        /* From afar: a direction by the light's distribution, a point on the disk facing it
         * about the casters' centre, toward the scene (light_emit.comp:31-62). */
        double share;
        uint32_t l = pick_distant(r, u_pick[1] / afar, &share);
        if (l == NONE || share <= 0.0 || !emits_from_afar(r, l)) return;
        lsample s;
        if (!sample_light(r, l, v3(0, 0, 0), u_point[0], u_point[1], &s)) return;
        d3 w = s.direction, t, b;
        double radius = r->emit_radius, dx, dy;
        onb(w, &t, &b);
        concentric(u_point[2], u_point[3], &dx, &dy);
        d3 start = add(add(add(v3(r->emit_center[0], r->emit_center[1], r->emit_center[2]), mul(w, 2.0 * radius)),
                           mul(t, dx * radius)), mul(b, dy * radius));
        double chance = afar * share * s.pdf;
        throughput = spec_scale(far_radiance(r, l, w, lambda), PI * radius * radius / chance);
        double most = spec_max(r, throughput);
        if (!(most > 0.0)) return;
        /* The light "point" is a direction: its density is the chance, and the camera's
         * density of it is its BSDF pdf alone (back_reach 1). */
        emitter = AFAR_EMITTER | l;
        origin = start, vertex = start, dir = neg(w);
        survival = 1.0 / most;
        ray_pdf = 0.0;
        mis[0] = 1.0, mis[1] = chance, mis[2] = 1.0, mis[3] = -1.0;
    } else {
        double chance;
        if (!emitter_by_power(r, (u_pick[1] - afar) / fmax(1e-7, 1.0 - afar), &emitter, &chance)) return;
        chance *= 1.0 - afar;
        code = r->tree_records[emitter * 4];
        d3 q, n;
        spec radiance;
        double area;
        int two_sided = 0;
        if (code & 0x80000000u) {
            uint32_t t = code & 0x7fffffffu;
            d3 a = point(r, r->indices[t * 3]), b = point(r, r->indices[t * 3 + 1]), c = point(r, r->indices[t * 3 + 2]);
            double rr = sqrt(u_point[0]);
            q = add(add(mul(a, 1.0 - rr), mul(b, rr * (1.0 - u_point[1]))), mul(c, rr * u_point[1]));
            d3 cr = cross(sub(b, a), sub(c, a));
            area = 0.5 * len(cr);
            n = mul(cr, 1.0 / fmax(2.0 * area, 1e-30));
            if (u_pick[2] < 0.5) n = neg(n);
            two_sided = 1;
            uint32_t tm = r->shading[t * 4 + 3];
            radiance = spec_of(r, material(r, tm, 6), material(r, tm, 7), lambda);
        } else {
            uint32_t type = light_type(r, code);
            const float *r0 = row(r, code, 0);
            if (type == 2) {
                double rad = row(r, code, 1)[3];
                double z = 1.0 - 2.0 * u_point[0], sz = sqrt(fmax(0.0, 1.0 - z * z)), phi = 2.0 * PI * u_point[1];
                n = v3(sz * cos(phi), sz * sin(phi), z);
                q = add(rv(r0), mul(n, rad));
                area = 4.0 * PI * rad * rad;
            } else {
                double ax, ay;
                if (type == 0) ax = 2.0 * u_point[0] - 1.0, ay = 2.0 * u_point[1] - 1.0;
                else concentric(u_point[0], u_point[1], &ax, &ay);
                q = add(add(rv(r0), mul(rv(row(r, code, 1)), ax)), mul(rv(row(r, code, 2)), ay));
                n = rv(row(r, code, 3));
                area = row(r, code, 3)[3];
            }
            radiance = light_radiance(r, code, lambda);
        }
        if (area <= 0.0) return;
        double dx, dy;
        concentric(u_point[2], u_point[3], &dx, &dy);
        double cos_n = sqrt(fmax(0.0, 1.0 - (dx * dx + dy * dy)));
        if (cos_n <= 0.0) return;
        d3 tg, bt;
        onb(n, &tg, &bt);
        dir = norm(add(add(mul(tg, dx), mul(bt, dy)), mul(n, cos_n)));
        double point_pdf = chance / area;
        ray_pdf = cos_n / (two_sided ? 2.0 * PI : PI);
        throughput = spec_scale(radiance, cos_n / (point_pdf * ray_pdf));
        double largest = spec_max(r, throughput);
        if (!(largest > 0.0)) return;
        origin = offset_origin(q, n), vertex = q;
        survival = 1.0 / largest;
        mis[0] = 1.0, mis[1] = point_pdf, mis[2] = cos_n, mis[3] = -1.0;
    }
    uint32_t bounces = 0;
    for (uint32_t round = 0; round < r->max_bounces + 1 + r->through; round++) {
        uint32_t total = bounces & 0xffu;
        double t, hu = 0, hv = 0;
        uint32_t what = trace64(r, origin, dir, INF, 0, &t, &hu, &hv);
        rays[0]++;
        for (uint32_t l = 0; l < r->light_count; l++) {
            if (total == 0 && !light_visible(r, l)) continue;
            double tl = intersect_light(r, l, origin, dir, t, 1);
            if (tl < t) {
                t = tl;
                what = LIGHT_HIT | l;
            }
        }
        if (what == NONE || (what & LIGHT_HIT)) return;
        uint32_t slot = what;
        d3 p0 = point(r, r->indices[slot * 3]);
        d3 geometric = norm(cross(sub(point(r, r->indices[slot * 3 + 1]), p0), sub(point(r, r->indices[slot * 3 + 2]), p0)));
        int back = dot(geometric, dir) > 0.0;
        if (back) geometric = neg(geometric);
        const uint32_t *attr = &r->shading[slot * 4];
        uint32_t m = attr[3];
        d3 p = add(origin, mul(dir, t));
        if (r->through) {
            double uo[4];
            or_sample4(r->seed, id, sample, 4 + 3 * total, uo);
            if (passes_through(r, m, (float)t, uo[0])) {
                origin = offset_origin(p, neg(geometric));
                continue;
            }
        }
        if (total >= r->max_bounces) return;
        /* Dispersion ends the secondary wavelengths, as on camera paths. */
        if (r->spectral && material(r, m, 12)[3] != 0.0f && lambda[1] >= 0.0) {
            throughput.s[0] *= 4.0, throughput.s[1] = throughput.s[2] = throughput.s[3] = 0.0;
            lambda[1] = -lambda[1], lambda[2] = -lambda[2], lambda[3] = -lambda[3];
        }
        d3 normal = norm(add(add(mul(oct_decode(attr[0]), 1.0 - hu - hv), mul(oct_decode(attr[1]), hu)), mul(oct_decode(attr[2]), hv)));
        if (dot(normal, geometric) < 0.0) normal = neg(normal);
        double ul[4];
        or_sample4(r->seed, id, sample, 2 + 3 * total, ul);
        d3 lens = lens_point(r, ul[0], ul[1]);
        uint32_t pixel = 0;
        d3 to_point;
        double camera_distance;
        int on_film = camera_pixel(r, p, lens, &pixel, &to_point, &camera_distance);
        /* The surface on the side light arrives from, read once: seen from the camera or the
         * next vertex on that side, it is only oriented (light_paths.glsl:93-96). */
        or_surface lit = or_surface_at(normal, geometric, m, back);
        d3 toward_light = neg(dir);
        or_read_material(&lit, r->materials, r->spectral && lambda[1] < 0.0 ? lambda[0] : 0.0);
        or_read_colors(&lit, r->materials, (int)r->spectral, lambda);
        double reach = len(sub(vertex, p));
        double cos_in = fabs(dot(dir, geometric));
        double density = ray_pdf * cos_in / (reach * reach);
        double back_reach = mis[2] / (reach * reach);
        /* The first surface of a path from afar: its density on the disk's shadow, and the
         * light's "point" is a direction (no distance to convert). */
        if (total == 0 && (emitter & AFAR_EMITTER)) {
            density = afar_first_density(r, p, neg(dir), cos_in);
            back_reach = 1.0;
            if (!(density > 0.0)) return;
        }
        double cos_shading_in = dot(toward_light, normal);
        if (cos_shading_in <= 0.0 || cos_in < 1e-6) return;
        double shading_in = cos_shading_in / cos_in;
        if (on_film) {
            d3 to_camera = neg(to_point);
            double side = dot(to_camera, geometric);
            or_surface seen = side > 0.0 ? lit : or_turned(&lit);
            d3 wo = or_to_local(&seen, to_camera), wi = or_to_local(&seen, toward_light);
            if ((dot(toward_light, seen.geometric) > 0.0) == (wi.z > 0.0) && wo.z > 0.0) {
                if (side > 0.0) or_orient_surface(&seen, wo);
                else or_prepare_surface(&seen, wo, r->materials, (int)r->spectral, lambda);
                double camera_bsdf_pdf;
                spec f = or_evaluate_surface(&seen, wi, wo, &camera_bsdf_pdf);
                double camera_density = camera_pdf(r, to_point) * fabs(side) / (camera_distance * camera_distance);
                spec contribution = spec_scale(spec_mul(throughput, f), shading_in * camera_density / L);
                if (spec_max(r, contribution) > 0.0) {
                    double last = mis[1] > 0.0 ? camera_bsdf_pdf * back_reach / mis[1] : 0.0;
                    double ratio = mis[0] * last * camera_density / density;
                    double sample_ratio = total == 0 ? light_sample_ratio(r, emitter, &seen, p, vertex, toward_light, camera_bsdf_pdf)
                                                     : fmax(mis[3], 0.0);
                    double weight = mis_weight(ratio / L, ratio * sample_ratio / L);
                    double margin = 4e-4 * fmax(1.0, fmax(fabs(p.x), fmax(fabs(p.y), fabs(p.z))));
                    d3 so = offset_origin(p, seen.geometric);
                    double sreach = fmax(0.0, camera_distance - margin);
                    int blocked = 0;
                    for (uint32_t l = 0; l < r->light_count && !blocked; l++)
                        if (light_visible(r, l) && intersect_light(r, l, so, to_camera, sreach, 1) < sreach) blocked = 1;
                    if (!blocked) {
                        rays[1]++;
                        double kept = shadow_kept(r, so, to_camera, sreach);
                        if (kept > 0.0) {
                            double v[3];
                            spec_to_film(r, spec_scale(contribution, weight * kept), lambda, v);
                            if (isfinite(v[0]) && isfinite(v[1]) && isfinite(v[2]))
                                for (int k = 0; k < 3; k++) splat[pixel * 3 + k] += v[k];
                        }
                    }
                }
            }
        }
        if (total + 1 >= r->max_bounces) return;
        double u[4];
        or_sample4(r->seed, id, sample, 3 + 3 * total, u);
        /* A direction by the lobe choice light paths sample with, weighed by the BSDF as a
         * camera arriving along it evaluates it (light_paths.glsl:147-178). */
        or_surface choosing = lit;
        or_light_lobes(&choosing);
        d3 wo_light = or_to_local(&lit, toward_light), wi_light;
        double light_pdf;
        uint32_t lobe;
        if (!or_sample_direction(&choosing, wo_light, u[0], u[1], u[3], &wi_light, &light_pdf, &lobe)) return;
        d3 direction = or_to_world(&lit, wi_light);
        double side = dot(direction, geometric);
        if ((side > 0.0) != (wi_light.z > 0.0)) return;
        or_surface seen = side > 0.0 ? lit : or_turned(&lit);
        d3 wo = or_to_local(&seen, direction), wi = or_to_local(&seen, toward_light);
        if ((dot(toward_light, seen.geometric) > 0.0) != (wi.z > 0.0)) return;
        if (side > 0.0) or_orient_surface(&seen, wo);
        else or_prepare_surface(&seen, wo, r->materials, (int)r->spectral, lambda);
        double camera_bsdf_pdf;
        spec f = or_evaluate_surface(&seen, wi, wo, &camera_bsdf_pdf);
        uint32_t kind = ((bounces >> (8u * (lobe + 1u))) & 0xffu) + 1u;
        if ((double)kind > r->limits[lobe] || (bounces & 0xffu) >= 255u) return;
        bounces = (bounces & ~(0xffu << (8u * (lobe + 1u)))) + (kind << (8u * (lobe + 1u))) + 1u;
        throughput = spec_scale(spec_mul(throughput, f), shading_in * fabs(side) / light_pdf);
        if (total + 1 >= 3) {
            double survive = fmin(0.95, spec_max(r, throughput) * survival);
            if (u[2] >= survive) return;
            throughput = spec_scale(throughput, 1.0 / survive);
        }
        if (!(spec_max(r, throughput) > 0.0)) return;
        double last = mis[1] > 0.0 ? camera_bsdf_pdf * back_reach / mis[1] : 0.0;
        double sample_ratio = total == 0 ? light_sample_ratio(r, emitter, &seen, p, vertex, toward_light, camera_bsdf_pdf) : mis[3];
        origin = offset_origin(p, side > 0.0 ? geometric : neg(geometric));
        vertex = p;
        dir = direction;
        ray_pdf = light_pdf;
        mis[0] *= last;
        mis[1] = density;
        mis[2] = fabs(side);
        mis[3] = sample_ratio;
    }
}

typedef struct {
    const or_render_desc *r;
    uint32_t samples, sample_first;
    size_t first;
    double *mean, *var;
    size_t next, n;
    uint64_t rays[2];
    pthread_mutex_t lock;
} render_job;

static void *render_worker(void *arg) {
    render_job *j = arg;
    uint64_t rays[2] = {0, 0};
    for (;;) {
        pthread_mutex_lock(&j->lock);
        size_t begin = j->next;
        j->next = begin + 16 < j->n ? begin + 16 : j->n;
        size_t end = j->next;
        pthread_mutex_unlock(&j->lock);
        if (begin >= end) break;
        for (size_t at = begin; at < end; at++) {
            double m[3] = {0, 0, 0}, m2[3] = {0, 0, 0};
            for (uint32_t s = 0; s < j->samples; s++) {
                double v[3];
                render_sample(j->r, (uint32_t)(j->first + at), j->sample_first + s, v, rays);
                for (int k = 0; k < 3; k++) {
                    double delta = v[k] - m[k];
                    m[k] += delta / (double)(s + 1);
                    m2[k] += delta * (v[k] - m[k]);
                }
            }
            for (int k = 0; k < 3; k++) {
                j->mean[at * 3 + k] = m[k];
                j->var[at * 3 + k] = j->samples > 1 ? m2[k] / (double)(j->samples - 1) : 0.0;
            }
        }
    }
    pthread_mutex_lock(&j->lock);
    j->rays[0] += rays[0];
    j->rays[1] += rays[1];
    pthread_mutex_unlock(&j->lock);
    return NULL;
}

void or_render_region(const or_render_desc *r, uint32_t samples, uint32_t sample_first, size_t first, size_t count,
                      double *mean, double *var, uint64_t rays[2], int threads) {
    if (threads <= 0) threads = (int)sysconf(_SC_NPROCESSORS_ONLN);
    if (threads > 256) threads = 256;
    render_job j;
    j.r = r;
    j.samples = samples;
    j.sample_first = sample_first;
    j.first = first;
    j.mean = mean;
    j.var = var;
    j.next = 0;
    j.n = count;
    j.rays[0] = j.rays[1] = 0;
    pthread_mutex_init(&j.lock, NULL);
    pthread_t ids[256];
    for (int i = 0; i < threads; i++) pthread_create(&ids[i], NULL, render_worker, &j);
    for (int i = 0; i < threads; i++) pthread_join(ids[i], NULL);
    pthread_mutex_destroy(&j.lock);
    if (rays) {
        rays[0] = j.rays[0];
        rays[1] = j.rays[1];
    }
}

void or_render(const or_render_desc *r, uint32_t samples, double *mean, double *var, int threads) {
    or_render_region(r, samples, 0, 0, (size_t)r->width * r->height, mean, var, NULL, threads);
}

/* ---- or_render_traced -------------------------------------------------------------- */

typedef struct {
    const or_render_desc *r;
    uint32_t sample;
    double *camera;             /* 3 per pixel */
    double *splats;             /* 3 per pixel per worker */
    size_t pixels;
    size_t next_pixel, next_light;
    uint64_t rays[2];
    pthread_mutex_t lock;
} traced_job;

typedef struct {
    traced_job *j;
    int worker;
} traced_arg;

static void *traced_worker(void *arg) {
    traced_arg *a = arg;
    traced_job *j = a->j;
    double *splat = j->splats + (size_t)a->worker * j->pixels * 3;
    uint64_t rays[2] = {0, 0};
    for (;;) {
        pthread_mutex_lock(&j->lock);
        size_t begin = j->next_pixel;
        j->next_pixel = begin + 64 < j->pixels ? begin + 64 : j->pixels;
        size_t end = j->next_pixel;
        pthread_mutex_unlock(&j->lock);
        if (begin >= end) break;
        for (size_t at = begin; at < end; at++) render_sample(j->r, (uint32_t)at, j->sample, &j->camera[at * 3], rays);
    }
    for (;;) {
        pthread_mutex_lock(&j->lock);
        size_t begin = j->next_light;
        j->next_light = begin + 64 < j->r->light_paths ? begin + 64 : j->r->light_paths;
        size_t end = j->next_light;
        pthread_mutex_unlock(&j->lock);
        if (begin >= end) break;
        for (size_t i = begin; i < end; i++) trace_light_path(j->r, j->sample, (uint32_t)i, splat, rays);
    }
    pthread_mutex_lock(&j->lock);
    j->rays[0] += rays[0];
    j->rays[1] += rays[1];
    pthread_mutex_unlock(&j->lock);
    return NULL;
}

void or_render_traced(const or_render_desc *r, uint32_t samples, uint32_t sample_first, double *mean, double *var,
                      uint64_t rays[2], int threads) {
    if (threads <= 0) threads = (int)sysconf(_SC_NPROCESSORS_ONLN);
    if (threads > 256) threads = 256;
    const size_t pixels = (size_t)r->width * r->height;
    traced_job j;
    j.r = r;
    j.pixels = pixels;
    j.camera = calloc(pixels * 3, sizeof(double));
    j.splats = calloc(pixels * 3 * (size_t)threads, sizeof(double));
    j.rays[0] = j.rays[1] = 0;
    double *m2 = calloc(pixels * 3, sizeof(double));
    for (size_t i = 0; i < pixels * 3; i++) mean[i] = 0.0;
    pthread_mutex_init(&j.lock, NULL);
    for (uint32_t s = 0; s < samples; s++) {
        j.sample = sample_first + s;
        j.next_pixel = j.next_light = 0;
        for (size_t i = 0; i < pixels * 3 * (size_t)threads; i++) j.splats[i] = 0.0;
        pthread_t ids[256];
        traced_arg args[256];
        for (int w = 0; w < threads; w++) {
            args[w].j = &j;
            args[w].worker = w;
            pthread_create(&ids[w], NULL, traced_worker, &args[w]);
        }
        for (int w = 0; w < threads; w++) pthread_join(ids[w], NULL);
        for (size_t px = 0; px < pixels; px++) {
            double sp[3] = {0, 0, 0};
            for (int w = 0; w < threads; w++)
                for (int k = 0; k < 3; k++) sp[k] += j.splats[((size_t)w * pixels + px) * 3 + k];
            double film_sp[3];
            if (r->spectral) {
                for (int k = 0; k < 3; k++) film_sp[k] = r->film[k * 3] * sp[0] + r->film[k * 3 + 1] * sp[1] + r->film[k * 3 + 2] * sp[2];
            } else {
                for (int k = 0; k < 3; k++) film_sp[k] = sp[k];
            }
            for (int k = 0; k < 3; k++) {
                double v = j.camera[px * 3 + k] + film_sp[k];
                double delta = v - mean[px * 3 + k];
                mean[px * 3 + k] += delta / (double)(s + 1);
                m2[px * 3 + k] += delta * (v - mean[px * 3 + k]);
            }
        }
    }
    for (size_t i = 0; i < pixels * 3; i++) var[i] = samples > 1 ? m2[i] / (double)(samples - 1) : 0.0;
    pthread_mutex_destroy(&j.lock);
    if (rays) {
        rays[0] = j.rays[0];
        rays[1] = j.rays[1];
    }
    free(m2);
    free(j.camera);
    free(j.splats);
}
