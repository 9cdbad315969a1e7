/*
 * Oracle (test infrastructure): ray frames (src/render/camera.lucb) and the probe's
 * pixel-centre rays (shaders/probe.comp), restated.
 */
#include <math.h>
#include <string.h>

#include "oracle.h"

static double len3(const double v[3]) { return sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]); }

static int normalized(const double v[3], double out[3]) {
    double l = len3(v);
    if (!(l > 0.0) || !isfinite(l)) return 400;
    for (int k = 0; k < 3; k++) out[k] = v[k] / l;
    return 0;
}

static void cross_d(const double a[3], const double b[3], double out[3]) {
    out[0] = a[1] * b[2] - a[2] * b[1];
    out[1] = a[2] * b[0] - a[0] * b[2];
    out[2] = a[0] * b[1] - a[1] * b[0];
}

/* ray_frame (camera.lucb:57-76) */
int or_ray_frame(const double m[12], int projection, double focal_length,
                 double horizontal_aperture, double f_stop, double focus_distance, uint32_t width,
                 uint32_t height, or_frame *out) {
    if (width == 0 || height == 0) return 400;
    double right[3], up[3], back[3];
    if (normalized(&m[0], right) || normalized(&m[3], up) || normalized(&m[6], back)) return 400;
    memset(out, 0, sizeof *out);
    double aspect = (double)height / (double)width;
    int ortho = projection == 1;
    double half_width = ortho ? 0.05 * horizontal_aperture : 0.5 * horizontal_aperture / focal_length;
    double half_height = half_width * aspect;
    for (int k = 0; k < 3; k++) {
        double forward = -back[k];
        out->forward[k] = forward;
        out->corner[k] = right[k] * -half_width + up[k] * half_height + (ortho ? 0.0 : forward);
        out->du[k] = right[k] * (2.0 * half_width / (double)width);
        out->dv[k] = up[k] * (-2.0 * half_height / (double)height);
        out->position[k] = m[9 + k];
    }
    out->orthographic = ortho;
    out->width = width;
    out->height = height;
    out->lens_radius = (f_stop > 0.0 && !ortho) ? 0.0005 * focal_length / f_stop : 0.0;
    out->focus_distance = focus_distance;
    return 0;
}

/* look_frame (camera.lucb:84-95) */
int or_look_frame(const double position[3], const double forward[3], const double up[3],
                  double tan_half_height, uint32_t width, uint32_t height, int orthographic,
                  or_frame *out) {
    if (width == 0 || height == 0) return 400;
    if (!(tan_half_height > 0.0 && tan_half_height < 1e6)) return 400;
    double ahead[3], side[3], right[3], above[3];
    if (normalized(forward, ahead)) return 400;
    cross_d(ahead, up, side);
    if (normalized(side, right)) return 400;
    cross_d(right, ahead, above);
    memset(out, 0, sizeof *out);
    double half_height = tan_half_height;
    double half_width = half_height * (double)width / (double)height;
    for (int k = 0; k < 3; k++) {
        out->corner[k] = right[k] * -half_width + above[k] * half_height + (orthographic ? 0.0 : ahead[k]);
        out->du[k] = right[k] * (2.0 * half_width / (double)width);
        out->dv[k] = above[k] * (-2.0 * half_height / (double)height);
        out->position[k] = position[k];
        out->forward[k] = ahead[k];
    }
    out->orthographic = orthographic;
    out->width = width;
    out->height = height;
    out->lens_radius = 0.0;
    out->focus_distance = 1.0;
    return 0;
}

/* RayFrame.pack (camera.lucb:41-47) */
void or_frame_pack(const or_frame *f, float out[16]) {
    double v[16] = {f->position[0], f->position[1], f->position[2], f->orthographic ? 1.0 : 0.0,
                    f->corner[0],   f->corner[1],   f->corner[2],   0.0,
                    f->du[0],       f->du[1],       f->du[2],       (double)f->width,
                    f->dv[0],       f->dv[1],       f->dv[2],       (double)f->height};
    for (int k = 0; k < 16; k++) out[k] = (float)v[k];
}

/* RayFrame.ray (camera.lucb:51-54) */
void or_frame_ray(const or_frame *f, double x, double y, double origin[3], double direction[3]) {
    for (int k = 0; k < 3; k++) {
        double film = f->corner[k] + f->du[k] * x + f->dv[k] * y;
        if (f->orthographic) {
            origin[k] = f->position[k] + film;
            direction[k] = f->forward[k];
        } else {
            origin[k] = f->position[k];
            direction[k] = film;
        }
    }
}

/* probe.comp:21-34, in f32: the pixel-centre ray of every pixel, row by row from the
 * top. normalize is v / sqrt(dot(v, v)), the form the CUDA kernel uses. */
void or_probe_rays(const float b[16], float *rays) {
    uint32_t width = (uint32_t)b[11], height = (uint32_t)b[15];
    const float *position = &b[0], *corner = &b[4], *du = &b[8], *dv = &b[12];
    int ortho = b[3] > 0.5f;
    float forward[3] = {du[1] * dv[2] - du[2] * dv[1], du[2] * dv[0] - du[0] * dv[2],
                        du[0] * dv[1] - du[1] * dv[0]};
    float fl = sqrtf(forward[0] * forward[0] + forward[1] * forward[1] + forward[2] * forward[2]);
    for (uint32_t y = 0; y < height; y++) {
        for (uint32_t x = 0; x < width; x++) {
            float *r = &rays[((size_t)y * width + x) * 8];
            float fx = (float)x + 0.5f, fy = (float)y + 0.5f;
            for (int k = 0; k < 3; k++) {
                float film = corner[k] + fx * du[k];
                film = film + fy * dv[k];
                r[k] = ortho ? position[k] + film : position[k];
                r[4 + k] = ortho ? forward[k] / fl : film;
            }
            r[3] = 0.0f;
            r[7] = 3.0e38f;
        }
    }
}
