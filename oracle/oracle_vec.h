/*
 * Oracle (test infrastructure): f64 vectors and four-lane spectra shared by the
 * integrator's restatement (integrator.c) and the OpenPBR surface's (openpbr.c).
 */
#ifndef LUCE_ORACLE_VEC_H
#define LUCE_ORACLE_VEC_H

#include <math.h>

#define PI 3.14159265358979323846

typedef struct {
    double x, y, z;
} d3;

static inline d3 v3(double x, double y, double z) { d3 r = {x, y, z}; return r; }
static inline d3 add(d3 a, d3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline d3 sub(d3 a, d3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline d3 mul(d3 a, double s) { return v3(a.x * s, a.y * s, a.z * s); }
static inline double dot(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline d3 cross(d3 a, d3 b) { return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
static inline double len(d3 a) { return sqrt(dot(a, a)); }
static inline d3 norm(d3 a) { return mul(a, 1.0 / len(a)); }
static inline d3 neg(d3 a) { return v3(-a.x, -a.y, -a.z); }

typedef struct {
    double s[4];
} spec;

static inline spec spec_scale(spec a, double k) { for (int i = 0; i < 4; i++) a.s[i] *= k; return a; }
static inline spec spec_mul(spec a, spec b) { for (int i = 0; i < 4; i++) a.s[i] *= b.s[i]; return a; }
static inline spec spec_add(spec a, spec b) { for (int i = 0; i < 4; i++) a.s[i] += b.s[i]; return a; }
static inline spec spec_zero(void) { spec z = {{0, 0, 0, 0}}; return z; }
static inline spec spec_all(double v) { spec z = {{v, v, v, v}}; return z; }

/* A color as a spectrum at the path's wavelengths (spectrum.glsl spec_of): the sigmoid
 * polynomial fit at each lane's wavelength, or the RGB itself in the RGB build. */
static inline spec spec_fit(int spectral, const float fit[4], const float rgb[3], const double lambda[4]) {
    spec s;
    if (!spectral) {
        s.s[0] = rgb[0], s.s[1] = rgb[1], s.s[2] = rgb[2], s.s[3] = 0.0;
        return s;
    }
    for (int i = 0; i < 4; i++) {
        double x = (lambda[i] - 360.0) / (830.0 - 360.0);
        double z = ((double)fit[0] * x + fit[1]) * x + fit[2];
        s.s[i] = fit[3] * (0.5 + z / (2.0 * sqrt(1.0 + z * z)));
    }
    return s;
}

/* An orthonormal basis around n (Duff et al. 2017; common.glsl:270-276). */
static inline void onb(d3 n, d3 *t, d3 *b) {
    double s = n.z >= 0.0 ? 1.0 : -1.0, a = -1.0 / (s + n.z), c = n.x * n.y * a;
    *t = v3(1.0 + s * n.x * n.x * a, s * c, -s * n.x);
    *b = v3(c, s + n.y * n.y * a, -n.y);
}

/* Shirley and Chiu's concentric map of the unit square onto the disk. */
static inline void concentric(double u0, double u1, double *x, double *y) {
    double ox = 2.0 * u0 - 1.0, oy = 2.0 * u1 - 1.0, rr, th;
    if (ox == 0.0 && oy == 0.0) { *x = *y = 0.0; return; }
    if (fabs(ox) > fabs(oy)) { rr = ox; th = (PI / 4.0) * (oy / ox); }
    else { rr = oy; th = (PI / 2.0) - (PI / 4.0) * (ox / oy); }
    *x = rr * cos(th);
    *y = rr * sin(th);
}

#endif
