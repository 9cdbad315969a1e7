/*
 * Oracle (test infrastructure): colour science of src/render/spectrum.lucb (host, f64)
 * and the kernels' wavelength sampling of shaders/spectrum.glsl, restated in f64.
 * Also the octahedral normal encoding of src/render/scene.lucb:400-412 and its decode.
 */
#include <math.h>
#include <string.h>

#include "oracle.h"

#define LAMBDA_MIN 360.0
#define LAMBDA_MAX 830.0

typedef struct {
    double m[9];
} mat3;

static void apply(const mat3 *a, const double v[3], double out[3]) {
    double r[3];
    for (int i = 0; i < 3; i++) r[i] = a->m[i * 3] * v[0] + a->m[i * 3 + 1] * v[1] + a->m[i * 3 + 2] * v[2];
    memcpy(out, r, sizeof r);
}

/* Matrix3.times (spectrum.lucb:38-45) */
static mat3 times(const mat3 *a, const mat3 *b) {
    mat3 out;
    for (int row = 0; row < 3; row++)
        for (int col = 0; col < 3; col++) {
            double sum = 0.0;
            for (int k = 0; k < 3; k++) sum += a->m[row * 3 + k] * b->m[k * 3 + col];
            out.m[row * 3 + col] = sum;
        }
    return out;
}

/* Matrix3.inverse (spectrum.lucb:47-55) */
static mat3 inverse(const mat3 *x) {
    const double *a = x->m;
    double c0 = a[4] * a[8] - a[5] * a[7];
    double c1 = a[5] * a[6] - a[3] * a[8];
    double c2 = a[3] * a[7] - a[4] * a[6];
    double d = 1.0 / (a[0] * c0 + a[1] * c1 + a[2] * c2);
    mat3 r = {{c0 * d, (a[2] * a[7] - a[1] * a[8]) * d, (a[1] * a[5] - a[2] * a[4]) * d,
               c1 * d, (a[0] * a[8] - a[2] * a[6]) * d, (a[2] * a[3] - a[0] * a[5]) * d,
               c2 * d, (a[1] * a[6] - a[0] * a[7]) * d, (a[0] * a[4] - a[1] * a[3]) * d}};
    return r;
}

/* acescg_to_xyz (spectrum.lucb:61-64) */
static mat3 acescg_to_xyz(void) {
    mat3 m = {{0.6624541811, 0.1340042065, 0.1561876870, 0.2722287168, 0.6740817658, 0.0536895174,
               -0.0055746495, 0.0040607335, 1.0103391003}};
    return m;
}

/* bradford (spectrum.lucb:67-71) */
static mat3 bradford(const double source[3], const double target[3]) {
    mat3 cone = {{0.8951, 0.2664, -0.1614, -0.7502, 1.7135, 0.0367, 0.0389, -0.0685, 1.0296}};
    double s[3], t[3];
    apply(&cone, source, s);
    apply(&cone, target, t);
    mat3 diag = {{t[0] / s[0], 0, 0, 0, t[1] / s[1], 0, 0, 0, t[2] / s[2]}};
    mat3 inv = inverse(&cone);
    mat3 a = times(&inv, &diag);
    return times(&a, &cone);
}

/* acescg_to_xyz_e (spectrum.lucb:74-76) */
static mat3 acescg_to_xyz_e_m(void) {
    mat3 to_xyz = acescg_to_xyz();
    double white[3] = {1.0, 1.0, 1.0}, w[3];
    apply(&to_xyz, white, w);
    mat3 b = bradford(w, white);
    return times(&b, &to_xyz);
}

void or_acescg_to_xyz_e(double out[9]) {
    mat3 m = acescg_to_xyz_e_m();
    memcpy(out, m.m, sizeof m.m);
}

/* film_matrix (spectrum.lucb:79-80) */
void or_film_matrix(double out[9]) {
    mat3 m = acescg_to_xyz_e_m();
    mat3 f = inverse(&m);
    memcpy(out, f.m, sizeof f.m);
}

/* lobe (spectrum.lucb:82-84) */
static double lobe(double x, double mean, double below, double above) {
    double t = (x - mean) / (x < mean ? below : above);
    return exp(-0.5 * t * t);
}

/* cmf (spectrum.lucb:87-91) */
void or_cmf(double lambda, double out[3]) {
    out[0] = 1.056 * lobe(lambda, 599.8, 37.9, 31.0) + 0.362 * lobe(lambda, 442.0, 16.0, 26.7) -
             0.065 * lobe(lambda, 501.1, 20.4, 26.2);
    out[1] = 0.821 * lobe(lambda, 568.8, 46.9, 40.5) + 0.286 * lobe(lambda, 530.9, 16.3, 31.1);
    out[2] = 1.217 * lobe(lambda, 437.0, 11.8, 36.0) + 0.681 * lobe(lambda, 459.0, 26.0, 13.8);
}

/* cmf_integrals (spectrum.lucb:94-100) */
void or_cmf_integrals(double out[3]) {
    double sum[3] = {0, 0, 0}, c[3];
    double lambda = LAMBDA_MIN;
    while (lambda <= LAMBDA_MAX) {
        or_cmf(lambda, c);
        for (int k = 0; k < 3; k++) sum[k] = sum[k] + c[k];
        lambda += 1.0;
    }
    memcpy(out, sum, sizeof sum);
}

/* basis_spectra (environment.lucb:27-35): blue, green, red at lambda nm. */
void or_basis_spectra(double lambda, double out[3]) {
    double blue = 1.0 - 1.0 / (1.0 + exp(-(lambda - 490.0) / 12.0));
    double red = 1.0 / (1.0 + exp(-(lambda - 595.0) / 12.0));
    out[0] = blue;
    out[1] = 1.0 - blue - red;
    out[2] = red;
}

/* basis_weights (environment.lucb:37-58): ACEScg to the basis spectra's weights, the
 * inverse of their colours through the film. */
void or_basis_weights(double out[9]) {
    double integrals[3], columns[3][3] = {{0}}, b[3], c[3];
    or_cmf_integrals(integrals);
    for (double lambda = LAMBDA_MIN; lambda <= LAMBDA_MAX; lambda += 1.0) {
        or_basis_spectra(lambda, b);
        or_cmf(lambda, c);
        for (int k = 0; k < 3; k++)
            for (int i = 0; i < 3; i++) columns[k][i] += c[i] * b[k];
    }
    mat3 film;
    or_film_matrix(film.m);
    double rgb[3][3];
    for (int k = 0; k < 3; k++) {
        double xyz[3] = {columns[k][0] / integrals[0], columns[k][1] / integrals[1], columns[k][2] / integrals[2]};
        apply(&film, xyz, rgb[k]);
    }
    mat3 colors = {{rgb[0][0], rgb[1][0], rgb[2][0], rgb[0][1], rgb[1][1], rgb[2][1], rgb[0][2], rgb[1][2], rgb[2][2]}};
    mat3 w = inverse(&colors);
    memcpy(out, w.m, sizeof w.m);
}

static double sigmoid(double z) { return 0.5 + z / (2.0 * sqrt(1.0 + z * z)); }

enum { FIT_SAMPLES = 95 };

/* fit_xyz (spectrum.lucb:122-129) */
static void fit_xyz(const double k[3], const double integrals[3], const double *observer, double out[3]) {
    double sum[3] = {0, 0, 0};
    for (int at = 0; at < FIT_SAMPLES; at++) {
        double lambda = LAMBDA_MIN + 5.0 * (double)at;
        double x = (lambda - LAMBDA_MIN) / (LAMBDA_MAX - LAMBDA_MIN);
        double s = sigmoid((k[0] * x + k[1]) * x + k[2]);
        for (int c = 0; c < 3; c++) sum[c] = sum[c] + observer[at * 3 + c] * (s * 5.0);
    }
    for (int c = 0; c < 3; c++) out[c] = sum[c] / integrals[c];
}

static double vlen(const double v[3]) { return sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]); }

/* fit_spectrum (spectrum.lucb:136-168) */
void or_fit_spectrum(const double rgb[3], double out[4]) {
    double largest = fmax(rgb[0], fmax(rgb[1], rgb[2]));
    if (largest <= 0.0) {
        out[0] = out[1] = out[2] = out[3] = 0.0;
        return;
    }
    if (fabs(rgb[0] - rgb[1]) < 1e-6 * largest && fabs(rgb[1] - rgb[2]) < 1e-6 * largest) {
        out[0] = out[1] = out[2] = 0.0;
        out[3] = 2.0 * largest;
        return;
    }
    mat3 to_e = acescg_to_xyz_e_m();
    double half[3] = {rgb[0] * (0.5 / largest), rgb[1] * (0.5 / largest), rgb[2] * (0.5 / largest)};
    double target[3], integrals[3], observer[FIT_SAMPLES * 3];
    apply(&to_e, half, target);
    or_cmf_integrals(integrals);
    for (int at = 0; at < FIT_SAMPLES; at++) or_cmf(LAMBDA_MIN + 5.0 * (double)at, &observer[at * 3]);
    double k[3] = {0, 0, 0};
    for (int iteration = 0; iteration < 40; iteration++) {
        double r[3], f[3];
        fit_xyz(k, integrals, observer, f);
        for (int c = 0; c < 3; c++) r[c] = f[c] - target[c];
        if (vlen(r) < 1e-7) break;
        const double h = 1e-4;
        double cols[3][3];
        for (int j = 0; j < 3; j++) {
            double kk[3] = {k[0], k[1], k[2]};
            kk[j] = k[j] + h;
            double g[3];
            fit_xyz(kk, integrals, observer, g);
            for (int c = 0; c < 3; c++) cols[j][c] = ((g[c] - target[c]) - r[c]) * (1.0 / h);
        }
        mat3 jm = {{cols[0][0], cols[1][0], cols[2][0], cols[0][1], cols[1][1], cols[2][1],
                    cols[0][2], cols[1][2], cols[2][2]}};
        mat3 ji = inverse(&jm);
        double step[3];
        apply(&ji, r, step);
        if (!isfinite(step[0]) || !isfinite(step[1]) || !isfinite(step[2])) break;
        double size = vlen(step);
        double longest = 20.0;
        double scale = size > longest ? longest / size : 1.0;
        for (int c = 0; c < 3; c++) k[c] = k[c] - step[c] * scale;
    }
    out[0] = k[0];
    out[1] = k[1];
    out[2] = k[2];
    out[3] = 2.0 * largest;
}

/* blackbody (spectrum.lucb:173-177) */
double or_blackbody(double lambda, double kelvin) {
    double peak = 2.8977721e6 / kelvin;
    double x = 1.4387769e7 / (lambda * kelvin);
    double r = peak / lambda;
    return r * r * r * r * r * ((exp(4.965114) - 1.0) / (exp(x) - 1.0));
}

/* blackbody_xyz (spectrum.lucb:180-187) */
void or_blackbody_xyz(double kelvin, double out[3]) {
    double integrals[3], sum[3] = {0, 0, 0}, c[3];
    or_cmf_integrals(integrals);
    double lambda = LAMBDA_MIN;
    while (lambda <= LAMBDA_MAX) {
        or_cmf(lambda, c);
        double b = or_blackbody(lambda, kelvin);
        for (int k = 0; k < 3; k++) sum[k] = sum[k] + c[k] * b;
        lambda += 1.0;
    }
    for (int k = 0; k < 3; k++) out[k] = sum[k] / integrals[k];
}

/* sample_wavelengths (spectrum.glsl:10-17), f64 */
void or_sample_wavelengths(double u, double out[4]) {
    for (int i = 0; i < 4; i++) {
        double v = u + (double)i * 0.25;
        v = v - floor(v);
        out[i] = 538.0 - 138.888889 * atanh(0.85691062 - 1.82750197 * v);
    }
}

/* wavelength_pdf (spectrum.glsl:19-23), f64 */
double or_wavelength_pdf(double lambda) {
    if (lambda < LAMBDA_MIN || lambda > LAMBDA_MAX) return 0.0;
    double c = cosh(0.0072 * (lambda - 538.0));
    return 0.0039398042 / (c * c);
}

/* octahedral (scene.lucb:400-412) */
uint32_t or_octahedral(const double n[3]) {
    double length = fabs(n[0]) + fabs(n[1]) + fabs(n[2]);
    if (length <= 0.0) {
        double up[3] = {0.0, 1.0, 0.0};
        return or_octahedral(up);
    }
    double x = n[0] / length, y = n[1] / length;
    if (n[2] < 0.0) {
        double fx = (1.0 - fabs(y)) * (x >= 0.0 ? 1.0 : -1.0);
        double fy = (1.0 - fabs(x)) * (y >= 0.0 ? 1.0 : -1.0);
        x = fx;
        y = fy;
    }
    int64_t qx = (int64_t)round(fmin(fmax(x, -1.0), 1.0) * 32767.0);
    int64_t qy = (int64_t)round(fmin(fmax(y, -1.0), 1.0) * 32767.0);
    return (uint32_t)(qx & 0xffff) | ((uint32_t)(qy & 0xffff) << 16);
}

/* octahedral_decode (common.glsl:262-267) in f64 */
void or_octahedral_decode(uint32_t packed, double out[3]) {
    double x = fmax(-1.0, (double)(int16_t)(uint16_t)(packed & 0xffff) / 32767.0);
    double y = fmax(-1.0, (double)(int16_t)(uint16_t)(packed >> 16) / 32767.0);
    double n[3] = {x, y, 1.0 - fabs(x) - fabs(y)};
    if (n[2] < 0.0) {
        double nx = (1.0 - fabs(y)) * (x >= 0.0 ? 1.0 : -1.0);
        double ny = (1.0 - fabs(x)) * (y >= 0.0 ? 1.0 : -1.0);
        n[0] = nx;
        n[1] = ny;
    }
    double l = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
    for (int k = 0; k < 3; k++) out[k] = n[k] / l;
}
