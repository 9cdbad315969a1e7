// Host colour science for the spectral build's constants and colour fits, after
// src/render/spectrum.lucb (f64): the ACEScg <-> XYZ-under-E matrices through a Bradford
// adaptation, Wyman-Sloan-Shirley's CIE 1931 fit and its per-channel integrals at 1 nm,
// Jakob-Hanika sigmoid fits by damped Gauss-Newton, peak-normalized blackbodies, and
// the octahedral normal encoding of scene.lucb:400-412.
#include <algorithm>
#include <array>
#include <cstring>
#include <mutex>
#include <unordered_map>

#include "common.hpp"

namespace lr {
namespace {

constexpr double kLambdaMin = 360.0, kLambdaMax = 830.0;

M3 mul(const M3 &a, const M3 &b) {
    M3 out{};
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) {
            double s = 0.0;
            for (int k = 0; k < 3; k++) s += a.m[r * 3 + k] * b.m[k * 3 + c];
            out.m[r * 3 + c] = s;
        }
    return out;
}

// The adjugate over the determinant, cofactors in the order spectrum.lucb:47-55 takes.
M3 inv(const M3 &x) {
    const double *a = x.m;
    double c0 = a[4] * a[8] - a[5] * a[7];
    double c1 = a[5] * a[6] - a[3] * a[8];
    double c2 = a[3] * a[7] - a[4] * a[6];
    double d = 1.0 / (a[0] * c0 + a[1] * c1 + a[2] * c2);
    return M3{{c0 * d, (a[2] * a[7] - a[1] * a[8]) * d, (a[1] * a[5] - a[2] * a[4]) * d,
               c1 * d, (a[0] * a[8] - a[2] * a[6]) * d, (a[2] * a[3] - a[0] * a[5]) * d,
               c2 * d, (a[1] * a[6] - a[0] * a[7]) * d, (a[0] * a[4] - a[1] * a[3]) * d}};
}

const M3 kAcescgToXyz{{0.6624541811, 0.1340042065, 0.1561876870, 0.2722287168, 0.6740817658,
                       0.0536895174, -0.0055746495, 0.0040607335, 1.0103391003}};
const M3 kBradfordCone{{0.8951, 0.2664, -0.1614, -0.7502, 1.7135, 0.0367, 0.0389, -0.0685, 1.0296}};

double lobe(double x, double mean, double below, double above) {
    double t = (x - mean) / (x < mean ? below : above);
    return std::exp(-0.5 * t * t);
}

V3 cmf(double l) {
    return {1.056 * lobe(l, 599.8, 37.9, 31.0) + 0.362 * lobe(l, 442.0, 16.0, 26.7) -
                0.065 * lobe(l, 501.1, 20.4, 26.2),
            0.821 * lobe(l, 568.8, 46.9, 40.5) + 0.286 * lobe(l, 530.9, 16.3, 31.1),
            1.217 * lobe(l, 437.0, 11.8, 36.0) + 0.681 * lobe(l, 459.0, 26.0, 13.8)};
}

double sigmoid(double z) { return 0.5 + z / (2.0 * std::sqrt(1.0 + z * z)); }

constexpr int kFitSamples = 95;  // 5 nm apart over 360..830 nm

V3 fit_xyz(const V3 &k, const V3 &integrals, const std::array<V3, kFitSamples> &observer) {
    V3 sum;
    for (int at = 0; at < kFitSamples; at++) {
        double lambda = kLambdaMin + 5.0 * (double)at;
        double x = (lambda - kLambdaMin) / (kLambdaMax - kLambdaMin);
        double s = sigmoid((k.x * x + k.y) * x + k.z);
        sum = sum + observer[at] * (s * 5.0);
    }
    return {sum.x / integrals.x, sum.y / integrals.y, sum.z / integrals.z};
}

double blackbody(double lambda, double kelvin) {
    double peak = 2.8977721e6 / kelvin;
    double x = 1.4387769e7 / (lambda * kelvin);
    double r = peak / lambda;
    return r * r * r * r * r * ((std::exp(4.965114) - 1.0) / (std::exp(x) - 1.0));
}

}  // namespace

M3 acescg_to_xyz_e() {
    V3 white = kAcescgToXyz.apply({1.0, 1.0, 1.0});
    V3 s = kBradfordCone.apply(white), t = kBradfordCone.apply({1.0, 1.0, 1.0});
    M3 diag{{t.x / s.x, 0, 0, 0, t.y / s.y, 0, 0, 0, t.z / s.z}};
    M3 bradford = mul(mul(inv(kBradfordCone), diag), kBradfordCone);
    return mul(bradford, kAcescgToXyz);
}

M3 film_matrix() { return inv(acescg_to_xyz_e()); }

V3 cmf_integrals() {
    V3 sum;
    for (double lambda = kLambdaMin; lambda <= kLambdaMax; lambda += 1.0) sum = sum + cmf(lambda);
    return sum;
}

namespace {

// The fit's fixed inputs, computed once: the observer at the fit's samples and its
// per-channel integrals at 1 nm.
struct FitTables {
    std::array<V3, kFitSamples> observer;
    V3 integrals;
    M3 to_xyz;
    FitTables() {
        for (int at = 0; at < kFitSamples; at++) observer[at] = cmf(kLambdaMin + 5.0 * (double)at);
        integrals = cmf_integrals();
        to_xyz = acescg_to_xyz_e();
    }
};

const FitTables &fit_tables() {
    static const FitTables tables;
    return tables;
}

void fit_spectrum_uncached(const V3 &rgb, double out[4]);

// Fits by their colour's exact bits: a scene's materials are loaded again for every
// render of it (a batch member, a server session), and a fit is a few hundred thousand
// operations; the memo keeps at most kFitMemo of them.
constexpr size_t kFitMemo = 1u << 18;

struct FitKey {
    uint64_t bits[3];
    bool operator==(const FitKey &o) const {
        return bits[0] == o.bits[0] && bits[1] == o.bits[1] && bits[2] == o.bits[2];
    }
};
struct FitKeyHash {
    size_t operator()(const FitKey &k) const {
        uint64_t h = 1469598103934665603ull;
        for (uint64_t b : k.bits) h = (h ^ b) * 1099511628211ull;
        return (size_t)h;
    }
};

}  // namespace

void fit_spectrum(const V3 &rgb, double out[4]) {
    static std::mutex lock;
    static std::unordered_map<FitKey, std::array<double, 4>, FitKeyHash> memo;
    FitKey key;
    std::memcpy(&key.bits[0], &rgb.x, 8);
    std::memcpy(&key.bits[1], &rgb.y, 8);
    std::memcpy(&key.bits[2], &rgb.z, 8);
    {
        std::lock_guard<std::mutex> guard(lock);
        auto it = memo.find(key);
        if (it != memo.end()) {
            for (int k = 0; k < 4; k++) out[k] = it->second[k];
            return;
        }
    }
    fit_spectrum_uncached(rgb, out);
    std::lock_guard<std::mutex> guard(lock);
    if (memo.size() >= kFitMemo) memo.clear();
    memo.emplace(key, std::array<double, 4>{out[0], out[1], out[2], out[3]});
}

namespace {

void fit_spectrum_uncached(const V3 &rgb, double out[4]) {
    double largest = std::max(rgb.x, std::max(rgb.y, rgb.z));
    if (largest <= 0.0) {
        out[0] = out[1] = out[2] = out[3] = 0.0;
        return;
    }
    if (std::fabs(rgb.x - rgb.y) < 1e-6 * largest && std::fabs(rgb.y - rgb.z) < 1e-6 * largest) {
        out[0] = out[1] = out[2] = 0.0;
        out[3] = 2.0 * largest;
        return;
    }
    const FitTables &tables = fit_tables();
    const V3 target = tables.to_xyz.apply(rgb * (0.5 / largest));
    const V3 &integrals = tables.integrals;
    const std::array<V3, kFitSamples> &observer = tables.observer;
    V3 k;
    for (int iteration = 0; iteration < 40; iteration++) {
        V3 r = fit_xyz(k, integrals, observer) - target;
        if (r.length() < 1e-7) break;
        const double h = 1e-4;
        V3 jx = ((fit_xyz({k.x + h, k.y, k.z}, integrals, observer) - target) - r) * (1.0 / h);
        V3 jy = ((fit_xyz({k.x, k.y + h, k.z}, integrals, observer) - target) - r) * (1.0 / h);
        V3 jz = ((fit_xyz({k.x, k.y, k.z + h}, integrals, observer) - target) - r) * (1.0 / h);
        M3 j{{jx.x, jy.x, jz.x, jx.y, jy.y, jz.y, jx.z, jy.z, jz.z}};
        V3 step = inv(j).apply(r);
        if (!std::isfinite(step.x) || !std::isfinite(step.y) || !std::isfinite(step.z)) break;
        double size = step.length();
        k = k - step * (size > 20.0 ? 20.0 / size : 1.0);
    }
    out[0] = k.x;
    out[1] = k.y;
    out[2] = k.z;
    out[3] = 2.0 * largest;
}

}  // namespace

V3 blackbody_xyz(double kelvin) {
    V3 integrals = cmf_integrals(), sum;
    for (double lambda = kLambdaMin; lambda <= kLambdaMax; lambda += 1.0)
        sum = sum + cmf(lambda) * blackbody(lambda, kelvin);
    return {sum.x / integrals.x, sum.y / integrals.y, sum.z / integrals.z};
}

// The three smooth spectra a dome's texel is made of (environment.lucb:27-35): blue below
// ~490 nm, red above ~595 nm, green between; they sum to the flat spectrum.
V3 basis_spectra(double lambda) {
    const double blue = 1.0 - 1.0 / (1.0 + std::exp(-(lambda - 490.0) / 12.0));
    const double red = 1.0 / (1.0 + std::exp(-(lambda - 595.0) / 12.0));
    return {blue, 1.0 - blue - red, red};
}

// basis_weights (environment.lucb:37-58): ACEScg -> the basis spectra's weights, the
// inverse of the matrix whose columns are the basis spectra's colours through the film.
M3 basis_weights() {
    const V3 integrals = cmf_integrals();
    V3 columns[3];
    for (double lambda = kLambdaMin; lambda <= kLambdaMax; lambda += 1.0) {
        const V3 b = basis_spectra(lambda), matching = cmf(lambda);
        for (int k = 0; k < 3; k++) columns[k] = columns[k] + matching * b[k];
    }
    const M3 film = film_matrix();
    V3 rgb[3];
    for (int k = 0; k < 3; k++)
        rgb[k] = film.apply({columns[k].x / integrals.x, columns[k].y / integrals.y, columns[k].z / integrals.z});
    const M3 colors{{rgb[0].x, rgb[1].x, rgb[2].x, rgb[0].y, rgb[1].y, rgb[2].y, rgb[0].z, rgb[1].z, rgb[2].z}};
    return inv(colors);
}

uint32_t octahedral(const V3 &n) {
    double length = std::fabs(n.x) + std::fabs(n.y) + std::fabs(n.z);
    if (length <= 0.0) return octahedral({0.0, 1.0, 0.0});
    double x = n.x / length, y = n.y / length;
    if (n.z < 0.0) {
        double fx = (1.0 - std::fabs(y)) * (x >= 0.0 ? 1.0 : -1.0);
        double fy = (1.0 - std::fabs(x)) * (y >= 0.0 ? 1.0 : -1.0);
        x = fx;
        y = fy;
    }
    int64_t qx = (int64_t)std::round(std::min(std::max(x, -1.0), 1.0) * 32767.0);
    int64_t qy = (int64_t)std::round(std::min(std::max(y, -1.0), 1.0) * 32767.0);
    return (uint32_t)(qx & 0xffff) | ((uint32_t)(qy & 0xffff) << 16);
}

}  // namespace lr
