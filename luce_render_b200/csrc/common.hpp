// Shared host-side plumbing: status codes with a per-thread message, small f64 vector
// math, and the compiled scene held behind the C ABI's lr_scene handle.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/luce_render_b200.h"

namespace lr {

// An error that crosses the C ABI as a status code and lr_last_error()'s text.
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string &message) : std::runtime_error(message), code(c) {}
};

[[noreturn]] inline void fail(int code, const std::string &message) { throw Error(code, message); }

void set_last_error(const char *message);

// Runs `body`, turning exceptions into a status code and the thread's last error.
template <class F>
int guarded(F &&body) {
    try {
        body();
        set_last_error("");
        return LR_OK;
    } catch (const Error &e) {
        set_last_error(e.what());
        return e.code;
    } catch (const std::bad_alloc &) {
        set_last_error("out of host memory");
        return LR_LIMIT;
    } catch (const std::exception &e) {
        set_last_error(e.what());
        return LR_INVALID;
    }
}

struct V3 {
    double x = 0, y = 0, z = 0;
    V3() = default;
    V3(double a, double b, double c) : x(a), y(b), z(c) {}
    double operator[](int k) const { return k == 0 ? x : (k == 1 ? y : z); }
    double &operator[](int k) { return k == 0 ? x : (k == 1 ? y : z); }
    V3 operator+(const V3 &o) const { return {x + o.x, y + o.y, z + o.z}; }
    V3 operator-(const V3 &o) const { return {x - o.x, y - o.y, z - o.z}; }
    V3 operator*(double s) const { return {x * s, y * s, z * s}; }
    double dot(const V3 &o) const { return x * o.x + y * o.y + z * o.z; }
    V3 cross(const V3 &o) const { return {y * o.z - z * o.y, z * o.x - x * o.z, x * o.y - y * o.x}; }
    double length() const { return std::sqrt(x * x + y * y + z * z); }
};

// Normalized, or an `invalid` error for a zero or non-finite vector.
inline V3 unit(const V3 &v, const char *what) {
    double l = v.length();
    if (!(l > 0.0) || !std::isfinite(l)) fail(LR_INVALID, std::string(what) + " has no direction");
    return {v.x / l, v.y / l, v.z / l};
}

// A 3x3 matrix by rows (spectrum.lucb's Matrix3).
struct M3 {
    double m[9];
    V3 apply(const V3 &v) const {
        return {m[0] * v.x + m[1] * v.y + m[2] * v.z, m[3] * v.x + m[4] * v.y + m[5] * v.z,
                m[6] * v.x + m[7] * v.y + m[8] * v.z};
    }
};

// Colour science (spectrum.cpp).
M3 film_matrix();       // XYZ under E -> ACEScg
M3 acescg_to_xyz_e();   // ACEScg -> XYZ under E
V3 cmf_integrals();     // each CIE channel's sum over 360..830 nm at 1 nm
void fit_spectrum(const V3 &rgb, double out[4]);
V3 blackbody_xyz(double kelvin);
M3 basis_weights();     // ACEScg -> weights of a dome texel's three basis spectra
uint32_t octahedral(const V3 &n);
// The flat shading normal a compile gives a triangle without authored normals: its own
// geometric normal (b - a) x (c - a), octahedrally encoded.
uint32_t flat_normal(const float *a, const float *b, const float *c);

// sampler.cpp: the 128 Sobol direction numbers (4 dimensions x 32 bits).
const uint32_t *sobol_table();

// The compiled scene (src/render/scene.lucb:31-63).
struct Scene {
    std::vector<float> positions;        // xyz per point, world space
    std::vector<uint32_t> indices;       // 3 per triangle, leaf order
    std::vector<uint32_t> faces;         // polygon per triangle, leaf order
    std::vector<uint32_t> shading;       // 3 octahedral normals + material, leaf order
    std::vector<uint8_t> flat;           // 1 where the normals are the triangle's own (no authored ones)
    std::vector<lr_bvh_node> nodes;      // binned-SAH BVH2
    std::vector<uint32_t> order;         // source triangle at each leaf slot
    std::vector<lr_camera> cameras;
    std::vector<lr_light> lights;        // image pointers cleared: the pixels are in light_images
    std::vector<std::vector<float>> light_images;  // per light: a dome's RGB pixels (else empty)
    std::vector<lr_openpbr> materials;   // the library (material k+1 of the triangles)
    std::vector<uint8_t> used;           // which materials (0: default) triangles use
    uint32_t face_count = 0;
    uint32_t bvh_depth = 0;
    size_t triangle_count() const { return indices.size() / 3; }
    size_t point_count() const { return positions.size() / 3; }
};

// bvh.cpp: the binned-SAH build of bvh.lucb:66-217, reordering the scene's triangles
// into leaf order.
void build_bvh(Scene &scene);
// Moves the scene's points (same triangles) and refits its BVH2 and flat normals (scene.cpp).
void move_points(Scene &scene, const float *positions);
uint32_t bvh_depth(const std::vector<lr_bvh_node> &nodes);

// camera.cpp
void camera_frame(const lr_camera &camera, uint32_t width, uint32_t height, lr_frame &out);
void look_frame(const double position[3], const double forward[3], const double up[3],
                double tan_half_height, uint32_t width, uint32_t height, bool orthographic,
                lr_frame &out);
void pack_frame(const lr_frame &frame, float out[16]);

}  // namespace lr

// The opaque handle types of the C ABI.
struct lr_scene : lr::Scene {};
