// Host-side loading of a renderer's lights, light tree, materials and constants.
#pragma once

#include <vector>

#include "common.hpp"

namespace lr {

// Light records: 7 vec4 (28 floats) per light, as shaders/lights.glsl:1-22 lays them out,
// then the textured dome's texels and cumulative weights (pack_lights says where).
struct LightRecords {
    std::vector<float> rows;
    size_t count = 0;
    double distant_power = 0.0;  // distant lights' and domes' power
    int32_t dome = -1;           // the light whose image the records hold (-1: none)
};

// A dome's image sampled by importance (environment.lucb:60-156): per texel its colour
// (ACEScg, or in the spectral build its three basis spectra's weights) and its weight
// (luminance x sin theta); each row's cumulative weights, then the rows'; their sum and
// the mean luminance over the sphere.
struct Environment {
    uint32_t width = 0, height = 0;
    std::vector<float> texels, cdf;
    double total = 0.0, average = 0.0;
};

// The light tree (light_tree.lucb:16-20): 12 floats per node (lo, energy; hi, cos theta_o;
// axis, cos theta_e), 2 links per node, 4 words per emitter (code, trail, depth, 0) and
// one emitter per triangle slot (0xffffffff: none).
struct LightTree {
    std::vector<float> nodes;
    std::vector<uint32_t> links, records, triangle_map;
    size_t node_count = 0, emitter_count = 0;
    double energy = 0.0;
};

struct Loaded {
    std::vector<lr_openpbr> library;  // the default material first
    LightRecords lights;
    LightTree tree;
    std::vector<float> materials;     // 64 floats per material
    double radius = 1.0, p_distant = 0.0;
    bool glossy = false;              // a used material has more than EON diffuse
    bool cutouts = false;             // a used material has geometry_opacity below 1
    // Light paths from afar (lights.glsl:283-308): the chance a light path starts at a
    // distant light with a size, and the disk it starts on (centre, radius) around what
    // casts caustics; share 0 when none do.
    double emit_share = 0.0, emit_radius = 1.0;
    V3 emit_center;
    double background_fit[4] = {0, 0, 0, 0};
    M3 film{};
    V3 cmf_integrals;
};

// The lights as the integrator's kernels read them (emitters.cuh DeviceLight: 32 floats a
// light; the bits of integers are stored as floats where a field is one), the finite
// lights and the lights from afar by index, and the textured dome's image apart.
struct DeviceLights {
    std::vector<float> records;
    std::vector<uint32_t> finite, afar;
    std::vector<float> dome_texels, dome_cdf;  // 4 floats a texel; cumulative weights
    uint32_t dome_light = 0xffffffffu, dome_width = 0, dome_height = 0;
    float dome_weight_sum = 0.0f;
};

// The light tree as the kernels walk it (lighttree.cuh TreePair: 24 floats per interior
// node, both children's bounds in the importance test's form), and where a walk starts.
struct DeviceTree {
    std::vector<float> pairs;
    uint32_t root = 0xffffffffu;
};

// A material as the kernels read it (surface.cuh MaterialCode: 64 floats): what does not
// depend on the hit, worked out once.
void material_code(const lr_openpbr &m, std::vector<float> &out);

DeviceLights device_lights(const LightRecords &records);
DeviceTree device_tree(const LightTree &tree);

Environment environment_of(const std::vector<float> &pixels, uint32_t width, uint32_t height, bool spectral);
LightRecords pack_lights(const std::vector<lr_light> &lights, const std::vector<std::vector<float>> &images,
                         double radius, bool spectral);
LightTree build_light_tree(const Scene &scene, const LightRecords &lights, const std::vector<lr_openpbr> &library);
void pack_material(const lr_openpbr &m, float program, std::vector<float> &out);
double scene_radius(const Scene &scene);
Loaded load(const Scene &scene, const lr_settings &settings);
bool casts_caustics(const lr_openpbr &m);
// Whether a material the scene uses (the settings' default included) is a cut-out: its
// passes trace 8 rounds more (loading.lucb:121-124, 161).
bool has_cutouts(const Scene &scene, const lr_settings &settings);

}  // namespace lr
