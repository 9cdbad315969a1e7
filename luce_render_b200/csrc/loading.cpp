// What a renderer loads besides geometry (src/render/loading.lucb:51-161): the UsdLux
// light records (lights.lucb:29-131), the light tree over placed lights and emissive
// triangles (light_tree.lucb:41-244), the OpenPBR material records
// (materials.lucb:105-119), and the scene-wide constants (loading.lucb:253-272).
#include "loading.hpp"

#include <algorithm>
#include <cstring>
#include <numeric>

namespace lr {
namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr uint32_t kEmitterTriangle = 0x80000000u;
constexpr uint32_t kLeafNode = 0x80000000u;

double luminance(const V3 &rgb) { return 0.2722287168 * rgb.x + 0.6740817658 * rgb.y + 0.0536895174 * rgb.z; }

struct Emitter {
    V3 lo, hi, axis;
    double theta_o, theta_e, energy;
    uint32_t code;
    double center(int k) const { return (lo[k] + hi[k]) * 0.5; }
};

// The cone holding both cones of normals (pbrt-v4's DirectionCone::Union;
// light_tree.lucb:41-56).
void cone_union(V3 &axis, double &theta, const V3 &b_axis, double b_theta) {
    double theta_d = std::acos(std::min(std::max(axis.dot(b_axis), -1.0), 1.0));
    if (std::min(theta_d + b_theta, kPi) <= theta) return;
    if (std::min(theta_d + theta, kPi) <= b_theta) {
        axis = b_axis;
        theta = b_theta;
        return;
    }
    double theta_o = 0.5 * (theta + theta_d + b_theta);
    if (theta_o >= kPi) {
        theta = kPi;
        return;
    }
    double rotate = theta_o - theta;
    V3 w = axis.cross(b_axis);
    double wl = w.length();
    if (wl < 1e-12) {
        theta = kPi;
        return;
    }
    V3 k = w * (1.0 / wl);
    V3 turned = axis * std::cos(rotate) + k.cross(axis) * std::sin(rotate) + k * (k.dot(axis) * (1.0 - std::cos(rotate)));
    double tl = turned.length();
    if (tl > 0.0 && std::isfinite(tl)) axis = {turned.x / tl, turned.y / tl, turned.z / tl};
    theta = theta_o;
}

// Three-way quickselect of the k-th emitter by centre along `axis`
// (light_tree.lucb:217-239): the same partition steps, so the same tree.
void select_kth(const std::vector<Emitter> &e, uint32_t *order, size_t length, size_t k, int axis) {
    size_t low = 0, high = length;
    while (high - low > 1) {
        double pivot = e[order[(low + high) / 2]].center(axis);
        size_t less = low, at = low, more = high;
        while (at < more) {
            double key = e[order[at]].center(axis);
            if (key < pivot) {
                std::swap(order[at], order[less]);
                less++;
                at++;
            } else if (key > pivot) {
                more--;
                std::swap(order[at], order[more]);
            } else {
                at++;
            }
        }
        if (k < less) high = less;
        else if (k >= more) low = more;
        else return;
    }
}

}  // namespace

Environment environment_of(const std::vector<float> &pixels, uint32_t width, uint32_t height, bool spectral) {
    // Linear Rec.709 (sRGB primaries, D65) to ACEScg, Bradford-adapted (environment.lucb:21-25).
    static const M3 kRec709ToAcescg{{0.613097, 0.339523, 0.047379, 0.070194, 0.916354, 0.013452, 0.020616, 0.109570,
                                     0.869815}};
    const M3 basis = basis_weights();
    Environment e;
    e.width = width;
    e.height = height;
    e.texels.reserve((size_t)width * height * 4);
    e.cdf.reserve((size_t)width * height + height);
    std::vector<double> rows(height);
    double luminance_sum = 0.0, solid_angle = 0.0;
    for (uint32_t y = 0; y < height; y++) {
        const double sin_theta = std::sin(kPi * ((double)y + 0.5) / (double)height);
        double row = 0.0;
        const size_t start = e.cdf.size();
        for (uint32_t x = 0; x < width; x++) {
            const float *p = &pixels[((size_t)y * width + x) * 3];
            const V3 raw = kRec709ToAcescg.apply(V3(p[0], p[1], p[2]));
            const V3 rgb(std::max(0.0, raw.x), std::max(0.0, raw.y), std::max(0.0, raw.z));
            const double lum = luminance(rgb);
            const double weight = lum * sin_theta;
            // The spectral build keeps each texel as its basis spectra's weights, the
            // 3 x 3 product spec_of_texel (spectrum.glsl:67-80) makes, done once here.
            const V3 stored = spectral ? basis.apply(rgb) : rgb;
            for (double value : {stored.x, stored.y, stored.z, weight}) e.texels.push_back((float)value);
            row += weight;
            e.cdf.push_back((float)row);
            luminance_sum += lum * sin_theta;
            solid_angle += sin_theta;
        }
        // Each row's cumulative weights end at 1 (uniform across an empty row).
        for (uint32_t x = 0; x < width; x++)
            e.cdf[start + x] = (float)(row > 0.0 ? (double)e.cdf[start + x] / row : (double)(x + 1) / (double)width);
        rows[y] = row;
    }
    double total = 0.0;
    for (double row : rows) total += row;
    double running = 0.0;
    for (uint32_t y = 0; y < height; y++) {
        running += rows[y];
        e.cdf.push_back((float)(total > 0.0 ? running / total : (double)(y + 1) / (double)height));
    }
    e.total = total;
    e.average = solid_angle > 0.0 ? luminance_sum / solid_angle : 0.0;
    return e;
}

LightRecords pack_lights(const std::vector<lr_light> &lights, const std::vector<std::vector<float>> &images,
                         double radius, bool spectral) {
    LightRecords out;
    const M3 to_acescg = film_matrix();
    std::vector<double> powers;
    // The first dome with an image lights by it (loading.lucb:55-61).
    Environment environment;
    int32_t textured = -1;
    for (size_t i = 0; i < lights.size(); i++)
        if (lights[i].shape == LR_LIGHT_DOME && i < images.size() && !images[i].empty()) {
            environment = environment_of(images[i], lights[i].image_width, lights[i].image_height, spectral);
            textured = (int32_t)i;
            break;
        }
    int32_t textured_record = -1;
    for (size_t index = 0; index < lights.size(); index++) {
        const lr_light &light = lights[index];
        const double *m = light.matrix;
        V3 position(m[9], m[10], m[11]);
        V3 mz(-m[6], -m[7], -m[8]);
        double l = mz.length();
        if (!(l > 0.0)) fail(LR_INVALID, "a light's placement has no z axis");
        V3 emits(mz.x / l, mz.y / l, mz.z / l);
        V3 u, v;
        double size = 0.0, area = 0.0, cos_half = 1.0, kind = 0.0;
        if (light.shape == LR_LIGHT_RECT) {
            u = V3(m[0], m[1], m[2]) * (0.5 * light.width);
            v = V3(m[3], m[4], m[5]) * (0.5 * light.height);
            area = 4.0 * u.cross(v).length();
        } else if (light.shape == LR_LIGHT_DISK) {
            kind = 1.0;
            u = V3(m[0], m[1], m[2]) * light.radius;
            v = V3(m[3], m[4], m[5]) * light.radius;
            area = kPi * u.cross(v).length();
        } else if (light.shape == LR_LIGHT_SPHERE) {
            kind = 2.0;
            double det = V3(m[0], m[1], m[2]).dot(V3(m[3], m[4], m[5]).cross(V3(m[6], m[7], m[8])));
            size = light.radius * std::cbrt(std::fabs(det));
            area = 4.0 * kPi * size * size;
        } else if (light.shape == LR_LIGHT_DOME) {
            kind = 4.0;
            u = unit(V3(m[0], m[1], m[2]), "a dome's x axis");
            v = unit(V3(m[3], m[4], m[5]), "a dome's y axis");
            // Rows 1-3 are the dome's axes (X, Y, Z): world to its frame.
            emits = unit(V3(m[6], m[7], m[8]), "a dome's z axis");
        } else {
            kind = 3.0;
            cos_half = std::cos(0.5 * light.angle * kPi / 180.0);
        }
        double scale = light.intensity * std::exp2(light.exposure);
        if (kind < 3.0 && light.normalize) {
            if (area <= 0.0) continue;
            scale = scale / area;
        }
        if (kind == 3.0 && cos_half < 1.0 - 1e-7) scale = scale / (2.0 * kPi * (1.0 - cos_half));
        V3 color(light.color[0], light.color[1], light.color[2]);
        V3 rgb = color * scale;
        double fit[4];
        fit_spectrum(color, fit);
        fit[3] = fit[3] * scale;
        double flags = light.visible ? 1.0 : 0.0;
        if (light.temperature > 0.0) {
            V3 tint = blackbody_xyz(light.temperature);
            fit[3] = fit[3] / tint.y;
            V3 tinted = to_acescg.apply(tint * (1.0 / tint.y));
            rgb = V3(rgb.x * tinted.x, rgb.y * tinted.y, rgb.z * tinted.z);
            flags += 2.0;
        }
        double power = -1.0;
        if (kind == 3.0)
            power = std::max(0.0, luminance(rgb)) * (cos_half < 1.0 - 1e-7 ? 2.0 * kPi * (1.0 - cos_half) : 1.0) * kPi *
                    radius * radius;
        // A dome's power: what a sphere of its mean radiance pours into the scene's disk.
        if (kind == 4.0) {
            double mean = 1.0;
            if ((int32_t)index == textured) {
                mean = environment.average;
                textured_record = (int32_t)powers.size();
            }
            power = std::max(0.0, luminance(rgb)) * mean * kPi * kPi * radius * radius;
        }
        powers.push_back(power);
        const double rows[28] = {position.x, position.y, position.z, kind,   u.x,    u.y,    u.z,    size,
                                 v.x,        v.y,        v.z,        cos_half, emits.x, emits.y, emits.z, area,
                                 fit[0],     fit[1],     fit[2],     fit[3], rgb.x,  rgb.y,  rgb.z,  flags,
                                 light.temperature, 0.0, 0.0, 0.0};
        for (double value : rows) out.rows.push_back((float)value);
    }
    out.count = powers.size();
    double total = 0.0;
    size_t distant = 0;
    for (double p : powers)
        if (p >= 0.0) {
            total += p;
            distant++;
        }
    double running = 0.0;
    uint32_t emitter = 0;
    for (size_t i = 0; i < powers.size(); i++) {
        float *row6 = &out.rows[i * 28 + 24];
        if (powers[i] < 0.0) {
            row6[3] = (float)emitter++;
            continue;
        }
        double share = total > 0.0 ? powers[i] / total : 1.0 / (double)distant;
        running += share;
        row6[1] = (float)share;
        row6[2] = (float)running;
    }
    out.distant_power = total;
    // The textured dome's texels (a float4 each), then its cumulative weights, after the
    // records. The reference keeps where they start in two constant rows (K_DOME,
    // K_DOME_CDF); here the dome's own record holds them, in slots a dome leaves unused:
    // row 0 x the weights' sum, rows 1-3 w the texels' first float4, the width and the
    // height, row 6 w the cumulative weights' first float (the integers as their bits).
    if (textured_record >= 0) {
        auto bits = [](size_t v) {
            const uint32_t u = (uint32_t)v;
            float f;
            std::memcpy(&f, &u, 4);
            return f;
        };
        const size_t texel_base = out.rows.size() / 4;
        out.rows.insert(out.rows.end(), environment.texels.begin(), environment.texels.end());
        const size_t cdf_base = out.rows.size();
        out.rows.insert(out.rows.end(), environment.cdf.begin(), environment.cdf.end());
        while (out.rows.size() % 4 != 0) out.rows.push_back(0.0f);
        if (out.rows.size() >= ((size_t)1 << 32)) fail(LR_LIMIT, "a dome's image does not fit the light records");
        float *record = &out.rows[(size_t)textured_record * 28];  // after the inserts, which may move the rows
        record[0] = (float)environment.total;
        record[1] = record[2] = 0.0f;
        record[7] = bits(texel_base);
        record[11] = bits(environment.width);
        record[15] = bits(environment.height);
        record[27] = bits(cdf_base);
        out.dome = textured_record;
    }
    return out;
}

LightTree build_light_tree(const Scene &scene, const LightRecords &lights, const std::vector<lr_openpbr> &library) {
    LightTree tree;
    std::vector<Emitter> emitters;
    for (size_t index = 0; index < lights.count; index++) {
        const float *row = &lights.rows[index * 28];
        double kind = row[3];
        if (kind >= 3.0) continue;
        V3 position(row[0], row[1], row[2]), u(row[4], row[5], row[6]), v(row[8], row[9], row[10]);
        V3 normal(row[12], row[13], row[14]);
        double area = row[15];
        V3 rgb(row[20], row[21], row[22]);
        V3 extent(std::fabs(u.x) + std::fabs(v.x), std::fabs(u.y) + std::fabs(v.y), std::fabs(u.z) + std::fabs(v.z));
        double theta_o = 0.0;
        if (kind == 2.0) {
            double r = row[7];
            extent = V3(r, r, r);
            theta_o = kPi;
        }
        emitters.push_back({position - extent, position + extent, normal, theta_o, 0.5 * kPi,
                            std::max(0.0, luminance(rgb)) * area * kPi, (uint32_t)index});
    }
    bool emissive = false;
    for (const auto &m : library) emissive = emissive || m.emission_luminance > 0.0;
    const size_t T = scene.triangle_count();
    const float *p = scene.positions.data();
    for (size_t t = 0; emissive && t < T; t++) {
        uint32_t material = scene.shading[t * 4 + 3];
        if ((size_t)material >= library.size()) continue;
        const lr_openpbr &m = library[material];
        if (m.emission_luminance <= 0.0) continue;
        V3 c[3];
        for (int k = 0; k < 3; k++) {
            const float *q = &p[(size_t)scene.indices[t * 3 + k] * 3];
            c[k] = V3(q[0], q[1], q[2]);
        }
        V3 cross = (c[1] - c[0]).cross(c[2] - c[0]);
        double area = 0.5 * cross.length();
        if (area <= 0.0) continue;
        V3 lo(std::min(c[0].x, std::min(c[1].x, c[2].x)), std::min(c[0].y, std::min(c[1].y, c[2].y)),
              std::min(c[0].z, std::min(c[1].z, c[2].z)));
        V3 hi(std::max(c[0].x, std::max(c[1].x, c[2].x)), std::max(c[0].y, std::max(c[1].y, c[2].y)),
              std::max(c[0].z, std::max(c[1].z, c[2].z)));
        V3 emission = V3(m.emission_color[0], m.emission_color[1], m.emission_color[2]) * m.emission_luminance;
        emitters.push_back({lo, hi, cross * (0.5 / area), kPi, 0.5 * kPi,
                            std::max(0.0, luminance(emission)) * area * 2.0 * kPi, kEmitterTriangle | (uint32_t)t});
    }
    const size_t count = emitters.size();
    tree.emitter_count = count;
    tree.records.assign(count * 4, 0u);
    tree.triangle_map.assign(T, 0xffffffffu);
    for (size_t i = 0; i < count; i++) {
        uint32_t code = emitters[i].code;
        tree.records[i * 4] = code;
        if (code & kEmitterTriangle) tree.triangle_map[code & ~kEmitterTriangle] = (uint32_t)i;
    }
    if (count == 0) return tree;
    std::vector<uint32_t> order(count);
    std::iota(order.begin(), order.end(), 0u);
    tree.nodes.assign(12, 0.0f);
    tree.links.assign(2, 0u);
    struct Job {
        size_t node, first, count;
        uint32_t trail, depth;
    };
    std::vector<Job> stack{{0, 0, count, 0, 0}};
    while (!stack.empty()) {
        Job job = stack.back();
        stack.pop_back();
        uint32_t *range = order.data() + job.first;
        const Emitter &head = emitters[range[0]];
        V3 lo = head.lo, hi = head.hi, axis = head.axis;
        double theta_o = head.theta_o, theta_e = head.theta_e, energy = 0.0;
        for (size_t i = 0; i < job.count; i++) {
            const Emitter &e = emitters[range[i]];
            for (int k = 0; k < 3; k++) {
                lo[k] = std::min(lo[k], e.lo[k]);
                hi[k] = std::max(hi[k], e.hi[k]);
            }
            cone_union(axis, theta_o, e.axis, e.theta_o);
            theta_e = std::max(theta_e, e.theta_e);
            energy += e.energy;
        }
        const double values[12] = {lo.x, lo.y, lo.z, energy, hi.x, hi.y, hi.z, std::cos(theta_o),
                                   axis.x, axis.y, axis.z, std::cos(theta_e)};
        for (int k = 0; k < 12; k++) tree.nodes[job.node * 12 + k] = (float)values[k];
        if (job.node == 0) tree.energy = energy;
        if (job.count == 1) {
            uint32_t emitter = range[0];
            tree.links[job.node * 2] = emitter;
            tree.links[job.node * 2 + 1] = kLeafNode;
            tree.records[emitter * 4 + 1] = job.trail;
            tree.records[emitter * 4 + 2] = job.depth;
            continue;
        }
        V3 size = hi - lo;
        int axis_index = 0;
        if (size.y > size.x && size.y >= size.z) axis_index = 1;
        else if (size.z > size.x && size.z > size.y) axis_index = 2;
        size_t half = job.count / 2;
        select_kth(emitters, range, job.count, half, axis_index);
        size_t child = tree.links.size() / 2;
        tree.nodes.resize(tree.nodes.size() + 24, 0.0f);
        tree.links.resize(tree.links.size() + 4, 0u);
        tree.links[job.node * 2] = (uint32_t)child;
        tree.links[job.node * 2 + 1] = 0;
        stack.push_back({child + 1, job.first + half, job.count - half, job.trail | (1u << job.depth), job.depth + 1});
        stack.push_back({child, job.first, half, job.trail, job.depth + 1});
    }
    tree.node_count = tree.links.size() / 2;
    return tree;
}

namespace {

float bits_of(uint32_t v) {
    float f;
    std::memcpy(&f, &v, 4);
    return f;
}

uint32_t uint_of(float f) {
    uint32_t v;
    std::memcpy(&v, &f, 4);
    return v;
}

}  // namespace

DeviceLights device_lights(const LightRecords &records) {
    DeviceLights out;
    out.records.assign(records.count * 32, 0.0f);
    for (size_t i = 0; i < records.count; i++) {
        const float *row = &records.rows[i * 28];
        float *d = &out.records[i * 32];
        const uint32_t shape = (uint32_t)row[3];
        const V3 u(row[4], row[5], row[6]), v(row[8], row[9], row[10]);
        for (int k = 0; k < 3; k++) {
            d[k] = row[k];          // centre
            d[4 + k] = row[4 + k];  // half edge u, or the dome frame's x axis
            d[8 + k] = row[8 + k];  // half edge v, or its y axis
            d[12 + k] = row[12 + k];  // the direction light leaves along, or the frame's z axis
        }
        d[3] = bits_of(shape);
        d[15] = row[15];  // area
        if (shape == 0u || shape == 1u) {
            const double uu = u.dot(u), vv = v.dot(v);
            d[7] = uu > 0.0 ? (float)(1.0 / uu) : 0.0f;
            d[11] = vv > 0.0 ? (float)(1.0 / vv) : 0.0f;
            out.finite.push_back((uint32_t)i);
        } else if (shape == 2u) {
            const float r = row[7];
            d[16] = r;
            d[17] = r * r;
            out.finite.push_back((uint32_t)i);
        } else {
            out.afar.push_back((uint32_t)i);
            if (shape == 3u) {
                const float cos_half = row[11];
                const bool delta = cos_half >= 1.0f - 1e-7f;
                d[16] = cos_half;
                d[17] = delta ? 1.0f : (float)(1.0 / (2.0 * kPi * (1.0 - (double)cos_half)));
                d[18] = delta ? 1.0f : 0.0f;
            }
        }
        for (int k = 0; k < 4; k++) d[20 + k] = row[16 + k];  // spectral fit
        for (int k = 0; k < 3; k++) d[24 + k] = row[20 + k];  // ACEScg radiance
        d[27] = bits_of((uint32_t)row[23]);                   // flags
        d[28] = row[24];                                      // kelvin
        d[29] = row[25];                                      // share among lights from afar
        d[30] = row[26];                                      // cumulative share
        d[31] = bits_of(shape < 3u ? (uint32_t)row[27] : 0u);  // the tree's emitter (finite lights)
    }
    if (records.dome >= 0) {
        // pack_lights keeps the textured dome's image after the records and says where in
        // the dome's own record (see there).
        const float *row = &records.rows[(size_t)records.dome * 28];
        out.dome_light = (uint32_t)records.dome;
        out.dome_weight_sum = row[0];
        out.dome_width = uint_of(row[11]);
        out.dome_height = uint_of(row[15]);
        const size_t texel_base = (size_t)uint_of(row[7]) * 4, cdf_base = uint_of(row[27]);
        const size_t texels = (size_t)out.dome_width * out.dome_height;
        out.dome_texels.assign(records.rows.begin() + (long)texel_base, records.rows.begin() + (long)(texel_base + texels * 4));
        out.dome_cdf.assign(records.rows.begin() + (long)cdf_base,
                            records.rows.begin() + (long)(cdf_base + texels + out.dome_height));
        float *d = &out.records[(size_t)records.dome * 32];
        d[0] = d[1] = d[2] = 0.0f;  // the slots pack_lights borrowed
        d[7] = d[11] = d[15] = 0.0f;
        d[31] = 0.0f;  // a dome is no emitter of the tree
    }
    return out;
}

DeviceTree device_tree(const LightTree &tree) {
    DeviceTree out;
    if (tree.node_count == 0) return out;
    // Pair slots for the interior nodes, in node order.
    std::vector<uint32_t> slot(tree.node_count, 0xffffffffu);
    uint32_t pairs = 0;
    for (size_t n = 0; n < tree.node_count; n++)
        if (!(tree.links[n * 2 + 1] & kLeafNode)) slot[n] = pairs++;
    auto lead = [&](size_t n) {
        return (tree.links[n * 2 + 1] & kLeafNode) ? (0x80000000u | tree.links[n * 2]) : slot[n];
    };
    out.root = lead(0);
    out.pairs.assign((size_t)pairs * 24, 0.0f);
    for (size_t n = 0; n < tree.node_count; n++) {
        if (slot[n] == 0xffffffffu) continue;
        float *pair = &out.pairs[(size_t)slot[n] * 24];
        for (int side = 0; side < 2; side++) {
            const size_t child = tree.links[n * 2] + (size_t)side;
            const float *b = &tree.nodes[child * 12];  // lo, power; hi, cos theta_o; axis, cos theta_e
            const V3 lo(b[0], b[1], b[2]), hi(b[4], b[5], b[6]);
            const V3 centre = (lo + hi) * 0.5;
            float *c = pair + side * 4, *a = pair + 8 + side * 4, *k = pair + 16 + side * 4;
            c[0] = (float)centre.x;
            c[1] = (float)centre.y;
            c[2] = (float)centre.z;
            c[3] = (float)(0.5 * (hi - lo).length());
            a[0] = b[8];
            a[1] = b[9];
            a[2] = b[10];
            a[3] = b[3];
            const double cos_o = b[7];
            k[0] = b[7];
            k[1] = (float)std::sqrt(std::max(0.0, 1.0 - cos_o * cos_o));
            k[2] = b[11];
            k[3] = bits_of(lead(child));
        }
    }
    return out;
}

namespace {

double clamp01(double v) { return std::min(std::max(v, 0.0), 1.0); }

// OpenPBR's GGX widths (x, y) from roughness and anisotropy.
void ggx_widths(double roughness, double anisotropy, float out[2]) {
    const double squeeze = 1.0 - anisotropy;
    const double t = roughness * roughness * std::sqrt(2.0 / (1.0 + squeeze * squeeze));
    out[0] = (float)std::max(t, 1e-4);
    out[1] = (float)std::max(squeeze * t, 1e-4);
}

// The hemispherical average of a dielectric's Fresnel reflectance (the closed fit of
// OpenPBR's reference code), computed in single precision as the kernels would.
float fresnel_mean(float eta) {
    return std::log((10893.0f * eta - 1438.2f) / (-774.4f * eta * eta + 10212.0f * eta + 1.0f));
}

}  // namespace

void material_code(const lr_openpbr &m, std::vector<float> &out) {
    const size_t at = out.size();
    out.resize(at + 64, 0.0f);
    float *c = &out[at];
    auto colour = [&](int slot, const V3 &rgb, double scale, float luma_w) {
        double fit[4];
        fit_spectrum(V3(std::max(rgb.x, 0.0), std::max(rgb.y, 0.0), std::max(rgb.z, 0.0)), fit);
        float *f = c + slot * 8;
        for (int k = 0; k < 3; k++) f[k] = (float)fit[k];
        f[3] = (float)(fit[3] * scale);
        f[4] = (float)(rgb.x * scale);
        f[5] = (float)(rgb.y * scale);
        f[6] = (float)(rgb.z * scale);
        f[7] = luma_w;
    };
    const V3 base(m.base_color[0], m.base_color[1], m.base_color[2]);
    const V3 spec(m.specular_color[0], m.specular_color[1], m.specular_color[2]);
    const V3 trans(m.transmission_color[0], m.transmission_color[1], m.transmission_color[2]);
    const V3 coat(m.coat_color[0], m.coat_color[1], m.coat_color[2]);
    const V3 glow = V3(m.emission_color[0], m.emission_color[1], m.emission_color[2]) * m.emission_luminance;
    auto lum = [](const V3 &v) { return (float)luminance(v); };
    colour(0, base, m.base_weight, std::max(lum(base * m.base_weight), 0.0f));
    colour(1, spec, 1.0, std::max(lum(spec), 0.0f));
    colour(2, trans, 1.0, std::max(lum(trans), 0.05f));
    colour(3, coat, 1.0, lum(coat));
    colour(4, glow, 1.0, (float)m.emission_luminance);
    const double coat_w = clamp01(m.coat_weight);
    float *w = c + 40;  // weights
    w[0] = (float)clamp01(m.base_metalness);
    w[1] = (float)std::max(m.specular_weight, 0.0);
    w[2] = (float)clamp01(m.transmission_weight);
    w[3] = (float)coat_w;
    const double rough = clamp01(m.specular_roughness), coat_rough = clamp01(m.coat_roughness);
    float *r = c + 44;  // roughnesses
    r[0] = (float)m.base_diffuse_roughness;
    r[1] = (float)rough;
    r[2] = (float)coat_rough;
    r[3] = (float)clamp01(m.coat_darkening);
    const double aniso = clamp01(m.specular_roughness_anisotropy);
    const float coat_eta = (float)std::max(m.coat_ior, 1.0001);
    const double eta = std::max(m.specular_ior, 1.0001);
    // The base under the coat: roughened (r^4 + 2 c^4)^(1/4), its index relative to the
    // coat's; and bare.
    const double r4 = std::pow(rough, 4.0), c4 = std::pow(coat_rough, 4.0);
    const double coated_rough = rough * (1.0 - coat_w) + std::min(1.0, std::pow(r4 + 2.0 * c4, 0.25)) * coat_w;
    double relative = eta / coat_eta;
    if (relative < 1.0) relative = 1.0 / relative;
    const float coated_ior = (float)std::max(eta * (1.0 - coat_w) + relative * coat_w, 1.0001);
    float *coated = c + 48, *bare = c + 52, *coat_lobe = c + 56, *extra = c + 60;
    ggx_widths(coated_rough, aniso, coated);
    coated[2] = coated_ior;
    coated[3] = fresnel_mean(coated_ior);
    ggx_widths(rough, aniso, bare);
    bare[2] = (float)eta;
    bare[3] = fresnel_mean((float)eta);
    ggx_widths(coat_rough, clamp01(m.coat_roughness_anisotropy), coat_lobe);
    coat_lobe[2] = coat_eta;
    coat_lobe[3] = fresnel_mean(coat_eta);
    double cauchy = 0.0;
    if (m.transmission_dispersion_scale > 0.0 && m.transmission_dispersion_abbe_number > 0.0 && m.transmission_weight > 0.0)
        cauchy = (m.specular_ior - 1.0) * m.transmission_dispersion_scale /
                 (m.transmission_dispersion_abbe_number * (1.0 / (486.1 * 486.1) - 1.0 / (656.3 * 656.3)));
    extra[0] = (float)m.geometry_opacity;
    extra[1] = (float)cauchy;
    extra[2] = (float)eta;
    extra[3] = (float)aniso;
}

void pack_material(const lr_openpbr &m, float program, std::vector<float> &out) {
    const V3 colors[5] = {V3(m.base_color[0], m.base_color[1], m.base_color[2]),
                          V3(m.specular_color[0], m.specular_color[1], m.specular_color[2]),
                          V3(m.coat_color[0], m.coat_color[1], m.coat_color[2]),
                          V3(m.emission_color[0], m.emission_color[1], m.emission_color[2]) * m.emission_luminance,
                          V3(m.transmission_color[0], m.transmission_color[1], m.transmission_color[2])};
    const double weights[5] = {m.base_weight, m.specular_weight, m.coat_weight, m.emission_luminance,
                               m.transmission_weight};
    for (int i = 0; i < 5; i++) {
        const V3 &c = colors[i];
        double fit[4];
        fit_spectrum(V3(std::max(c.x, 0.0), std::max(c.y, 0.0), std::max(c.z, 0.0)), fit);
        const double row[8] = {fit[0], fit[1], fit[2], fit[3], c.x, c.y, c.z, weights[i]};
        for (double v : row) out.push_back((float)v);
    }
    double cauchy = 0.0;
    if (m.transmission_dispersion_scale > 0.0 && m.transmission_dispersion_abbe_number > 0.0 && m.transmission_weight > 0.0)
        cauchy = (m.specular_ior - 1.0) * m.transmission_dispersion_scale /
                 (m.transmission_dispersion_abbe_number * (1.0 / (486.1 * 486.1) - 1.0 / (656.3 * 656.3)));
    const double rest[24] = {m.base_metalness, m.base_diffuse_roughness, m.specular_roughness,
                             m.specular_roughness_anisotropy, m.specular_ior, m.coat_roughness, m.coat_ior,
                             m.coat_darkening, m.geometry_opacity, m.geometry_thin_walled ? 1.0 : 0.0,
                             m.coat_roughness_anisotropy, cauchy, (double)program, 0, 0, 0,
                             0, 0, 0, 0, 0, 0, 0, 0};
    for (double v : rest) out.push_back((float)v);
}

// Materials this build shades: OpenPBR Surface's lobes (EON diffuse, GGX specular, F82
// metal, coat, rough transmission with dispersion, emission) and cut-outs.
void check_material(const lr_openpbr &m, size_t index, bool spectral) {
    auto bad = [&](const char *what) {
        fail(LR_INVALID, "material " + std::to_string(index) + ": " + what + " is not part of this build's shading");
    };
    if (m.base_diffuse_roughness < 0.0 || m.base_diffuse_roughness > 1.0) bad("base_diffuse_roughness outside 0..1");
}

bool has_cutouts(const Scene &scene, const lr_settings &settings) {
    if (settings.material.geometry_opacity < 1.0 && (scene.used.empty() || scene.used[0])) return true;
    for (size_t i = 0; i < scene.materials.size(); i++)
        if (scene.materials[i].geometry_opacity < 1.0 && (i + 1 >= scene.used.size() || scene.used[i + 1])) return true;
    return false;
}

// Whether a material has a lobe besides EON diffuse (openpbr.glsl's HAS_COAT,
// HAS_TRANSMISSION, HAS_METAL and a specular layer).
bool is_glossy(const lr_openpbr &m) {
    return m.specular_weight > 0.0 || m.base_metalness > 0.0 || m.transmission_weight > 0.0 || m.coat_weight > 0.0;
}

double scene_radius(const Scene &scene) {
    if (scene.point_count() == 0 || scene.nodes.empty()) return 1.0;
    const lr_bvh_node &root = scene.nodes[0];
    if (root.lo[0] > root.hi[0]) return 1.0;
    V3 d((double)(root.hi[0] - root.lo[0]), (double)(root.hi[1] - root.lo[1]), (double)(root.hi[2] - root.lo[2]));
    return std::max(1.0, 0.5 * d.length());
}

// casts_caustics (loading.lucb:215-219): it refracts, or reflects sharply enough (metal,
// glossy specular or a clear coat) to focus light.
bool casts_caustics(const lr_openpbr &m) {
    if (m.transmission_weight > 0.0) return true;
    if (m.base_metalness > 0.0 && m.specular_roughness < 0.3) return true;
    if (m.coat_weight > 0.0 && m.coat_roughness < 0.3) return true;
    return m.specular_weight > 0.0 && m.specular_roughness < 0.1;
}

namespace {

// caster_bounds (loading.lucb:224-241): the sphere around the triangles that cast
// caustics (centre, radius at least 1e-3), or false when none does.
bool caster_bounds(const Scene &scene, const std::vector<lr_openpbr> &library, V3 &center, double &reach) {
    V3 lo(1e30, 1e30, 1e30), hi(-1e30, -1e30, -1e30);
    bool any = false;
    for (size_t t = 0; t < scene.triangle_count(); t++) {
        const size_t material = scene.shading[t * 4 + 3];
        if (material >= library.size() || !casts_caustics(library[material])) continue;
        for (int corner = 0; corner < 3; corner++) {
            const size_t at = (size_t)scene.indices[t * 3 + corner] * 3;
            const V3 point(scene.positions[at], scene.positions[at + 1], scene.positions[at + 2]);
            lo = V3(std::min(lo.x, point.x), std::min(lo.y, point.y), std::min(lo.z, point.z));
            hi = V3(std::max(hi.x, point.x), std::max(hi.y, point.y), std::max(hi.z, point.z));
        }
        any = true;
    }
    if (!any) return false;
    center = (lo + hi) * 0.5;
    reach = std::max(1e-3, 0.5 * (hi - lo).length());
    return true;
}

}  // namespace

Loaded load(const Scene &scene, const lr_settings &settings) {
    Loaded L;
    L.library.push_back(settings.material);
    for (const auto &m : scene.materials) L.library.push_back(m);
    for (size_t i = 0; i < L.library.size(); i++)
        if (i >= scene.used.size() || scene.used[i]) {
            check_material(L.library[i], i, settings.spectral != 0);
            L.glossy = L.glossy || is_glossy(L.library[i]);
            L.cutouts = L.cutouts || L.library[i].geometry_opacity < 1.0;
        }
    L.radius = scene_radius(scene);
    L.lights = pack_lights(scene.lights, scene.light_images, L.radius, settings.spectral != 0);
    L.tree = build_light_tree(scene, L.lights, L.library);
    for (size_t i = 0; i < L.library.size(); i++) pack_material(L.library[i], -1.0f, L.materials);
    // Domes and distant lights with a size start light paths too, on a disk around what
    // casts caustics, sharing them with the tree's emitters by power (loading.lucb:127-146);
    // looked for only when such a light would aim light paths at it. An orthographic
    // view takes no light paths at all (the member drops the share).
    bool sized = false;
    for (size_t i = 0; i < L.lights.count; i++)
        sized = sized || L.lights.rows[i * 28 + 3] == 4.0f ||
                (L.lights.rows[i * 28 + 3] == 3.0f && L.lights.rows[i * 28 + 11] < 1.0f - 1e-7f);
    if (sized && settings.light_tracing > 0.0) {
        V3 center;
        double reach = 1.0;
        if (caster_bounds(scene, L.library, center, reach)) {
            const double afar_power = L.lights.distant_power * (reach / L.radius) * (reach / L.radius);
            const double both = afar_power + L.tree.energy;
            L.emit_share = both > 0.0 ? afar_power / both : 0.0;
            L.emit_radius = reach;
            L.emit_center = center;
        }
    }
    const double total = L.lights.distant_power + L.tree.energy;
    L.p_distant = L.tree.emitter_count > 0 ? (total > 0.0 ? L.lights.distant_power / total : 0.0)
                                           : (L.lights.distant_power > 0.0 ? 1.0 : 0.0);
    fit_spectrum(V3(settings.background[0], settings.background[1], settings.background[2]), L.background_fit);
    L.film = film_matrix();
    L.cmf_integrals = cmf_integrals();
    return L;
}

}  // namespace lr
