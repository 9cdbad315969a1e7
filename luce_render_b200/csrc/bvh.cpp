// The binned-SAH BVH2 of src/render/bvh.lucb:66-217 (12 bins per axis, leaves of at most
// 4 triangles unless SAH keeps up to 16 together, children stored as a pair), built on
// the host. The build is node-for-node the reference's: same split choices, same node
// numbering (a depth-first stack that takes the left child first), same leaf order, so
// triangle slots and node ids match the reference's buffers. Only the work is laid
// out differently: boxes and centroids in structure-of-arrays form, all three axes
// binned in one pass over a node's triangles, and large nodes binned by several
// threads (bounds are min/max, which merge exactly in any order).
#include <algorithm>
#include <thread>

#include "common.hpp"

namespace lr {
namespace {

constexpr int kBins = 12;       // bvh.lucb:29
constexpr size_t kLeafSize = 4; // bvh.lucb:30
constexpr size_t kLeafLimit = 16; // bvh.lucb:32
constexpr float kBig = 3.0e38f;

struct Box {
    float lo[3] = {kBig, kBig, kBig};
    float hi[3] = {-kBig, -kBig, -kBig};
    void grow(const float l[3], const float h[3]) {
        for (int k = 0; k < 3; k++) {
            lo[k] = lo[k] < l[k] ? lo[k] : l[k];
            hi[k] = hi[k] > h[k] ? hi[k] : h[k];
        }
    }
    void grow(const Box &b) { grow(b.lo, b.hi); }
    // Box.area (bvh.lucb:48-53), f32.
    float area() const {
        float x = hi[0] - lo[0], y = hi[1] - lo[1], z = hi[2] - lo[2];
        if (x < 0.0f || y < 0.0f || z < 0.0f) return 0.0f;
        return 2.0f * (x * y + y * z + z * x);
    }
};

// bin_of (bvh.lucb:136-142), f32.
inline int bin_of(float c, float lo, float extent) {
    if (extent <= 0.0f) return 0;
    long at = (long)((float)kBins * (c - lo) / extent);
    if (at < 0) return 0;
    return at < kBins ? (int)at : kBins - 1;
}

struct Bins {
    uint32_t count[3][kBins];
    Box bounds[3][kBins];
    void clear() {
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < kBins; b++) {
                count[a][b] = 0;
                bounds[a][b] = Box();
            }
    }
    void merge(const Bins &o) {
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < kBins; b++) {
                count[a][b] += o.count[a][b];
                bounds[a][b].grow(o.bounds[a][b]);
            }
    }
};

struct Builder {
    // Per source triangle: box and centroid, structure of arrays.
    std::vector<float> lo[3], hi[3], center[3];
    std::vector<uint32_t> order;
    unsigned threads = 1;

    void bin_range(const uint32_t *ids, size_t n, const Box &middle, Bins &out) const {
        out.clear();
        float base[3], extent[3];
        for (int a = 0; a < 3; a++) {
            base[a] = middle.lo[a];
            extent[a] = middle.hi[a] - middle.lo[a];
        }
        for (size_t i = 0; i < n; i++) {
            uint32_t t = ids[i];
            float l[3] = {lo[0][t], lo[1][t], lo[2][t]};
            float h[3] = {hi[0][t], hi[1][t], hi[2][t]};
            for (int a = 0; a < 3; a++) {
                if (extent[a] <= 0.0f) continue;
                int b = bin_of(center[a][t], base[a], extent[a]);
                out.count[a][b] += 1;
                out.bounds[a][b].grow(l, h);
            }
        }
    }

    // best_split (bvh.lucb:147-182). Returns axis (-1 none), bin and cost.
    void best_split(const uint32_t *ids, size_t n, const Box &parent, const Box &middle, int &axis_out,
                    int &bin_out, float &cost_out) const {
        axis_out = -1;
        bin_out = 0;
        cost_out = kBig;
        float area = parent.area();
        if (area <= 0.0f) return;
        Bins bins;
        if (n >= (1u << 16) && threads > 1) {
            unsigned parts = std::min<unsigned>(threads, (unsigned)(n >> 14));
            std::vector<Bins> partial(parts);
            std::vector<std::thread> pool;
            size_t chunk = (n + parts - 1) / parts;
            for (unsigned p = 0; p < parts; p++) {
                size_t b = p * chunk, e = std::min(n, b + chunk);
                pool.emplace_back([&, p, b, e] { bin_range(ids + b, e - b, middle, partial[p]); });
            }
            for (auto &t : pool) t.join();
            bins = partial[0];
            for (unsigned p = 1; p < parts; p++) bins.merge(partial[p]);
        } else {
            bin_range(ids, n, middle, bins);
        }
        for (int axis = 0; axis < 3; axis++) {
            if (middle.hi[axis] - middle.lo[axis] <= 0.0f) continue;
            float right_area[kBins];
            uint64_t right_count[kBins];
            Box sweep;
            uint64_t total = 0;
            for (int b = kBins - 1; b > 0; b--) {
                sweep.grow(bins.bounds[axis][b]);
                total += bins.count[axis][b];
                right_area[b] = sweep.area();
                right_count[b] = total;
            }
            Box left;
            uint64_t left_count = 0;
            for (int s = 1; s < kBins; s++) {
                left.grow(bins.bounds[axis][s - 1]);
                left_count += bins.count[axis][s - 1];
                if (left_count == 0 || right_count[s] == 0) continue;
                float cost = 1.0f + (left.area() * (float)left_count + right_area[s] * (float)right_count[s]) / area;
                if (cost < cost_out) {
                    axis_out = axis;
                    bin_out = s;
                    cost_out = cost;
                }
            }
        }
    }

    // partition (bvh.lucb:185-196): the same swaps, so the same leaf order.
    size_t partition(uint32_t *ids, size_t n, const Box &middle, int axis, int bin) const {
        size_t low = 0, high = n;
        const float base = middle.lo[axis], extent = middle.hi[axis] - middle.lo[axis];
        const float *c = center[axis].data();
        while (low < high) {
            if (bin_of(c[ids[low]], base, extent) < bin) {
                low++;
            } else {
                high--;
                std::swap(ids[low], ids[high]);
            }
        }
        return low;
    }

    void bounds_of(const uint32_t *ids, size_t n, Box &bounds, Box &middle) const {
        for (size_t i = 0; i < n; i++) {
            uint32_t t = ids[i];
            float l[3] = {lo[0][t], lo[1][t], lo[2][t]}, h[3] = {hi[0][t], hi[1][t], hi[2][t]};
            float c[3] = {center[0][t], center[1][t], center[2][t]};
            bounds.grow(l, h);
            middle.grow(c, c);
        }
    }
};

void set_node(lr_bvh_node &node, const Box &b, uint32_t first, uint32_t count) {
    for (int k = 0; k < 3; k++) {
        node.lo[k] = b.lo[k];
        node.hi[k] = b.hi[k];
    }
    node.first = first;
    node.count = count;
}

}  // namespace

uint32_t bvh_depth(const std::vector<lr_bvh_node> &nodes) {
    if (nodes.empty() || nodes[0].lo[0] > nodes[0].hi[0]) return 0;
    uint32_t deepest = 0;
    std::vector<std::pair<uint32_t, uint32_t>> stack{{0u, 0u}};
    while (!stack.empty()) {
        auto [node, depth] = stack.back();
        stack.pop_back();
        if (nodes[node].count > 0) {
            deepest = std::max(deepest, depth);
            continue;
        }
        stack.push_back({nodes[node].first, depth + 1});
        stack.push_back({nodes[node].first + 1, depth + 1});
    }
    return deepest;
}

// build_bvh (bvh.lucb:66-82) with build_tree (85-129) and reorder (198-217).
void build_bvh(Scene &scene) {
    const size_t count = scene.triangle_count();
    scene.nodes.clear();
    scene.order.clear();
    if (count == 0) {
        lr_bvh_node empty{{1.0f, 1.0f, 1.0f}, 0, {-1.0f, -1.0f, -1.0f}, 0};
        scene.nodes.push_back(empty);
        scene.bvh_depth = 0;
        return;
    }
    if (count > 0x7fffffffull) fail(LR_LIMIT, "a scene holds at most 2^31 triangles");
    Builder b;
    b.threads = std::max(1u, std::thread::hardware_concurrency());
    for (int k = 0; k < 3; k++) {
        b.lo[k].resize(count);
        b.hi[k].resize(count);
        b.center[k].resize(count);
    }
    const float *p = scene.positions.data();
    for (size_t t = 0; t < count; t++) {
        Box box;
        for (int c = 0; c < 3; c++) {
            const float *v = &p[(size_t)scene.indices[t * 3 + c] * 3];
            box.grow(v, v);
        }
        for (int k = 0; k < 3; k++) {
            b.lo[k][t] = box.lo[k];
            b.hi[k][t] = box.hi[k];
            b.center[k][t] = 0.5f * (box.lo[k] + box.hi[k]);
        }
    }
    b.order.resize(count);
    for (size_t t = 0; t < count; t++) b.order[t] = (uint32_t)t;

    std::vector<lr_bvh_node> &nodes = scene.nodes;
    nodes.reserve(2 * count);
    nodes.push_back(lr_bvh_node{});
    struct Job {
        size_t node, first, count;
    };
    std::vector<Job> stack{{0, 0, count}};
    while (!stack.empty()) {
        Job job = stack.back();
        stack.pop_back();
        uint32_t *ids = b.order.data() + job.first;
        Box bounds, middle;
        b.bounds_of(ids, job.count, bounds, middle);
        size_t left_count = 0;
        int axis = -1, bin = 0;
        float cost = kBig;
        if (job.count > kLeafSize) b.best_split(ids, job.count, bounds, middle, axis, bin, cost);
        if (job.count > kLeafSize && (cost < (float)job.count || job.count > kLeafLimit)) {
            if (axis >= 0 && cost < kBig) left_count = b.partition(ids, job.count, middle, axis, bin);
            if (left_count == 0 || left_count == job.count) left_count = job.count / 2;
        }
        if (left_count == 0) {
            set_node(nodes[job.node], bounds, (uint32_t)job.first, (uint32_t)job.count);
            continue;
        }
        size_t child = nodes.size();
        nodes.push_back(lr_bvh_node{});
        nodes.push_back(lr_bvh_node{});
        set_node(nodes[job.node], bounds, (uint32_t)child, 0);
        stack.push_back({child + 1, job.first + left_count, job.count - left_count});
        stack.push_back({child, job.first, left_count});
    }

    // reorder (bvh.lucb:198-217)
    scene.order = b.order;
    std::vector<uint32_t> indices(count * 3), faces(count), shading(count * 4);
    std::vector<uint8_t> flat(count);
    for (size_t at = 0; at < count; at++) {
        size_t s = scene.order[at];
        for (int k = 0; k < 3; k++) indices[at * 3 + k] = scene.indices[s * 3 + k];
        for (int k = 0; k < 4; k++) shading[at * 4 + k] = scene.shading[s * 4 + k];
        faces[at] = scene.faces[s];
        flat[at] = scene.flat[s];
    }
    scene.indices.swap(indices);
    scene.faces.swap(faces);
    scene.shading.swap(shading);
    scene.flat.swap(flat);
    scene.bvh_depth = bvh_depth(nodes);
}

}  // namespace lr
