// A wide BVH for the watertight traversal path, collapsed from the reference's BVH2: each
// wide node holds up to W (4 or 8) children, taken by repeatedly opening the child with the
// largest surface area (the greedy collapse of Wald et al. 2008 and Ylitie et al. 2017).
// Leaves are the BVH2's leaves unchanged, so the wide tree reaches the same triangle
// records in the same leaf order; only interior levels are merged, which cuts the
// dependent node fetches along a ray by about log2(W).
//
// Node layouts. W = 4: float4s, structure of arrays over the children so one load brings
// a plane of every child: 7 float4 = 112 bytes -- lo.x, hi.x, lo.y, hi.y, lo.z, hi.z of
// the 4 children, then their 4 links; an empty slot has an inverted box (lo +inf, hi
// -inf). W = 8: compressed, 96 bytes -- the node's origin and per-axis power-of-two steps,
// 8 child links, and each child's planes as 8-bit multiples of the steps, rounded outward
// (quantize.hpp). Links: >= 0 a wide node, < 0 a leaf (-1 - (first << 4 | count - 1)).
// The 8-wide node's children take slots by direction octant (Ylitie et al. 2017, section
// 3.2): slot s stands for the direction whose component k is negative where bit k of s is
// set, and children are placed greedily, the (child, slot) pair whose centroid lies
// furthest back along the slot's direction first. A ray whose direction signs make octant
// o then visits its hit children in the order of slot ^ o, nearest-first approximately,
// without sorting them.
// Boxes are widened outward like the BVH2 path's before they are stored or quantized.
#include "wide.hpp"

#include "quantize.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace lr {
namespace {

float area_of(const lr_bvh_node &n) {
    const float x = n.hi[0] - n.lo[0], y = n.hi[1] - n.lo[1], z = n.hi[2] - n.lo[2];
    return 2.0f * (x * y + y * z + z * x);
}

float bits(int v) {
    float f;
    std::memcpy(&f, &v, sizeof f);
    return f;
}

// The slot of each of `m` (<= 8) children of a node by direction octant: repeatedly the
// free (child, slot) pair with the smallest projection of the child's centroid, taken
// from the node's centre, on the slot's direction (ties: lower child, then lower slot).
void octant_slots(const lr_bvh_node *const *children, int m, int *slot_of) {
    float centre[3];
    for (int k = 0; k < 3; k++) {
        float lo = children[0]->lo[k], hi = children[0]->hi[k];
        for (int i = 1; i < m; i++) {
            lo = std::min(lo, children[i]->lo[k]);
            hi = std::max(hi, children[i]->hi[k]);
        }
        centre[k] = 0.5f * (lo + hi);
    }
    float cost[8][8];
    for (int i = 0; i < m; i++)
        for (int s = 0; s < 8; s++) {
            float c = 0.0f;
            for (int k = 0; k < 3; k++) {
                const float offset = 0.5f * (children[i]->lo[k] + children[i]->hi[k]) - centre[k];
                c += ((s >> k) & 1) ? -offset : offset;
            }
            cost[i][s] = c;
        }
    bool child_done[8] = {false}, slot_taken[8] = {false};
    for (int round = 0; round < m; round++) {
        int bi = -1, bs = -1;
        for (int i = 0; i < m; i++) {
            if (child_done[i]) continue;
            for (int s = 0; s < 8; s++)
                if (!slot_taken[s] && (bi < 0 || cost[i][s] < cost[bi][bs])) {
                    bi = i;
                    bs = s;
                }
        }
        child_done[bi] = true;
        slot_taken[bs] = true;
        slot_of[bi] = bs;
    }
}

}  // namespace

WideBvh build_wide(const std::vector<lr_bvh_node> &nodes, int width, float delta,
                   float (*widen_down)(float, float), float (*widen_up)(float, float),
                   int (*leaf_link)(const lr_bvh_node &)) {
    WideBvh w;
    w.width = width;
    const int per_node = width == 4 ? 7 : 14;
    w.floats_per_node = per_node;
    if (nodes.empty() || nodes[0].lo[0] > nodes[0].hi[0]) return w;  // no triangles
    struct Job {
        uint32_t bvh2;    // the BVH2 node this wide node stands for
        uint32_t wide;    // its index
    };
    std::vector<Job> queue;
    std::vector<std::vector<uint32_t>> children_of;  // per wide node, the BVH2 nodes it holds
    auto collapse = [&](uint32_t n) {
        std::vector<uint32_t> list;
        if (nodes[n].count > 0) {
            list.push_back(n);  // a leaf root: one leaf child
            return list;
        }
        list = {nodes[n].first, nodes[n].first + 1};
        while ((int)list.size() < width) {
            int best = -1;
            float best_area = -1.0f;
            for (size_t i = 0; i < list.size(); i++) {
                const lr_bvh_node &c = nodes[list[i]];
                if (c.count > 0) continue;
                const float a = area_of(c);
                if (a > best_area) {
                    best_area = a;
                    best = (int)i;
                }
            }
            if (best < 0) break;
            const uint32_t open = list[best];
            list.erase(list.begin() + best);
            list.insert(list.begin() + best, {nodes[open].first, nodes[open].first + 1});
        }
        return list;
    };
    // Breadth first: a node's interior children get consecutive indices.
    children_of.push_back(collapse(0));
    queue.push_back({0, 0});
    for (size_t head = 0; head < queue.size(); head++) {
        const uint32_t wide = queue[head].wide;
        for (uint32_t c : children_of[wide]) {
            if (nodes[c].count > 0) continue;
            const uint32_t index = (uint32_t)children_of.size();
            children_of.push_back(collapse(c));
            queue.push_back({c, index});
        }
    }
    const size_t count = children_of.size();
    w.node_count = count;
    w.sources.assign(count * width, 0xffffffffu);
    std::vector<uint32_t> index_of_bvh2(nodes.size(), 0xffffffffu);
    for (const Job &j : queue) index_of_bvh2[j.bvh2] = j.wide;
    // The wide root stands for BVH2 node 0 even when it is a leaf.
    std::vector<uint32_t> bound(count, 0);
    if (width == 8) {
        // Compressed: quantized child boxes (quantize.hpp), 96 bytes a node.
        w.floats_per_node = kQNodeFloat4s;
        w.nodes.assign(count * kQNodeFloat4s * 4, 0.0f);
        for (size_t n = 0; n < count; n++) {
            const auto &list = children_of[n];
            const int m = (int)list.size();
            const lr_bvh_node *kids[8];
            int slot_of[8];
            for (int i = 0; i < m; i++) kids[i] = &nodes[list[i]];
            octant_slots(kids, m, slot_of);
            float lo[8][3] = {}, hi[8][3] = {};
            int links[8] = {0};
            uint32_t occupied = 0;
            for (int i = 0; i < m; i++) {
                const int slot = slot_of[i];
                occupied |= 1u << slot;
                w.sources[n * width + slot] = list[i];
                const lr_bvh_node &c = *kids[i];
                for (int k = 0; k < 3; k++) {
                    lo[slot][k] = widen_down(c.lo[k], delta);
                    hi[slot][k] = widen_up(c.hi[k], delta);
                }
                links[slot] = c.count > 0 ? leaf_link(c) : (int)index_of_bvh2[list[i]];
            }
            quantize_node(occupied, lo, hi, links, &w.nodes[n * kQNodeFloat4s * 4]);
        }
        // A traversal keeps one group of a node's unvisited children a level: the stack
        // holds at most the tree's interior depth.
        for (size_t n = count; n-- > 0;) {
            uint32_t deepest = 0;
            for (uint32_t c : children_of[n])
                if (nodes[c].count == 0) deepest = std::max(deepest, bound[index_of_bvh2[c]]);
            bound[n] = 1 + deepest;
        }
        w.max_stack = bound[0];
        return w;
    }
    w.nodes.assign(count * per_node * 4, 0.0f);
    for (size_t n = 0; n < count; n++) {
        float *base = &w.nodes[n * per_node * 4];
        const auto &list = children_of[n];
        const int planes = width / 4;  // float4s per plane
        for (int slot = 0; slot < width; slot++) {
            float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
            int link = 0;
            if (slot < (int)list.size()) {
                w.sources[n * width + slot] = list[slot];
                const lr_bvh_node &c = nodes[list[slot]];
                for (int k = 0; k < 3; k++) {
                    lo[k] = widen_down(c.lo[k], delta);
                    hi[k] = widen_up(c.hi[k], delta);
                }
                link = c.count > 0 ? leaf_link(c) : (int)index_of_bvh2[list[slot]];
            }
            for (int k = 0; k < 3; k++) {
                base[((2 * k) * planes) * 4 + slot] = lo[k];
                base[((2 * k + 1) * planes) * 4 + slot] = hi[k];
            }
            base[(6 * planes) * 4 + slot] = bits(link);
        }
    }
    // The deepest stack a traversal can need: at each node it keeps all but one of the
    // hit children, so along a path the entries add up to sum(children - 1).
    for (size_t n = count; n-- > 0;) {
        uint32_t deepest = 0;
        for (uint32_t c : children_of[n])
            if (nodes[c].count == 0) deepest = std::max(deepest, bound[index_of_bvh2[c]]);
        bound[n] = (uint32_t)children_of[n].size() - 1 + deepest;
    }
    w.max_stack = bound[0];
    return w;
}

}  // namespace lr
