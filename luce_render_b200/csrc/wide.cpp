// A wide BVH for the watertight traversal path, collapsed from the reference's BVH2: each
// wide node holds up to W (4 or 8) children. Which BVH2 nodes become wide nodes is chosen
// by the surface area heuristic over the BVH2's own topology (Ylitie, Karras and Laine,
// HPG 2017, section 3.1, after Pinto 2010): a dynamic program gives every BVH2 node its
// least cost when it fills 1 to W child slots of its parent -- as one child (a wide node
// of its own, or a leaf) or opened, its two children sharing the slots -- and the tree is
// read back from the root. A leaf child is a BVH2 leaf, or a BVH2 subtree of at most
// `max_leaf` triangles taken whole (a subtree's triangles are one contiguous range of
// the leaf order): the wide tree reaches the same triangle records, and since a closest
// hit does not depend on the visiting order, the same hits.
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
#include <cstdlib>
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

// The SAH collapse: per BVH2 node its triangle range and, for 1 to W slots, its least
// cost and how it fills them.
struct Collapse {
    static constexpr float kNodeCost = 1.0f, kTriangleCost = 0.3f;
    const std::vector<lr_bvh_node> &nodes;
    int width, max_leaf;
    std::vector<uint32_t> first, tris;  // the subtree's triangles: [first, first + tris)
    std::vector<float> cost;            // per node, W entries: C(n, 1 .. W slots)
    std::vector<uint8_t> split;         // per node and slots: the left child's share when opened, 0 whole
    std::vector<uint8_t> leaf;          // taken whole, the node is a leaf (else a wide node)

    Collapse(const std::vector<lr_bvh_node> &n, int w, int m) : nodes(n), width(w), max_leaf(m) {
        const size_t N = nodes.size();
        first.assign(N, 0);
        tris.assign(N, 0);
        cost.assign(N * width, 0.0f);
        split.assign(N * width, 0);
        leaf.assign(N, 0);
        // Children come after their parent in the BVH2's numbering: a reverse sweep is a
        // post-order.
        for (size_t i = N; i-- > 0;) solve((uint32_t)i);
    }

    float C(uint32_t n, int slots) const { return cost[(size_t)n * width + slots - 1]; }

    void solve(uint32_t n) {
        const lr_bvh_node &node = nodes[n];
        const float area = area_of(node);
        float *c = &cost[(size_t)n * width];
        if (node.count > 0) {
            first[n] = node.first;
            tris[n] = node.count;
            leaf[n] = 1;
            for (int i = 0; i < width; i++) c[i] = area * kTriangleCost * (float)node.count;
            return;
        }
        const uint32_t l = node.first, r = node.first + 1;
        if (l <= n || r >= nodes.size()) fail(LR_INVALID, "a BVH2 node's children must follow it");
        first[n] = std::min(first[l], first[r]);
        tris[n] = tris[l] + tris[r];
        // Opened: the two children share i slots.
        float opened[9];
        uint8_t share[9] = {0};
        for (int i = 2; i <= width; i++) {
            opened[i] = INFINITY;
            for (int k = 1; k < i; k++) {
                const float v = C(l, k) + C(r, i - k);
                if (v < opened[i]) {
                    opened[i] = v;
                    share[i] = (uint8_t)k;
                }
            }
        }
        const float as_node = area * kNodeCost + opened[width];
        const float as_leaf = (int)tris[n] <= max_leaf ? area * kTriangleCost * (float)tris[n] : INFINITY;
        leaf[n] = as_leaf < as_node;
        c[0] = std::min(as_node, as_leaf);
        split[(size_t)n * width + width - 1] = share[width];  // a wide node's own children
        for (int i = 2; i <= width; i++) {
            const bool whole = c[0] <= opened[i];
            c[i - 1] = whole ? c[0] : opened[i];
            if (i < width) split[(size_t)n * width + i - 1] = whole ? 0 : share[i];
        }
    }

    // The children of wide node n: its two BVH2 children sharing W slots.
    void children(uint32_t n, std::vector<uint32_t> &out) const {
        const uint32_t k = split[(size_t)n * width + width - 1];
        gather(nodes[n].first, (int)k, out);
        gather(nodes[n].first + 1, width - (int)k, out);
    }

    // Node n in `slots` slots: whole (one child), or opened.
    void gather(uint32_t n, int slots, std::vector<uint32_t> &out) const {
        const uint32_t k = slots >= 2 && slots < width ? split[(size_t)n * width + slots - 1] : 0;
        if (slots == 1 || nodes[n].count > 0 || k == 0) {
            out.push_back(n);
            return;
        }
        gather(nodes[n].first, (int)k, out);
        gather(nodes[n].first + 1, slots - (int)k, out);
    }

    // Taken whole, node n is a leaf child.
    bool is_leaf(uint32_t n) const { return leaf[n] != 0; }
};

}  // namespace

int wide_leaf_triangles() {
    if (const char *env = std::getenv("LUCE_RENDER_B200_WIDE_LEAF")) {
        const int v = std::atoi(env);
        if (v >= 0 && v <= 16) return v;
    }
    return kWideLeafTriangles;
}

WideBvh build_wide(const std::vector<lr_bvh_node> &nodes, int width, float delta,
                   float (*widen_down)(float, float), float (*widen_up)(float, float),
                   int (*leaf_link)(const lr_bvh_node &)) {
    WideBvh w;
    w.width = width;
    const int per_node = width == 4 ? 7 : 14;
    w.floats_per_node = per_node;
    if (nodes.empty() || nodes[0].lo[0] > nodes[0].hi[0]) return w;  // no triangles
    const Collapse plan(nodes, width, wide_leaf_triangles());
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
        plan.children(n, list);
        return list;
    };
    // A child taken as a leaf: a BVH2 leaf, or a subtree's triangle range.
    auto is_leaf = [&](uint32_t c) { return plan.is_leaf(c); };
    auto link_of_leaf = [&](uint32_t c) {
        lr_bvh_node range = nodes[c];
        range.first = plan.first[c];
        range.count = plan.tris[c];
        return leaf_link(range);
    };
    // Breadth first: a node's interior children get consecutive indices.
    children_of.push_back(collapse(0));
    queue.push_back({0, 0});
    for (size_t head = 0; head < queue.size(); head++) {
        const uint32_t wide = queue[head].wide;
        for (uint32_t c : children_of[wide]) {
            if (is_leaf(c)) continue;
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
                links[slot] = is_leaf(list[i]) ? link_of_leaf(list[i]) : (int)index_of_bvh2[list[i]];
            }
            quantize_node(occupied, lo, hi, links, &w.nodes[n * kQNodeFloat4s * 4]);
        }
        // A traversal keeps one group of a node's unvisited children a level: the stack
        // holds at most the tree's interior depth.
        for (size_t n = count; n-- > 0;) {
            uint32_t deepest = 0;
            for (uint32_t c : children_of[n])
                if (!is_leaf(c)) deepest = std::max(deepest, bound[index_of_bvh2[c]]);
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
                link = is_leaf(list[slot]) ? link_of_leaf(list[slot]) : (int)index_of_bvh2[list[slot]];
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
            if (!is_leaf(c)) deepest = std::max(deepest, bound[index_of_bvh2[c]]);
        bound[n] = (uint32_t)children_of[n].size() - 1 + deepest;
    }
    w.max_stack = bound[0];
    return w;
}

}  // namespace lr
