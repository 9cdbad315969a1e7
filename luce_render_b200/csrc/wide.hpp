// The wide BVH of the watertight traversal path (wide.cpp).
#pragma once

#include <vector>

#include "common.hpp"

namespace lr {

struct WideBvh {
    int width = 4;
    int floats_per_node = 7;  // float4s per node
    size_t node_count = 0;
    std::vector<float> nodes;  // node_count * floats_per_node float4s
    uint32_t max_stack = 0;    // the most stack entries a traversal can hold
    // Per node and child slot, the BVH2 node whose box the slot holds (0xffffffff: an
    // empty slot), so a refit can copy the boxes again.
    std::vector<uint32_t> sources;
};

// The most triangles of a BVH2 subtree the collapse may take as one leaf of a wide tree.
// The environment variable LUCE_RENDER_B200_WIDE_LEAF (0 to 16; 0 keeps the BVH2's leaves)
// overrides it, for tuning.
constexpr int kWideLeafTriangles = 0;
int wide_leaf_triangles();

// Collapses the BVH2 `nodes` into a `width`-wide BVH (4 or 8). Child boxes are widened by
// `delta` with the given rounding, leaves encoded by `leaf_link`.
WideBvh build_wide(const std::vector<lr_bvh_node> &nodes, int width, float delta, float (*widen_down)(float, float),
                   float (*widen_up)(float, float), int (*leaf_link)(const lr_bvh_node &));

}  // namespace lr
