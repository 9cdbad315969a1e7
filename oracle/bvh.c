/*
 * Oracle (test infrastructure): the reference's binned-SAH BVH2 build, restated.
 * Follows src/render/bvh.lucb line by line; f32 arithmetic as the reference has it.
 */
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

enum { BINS = 12, LEAF_SIZE = 4, LEAF_LIMIT = 16 }; /* bvh.lucb:29-32 */

typedef struct {
    float lo[3], hi[3];
} box;

/* Box.empty (bvh.lucb:38-39) */
static box box_empty(void) {
    box b = {{3.0e38f, 3.0e38f, 3.0e38f}, {-3.0e38f, -3.0e38f, -3.0e38f}};
    return b;
}

static float fmin32(float a, float b) { return a < b ? a : b; }
static float fmax32(float a, float b) { return a > b ? a : b; }

/* Box.grow (bvh.lucb:41-43) */
static box box_grow(box a, const box *b) {
    for (int k = 0; k < 3; k++) {
        a.lo[k] = fmin32(a.lo[k], b->lo[k]);
        a.hi[k] = fmax32(a.hi[k], b->hi[k]);
    }
    return a;
}

static box box_grow_point(box a, const float p[3]) {
    box b = {{p[0], p[1], p[2]}, {p[0], p[1], p[2]}};
    return box_grow(a, &b);
}

/* Box.area (bvh.lucb:48-53) */
static float box_area(const box *b) {
    float x = b->hi[0] - b->lo[0];
    float y = b->hi[1] - b->lo[1];
    float z = b->hi[2] - b->lo[2];
    if (x < 0.0f || y < 0.0f || z < 0.0f) return 0.0f;
    return 2.0f * (x * y + y * z + z * x);
}

typedef struct {
    long axis;
    size_t bin;
    float cost;
} split_t;

/* bin_of (bvh.lucb:136-142) */
static size_t bin_of(const float c[3], const box *middle, int axis) {
    float lo = middle->lo[axis];
    float extent = middle->hi[axis] - lo;
    if (extent <= 0.0f) return 0;
    long at = (long)((float)BINS * (c[axis] - lo) / extent);
    if (at < 0) return 0;
    return at < (long)BINS ? (size_t)at : BINS - 1;
}

/* best_split (bvh.lucb:147-182) */
static split_t best_split(const box *boxes, const float (*centers)[3], const uint32_t *order,
                          size_t n, const box *parent, const box *middle) {
    split_t best = {-1, 0, 3.0e38f};
    float area = box_area(parent);
    if (area <= 0.0f) return best;
    for (int axis = 0; axis < 3; axis++) {
        if (middle->hi[axis] - middle->lo[axis] <= 0.0f) continue;
        size_t counts[BINS];
        box bounds[BINS];
        for (int b = 0; b < BINS; b++) {
            counts[b] = 0;
            bounds[b] = box_empty();
        }
        for (size_t i = 0; i < n; i++) {
            uint32_t index = order[i];
            size_t b = bin_of(centers[index], middle, axis);
            counts[b] += 1;
            bounds[b] = box_grow(bounds[b], &boxes[index]);
        }
        float right_area[BINS];
        size_t right_count[BINS];
        box sweep = box_empty();
        size_t total = 0;
        for (size_t b = BINS - 1; b > 0; b--) {
            sweep = box_grow(sweep, &bounds[b]);
            total += counts[b];
            right_area[b] = box_area(&sweep);
            right_count[b] = total;
        }
        box left = box_empty();
        size_t left_count = 0;
        for (size_t s = 1; s < BINS; s++) {
            left = box_grow(left, &bounds[s - 1]);
            left_count += counts[s - 1];
            if (left_count == 0 || right_count[s] == 0) continue;
            float cost = 1.0f + (box_area(&left) * (float)left_count +
                                 right_area[s] * (float)right_count[s]) /
                                    area;
            if (cost < best.cost) {
                best.axis = axis;
                best.bin = s;
                best.cost = cost;
            }
        }
    }
    return best;
}

/* partition (bvh.lucb:185-196) */
static size_t partition(const float (*centers)[3], uint32_t *order, size_t n, const box *middle,
                        int axis, size_t bin) {
    size_t low = 0, high = n;
    while (low < high) {
        if (bin_of(centers[order[low]], middle, axis) < bin) {
            low += 1;
        } else {
            high -= 1;
            uint32_t held = order[low];
            order[low] = order[high];
            order[high] = held;
        }
    }
    return low;
}

typedef struct {
    size_t node, first, count;
} pending;

static void set_node(or_node *n, const box *b, uint32_t first, uint32_t count) {
    for (int k = 0; k < 3; k++) {
        n->lo[k] = b->lo[k];
        n->hi[k] = b->hi[k];
    }
    n->first = first;
    n->count = count;
}

/* build_tree (bvh.lucb:85-129) */
static size_t build_tree(const box *boxes, size_t count, uint32_t *order, or_node *nodes) {
    size_t node_count = 0;
    if (count == 0) {
        or_node empty = {{1.0f, 1.0f, 1.0f}, 0, {-1.0f, -1.0f, -1.0f}, 0};
        nodes[0] = empty;
        return 1;
    }
    float (*centers)[3] = malloc(sizeof(float[3]) * count);
    for (size_t at = 0; at < count; at++) {
        for (int k = 0; k < 3; k++) centers[at][k] = 0.5f * (boxes[at].lo[k] + boxes[at].hi[k]);
        order[at] = (uint32_t)at;
    }
    memset(&nodes[0], 0, sizeof(or_node));
    node_count = 1;
    pending *stack = malloc(sizeof(pending) * (2 * count + 2));
    size_t depth = 0;
    stack[depth++] = (pending){0, 0, count};
    while (depth > 0) {
        pending job = stack[--depth];
        box bounds = box_empty(), middle = box_empty();
        for (size_t at = job.first; at < job.first + job.count; at++) {
            bounds = box_grow(bounds, &boxes[order[at]]);
            middle = box_grow_point(middle, centers[order[at]]);
        }
        float leaf_cost = (float)job.count;
        size_t left_count = 0;
        split_t split = {-1, 0, 3.0e38f};
        if (job.count > LEAF_SIZE)
            split = best_split(boxes, (const float (*)[3])centers, order + job.first, job.count,
                               &bounds, &middle);
        if (job.count > LEAF_SIZE && (split.cost < leaf_cost || job.count > LEAF_LIMIT)) {
            if (split.axis >= 0 && split.cost < 3.0e38f)
                left_count = partition((const float (*)[3])centers, order + job.first, job.count,
                                       &middle, (int)split.axis, split.bin);
            if (left_count == 0 || left_count == job.count) left_count = job.count / 2;
        }
        if (left_count == 0) {
            set_node(&nodes[job.node], &bounds, (uint32_t)job.first, (uint32_t)job.count);
            continue;
        }
        size_t child = node_count;
        memset(&nodes[child], 0, 2 * sizeof(or_node));
        node_count += 2;
        set_node(&nodes[job.node], &bounds, (uint32_t)child, 0);
        stack[depth++] = (pending){child + 1, job.first + left_count, job.count - left_count};
        stack[depth++] = (pending){child, job.first, left_count};
    }
    free(stack);
    free(centers);
    return node_count;
}

/* build_bvh (bvh.lucb:66-82), without the reorder. */
size_t or_build_bvh(const float *positions, const uint32_t *indices, size_t triangle_count,
                    or_node *nodes, uint32_t *order) {
    box *boxes = malloc(sizeof(box) * (triangle_count ? triangle_count : 1));
    for (size_t at = 0; at < triangle_count; at++) {
        box b = box_empty();
        for (int k = 0; k < 3; k++) b = box_grow_point(b, &positions[(size_t)indices[at * 3 + k] * 3]);
        boxes[at] = b;
    }
    size_t n = build_tree(boxes, triangle_count, order, nodes);
    free(boxes);
    return n;
}

/* reorder (bvh.lucb:198-217) */
void or_reorder(const uint32_t *order, size_t count, uint32_t *indices, uint32_t *faces,
                uint32_t *shading, float *uvs) {
    uint32_t *i2 = indices ? malloc(sizeof(uint32_t) * 3 * count + 4) : NULL;
    uint32_t *f2 = faces ? malloc(sizeof(uint32_t) * count + 4) : NULL;
    uint32_t *s2 = shading ? malloc(sizeof(uint32_t) * 4 * count + 4) : NULL;
    float *u2 = uvs ? malloc(sizeof(float) * 6 * count + 4) : NULL;
    for (size_t at = 0; at < count; at++) {
        size_t source = order[at];
        if (i2)
            for (int k = 0; k < 3; k++) i2[at * 3 + k] = indices[source * 3 + k];
        if (s2)
            for (int k = 0; k < 4; k++) s2[at * 4 + k] = shading[source * 4 + k];
        if (u2)
            for (int k = 0; k < 6; k++) u2[at * 6 + k] = uvs[source * 6 + k];
        if (f2) f2[at] = faces[source];
    }
    if (i2) memcpy(indices, i2, sizeof(uint32_t) * 3 * count), free(i2);
    if (f2) memcpy(faces, f2, sizeof(uint32_t) * count), free(f2);
    if (s2) memcpy(shading, s2, sizeof(uint32_t) * 4 * count), free(s2);
    if (u2) memcpy(uvs, u2, sizeof(float) * 6 * count), free(u2);
}

static uint32_t depth_of(const or_node *nodes, uint32_t node, uint32_t depth) {
    if (nodes[node].count > 0) return depth;
    uint32_t a = depth_of(nodes, nodes[node].first, depth + 1);
    uint32_t b = depth_of(nodes, nodes[node].first + 1, depth + 1);
    return a > b ? a : b;
}

uint32_t or_bvh_depth(const or_node *nodes, size_t node_count) {
    if (node_count == 0 || nodes[0].lo[0] > nodes[0].hi[0]) return 0;
    return depth_of(nodes, 0, 0);
}
