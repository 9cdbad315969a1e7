// Device-side state shared by the CUDA translation units: the context (device + stream
// + timing events), the scene as it lives in HBM, and CUDA error checking.
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "common.hpp"

namespace lr {

#define LR_CUDA(call)                                                                      \
    do {                                                                                   \
        cudaError_t lr_status_ = (call);                                                   \
        if (lr_status_ != cudaSuccess)                                                     \
            ::lr::fail(LR_DEVICE, std::string(#call) + ": " + cudaGetErrorString(lr_status_)); \
    } while (0)

// Leaf links: a child link >= 0 is an interior entry; a negative link is a leaf whose
// triangles are `first .. first + count` in leaf order, packed as -1 - (first << 4 | count - 1).
constexpr int kLeafShift = 4;
constexpr uint32_t kMaxLeafFirst = (1u << (31 - kLeafShift)) - 1;

// The BVH2 in traversal form: one 64-byte entry per interior node holding both children's
// boxes and links (the 64 bytes an interior visit reads), plus the root's box and link.
struct DeviceBvh {
    const float4 *entries = nullptr;  // 4 float4 per interior node
    float root_lo[3] = {1, 1, 1}, root_hi[3] = {-1, -1, -1};
    int root = 0;                      // root link (entry 0, or a leaf link)
    int empty = 1;                     // no triangles: every ray misses
};

// A wide BVH (wide.cpp) in HBM: `width` children a node, nodes of 7 (W=4) or 14 (W=8)
// float4s; the root is node 0.
struct DeviceWide {
    const float4 *nodes = nullptr;
    int width = 0;
    uint32_t max_stack = 0;   // the most stack entries a traversal can hold
    uint64_t node_count = 0;
};

// A scene in HBM (GpuScene, device.lucb:16-38).
struct DeviceScene {
    DeviceBvh bvh;        // boxes widened outward for the watertight path
    DeviceBvh ref_bvh;    // the reference's exact boxes (LR_TRACE_REFERENCE)
    DeviceWide wide4, wide8;  // the watertight path's 4- and 8-wide collapses of bvh
    const float4 *tris = nullptr;      // 3 float4 per leaf slot: v0 (w: source id bits), v1, v2
    const float *positions = nullptr;  // xyz per point
    const uint32_t *indices = nullptr; // 3 per leaf slot
    const uint32_t *faces = nullptr;   // polygon per leaf slot
    const uint32_t *ids = nullptr;     // source triangle per leaf slot
    const uint4 *shading = nullptr;    // 3 octahedral normals + material per leaf slot
    uint64_t triangle_count = 0, point_count = 0, entry_count = 0;
    uint32_t depth = 0;                // the BVH2's deepest leaf
};

}  // namespace lr

struct lr_context {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t start = nullptr, stop = nullptr;
    int sm_count = 148;
    // Device status words: [0] traversal stack pushes lost, [1] bounded waits that gave up.
    int *status = nullptr;
    // Traversal work of counted ray queries: interior visits, triangle tests.
    unsigned long long *counts = nullptr;
};

namespace lr {
// Reads and clears the context's status words; fails when one is set.
void check_status(lr_context *ctx);
// lr_probe_static's set-up on `device` (the device address of its static array, looked up
// once per device, which may load the module there); returns the address.
void *probe_static_setup(int device);
}  // namespace lr

struct lr_gpu_scene {
    lr_context *ctx = nullptr;
    lr::DeviceScene scene;
    void *allocation = nullptr;  // one device block holds every array
    size_t bytes = 0;
    size_t wide4_nodes = 0, wide8_nodes = 0;
    // What a refit (refit.cu) reads besides the traversal arrays: per interior entry its
    // parent (entry << 1 | side; 0xffffffff the root) and a climb counter; per wide child
    // slot the BVH2 box it holds (entry << 1 | side; kRefitRoot the root's; 0xffffffff
    // none); per leaf slot whether its normals are its own flat one; the exact root box.
    uint32_t *parents = nullptr, *counters = nullptr, *wide4_sources = nullptr, *wide8_sources = nullptr;
    uint8_t *flat = nullptr;
    float *root_box = nullptr;
    uint64_t topology = 0;  // a hash of the triangles (leaf order) a refit must keep
    uint64_t refits = 0;    // refits so far: batch members borrowing the scene follow them
    bool any_flat = false;  // some triangle's normals are its own flat one
    // Built on the device (build.cu): a linear BVH in its own leaf order, no wide collapses;
    // its leaf order is not the compiled scene's, so renders do not take it.
    bool device_built = false;
};

namespace lr {
constexpr uint32_t kRefitRoot = 0xfffffffeu;
// refit.cu: with the uploaded scene's points already moved (its `positions` array),
// refits its triangle records, flat normals and every BVH's boxes on `stream`; waits.
void refit_scene(lr_gpu_scene *gs, cudaStream_t stream);
// FNV-1a over a scene's triangle count and leaf-order indices.
uint64_t topology_hash(const Scene &scene);
}  // namespace lr

namespace lr {
// The traversal the watertight path uses for a scene: BVH width 2, 4 or 8 and stack
// entries (`requested` 0 picks the widest whose stack bound fits shared memory).
struct TraversalChoice {
    int width;
    int stack;
};
TraversalChoice choose_traversal(const DeviceScene &s, int requested);
}  // namespace lr
