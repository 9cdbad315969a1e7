// Building an uploaded scene's BVH2 on the device: the analogue of the reference's
// `GpuScene.upload(accelerate = true)` (device.lucb:41-89), where a device that traces rays
// in hardware builds its own acceleration structure from the uploaded triangles and the
// host compiles without software trees (`compile_scene(trees = false)`, scene.lucb:111-129).
// B200 has no ray-tracing cores, so the device builds the BVH2 the watertight path walks:
//   1. the bounds of the triangles' centroids (one reduction launch);
//   2. a triangle's 30-bit Morton code of its centroid over those bounds;
//   3. the codes sorted stably with the triangles' indices (a least-significant-digit radix
//      sort of this file's own, four passes of 8 bits), which leaves the 64-bit keys
//      code << 32 | index -- unique, in ascending order;
//   4. the triangles' indices, polygons, shading words, flat flags and source ids gathered
//      into the sorted (leaf) order, one triangle a leaf;
//   5. the hierarchy over the sorted keys (Karras, "Maximizing Parallelism in the
//      Construction of BVHs, Octrees, and k-d Trees", HPG 2012): interior node i covers a
//      key range found from the longest common prefixes around i, split where the range's
//      keys first differ in the range's highest differing bit; links and parent slots in
//      the traversal layout;
//   6. the deepest leaf (the traversal's stack bound);
//   7. the boxes, the triangle records, flat normals and widened boxes by the refit of
//      refit.cu (the same bottom-up climb), since a refit is exactly "boxes for a topology".
// Closest hits stay exact: the watertight triangle test and the conservative widened boxes
// do not depend on the tree, so ids and distances equal the brute force bit for bit. The
// tree is a linear BVH, shallower to build but slower to trace than the host's binned SAH,
// and has no 4- or 8-wide collapse: every query on it takes the BVH2.
#include <algorithm>
#include <cmath>
#include <memory>
#include <vector>

#include "device.hpp"

namespace lr {
namespace {

// Floats as unsigned integers whose order is the floats' order (for atomicMin / atomicMax).
__device__ __forceinline__ uint32_t ordered(float f) {
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float unordered(uint32_t u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

__device__ __forceinline__ float3 centroid(const float *positions, const uint32_t *indices, uint64_t t) {
    const float *a = &positions[(size_t)indices[t * 3] * 3];
    const float *b = &positions[(size_t)indices[t * 3 + 1] * 3];
    const float *c = &positions[(size_t)indices[t * 3 + 2] * 3];
    return make_float3((a[0] + b[0] + c[0]) * (1.0f / 3.0f), (a[1] + b[1] + c[1]) * (1.0f / 3.0f),
                       (a[2] + b[2] + c[2]) * (1.0f / 3.0f));
}

// Step 1: bounds[0..2] the ordered minima, bounds[3..5] the maxima (set to the extremes first).
__global__ void bounds_kernel(uint64_t count, const float *positions, const uint32_t *indices, uint32_t *bounds) {
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < count; t += (uint64_t)gridDim.x * blockDim.x) {
        const float3 c = centroid(positions, indices, t);
        lo[0] = fminf(lo[0], c.x), lo[1] = fminf(lo[1], c.y), lo[2] = fminf(lo[2], c.z);
        hi[0] = fmaxf(hi[0], c.x), hi[1] = fmaxf(hi[1], c.y), hi[2] = fmaxf(hi[2], c.z);
    }
    for (int k = 0; k < 3; k++)
        for (int step = 16; step > 0; step >>= 1) {
            lo[k] = fminf(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], step));
            hi[k] = fmaxf(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], step));
        }
    if ((threadIdx.x & 31) == 0)
        for (int k = 0; k < 3; k++) {
            atomicMin(&bounds[k], ordered(lo[k]));
            atomicMax(&bounds[3 + k], ordered(hi[k]));
        }
}

// 10 bits spread to every third bit.
__device__ __forceinline__ uint32_t spread(uint32_t v) {
    v = (v | (v << 16)) & 0x030000ffu;
    v = (v | (v << 8)) & 0x0300f00fu;
    v = (v | (v << 4)) & 0x030c30c3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

// Step 2.
__global__ void keys_kernel(uint64_t count, const float *positions, const uint32_t *indices, const uint32_t *bounds,
                            uint32_t *codes) {
    float lo[3], scale[3];
    for (int k = 0; k < 3; k++) {
        lo[k] = unordered(bounds[k]);
        const float extent = unordered(bounds[3 + k]) - lo[k];
        scale[k] = extent > 0.0f ? 1024.0f / extent : 0.0f;
    }
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < count; t += (uint64_t)gridDim.x * blockDim.x) {
        const float3 c = centroid(positions, indices, t);
        const float v[3] = {c.x, c.y, c.z};
        uint32_t q[3];
        for (int k = 0; k < 3; k++) q[k] = (uint32_t)fminf(fmaxf((v[k] - lo[k]) * scale[k], 0.0f), 1023.0f);
        codes[t] = (spread(q[0]) << 2) | (spread(q[1]) << 1) | spread(q[2]);
    }
}

// Step 3: a stable LSD radix sort of the codes with their indices, 8 bits a pass. A pass
// is three launches over tiles of kSortTile codes (kSortThreads threads, kSortItems codes
// each): every tile counts its digits (digit_counts_kernel); one block a digit turns that
// digit's counts over the tiles into exclusive offsets and the digit's total (row_scan_kernel);
// every tile then ranks its codes within each digit in input order and writes them after
// the digits below and the tiles before (scatter_kernel). Inside a tile, warp w holds codes
// w*256 .. w*256+255 with item k of lane l at k*32 + l, so the order (warp, item, lane) is the
// input order; a warp ranks equal digits of one item with __match_any_sync and keeps a
// count a digit in shared memory.
constexpr int kSortThreads = 256, kSortItems = 8, kSortTile = kSortThreads * kSortItems, kRadix = 256;

__global__ void __launch_bounds__(kSortThreads) digit_counts_kernel(uint64_t count, const uint32_t *codes, int shift,
                                                                    uint32_t *counts) {
    __shared__ uint32_t hist[kRadix];
    hist[threadIdx.x] = 0;
    __syncthreads();
    const uint64_t base = (uint64_t)blockIdx.x * kSortTile;
    for (int k = 0; k < kSortItems; k++) {
        const uint64_t i = base + (uint64_t)k * kSortThreads + threadIdx.x;
        if (i < count) atomicAdd(&hist[(codes[i] >> shift) & (kRadix - 1)], 1u);
    }
    __syncthreads();
    counts[(size_t)threadIdx.x * gridDim.x + blockIdx.x] = hist[threadIdx.x];
}

// Exclusive scan of a block's values (one a thread, kSortThreads of them); *total the sum.
__device__ __forceinline__ uint32_t block_exclusive(uint32_t v, uint32_t *warp_sums, uint32_t &total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
        if (lane >= d) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    uint32_t before = 0;
    total = 0;
    for (int w = 0; w < kSortThreads / 32; w++) {
        const uint32_t s = warp_sums[w];
        if (w < warp) before += s;
        total += s;
    }
    __syncthreads();
    return before + x - v;
}

// Digit `blockIdx.x`'s counts over the `tiles` tiles become exclusive offsets; totals[d]
// the digit's count.
__global__ void __launch_bounds__(kSortThreads) row_scan_kernel(uint32_t tiles, uint32_t *counts, uint32_t *totals) {
    __shared__ uint32_t warp_sums[kSortThreads / 32];
    uint32_t *row = counts + (size_t)blockIdx.x * tiles;
    uint32_t carry = 0;
    for (uint32_t at = 0; at < tiles; at += kSortThreads) {
        const uint32_t i = at + threadIdx.x;
        const uint32_t v = i < tiles ? row[i] : 0u;
        uint32_t total;
        const uint32_t before = block_exclusive(v, warp_sums, total);
        if (i < tiles) row[i] = carry + before;
        carry += total;
    }
    if (threadIdx.x == 0) totals[blockIdx.x] = carry;
}

// One pass's scatter. `values` null: the indices are the positions (the first pass). With
// `keys` the pass writes code << 32 | index there instead of codes and values (the last).
__global__ void __launch_bounds__(kSortThreads) scatter_kernel(uint64_t count, const uint32_t *codes_in,
                                                               const uint32_t *values_in, int shift,
                                                               const uint32_t *counts, const uint32_t *totals,
                                                               uint32_t *codes_out, uint32_t *values_out,
                                                               uint64_t *keys) {
    constexpr int kWarps = kSortThreads / 32;
    __shared__ uint32_t warp_count[kWarps][kRadix];
    __shared__ uint32_t tile_base[kRadix];
    __shared__ uint32_t warp_sums[kWarps];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int w = 0; w < kWarps; w++) warp_count[w][threadIdx.x] = 0;
    // The digit's start: the digits below it, then the tiles before this one.
    uint32_t total;
    const uint32_t below = block_exclusive(totals[threadIdx.x], warp_sums, total);
    tile_base[threadIdx.x] = below + counts[(size_t)threadIdx.x * gridDim.x + blockIdx.x];
    __syncthreads();
    const uint64_t base = (uint64_t)blockIdx.x * kSortTile + (uint64_t)warp * (32 * kSortItems);
    const uint32_t lower = (1u << lane) - 1u;
    uint32_t code[kSortItems], value[kSortItems], rank[kSortItems];
#pragma unroll
    for (int k = 0; k < kSortItems; k++) {
        const uint64_t i = base + (uint64_t)k * 32 + lane;
        const bool valid = i < count;
        code[k] = valid ? codes_in[i] : 0u;
        value[k] = valid ? (values_in ? values_in[i] : (uint32_t)i) : 0u;
        const uint32_t digit = (code[k] >> shift) & (kRadix - 1);
        // Lanes past the end get keys of their own, so they match no one.
        const uint32_t peers = __match_any_sync(0xffffffffu, valid ? digit : kRadix + (uint32_t)lane);
        const uint32_t seen = warp_count[warp][digit];
        rank[k] = seen + __popc(peers & lower);
        __syncwarp();
        if (valid && lane == __ffs(peers) - 1) warp_count[warp][digit] = seen + __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    // Each digit's count over the warps before, in place.
    {
        uint32_t running = 0;
        for (int w = 0; w < kWarps; w++) {
            const uint32_t c = warp_count[w][threadIdx.x];
            warp_count[w][threadIdx.x] = running;
            running += c;
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kSortItems; k++) {
        const uint64_t i = base + (uint64_t)k * 32 + lane;
        if (i >= count) continue;
        const uint32_t digit = (code[k] >> shift) & (kRadix - 1);
        const uint64_t at = (uint64_t)tile_base[digit] + warp_count[warp][digit] + rank[k];
        if (keys) {
            keys[at] = (uint64_t)code[k] << 32 | value[k];
        } else {
            codes_out[at] = code[k];
            values_out[at] = value[k];
        }
    }
}

// Step 4.
__global__ void gather_kernel(uint64_t count, const uint64_t *keys, const uint32_t *indices_in, const uint32_t *faces_in,
                              const uint4 *shading_in, const uint8_t *flat_in, const uint32_t *ids_in, uint32_t *indices,
                              uint32_t *faces, uint4 *shading, uint8_t *flat, uint32_t *ids) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < count; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t j = (uint32_t)keys[i];
        indices[i * 3] = indices_in[(size_t)j * 3];
        indices[i * 3 + 1] = indices_in[(size_t)j * 3 + 1];
        indices[i * 3 + 2] = indices_in[(size_t)j * 3 + 2];
        faces[i] = faces_in[j];
        shading[i] = shading_in[j];
        flat[i] = flat_in[j];
        ids[i] = ids_in[j];
    }
}

// The length of the common prefix of keys a and b; -1 when b lies outside the keys.
__device__ __forceinline__ int prefix(const uint64_t *keys, int64_t count, int64_t a, int64_t b) {
    if (b < 0 || b >= count) return -1;
    return __clzll((long long)(keys[a] ^ keys[b]));
}

// Step 5: interior node i (0 the root) of count - 1. A child link is the child's interior
// index, or for a leaf -1 - (slot << kLeafShift) (one triangle). Both entry arrays get the
// links (refit.cu fills their boxes); interior children record their parent slot
// (node << 1 | side), leaves theirs in `leaf_parents`.
__global__ void hierarchy_kernel(int64_t count, const uint64_t *keys, float4 *exact, float4 *widened,
                                 uint32_t *parents, uint32_t *leaf_parents) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= count - 1) return;
    const int d = prefix(keys, count, i, i + 1) > prefix(keys, count, i, i - 1) ? 1 : -1;
    const int bottom = prefix(keys, count, i, i - d);
    int64_t reach = 2;
    while (prefix(keys, count, i, i + reach * d) > bottom) reach <<= 1;
    int64_t length = 0;
    for (int64_t step = reach >> 1; step >= 1; step >>= 1)
        if (prefix(keys, count, i, i + (length + step) * d) > bottom) length += step;
    const int64_t j = i + length * d;
    const int shared = prefix(keys, count, i, j);
    int64_t split = 0;
    for (int64_t divisor = 2;; divisor <<= 1) {
        const int64_t step = (length + divisor - 1) / divisor;
        if (prefix(keys, count, i, i + (split + step) * d) > shared) split += step;
        if (step <= 1) break;
    }
    const int64_t gamma = i + split * d + (d < 0 ? -1 : 0);
    const int64_t child[2] = {gamma, gamma + 1};
    const bool leaf[2] = {(i < j ? i : j) == gamma, (i < j ? j : i) == gamma + 1};
    int link[2];
    for (int side = 0; side < 2; side++) {
        const uint32_t slot = (uint32_t)i << 1 | (uint32_t)side;
        if (leaf[side]) {
            link[side] = -1 - (int)((uint32_t)child[side] << kLeafShift);
            leaf_parents[child[side]] = slot;
        } else {
            link[side] = (int)child[side];
            parents[child[side]] = slot;
        }
    }
    const float4 links = make_float4(__int_as_float(link[0]), __int_as_float(link[1]), 0.0f, 0.0f);
    exact[i * 4 + 3] = links;
    widened[i * 4 + 3] = links;
    if (i == 0) parents[0] = 0xffffffffu;
}

// Step 6: each leaf's depth (the root's children at 1), bounded by `limit` steps.
__global__ void depth_kernel(uint64_t count, const uint32_t *leaf_parents, const uint32_t *parents, uint32_t limit,
                             uint32_t *deepest) {
    uint32_t best = 0;
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < count; t += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t depth = 1, at = leaf_parents[t] >> 1;
        while (depth < limit && parents[at] != 0xffffffffu) {
            at = parents[at] >> 1;
            depth++;
        }
        best = max(best, depth);
    }
    for (int step = 16; step > 0; step >>= 1) best = max(best, __shfl_xor_sync(0xffffffffu, best, step));
    if ((threadIdx.x & 31) == 0) atomicMax(deepest, best);
}

unsigned grid_of(uint64_t items, int sm_count) {
    const uint64_t blocks = (items + 255) / 256;
    return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(blocks, (uint64_t)sm_count * 8));
}

size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

// Device scratch of one build, freed however the build ends.
struct Scratch {
    void *p = nullptr;
    ~Scratch() {
        if (p) cudaFree(p);
    }
};

}  // namespace
}  // namespace lr

using namespace lr;

extern "C" {

int lr_gpu_scene_build(lr_context *ctx, const lr_scene *scene, lr_gpu_scene **out) {
    return guarded([&] {
        if (!ctx || !scene || !out) fail(LR_INVALID, "a device build needs a context and a scene");
        *out = nullptr;
        const uint64_t T = scene->triangle_count(), P = scene->point_count();
        if (T > kMaxLeafFirst) fail(LR_LIMIT, "a device build takes at most 2^27 triangles");
        LR_CUDA(cudaSetDevice(ctx->device));
        const uint64_t E = T > 1 ? T - 1 : 0;
        // The scene's block, laid out as lr_gpu_scene_upload's (no wide collapses).
        size_t offsets[12], total = 0;
        const size_t sizes[12] = {E * 4 * sizeof(float4), E * 4 * sizeof(float4), T * 3 * sizeof(float4),
                                  P * 3 * sizeof(float), T * 3 * sizeof(uint32_t), T * sizeof(uint32_t),
                                  T * sizeof(uint32_t), T * sizeof(uint4), E * sizeof(uint32_t),
                                  E * sizeof(uint32_t), T, 8 * sizeof(float)};
        for (int i = 0; i < 12; i++) {
            offsets[i] = total;
            total += align256(std::max<size_t>(sizes[i], 64));
        }
        // Freed (after the stream drains) if the build fails part way.
        std::unique_ptr<lr_gpu_scene, void (*)(lr_gpu_scene *)> gs(new lr_gpu_scene(), lr_gpu_scene_destroy);
        gs->ctx = ctx;
        LR_CUDA(cudaMalloc(&gs->allocation, total));
        gs->bytes = total;
        char *base = (char *)gs->allocation;
        cudaStream_t stream = ctx->stream;
        LR_CUDA(cudaMemsetAsync(base, 0, total, stream));
        DeviceScene &s = gs->scene;
        float4 *widened = (float4 *)(base + offsets[0]), *exact = (float4 *)(base + offsets[1]);
        float *positions = (float *)(base + offsets[3]);
        uint32_t *indices = (uint32_t *)(base + offsets[4]), *faces = (uint32_t *)(base + offsets[5]);
        uint32_t *ids = (uint32_t *)(base + offsets[6]);
        uint4 *shading = (uint4 *)(base + offsets[7]);
        s.bvh.entries = widened;
        s.ref_bvh.entries = exact;
        s.tris = (const float4 *)(base + offsets[2]);
        s.positions = positions;
        s.indices = indices;
        s.faces = faces;
        s.ids = ids;
        s.shading = shading;
        s.wide4 = DeviceWide{nullptr, 0, 0};
        s.wide8 = DeviceWide{nullptr, 0, 0};
        gs->parents = (uint32_t *)(base + offsets[8]);
        gs->counters = (uint32_t *)(base + offsets[9]);
        gs->flat = (uint8_t *)(base + offsets[10]);
        gs->root_box = (float *)(base + offsets[11]);
        gs->device_built = true;
        gs->any_flat = std::any_of(scene->flat.begin(), scene->flat.end(), [](uint8_t f) { return f != 0; });
        s.triangle_count = T;
        s.point_count = P;
        s.entry_count = E;
        if (P) LR_CUDA(cudaMemcpyAsync(positions, scene->positions.data(), P * 3 * sizeof(float), cudaMemcpyHostToDevice, stream));
        if (T == 0) {
            LR_CUDA(cudaStreamSynchronize(stream));
            *out = gs.release();  // every ray misses: the default root box is inverted and empty is set
            return;
        }
        // Scratch: the compiled scene's triangles in their own order, the sort's two code
        // and index arrays, its per-tile digit counts and digit totals, the sorted keys,
        // the leaves' parents, and the bounds and the depth.
        const uint64_t tiles = (T + kSortTile - 1) / kSortTile;
        size_t so[12], scratch_total = 0;
        const size_t ss[12] = {T * 3 * sizeof(uint32_t), T * sizeof(uint32_t), T * sizeof(uint4), T,
                               T * sizeof(uint32_t), 4 * T * sizeof(uint32_t), tiles * kRadix * sizeof(uint32_t),
                               T * sizeof(uint64_t), T * sizeof(uint32_t), 8 * sizeof(uint32_t),
                               kRadix * sizeof(uint32_t), 64};
        for (int i = 0; i < 12; i++) {
            so[i] = scratch_total;
            scratch_total += align256(std::max<size_t>(ss[i], 64));
        }
        Scratch scratch;
        LR_CUDA(cudaMalloc(&scratch.p, scratch_total));
        char *sb = (char *)scratch.p;
        uint32_t *indices_in = (uint32_t *)(sb + so[0]), *faces_in = (uint32_t *)(sb + so[1]);
        uint4 *shading_in = (uint4 *)(sb + so[2]);
        uint8_t *flat_in = (uint8_t *)(sb + so[3]);
        uint32_t *ids_in = (uint32_t *)(sb + so[4]);
        uint32_t *codes[2] = {(uint32_t *)(sb + so[5]), (uint32_t *)(sb + so[5]) + T};
        uint32_t *values[2] = {(uint32_t *)(sb + so[5]) + 2 * T, (uint32_t *)(sb + so[5]) + 3 * T};
        uint32_t *counts = (uint32_t *)(sb + so[6]), *totals = (uint32_t *)(sb + so[10]);
        uint64_t *sorted = (uint64_t *)(sb + so[7]);
        uint32_t *leaf_parents = (uint32_t *)(sb + so[8]), *words = (uint32_t *)(sb + so[9]);
        LR_CUDA(cudaMemcpyAsync(indices_in, scene->indices.data(), T * 3 * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
        LR_CUDA(cudaMemcpyAsync(faces_in, scene->faces.data(), T * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
        LR_CUDA(cudaMemcpyAsync(shading_in, scene->shading.data(), T * sizeof(uint4), cudaMemcpyHostToDevice, stream));
        LR_CUDA(cudaMemcpyAsync(flat_in, scene->flat.data(), T, cudaMemcpyHostToDevice, stream));
        LR_CUDA(cudaMemcpyAsync(ids_in, scene->order.data(), T * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
        // words[0..2]: ordered +inf (the minima start there), [3..5]: ordered -inf, [6]: depth.
        const uint32_t init[8] = {0xff800000u, 0xff800000u, 0xff800000u, 0x007fffffu, 0x007fffffu, 0x007fffffu, 0u, 0u};
        LR_CUDA(cudaMemcpyAsync(words, init, sizeof init, cudaMemcpyHostToDevice, stream));
        // Every leaf gets its parent from the hierarchy; zeros keep a walk in bounds regardless.
        LR_CUDA(cudaMemsetAsync(leaf_parents, 0, T * sizeof(uint32_t), stream));
        const int sms = ctx->sm_count;
        bounds_kernel<<<grid_of(T, sms), 256, 0, stream>>>(T, positions, indices_in, words);
        keys_kernel<<<grid_of(T, sms), 256, 0, stream>>>(T, positions, indices_in, words, codes[0]);
        LR_CUDA(cudaGetLastError());
        if (tiles > 0xffffffffull) fail(LR_LIMIT, "too many triangles to sort on the device");
        for (int pass = 0; pass < 4; pass++) {
            const int in = pass & 1, out = in ^ 1, shift = 8 * pass;
            digit_counts_kernel<<<(unsigned)tiles, kSortThreads, 0, stream>>>(T, codes[in], shift, counts);
            row_scan_kernel<<<kRadix, kSortThreads, 0, stream>>>((uint32_t)tiles, counts, totals);
            scatter_kernel<<<(unsigned)tiles, kSortThreads, 0, stream>>>(
                T, codes[in], pass == 0 ? nullptr : values[in], shift, counts, totals, codes[out], values[out],
                pass == 3 ? sorted : nullptr);
        }
        LR_CUDA(cudaGetLastError());
        gather_kernel<<<grid_of(T, sms), 256, 0, stream>>>(T, sorted, indices_in, faces_in, shading_in, flat_in, ids_in,
                                                           indices, faces, shading, gs->flat, ids);
        LR_CUDA(cudaGetLastError());
        uint32_t depth = 0;
        if (E > 0) {
            hierarchy_kernel<<<(unsigned)((E + 127) / 128), 128, 0, stream>>>((int64_t)T, sorted, exact, widened,
                                                                               gs->parents, leaf_parents);
            depth_kernel<<<grid_of(T, sms), 256, 0, stream>>>(T, leaf_parents, gs->parents, 128u, words + 6);
            LR_CUDA(cudaGetLastError());
            LR_CUDA(cudaMemcpyAsync(&depth, words + 6, sizeof depth, cudaMemcpyDeviceToHost, stream));
        }
        LR_CUDA(cudaStreamSynchronize(stream));
        if (depth + 2 > 96) fail(LR_LIMIT, "the device-built BVH is deeper than 94 levels");
        s.depth = depth;
        const int root = E > 0 ? 0 : -1;  // one triangle: the root is the leaf of slot 0
        s.bvh.root = s.ref_bvh.root = root;
        s.bvh.empty = s.ref_bvh.empty = 0;
        refit_scene(gs.get(), stream);
        gs->refits = 0;
        *out = gs.release();
    });
}

}  // extern "C"
