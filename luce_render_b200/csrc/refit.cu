// Refitting an uploaded scene on the device after its points move (the triangles, their
// leaf order and the BVH topology kept): a deforming mesh, or points a simulation writes
// straight into device memory, traced again without a host rebuild or a re-upload.
//
// The reference rebuilds its BVH2 on the host for every geometry change (bvh.lucb:66-82,
// called from compile_scene); this keeps the reference's tree and recomputes its boxes:
//   1. every leaf slot's triangle record (3 float4) from the moved points, and the flat
//      shading normal of triangles that had no authored normals;
//   2. the BVH2's exact boxes bottom-up in one launch: a thread per interior entry writes
//      its leaf children's boxes, then climbs -- at each entry the second child to finish
//      (an atomic count of finished children) unions both boxes into its parent's slot, the
//      first stops -- so every box is written once, after both of its children, with no
//      thread waiting on another;
//   3. the watertight path's widened boxes from the exact ones, with the widening taken
//      again from the new root box (2^-16 of the scene's scale, one more float step);
//   4. the 4-wide collapse's child boxes, copied from the BVH2 slots they came from, and the
//      compressed 8-wide nodes quantized again from those boxes (quantize.hpp).
// With the points unchanged a refit leaves every array bit for bit as the upload made it,
// and the boxes equal the host refit (lr_scene_move_points) of the same move exactly: boxes
// are minima and maxima of the same floats, and the widening is the same float arithmetic.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "device.hpp"
#include "quantize.hpp"

namespace lr {
namespace {

struct Box {
    float lo[3], hi[3];
};

// Entry e's child `side` box in the traversal layout: side 0 in float4 0 (x, y) and the
// first half of float4 2 (z); side 1 in float4 1 and the second half of float4 2. Reads and
// writes go through L2 (other threads' boxes are read after an atomic, never from L1).
__device__ __forceinline__ Box read_side(const float4 *entries, uint32_t e, uint32_t side) {
    const float4 xy = __ldcg(&entries[(size_t)e * 4 + side]);
    const float2 z = __ldcg(reinterpret_cast<const float2 *>(&entries[(size_t)e * 4 + 2]) + side);
    return Box{{xy.x, xy.z, z.x}, {xy.y, xy.w, z.y}};
}

__device__ __forceinline__ void write_side(float4 *entries, uint32_t e, uint32_t side, const Box &b) {
    __stcg(&entries[(size_t)e * 4 + side], make_float4(b.lo[0], b.hi[0], b.lo[1], b.hi[1]));
    __stcg(reinterpret_cast<float2 *>(&entries[(size_t)e * 4 + 2]) + side, make_float2(b.lo[2], b.hi[2]));
}

// A leaf's box from its triangles' corners: 12 bytes of indices a triangle and the points
// (which stay in L2), not the 48-byte triangle records.
__device__ __forceinline__ Box leaf_box(const float *positions, const uint32_t *indices, int link) {
    const uint32_t code = (uint32_t)(-1 - link);
    const uint32_t first = code >> kLeafShift, count = (code & ((1u << kLeafShift) - 1u)) + 1u;
    Box b{{INFINITY, INFINITY, INFINITY}, {-INFINITY, -INFINITY, -INFINITY}};
    for (uint32_t t = first; t < first + count; t++)
        for (uint32_t c = 0; c < 3; c++) {
            const float *v = &positions[(size_t)__ldg(&indices[(size_t)t * 3 + c]) * 3];
            const float x = __ldg(v), y = __ldg(v + 1), z = __ldg(v + 2);
            b.lo[0] = fminf(b.lo[0], x);
            b.lo[1] = fminf(b.lo[1], y);
            b.lo[2] = fminf(b.lo[2], z);
            b.hi[0] = fmaxf(b.hi[0], x);
            b.hi[1] = fmaxf(b.hi[1], y);
            b.hi[2] = fmaxf(b.hi[2], z);
        }
    return b;
}

__device__ __forceinline__ Box join(const Box &a, const Box &b) {
    return Box{{fminf(a.lo[0], b.lo[0]), fminf(a.lo[1], b.lo[1]), fminf(a.lo[2], b.lo[2])},
               {fmaxf(a.hi[0], b.hi[0]), fmaxf(a.hi[1], b.hi[1]), fmaxf(a.hi[2], b.hi[2])}};
}

// The host's widen_down / widen_up (device.cu): `delta` outward, then one more float step.
__device__ __forceinline__ float widen_lo(float v, float delta) { return nextafterf(v - delta, -INFINITY); }
__device__ __forceinline__ float widen_hi(float v, float delta) { return nextafterf(v + delta, INFINITY); }

// The first corner's w holds the source triangle id (the upload's layout), taken from the
// 4-byte ids rather than by reading the old record back.
__global__ void tris_kernel(uint64_t count, const float *positions, const uint32_t *indices, const uint32_t *ids,
                            float4 *tris) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < count * 3; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t point = indices[i];
        const uint64_t t = i / 3;
        const float w = i - t * 3 == 0 ? __uint_as_float(ids[t]) : 0.0f;
        tris[i] = make_float4(positions[(size_t)point * 3], positions[(size_t)point * 3 + 1],
                              positions[(size_t)point * 3 + 2], w);
    }
}

// octahedral (scene.cpp, scene.lucb:400-412) of (b - a) x (c - a), in f64 with every
// operation rounded as the host's (no fused multiply-adds), so the codes are the host's.
__device__ uint32_t flat_code(const float *pa, const float *pb, const float *pc) {
    const double e1[3] = {__dsub_rn(pb[0], pa[0]), __dsub_rn(pb[1], pa[1]), __dsub_rn(pb[2], pa[2])};
    const double e2[3] = {__dsub_rn(pc[0], pa[0]), __dsub_rn(pc[1], pa[1]), __dsub_rn(pc[2], pa[2])};
    const double n[3] = {__dsub_rn(__dmul_rn(e1[1], e2[2]), __dmul_rn(e1[2], e2[1])),
                         __dsub_rn(__dmul_rn(e1[2], e2[0]), __dmul_rn(e1[0], e2[2])),
                         __dsub_rn(__dmul_rn(e1[0], e2[1]), __dmul_rn(e1[1], e2[0]))};
    const double length = __dadd_rn(__dadd_rn(fabs(n[0]), fabs(n[1])), fabs(n[2]));
    double x = 0.0, y = 1.0;  // a degenerate triangle's normal: +Y (octahedral of (0, 1, 0))
    if (length > 0.0) {
        x = __ddiv_rn(n[0], length);
        y = __ddiv_rn(n[1], length);
        if (n[2] < 0.0) {
            const double fx = __dmul_rn(__dsub_rn(1.0, fabs(y)), x >= 0.0 ? 1.0 : -1.0);
            const double fy = __dmul_rn(__dsub_rn(1.0, fabs(x)), y >= 0.0 ? 1.0 : -1.0);
            x = fx;
            y = fy;
        }
    }
    const long long qx = (long long)round(__dmul_rn(fmin(fmax(x, -1.0), 1.0), 32767.0));
    const long long qy = (long long)round(__dmul_rn(fmin(fmax(y, -1.0), 1.0), 32767.0));
    return (uint32_t)(qx & 0xffff) | ((uint32_t)(qy & 0xffff) << 16);
}

__global__ void flat_kernel(uint64_t count, const float *positions, const uint32_t *indices, const uint8_t *flat,
                            uint4 *shading) {
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < count; t += (uint64_t)gridDim.x * blockDim.x) {
        if (!flat[t]) continue;
        const uint32_t code = flat_code(&positions[(size_t)indices[t * 3] * 3], &positions[(size_t)indices[t * 3 + 1] * 3],
                                        &positions[(size_t)indices[t * 3 + 2] * 3]);
        const uint4 s = shading[t];
        shading[t] = make_uint4(code, code, code, s.w);
    }
}

// An atomic add with release and acquire semantics at device scope: the box stores before
// it are visible to the thread whose add comes after, and that thread's loads after its add
// see them (one atom.acq_rel in place of a full __threadfence on each side).
__device__ __forceinline__ uint32_t add_acq_rel(uint32_t *counter, uint32_t value) {
    uint32_t old;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(counter), "r"(value) : "memory");
    return old;
}

// Step 2. `levels` bounds a climb (the BVH2's depth + 1), so a damaged parent table can
// only end a climb early, never loop. The next parent link is fetched before the atomic
// (the table is read-only), so it is not on the climb's chain of dependent latencies.
__global__ void climb_kernel(uint32_t entries, const float *positions, const uint32_t *indices, float4 *exact,
                             const uint32_t *parents, uint32_t *counters, float *root_box, uint32_t levels) {
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= entries) return;
    const float4 links = exact[(size_t)e * 4 + 3];
    const int link[2] = {__float_as_int(links.x), __float_as_int(links.y)};
    uint32_t leaves = 0;
    for (uint32_t side = 0; side < 2; side++)
        if (link[side] < 0) {
            write_side(exact, e, side, leaf_box(positions, indices, link[side]));
            leaves++;
        }
    if (leaves == 0) return;
    uint32_t up = __ldg(&parents[e]);
    if (add_acq_rel(&counters[e], leaves) + leaves != 2u) return;
    uint32_t at = e;
    for (uint32_t level = 0; level < levels; level++) {
        const Box box = join(read_side(exact, at, 0), read_side(exact, at, 1));
        if (up == 0xffffffffu) {
            for (int k = 0; k < 3; k++) {
                __stcg(&root_box[k], box.lo[k]);
                __stcg(&root_box[4 + k], box.hi[k]);
            }
            return;
        }
        const uint32_t parent = up >> 1;
        const uint32_t next = __ldg(&parents[parent]);
        write_side(exact, parent, up & 1u, box);
        if (add_acq_rel(&counters[parent], 1u) == 0u) return;  // the sibling is still on its way
        at = parent;
        up = next;
    }
}

// A scene whose root is a leaf (at most 16 triangles): its box.
__global__ void leaf_root_kernel(const float *positions, const uint32_t *indices, int root, float *root_box) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const Box b = leaf_box(positions, indices, root);
    for (int k = 0; k < 3; k++) {
        root_box[k] = b.lo[k];
        root_box[4 + k] = b.hi[k];
    }
}

// Step 3: the float4s 0..2 of every entry hold (lo, hi, lo, hi) pairs.
__global__ void widen_kernel(uint64_t count, const float4 *exact, float4 *widened, float delta) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < count; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t e = i / 3, k = i % 3;
        const float4 v = exact[e * 4 + k];
        widened[e * 4 + k] = make_float4(widen_lo(v.x, delta), widen_hi(v.y, delta), widen_lo(v.z, delta),
                                         widen_hi(v.w, delta));
    }
}

// Step 4: 4-wide node n's child slot i from the BVH2 slot (or the root) it was collapsed
// from; empty slots keep their inverted boxes.
__global__ void wide_kernel(uint64_t slots, int width, const uint32_t *sources, const float4 *exact,
                            const float *root_box, float delta, float4 *nodes) {
    const int per_node = 7, planes = width / 4;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < slots; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t source = sources[i];
        if (source == 0xffffffffu) continue;
        Box b;
        if (source == kRefitRoot) {
            for (int k = 0; k < 3; k++) {
                b.lo[k] = root_box[k];
                b.hi[k] = root_box[4 + k];
            }
        } else {
            b = read_side(exact, source >> 1, source & 1u);
        }
        const uint64_t n = i / width;
        const int slot = (int)(i % width);
        float *base = reinterpret_cast<float *>(nodes + n * per_node);
        for (int k = 0; k < 3; k++) {
            base[((2 * k) * planes) * 4 + slot] = widen_lo(b.lo[k], delta);
            base[((2 * k + 1) * planes) * 4 + slot] = widen_hi(b.hi[k], delta);
        }
    }
}

// Step 4 for the compressed 8-wide tree: node n quantized again (quantize.hpp) from its
// children's BVH2 boxes (or the root's), widened as at upload; its links and occupied
// slots stay.
__global__ void quantize_kernel(uint64_t count, const uint32_t *sources, const float4 *exact, const float *root_box,
                                float delta, float4 *nodes) {
    for (uint64_t n = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; n < count; n += (uint64_t)gridDim.x * blockDim.x) {
        float *node = reinterpret_cast<float *>(nodes + n * kQNodeFloat4s);
        const uint32_t occupied = __float_as_uint(node[3]) >> 24;
        float lo[8][3], hi[8][3];
        int links[8];
        for (int c = 0; c < 8; c++) {
            links[c] = __float_as_int(node[4 + c]);
            if (!((occupied >> c) & 1u)) continue;
            const uint32_t source = sources[n * 8 + c];
            Box b;
            if (source == kRefitRoot) {
                for (int k = 0; k < 3; k++) {
                    b.lo[k] = root_box[k];
                    b.hi[k] = root_box[4 + k];
                }
            } else {
                b = read_side(exact, source >> 1, source & 1u);
            }
            for (int k = 0; k < 3; k++) {
                lo[c][k] = widen_lo(b.lo[k], delta);
                hi[c][k] = widen_hi(b.hi[k], delta);
            }
        }
        float out[kQNodeFloat4s * 4];
        quantize_node(occupied, lo, hi, links, out);
        for (int k = 0; k < kQNodeFloat4s * 4; k++) node[k] = out[k];
    }
}

unsigned grid_for(uint64_t items, int sm_count) {
    const uint64_t blocks = (items + 255) / 256;
    return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(blocks, (uint64_t)sm_count * 8));
}

float host_widen_down(float v, float delta) { return std::nextafter(v - delta, -INFINITY); }
float host_widen_up(float v, float delta) { return std::nextafter(v + delta, INFINITY); }

}  // namespace

uint64_t topology_hash(const Scene &scene) {
    uint64_t key = 14695981039346656037ull;
    auto mix = [&](const void *data, size_t bytes) {
        const unsigned char *p = (const unsigned char *)data;
        for (size_t i = 0; i < bytes; i++) key = (key ^ p[i]) * 1099511628211ull;
    };
    const uint64_t counts[2] = {scene.point_count(), scene.triangle_count()};
    mix(counts, sizeof counts);
    mix(scene.indices.data(), scene.indices.size() * sizeof(uint32_t));
    return key;
}

void refit_scene(lr_gpu_scene *gs, cudaStream_t stream) {
    DeviceScene &s = gs->scene;
    const uint64_t T = s.triangle_count;
    if (T == 0) return;
    const int sms = gs->ctx->sm_count;
    float4 *tris = const_cast<float4 *>(s.tris);
    float4 *exact = const_cast<float4 *>(s.ref_bvh.entries);
    float4 *widened = const_cast<float4 *>(s.bvh.entries);
    tris_kernel<<<grid_for(T * 3, sms), 256, 0, stream>>>(T, s.positions, s.indices, s.ids, tris);
    if (gs->any_flat)
        flat_kernel<<<grid_for(T, sms), 256, 0, stream>>>(T, s.positions, s.indices, gs->flat,
                                                         const_cast<uint4 *>(s.shading));
    const uint64_t E = s.entry_count;
    if (E > 0) {
        LR_CUDA(cudaMemsetAsync(gs->counters, 0, E * sizeof(uint32_t), stream));
        climb_kernel<<<(unsigned)((E + 127) / 128), 128, 0, stream>>>((uint32_t)E, s.positions, s.indices, exact,
                                                                       gs->parents, gs->counters, gs->root_box,
                                                                       s.depth + 2);
    } else {
        leaf_root_kernel<<<1, 32, 0, stream>>>(s.positions, s.indices, s.bvh.root, gs->root_box);
    }
    LR_CUDA(cudaGetLastError());
    float root[8];
    LR_CUDA(cudaMemcpyAsync(root, gs->root_box, sizeof root, cudaMemcpyDeviceToHost, stream));
    LR_CUDA(cudaStreamSynchronize(stream));
    // The widening as the upload takes it (device.cu's build_layout), from the new root box.
    double scale = 1.0;
    for (int k = 0; k < 3; k++) {
        scale = std::max(scale, (double)std::fabs(root[k]));
        scale = std::max(scale, (double)std::fabs(root[4 + k]));
        scale = std::max(scale, (double)(root[4 + k] - root[k]));
    }
    const float delta = (float)std::ldexp(scale, -16);
    for (int k = 0; k < 3; k++) {
        s.ref_bvh.root_lo[k] = root[k];
        s.ref_bvh.root_hi[k] = root[4 + k];
        s.bvh.root_lo[k] = host_widen_down(root[k], delta);
        s.bvh.root_hi[k] = host_widen_up(root[4 + k], delta);
    }
    if (E > 0) widen_kernel<<<grid_for(E * 3, sms), 256, 0, stream>>>(E * 3, exact, widened, delta);
    if (s.wide4.width)
        wide_kernel<<<grid_for(gs->wide4_nodes * 4, sms), 256, 0, stream>>>(
            gs->wide4_nodes * 4, 4, gs->wide4_sources, exact, gs->root_box, delta, const_cast<float4 *>(s.wide4.nodes));
    if (s.wide8.width)
        quantize_kernel<<<grid_for(gs->wide8_nodes, sms), 256, 0, stream>>>(
            gs->wide8_nodes, gs->wide8_sources, exact, gs->root_box, delta, const_cast<float4 *>(s.wide8.nodes));
    LR_CUDA(cudaGetLastError());
    LR_CUDA(cudaStreamSynchronize(stream));
    gs->refits++;
}

}  // namespace lr

using namespace lr;

extern "C" {

int lr_gpu_scene_refit(lr_context *ctx, lr_gpu_scene *gs, const void *positions, uint64_t point_count, uint32_t flags) {
    return guarded([&] {
        if (!ctx || !gs || (point_count && !positions)) fail(LR_INVALID, "a refit needs a context, a scene and its points");
        if (ctx->device != gs->ctx->device) fail(LR_INVALID, "a refit runs on the scene's device");
        if (flags & ~LR_REFIT_DEVICE) fail(LR_INVALID, "unknown refit flags");
        if (point_count != gs->scene.point_count) fail(LR_INVALID, "a refit keeps the scene's point count");
        LR_CUDA(cudaSetDevice(ctx->device));
        float *dst = const_cast<float *>(gs->scene.positions);
        const size_t bytes = point_count * 3 * sizeof(float);
        // The copy's direction follows the pointer (unified addressing), so a pointer given
        // with the wrong flag is still copied from where it lives rather than misread.
        if (bytes && dst != positions) LR_CUDA(cudaMemcpyAsync(dst, positions, bytes, cudaMemcpyDefault, ctx->stream));
        refit_scene(gs, ctx->stream);
    });
}

}  // extern "C"
