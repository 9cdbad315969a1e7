// The context, the scene in HBM (GpuScene.upload, src/render/device.lucb:41-89), the
// primary-ray probe (device.lucb:138-160, shaders/probe.comp) and ray-list queries.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "device.hpp"
#include "traverse.cuh"
#include "wide.hpp"

namespace lr {

thread_local std::string g_last_error;
void set_last_error(const char *message) { g_last_error = message; }

namespace {

constexpr int kBlock = 128;
// Where the ray queries' batch cursor sits among a context's status words (in ints).
constexpr int kBatchCursor = 8;

struct ProbeFrame {
    float b[16];
};

__device__ __forceinline__ void note_overflow(int *status, bool overflow) {
    if (overflow) atomicAdd(status, 1);
}

// probe.comp:21-34: one pixel-centre ray per pixel, row-major from the top.
template <bool kRef, int kStack>
__global__ void __launch_bounds__(kBlock) probe_kernel(DeviceScene s, ProbeFrame f, uint32_t *faces, float *ts,
                                                      int *status) {
    __shared__ int stack[kStack * kBlock];
    const uint32_t width = (uint32_t)f.b[11], height = (uint32_t)f.b[15];
    const uint64_t pixel = (uint64_t)blockIdx.x * kBlock + threadIdx.x;
    if (pixel >= (uint64_t)width * height) return;
    const uint32_t x = (uint32_t)(pixel % width), y = (uint32_t)(pixel / width);
    const float fx = fadd_((float)x, 0.5f), fy = fadd_((float)y, 0.5f);
    float film[3], o[3], d[3];
    const bool ortho = f.b[3] > 0.5f;
    for (int k = 0; k < 3; k++) film[k] = fadd_(fadd_(f.b[4 + k], fmul_(fx, f.b[8 + k])), fmul_(fy, f.b[12 + k]));
    float fw[3] = {fsub_(fmul_(f.b[9], f.b[14]), fmul_(f.b[10], f.b[13])),
                   fsub_(fmul_(f.b[10], f.b[12]), fmul_(f.b[8], f.b[14])),
                   fsub_(fmul_(f.b[8], f.b[13]), fmul_(f.b[9], f.b[12]))};
    const float fl = __fsqrt_rn(fadd_(fadd_(fmul_(fw[0], fw[0]), fmul_(fw[1], fw[1])), fmul_(fw[2], fw[2])));
    for (int k = 0; k < 3; k++) {
        o[k] = ortho ? fadd_(f.b[k], film[k]) : f.b[k];
        d[k] = ortho ? __fdiv_rn(fw[k], fl) : film[k];
    }
    Ray r{make_float3(o[0], o[1], o[2]), 0.0f, make_float3(d[0], d[1], d[2]), kNoHitT};
    bool overflow = false;
    Visits visits;
    Hit h = kRef ? trace_reference<false, kStack>(s, r, stack + threadIdx.x, kBlock, overflow, visits)
                 : trace_exact<false, kStack>(s, r, stack + threadIdx.x, kBlock, overflow, visits);
    note_overflow(status, overflow);
    faces[pixel] = h.slot >= 0 ? __ldg(&s.faces[h.slot]) : 0xffffffffu;
    ts[pixel] = h.t;
}

// A list of rays (two float4 each) to hits (t, source id bits, u, v). With kCount the
// traversal's interior visits and triangle tests add into counts[0..1].
template <bool kRef, bool kAny, int kStack, bool kCount>
__global__ void __launch_bounds__(kBlock) trace_kernel(DeviceScene s, const float4 *__restrict__ rays, uint64_t n,
                                                      float4 *__restrict__ hits, int *status,
                                                      unsigned long long *counts) {
    __shared__ int stack[kStack * kBlock];
    const uint64_t i = (uint64_t)blockIdx.x * kBlock + threadIdx.x;
    Visits visits;
    if (i < n) {
        const float4 a = __ldg(&rays[2 * i]), b = __ldg(&rays[2 * i + 1]);
        Ray r{make_float3(a.x, a.y, a.z), a.w, make_float3(b.x, b.y, b.z), b.w};
        bool overflow = false;
        Hit h = kRef ? trace_reference<kAny, kStack, kCount>(s, r, stack + threadIdx.x, kBlock, overflow, visits)
                     : trace_exact<kAny, kStack, kCount>(s, r, stack + threadIdx.x, kBlock, overflow, visits);
        note_overflow(status, overflow);
        hits[i] = make_float4(h.t, __int_as_float(h.id), h.u, h.v);
    }
    if (kCount) add_visits(counts, visits);
}

// The watertight path over a ray list: a grid sized to the GPU's resident blocks, each
// warp taking the next 32 consecutive rays (`next`, zeroed before the launch) as it
// finishes the last.
template <int W, bool kAny, int kStack, bool kCount>
__global__ void __launch_bounds__(kBlock) trace_resident_kernel(DeviceScene s, const float4 *__restrict__ rays,
                                                               uint32_t n, float4 *__restrict__ hits, int *status,
                                                               unsigned long long *counts, uint32_t *next) {
    __shared__ int stack[TracerOf<W, kAny, kStack, kCount>::kInts * kBlock];
    bool overflow = false;
    Visits visits;
    auto load = [&](uint32_t i) {
        const float4 a = __ldg(&rays[2 * i]), b = __ldg(&rays[2 * i + 1]);
        return Ray{make_float3(a.x, a.y, a.z), a.w, make_float3(b.x, b.y, b.z), b.w};
    };
    auto store = [&](uint32_t i, const Hit &h, const Ray &) {
        hits[i] = make_float4(h.t, __int_as_float(h.id), h.u, h.v);
    };
    trace_batched<W, kAny, kStack, kCount>(s, n, next, stack + threadIdx.x, kBlock, load, store, overflow, visits);
    note_overflow(status, overflow);
    if (kCount) add_visits(counts, visits);
}

// Does nothing (the sink is never written): launch-overhead measurements.
__global__ void idle_kernel(int *sink) {
    if (sink && threadIdx.x == 1023u) *sink = 0;
}

int stack_for(uint32_t depth) {
    if (depth + 2 <= 32) return 32;
    if (depth + 2 <= 64) return 64;
    if (depth + 2 <= 96) return 96;
    fail(LR_LIMIT, "the BVH is deeper than 94 levels");
}

}  // namespace

// The width the watertight path uses when the caller names none: the BVH2, which on
// sm_100a traces incoherent rays faster than the 4- and 8-wide collapses (1.96 against
// 1.49 Grays/s on the 1M-triangle scene). A wide request falls back to 4, then to the
// BVH2, when the scene's stack bound does not fit. The environment variable
// LUCE_RENDER_B200_BVH_WIDTH (2, 4 or 8) overrides the default, for tuning.
TraversalChoice choose_traversal(const DeviceScene &s, int requested) {
    if (requested == 0) {
        requested = 2;
        if (const char *env = std::getenv("LUCE_RENDER_B200_BVH_WIDTH")) {
            const int w = std::atoi(env);
            if (w == 2 || w == 4 || w == 8) requested = w;
        }
    }
    auto wide_stack = [](uint32_t bound) { return bound + 1 <= 32 ? 32 : (bound + 1 <= 48 ? 48 : 0); };
    // The compressed 8-wide tree's stack holds one group a level, a node index under 2^24
    // beside its child ranks in one word.
    auto group_stack = [](uint32_t bound) { return bound <= 16 ? 16 : (bound <= 32 ? 32 : 0); };
    // A scene built on the device has no wide collapses (null nodes).
    if (requested == 8 && s.wide8.nodes && s.wide8.node_count < (1ull << 24) && group_stack(s.wide8.max_stack))
        return {8, group_stack(s.wide8.max_stack)};
    if (requested >= 4 && s.wide4.nodes && wide_stack(s.wide4.max_stack)) return {4, wide_stack(s.wide4.max_stack)};
    return {2, stack_for(s.depth)};
}

namespace {

template <int W, bool kAny, int kStack, bool kCount>
void launch_resident(const lr_gpu_scene *gs, const float4 *rays, uint64_t n, float4 *hits, int *status,
                     unsigned long long *counts, cudaStream_t stream) {
    static int resident = 0;
    if (!resident) {
        int per_sm = 0, device = 0, sms = 0;
        LR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, trace_resident_kernel<W, kAny, kStack, kCount>,
                                                              kBlock, 0));
        LR_CUDA(cudaGetDevice(&device));
        LR_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
        resident = std::max(1, per_sm) * sms;
    }
    const uint64_t needed = (n + kBlock - 1) / kBlock;
    const unsigned grid = (unsigned)std::min<uint64_t>(needed, (uint64_t)resident);
    uint32_t *next = (uint32_t *)(status + kBatchCursor);
    LR_CUDA(cudaMemsetAsync(next, 0, sizeof(uint32_t), stream));
    trace_resident_kernel<W, kAny, kStack, kCount><<<grid, kBlock, 0, stream>>>(gs->scene, rays, (uint32_t)n, hits,
                                                                               status, counts, next);
}

template <bool kAny, bool kCount>
void dispatch_exact(const lr_gpu_scene *gs, const float4 *rays, uint64_t n, float4 *hits, int *status,
                    unsigned long long *counts, cudaStream_t stream, int requested_width) {
    if (n > 0xffffffffull) fail(LR_LIMIT, "a ray query holds at most 2^32 - 1 rays");
    const TraversalChoice c = choose_traversal(gs->scene, requested_width);
    switch (c.width * 1000 + c.stack) {
        case 8016: launch_resident<8, kAny, 16, kCount>(gs, rays, n, hits, status, counts, stream); break;
        case 8032: launch_resident<8, kAny, 32, kCount>(gs, rays, n, hits, status, counts, stream); break;
        case 4032: launch_resident<4, kAny, 32, kCount>(gs, rays, n, hits, status, counts, stream); break;
        case 4048: launch_resident<4, kAny, 48, kCount>(gs, rays, n, hits, status, counts, stream); break;
        case 2032: launch_resident<2, kAny, 32, kCount>(gs, rays, n, hits, status, counts, stream); break;
        case 2064: launch_resident<2, kAny, 64, kCount>(gs, rays, n, hits, status, counts, stream); break;
        default: launch_resident<2, kAny, 96, kCount>(gs, rays, n, hits, status, counts, stream); break;
    }
}

template <bool kRef, int kStack>
void launch_probe(const lr_gpu_scene *gs, const ProbeFrame &f, uint64_t count, uint32_t *faces, float *ts,
                  int *status, cudaStream_t stream) {
    const unsigned grid = (unsigned)((count + kBlock - 1) / kBlock);
    probe_kernel<kRef, kStack><<<grid, kBlock, 0, stream>>>(gs->scene, f, faces, ts, status);
}

template <bool kAny, int kStack, bool kCount>
void launch_reference(const lr_gpu_scene *gs, const float4 *rays, uint64_t n, float4 *hits, int *status,
                      unsigned long long *counts, cudaStream_t stream) {
    const unsigned grid = (unsigned)((n + kBlock - 1) / kBlock);
    trace_kernel<true, kAny, kStack, kCount><<<grid, kBlock, 0, stream>>>(gs->scene, rays, n, hits, status, counts);
}

template <bool kAny, bool kCount>
void dispatch_reference(const lr_gpu_scene *gs, const float4 *rays, uint64_t n, float4 *hits, int *status,
                        unsigned long long *counts, cudaStream_t stream) {
    switch (stack_for(gs->scene.depth)) {
        case 32: launch_reference<kAny, 32, kCount>(gs, rays, n, hits, status, counts, stream); break;
        case 64: launch_reference<kAny, 64, kCount>(gs, rays, n, hits, status, counts, stream); break;
        default: launch_reference<kAny, 96, kCount>(gs, rays, n, hits, status, counts, stream); break;
    }
}

template <bool kRef>
void dispatch_probe(const lr_gpu_scene *gs, const ProbeFrame &f, uint64_t count, uint32_t *faces, float *ts,
                    int *status, cudaStream_t stream) {
    switch (stack_for(gs->scene.depth)) {
        case 32: launch_probe<kRef, 32>(gs, f, count, faces, ts, status, stream); break;
        case 64: launch_probe<kRef, 64>(gs, f, count, faces, ts, status, stream); break;
        default: launch_probe<kRef, 96>(gs, f, count, faces, ts, status, stream); break;
    }
}

float bits_as_float(int v) {
    float f;
    std::memcpy(&f, &v, sizeof f);
    return f;
}

// Rounds outward by `delta`, then one more float step.
float widen_down(float v, float delta) { return std::nextafter(v - delta, -INFINITY); }
float widen_up(float v, float delta) { return std::nextafter(v + delta, INFINITY); }

struct HostLayout {
    std::vector<float4> entries, ref_entries, tris;
    std::vector<uint4> shading;
    int root = 0;
    float root_lo[3], root_hi[3];
    float delta = 0.0f;
    // For refits: per interior entry its parent slot; per BVH2 node the slot holding its box.
    std::vector<uint32_t> parents, slot_of_node;
};

int leaf_link(const lr_bvh_node &n) {
    if (n.count == 0 || n.count > 16) fail(LR_INVALID, "a BVH leaf holds 1 to 16 triangles");
    if (n.first > kMaxLeafFirst) fail(LR_LIMIT, "a scene holds at most 2^27 triangles");
    return -1 - (int)((n.first << kLeafShift) | (n.count - 1));
}

void build_layout(const lr::Scene &scene, HostLayout &L) {
    const auto &nodes = scene.nodes;
    const size_t T = scene.triangle_count();
    // The widening that keeps the box test conservative for the watertight triangle
    // test: 2^-16 of the scene's coordinate scale (its largest magnitude or extent).
    double scale = 1.0;
    for (int k = 0; k < 3; k++) {
        scale = std::max(scale, (double)std::fabs(nodes[0].lo[k]));
        scale = std::max(scale, (double)std::fabs(nodes[0].hi[k]));
        scale = std::max(scale, (double)(nodes[0].hi[k] - nodes[0].lo[k]));
    }
    L.delta = T ? (float)std::ldexp(scale, -16) : 0.0f;
    std::vector<int> entry(nodes.size(), -1);
    int interior = 0;
    for (size_t n = 0; n < nodes.size(); n++)
        if (T && nodes[n].count == 0) entry[n] = interior++;
    auto link = [&](uint32_t c) { return nodes[c].count == 0 ? entry[c] : leaf_link(nodes[c]); };
    L.entries.resize((size_t)interior * 4);
    L.ref_entries.resize((size_t)interior * 4);
    L.parents.assign((size_t)interior, 0xffffffffu);
    L.slot_of_node.assign(nodes.size(), kRefitRoot);
    for (size_t n = 0; n < nodes.size(); n++) {
        if (entry[n] < 0) continue;
        for (uint32_t side = 0; side < 2; side++) {
            const uint32_t c = nodes[n].first + side;
            L.slot_of_node[c] = (uint32_t)entry[n] << 1 | side;
            if (entry[c] >= 0) L.parents[(size_t)entry[c]] = (uint32_t)entry[n] << 1 | side;
        }
        const lr_bvh_node &a = nodes[nodes[n].first], &b = nodes[nodes[n].first + 1];
        const float d = L.delta;
        float4 *e = &L.entries[(size_t)entry[n] * 4];
        e[0] = make_float4(widen_down(a.lo[0], d), widen_up(a.hi[0], d), widen_down(a.lo[1], d), widen_up(a.hi[1], d));
        e[1] = make_float4(widen_down(b.lo[0], d), widen_up(b.hi[0], d), widen_down(b.lo[1], d), widen_up(b.hi[1], d));
        e[2] = make_float4(widen_down(a.lo[2], d), widen_up(a.hi[2], d), widen_down(b.lo[2], d), widen_up(b.hi[2], d));
        float4 links = make_float4(bits_as_float(link(nodes[n].first)), bits_as_float(link(nodes[n].first + 1)), 0.0f, 0.0f);
        e[3] = links;
        float4 *r = &L.ref_entries[(size_t)entry[n] * 4];
        r[0] = make_float4(a.lo[0], a.hi[0], a.lo[1], a.hi[1]);
        r[1] = make_float4(b.lo[0], b.hi[0], b.lo[1], b.hi[1]);
        r[2] = make_float4(a.lo[2], a.hi[2], b.lo[2], b.hi[2]);
        r[3] = links;
    }
    for (int k = 0; k < 3; k++) {
        L.root_lo[k] = nodes[0].lo[k];
        L.root_hi[k] = nodes[0].hi[k];
    }
    L.root = T == 0 ? 0 : link(0);
    L.tris.resize(T * 3);
    const float *p = scene.positions.data();
    for (size_t t = 0; t < T; t++) {
        for (int c = 0; c < 3; c++) {
            const float *v = &p[(size_t)scene.indices[t * 3 + c] * 3];
            float w = c == 0 ? bits_as_float((int)scene.order[t]) : 0.0f;
            L.tris[t * 3 + c] = make_float4(v[0], v[1], v[2], w);
        }
    }
    L.shading.resize(T);
    for (size_t t = 0; t < T; t++)
        L.shading[t] = make_uint4(scene.shading[t * 4], scene.shading[t * 4 + 1], scene.shading[t * 4 + 2],
                                  scene.shading[t * 4 + 3]);
}

size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

}  // namespace

}  // namespace lr

using namespace lr;

namespace lr {
void check_status(lr_context *ctx) {
    int words[2] = {0, 0};
    LR_CUDA(cudaMemcpyAsync(words, ctx->status, sizeof words, cudaMemcpyDeviceToHost, ctx->stream));
    LR_CUDA(cudaStreamSynchronize(ctx->stream));
    if (words[0] || words[1]) {
        LR_CUDA(cudaMemsetAsync(ctx->status, 0, sizeof words, ctx->stream));
        LR_CUDA(cudaStreamSynchronize(ctx->stream));
        if (words[0]) fail(LR_LIMIT, "a traversal stack overflowed: " + std::to_string(words[0]) + " pushes lost");
        fail(LR_TIMEOUT, "a device-side bounded wait gave up " + std::to_string(words[1]) + " times");
    }
}
}  // namespace lr

extern "C" {

const char *lr_last_error(void) { return lr::g_last_error.c_str(); }
const char *lr_version(void) { return "luce_render_b200 0.1 (sm_100a)"; }

int lr_context_create(int device, lr_context **out) { return lr_context_create_ex(device, 0, out); }

int lr_context_create_ex(int device, int priority, lr_context **out) {
    return guarded([&] {
        if (!out) fail(LR_INVALID, "no place for the context");
        *out = nullptr;
        if (priority != 0 && priority != 1) fail(LR_INVALID, "a context's priority is 0 (normal) or 1 (high)");
        int count = 0;
        LR_CUDA(cudaGetDeviceCount(&count));
        if (device < 0 || device >= count) fail(LR_INVALID, "no such CUDA device");
        LR_CUDA(cudaSetDevice(device));
        auto ctx = std::make_unique<lr_context>();
        ctx->device = device;
        LR_CUDA(cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device));
        int least = 0, greatest = 0;
        LR_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        LR_CUDA(cudaStreamCreateWithPriority(&ctx->stream, cudaStreamNonBlocking, priority ? greatest : least));
        LR_CUDA(cudaEventCreate(&ctx->start));
        LR_CUDA(cudaEventCreate(&ctx->stop));
        // Status words at byte 0, traversal counts at byte 16, the ray queries' batch
        // cursor at byte 32 (kBatchCursor ints in).
        LR_CUDA(cudaMalloc(&ctx->status, 64));
        LR_CUDA(cudaMemsetAsync(ctx->status, 0, 64, ctx->stream));
        ctx->counts = (unsigned long long *)((char *)ctx->status + 16);
        LR_CUDA(cudaStreamSynchronize(ctx->stream));
        *out = ctx.release();
    });
}

void lr_context_destroy(lr_context *ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (ctx->status) cudaFree(ctx->status);
    if (ctx->start) cudaEventDestroy(ctx->start);
    if (ctx->stop) cudaEventDestroy(ctx->stop);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

int lr_context_synchronize(lr_context *ctx) {
    return guarded([&] {
        if (!ctx) fail(LR_INVALID, "no context");
        LR_CUDA(cudaStreamSynchronize(ctx->stream));
        check_status(ctx);
    });
}

void *lr_context_stream(lr_context *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

int lr_device_alloc(lr_context *ctx, size_t bytes, void **out) {
    return guarded([&] {
        if (!ctx || !out) fail(LR_INVALID, "no context");
        *out = nullptr;
        LR_CUDA(cudaSetDevice(ctx->device));
        LR_CUDA(cudaMalloc(out, bytes ? bytes : 16));
    });
}

int lr_device_free(lr_context *ctx, void *ptr) {
    return guarded([&] {
        if (!ctx) fail(LR_INVALID, "no context");
        if (ptr) {
            LR_CUDA(cudaStreamSynchronize(ctx->stream));
            LR_CUDA(cudaFree(ptr));
        }
    });
}

int lr_memcpy_htod(lr_context *ctx, void *dst, const void *src, size_t bytes) {
    return guarded([&] {
        if (!ctx) fail(LR_INVALID, "no context");
        LR_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream));
        LR_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}

int lr_memcpy_dtoh(lr_context *ctx, void *dst, const void *src, size_t bytes) {
    return guarded([&] {
        if (!ctx) fail(LR_INVALID, "no context");
        LR_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->stream));
        LR_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}

int lr_memset_device(lr_context *ctx, void *dst, int value, size_t bytes) {
    return guarded([&] {
        if (!ctx) fail(LR_INVALID, "no context");
        LR_CUDA(cudaMemsetAsync(dst, value, bytes, ctx->stream));
    });
}

int lr_host_alloc_pinned(size_t bytes, void **out) {
    return guarded([&] {
        if (!out) fail(LR_INVALID, "no place for the pointer");
        LR_CUDA(cudaMallocHost(out, bytes ? bytes : 16));
    });
}

int lr_host_free_pinned(void *ptr) {
    return guarded([&] {
        if (ptr) LR_CUDA(cudaFreeHost(ptr));
    });
}

int lr_timer_start(lr_context *ctx) {
    return guarded([&] {
        if (!ctx) fail(LR_INVALID, "no context");
        LR_CUDA(cudaEventRecord(ctx->start, ctx->stream));
    });
}

int lr_timer_stop(lr_context *ctx, float *ms) {
    return guarded([&] {
        if (!ctx || !ms) fail(LR_INVALID, "no context");
        LR_CUDA(cudaEventRecord(ctx->stop, ctx->stream));
        LR_CUDA(cudaEventSynchronize(ctx->stop));
        LR_CUDA(cudaEventElapsedTime(ms, ctx->start, ctx->stop));
    });
}

int lr_launch_overhead(lr_context *ctx, uint32_t count, int32_t graph, double out[2]) {
    return guarded([&] {
        if (!ctx || !out || count == 0 || count > 100000) fail(LR_INVALID, "1 to 100000 launches, two results");
        LR_CUDA(cudaSetDevice(ctx->device));
        cudaGraph_t g = nullptr;
        cudaGraphExec_t exec = nullptr;
        auto chain = [&](cudaStream_t s) {
            for (uint32_t i = 0; i < count; i++) idle_kernel<<<1, 32, 0, s>>>(nullptr);
        };
        if (graph) {
            cudaStream_t s;
            LR_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
            LR_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
            chain(s);
            LR_CUDA(cudaStreamEndCapture(s, &g));
            LR_CUDA(cudaStreamDestroy(s));
            LR_CUDA(cudaGraphInstantiate(&exec, g, 0));
        }
        auto run = [&] {
            if (graph) LR_CUDA(cudaGraphLaunch(exec, ctx->stream));
            else chain(ctx->stream);
        };
        run();  // warm: module load, first launch
        LR_CUDA(cudaStreamSynchronize(ctx->stream));
        double best_device = 1e30, best_host = 1e30;
        for (int round = 0; round < 5; round++) {
            const auto t0 = std::chrono::steady_clock::now();
            LR_CUDA(cudaEventRecord(ctx->start, ctx->stream));
            run();
            LR_CUDA(cudaEventRecord(ctx->stop, ctx->stream));
            LR_CUDA(cudaEventSynchronize(ctx->stop));
            const double host = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
            float ms = 0.0f;
            LR_CUDA(cudaEventElapsedTime(&ms, ctx->start, ctx->stop));
            best_device = std::min(best_device, (double)ms);
            best_host = std::min(best_host, host);
        }
        if (exec) cudaGraphExecDestroy(exec);
        if (g) cudaGraphDestroy(g);
        LR_CUDA(cudaGetLastError());
        out[0] = best_device * 1e3 / count;
        out[1] = best_host * 1e3 / count;
    });
}

int lr_gpu_scene_upload(lr_context *ctx, const lr_scene *scene, lr_gpu_scene **out) {
    return guarded([&] {
        if (!ctx || !scene || !out) fail(LR_INVALID, "upload needs a context and a scene");
        *out = nullptr;
        if (scene->nodes.empty()) fail(LR_INVALID, "a scene compiled without its BVH");
        LR_CUDA(cudaSetDevice(ctx->device));
        HostLayout L;
        build_layout(*scene, L);
        const WideBvh w4 = build_wide(scene->nodes, 4, L.delta, widen_down, widen_up, leaf_link);
        const WideBvh w8 = build_wide(scene->nodes, 8, L.delta, widen_down, widen_up, leaf_link);
        const size_t T = scene->triangle_count(), P = scene->point_count();
        // The wide nodes' child slots as refit sources: the BVH2 slot (or root) of each box.
        std::vector<uint32_t> sources4(w4.sources.size()), sources8(w8.sources.size());
        for (auto [from, to] : {std::pair{&w4.sources, &sources4}, std::pair{&w8.sources, &sources8}})
            for (size_t i = 0; i < from->size(); i++)
                (*to)[i] = (*from)[i] == 0xffffffffu ? 0xffffffffu : L.slot_of_node[(*from)[i]];
        const float root_box[8] = {L.root_lo[0], L.root_lo[1], L.root_lo[2], 0.0f,
                                   L.root_hi[0], L.root_hi[1], L.root_hi[2], 0.0f};
        // One allocation, arrays at 256-byte offsets; empty arrays still get room.
        struct Part {
            const void *src;
            size_t bytes;
            size_t offset;
        };
        std::vector<Part> parts = {
            {L.entries.data(), L.entries.size() * sizeof(float4), 0},
            {L.ref_entries.data(), L.ref_entries.size() * sizeof(float4), 0},
            {L.tris.data(), L.tris.size() * sizeof(float4), 0},
            {scene->positions.data(), P * 3 * sizeof(float), 0},
            {scene->indices.data(), T * 3 * sizeof(uint32_t), 0},
            {scene->faces.data(), T * sizeof(uint32_t), 0},
            {scene->order.data(), T * sizeof(uint32_t), 0},
            {L.shading.data(), T * sizeof(uint4), 0},
            {w4.nodes.data(), w4.nodes.size() * sizeof(float), 0},
            {w8.nodes.data(), w8.nodes.size() * sizeof(float), 0},
            {L.parents.data(), L.parents.size() * sizeof(uint32_t), 0},
            {nullptr, L.parents.size() * sizeof(uint32_t), 0},  // climb counters
            {sources4.data(), sources4.size() * sizeof(uint32_t), 0},
            {sources8.data(), sources8.size() * sizeof(uint32_t), 0},
            {scene->flat.data(), scene->flat.size(), 0},
            {root_box, sizeof root_box, 0},
        };
        size_t total = 0;
        for (auto &p : parts) {
            p.offset = total;
            total += align256(std::max<size_t>(p.bytes, 64));
        }
        auto gs = std::make_unique<lr_gpu_scene>();
        gs->ctx = ctx;
        LR_CUDA(cudaMalloc(&gs->allocation, total));
        gs->bytes = total;
        char *base = (char *)gs->allocation;
        LR_CUDA(cudaMemsetAsync(base, 0, total, ctx->stream));
        for (auto &p : parts)
            if (p.bytes && p.src)
                LR_CUDA(cudaMemcpyAsync(base + p.offset, p.src, p.bytes, cudaMemcpyHostToDevice, ctx->stream));
        LR_CUDA(cudaStreamSynchronize(ctx->stream));
        DeviceScene &s = gs->scene;
        s.bvh.entries = (const float4 *)(base + parts[0].offset);
        s.ref_bvh.entries = (const float4 *)(base + parts[1].offset);
        s.tris = (const float4 *)(base + parts[2].offset);
        s.positions = (const float *)(base + parts[3].offset);
        s.indices = (const uint32_t *)(base + parts[4].offset);
        s.faces = (const uint32_t *)(base + parts[5].offset);
        s.ids = (const uint32_t *)(base + parts[6].offset);
        s.shading = (const uint4 *)(base + parts[7].offset);
        s.wide4 = DeviceWide{(const float4 *)(base + parts[8].offset), T ? 4 : 0, w4.max_stack, w4.node_count};
        s.wide8 = DeviceWide{(const float4 *)(base + parts[9].offset), T ? 8 : 0, w8.max_stack, w8.node_count};
        gs->wide4_nodes = w4.node_count;
        gs->wide8_nodes = w8.node_count;
        gs->parents = (uint32_t *)(base + parts[10].offset);
        gs->counters = (uint32_t *)(base + parts[11].offset);
        gs->wide4_sources = (uint32_t *)(base + parts[12].offset);
        gs->wide8_sources = (uint32_t *)(base + parts[13].offset);
        gs->flat = (uint8_t *)(base + parts[14].offset);
        gs->root_box = (float *)(base + parts[15].offset);
        gs->topology = topology_hash(*scene);
        gs->any_flat = std::any_of(scene->flat.begin(), scene->flat.end(), [](uint8_t f) { return f != 0; });
        for (DeviceBvh *b : {&s.bvh, &s.ref_bvh}) {
            b->root = L.root;
            b->empty = T == 0 ? 1 : 0;
            for (int k = 0; k < 3; k++) {
                b->root_lo[k] = L.root_lo[k];
                b->root_hi[k] = L.root_hi[k];
            }
        }
        for (int k = 0; k < 3; k++) {
            s.bvh.root_lo[k] = widen_down(L.root_lo[k], L.delta);
            s.bvh.root_hi[k] = widen_up(L.root_hi[k], L.delta);
        }
        s.triangle_count = T;
        s.point_count = P;
        s.entry_count = L.entries.size() / 4;
        s.depth = scene->bvh_depth;
        stack_for(s.depth);
        *out = gs.release();
    });
}

int lr_gpu_scene_info_get(const lr_gpu_scene *gs, lr_gpu_scene_info *out) {
    return guarded([&] {
        if (!gs || !out) fail(LR_INVALID, "no scene");
        out->bytes = gs->bytes;
        out->bvh2_depth = gs->scene.depth;
        out->wide4_nodes = gs->wide4_nodes;
        out->wide8_nodes = gs->wide8_nodes;
        out->wide4_stack = gs->scene.wide4.max_stack;
        out->wide8_stack = gs->scene.wide8.max_stack;
        const TraversalChoice c = choose_traversal(gs->scene, 0);
        out->width = (uint32_t)c.width;
        out->stack = (uint32_t)c.stack;
    });
}

void lr_gpu_scene_destroy(lr_gpu_scene *gs) {
    if (!gs) return;
    if (gs->ctx) {
        cudaSetDevice(gs->ctx->device);
        cudaStreamSynchronize(gs->ctx->stream);
    }
    if (gs->allocation) cudaFree(gs->allocation);
    delete gs;
}

int lr_probe(lr_context *ctx, const lr_gpu_scene *gs, const lr_frame *frame, uint32_t flags, uint32_t *faces,
             float *distances) {
    return guarded([&] {
        if (!ctx || !gs || !frame || !faces || !distances) fail(LR_INVALID, "a probe needs one result per pixel");
        if (frame->width == 0 || frame->height == 0) fail(LR_INVALID, "an image needs pixels");
        const uint64_t count = (uint64_t)frame->width * frame->height;
        ProbeFrame f;
        pack_frame(*frame, f.b);
        LR_CUDA(cudaSetDevice(ctx->device));
        void *buffer = nullptr;
        LR_CUDA(cudaMallocAsync(&buffer, count * 8, ctx->stream));
        uint32_t *d_faces = (uint32_t *)buffer;
        float *d_ts = (float *)((char *)buffer + count * 4);
        if (flags & LR_TRACE_REFERENCE)
            dispatch_probe<true>(gs, f, count, d_faces, d_ts, ctx->status, ctx->stream);
        else
            dispatch_probe<false>(gs, f, count, d_faces, d_ts, ctx->status, ctx->stream);
        LR_CUDA(cudaGetLastError());
        LR_CUDA(cudaMemcpyAsync(faces, d_faces, count * 4, cudaMemcpyDeviceToHost, ctx->stream));
        LR_CUDA(cudaMemcpyAsync(distances, d_ts, count * 4, cudaMemcpyDeviceToHost, ctx->stream));
        LR_CUDA(cudaFreeAsync(buffer, ctx->stream));
        LR_CUDA(cudaStreamSynchronize(ctx->stream));
        check_status(ctx);
    });
}

}  // extern "C"

// The device scratch of lr_probe_static: LR_PROBE_STATIC_PIXELS face ids, then as many
// distances (16 MiB), reserved when the module loads on a device and never freed.
static __device__ __align__(256) unsigned char g_probe_scratch[(size_t)LR_PROBE_STATIC_PIXELS * 8];

namespace {

constexpr int kScratchDevices = 64;
std::mutex g_scratch_mutex;
void *g_scratch_of[kScratchDevices] = {};
// One lock a device, held by a call from its launch until its results are on the host:
// calls from several host threads of this process take turns on the array.
std::mutex g_scratch_in_use[kScratchDevices];

}  // namespace

namespace lr {

// The address of g_probe_scratch on `device`, looked up once per device with that device
// current (the first lookup may load the module there). The address stays valid while
// the process keeps the device's primary context: the library is not to be used across a
// cudaDeviceReset.
void *probe_static_setup(int device) {
    if (device < 0 || device >= kScratchDevices) fail(LR_LIMIT, "lr_probe_static serves devices 0 to 63");
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_of[device]) {
        int current = -1;
        LR_CUDA(cudaGetDevice(&current));
        if (current != device) LR_CUDA(cudaSetDevice(device));
        void *address = nullptr;
        const cudaError_t looked = cudaGetSymbolAddress(&address, g_probe_scratch);
        if (current != device && current >= 0) cudaSetDevice(current);
        if (looked != cudaSuccess)
            fail(LR_DEVICE, std::string("cudaGetSymbolAddress(g_probe_scratch): ") + cudaGetErrorString(looked));
        if (!address) fail(LR_DEVICE, "no address for the static probe scratch");
        g_scratch_of[device] = address;
    }
    return g_scratch_of[device];
}

}  // namespace lr

extern "C" {

int lr_probe_static(lr_context *ctx, const lr_gpu_scene *gs, const lr_frame *frame, uint32_t flags,
                    uint32_t *faces, float *distances) {
    return guarded([&] {
        if (!ctx || !gs || !frame || !faces || !distances) fail(LR_INVALID, "a probe needs one result per pixel");
        if (frame->width == 0 || frame->height == 0) fail(LR_INVALID, "an image needs pixels");
        const uint64_t count = (uint64_t)frame->width * frame->height;
        if (count > LR_PROBE_STATIC_PIXELS)
            fail(LR_LIMIT, "lr_probe_static takes at most " + std::to_string(LR_PROBE_STATIC_PIXELS) +
                               " pixels (its static scratch); this frame has " + std::to_string(count) +
                               ": use lr_probe");
        ProbeFrame f;
        pack_frame(*frame, f.b);
        LR_CUDA(cudaSetDevice(ctx->device));
        char *scratch = (char *)probe_static_setup(ctx->device);
        std::lock_guard<std::mutex> turn(g_scratch_in_use[ctx->device]);
        // The kernel writes every pixel's face and distance, so nothing in the scratch has
        // to start at zero; the status words it may raise are the context's, kept at zero.
        uint32_t *d_faces = (uint32_t *)scratch;
        float *d_ts = (float *)(scratch + (size_t)LR_PROBE_STATIC_PIXELS * 4);
        try {
            if (flags & LR_TRACE_REFERENCE)
                dispatch_probe<true>(gs, f, count, d_faces, d_ts, ctx->status, ctx->stream);
            else
                dispatch_probe<false>(gs, f, count, d_faces, d_ts, ctx->status, ctx->stream);
            LR_CUDA(cudaGetLastError());
            LR_CUDA(cudaMemcpyAsync(faces, d_faces, count * 4, cudaMemcpyDeviceToHost, ctx->stream));
            LR_CUDA(cudaMemcpyAsync(distances, d_ts, count * 4, cudaMemcpyDeviceToHost, ctx->stream));
            LR_CUDA(cudaStreamSynchronize(ctx->stream));
        } catch (...) {
            // Whatever was queued finishes before the array is handed to the next call.
            cudaStreamSynchronize(ctx->stream);
            throw;
        }
        check_status(ctx);
    });
}

int lr_context_memory(lr_context *ctx, int32_t reset_high, uint64_t out[4]) {
    return guarded([&] {
        if (!ctx || !out) fail(LR_INVALID, "memory figures need a context and four words");
        LR_CUDA(cudaSetDevice(ctx->device));
        size_t free_bytes = 0, total_bytes = 0;
        LR_CUDA(cudaMemGetInfo(&free_bytes, &total_bytes));
        cudaMemPool_t pool;
        LR_CUDA(cudaDeviceGetDefaultMemPool(&pool, ctx->device));
        if (reset_high) {
            unsigned long long zero = 0;
            LR_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrUsedMemHigh, &zero));
        }
        unsigned long long used = 0, high = 0;
        LR_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used));
        LR_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemHigh, &high));
        out[0] = free_bytes;
        out[1] = total_bytes;
        out[2] = used;
        out[3] = high;
    });
}

}  // extern "C"

extern "C" {

static void trace_device(lr_context *ctx, const lr_gpu_scene *gs, const void *rays, uint64_t n, void *hits,
                         uint32_t flags) {
    if (n == 0) return;
    const float4 *r = (const float4 *)rays;
    float4 *h = (float4 *)hits;
    const bool any = flags & LR_TRACE_ANY, ref = flags & LR_TRACE_REFERENCE, count = flags & LR_TRACE_COUNT;
    const int width = (flags & LR_TRACE_BVH2) ? 2 : (flags & LR_TRACE_BVH4) ? 4 : (flags & LR_TRACE_BVH8) ? 8 : 0;
    unsigned long long *c = ctx->counts;
    int *st = ctx->status;
    cudaStream_t s = ctx->stream;
    if (ref) {
        if (any && count) dispatch_reference<true, true>(gs, r, n, h, st, c, s);
        else if (any) dispatch_reference<true, false>(gs, r, n, h, st, c, s);
        else if (count) dispatch_reference<false, true>(gs, r, n, h, st, c, s);
        else dispatch_reference<false, false>(gs, r, n, h, st, c, s);
    } else {
        if (any && count) dispatch_exact<true, true>(gs, r, n, h, st, c, s, width);
        else if (any) dispatch_exact<true, false>(gs, r, n, h, st, c, s, width);
        else if (count) dispatch_exact<false, true>(gs, r, n, h, st, c, s, width);
        else dispatch_exact<false, false>(gs, r, n, h, st, c, s, width);
    }
    LR_CUDA(cudaGetLastError());
}

int lr_trace_counts(lr_context *ctx, uint64_t out[2]) {
    return guarded([&] {
        if (!ctx || !out) fail(LR_INVALID, "trace counts need two words");
        unsigned long long words[2] = {0, 0};
        LR_CUDA(cudaMemcpyAsync(words, ctx->counts, sizeof words, cudaMemcpyDeviceToHost, ctx->stream));
        LR_CUDA(cudaMemsetAsync(ctx->counts, 0, sizeof words, ctx->stream));
        LR_CUDA(cudaStreamSynchronize(ctx->stream));
        out[0] = words[0];
        out[1] = words[1];
    });
}

int lr_trace_rays(lr_context *ctx, const lr_gpu_scene *gs, const float *rays, uint64_t count, float *hits,
                  uint32_t flags) {
    return guarded([&] {
        if (!ctx || !gs || (count && (!rays || !hits))) fail(LR_INVALID, "a ray query needs rays and room for hits");
        if (count == 0) return;
        LR_CUDA(cudaSetDevice(ctx->device));
        void *buffer = nullptr;
        LR_CUDA(cudaMallocAsync(&buffer, count * 48, ctx->stream));
        void *d_hits = (char *)buffer + count * 32;
        LR_CUDA(cudaMemcpyAsync(buffer, rays, count * 32, cudaMemcpyHostToDevice, ctx->stream));
        trace_device(ctx, gs, buffer, count, d_hits, flags);
        LR_CUDA(cudaMemcpyAsync(hits, d_hits, count * 16, cudaMemcpyDeviceToHost, ctx->stream));
        LR_CUDA(cudaFreeAsync(buffer, ctx->stream));
        LR_CUDA(cudaStreamSynchronize(ctx->stream));
        check_status(ctx);
    });
}

int lr_trace_rays_device(lr_context *ctx, const lr_gpu_scene *gs, const void *rays, uint64_t count, void *hits,
                         uint32_t flags) {
    return guarded([&] {
        if (!ctx || !gs || (count && (!rays || !hits))) fail(LR_INVALID, "a ray query needs rays and room for hits");
        if (((uintptr_t)rays & 15) || ((uintptr_t)hits & 15)) fail(LR_INVALID, "rays and hits must be 16-byte aligned");
        trace_device(ctx, gs, rays, count, hits, flags);
    });
}

}  // extern "C"
