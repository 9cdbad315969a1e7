// The wavefront path tracer (src/render/integrator.lucb, shaders/camera.comp,
// intersect_closest.comp, shade_surface.comp, shade_miss.comp, intersect_shadow.comp,
// finish.comp, film_convert.comp) on sm_100a, for one scene or many at once.
//
// A wave is a pool of paths shared by its members (a member: one scene seen through one
// camera into one film). Each pass traces one sample for a set of segments -- a segment
// is a range of one member's pixels at one sample index -- laid end to end in the pool:
//   camera -> (closest -> shade -> shadow) x rounds -> finish -> convert
// The host plans the segments of every pass and copies the plan (a few hundred bytes)
// ahead of it on the stream; the pass itself is one CUDA graph per traversal variant.
// Rays live in two ping-pong queues of structure-of-arrays float4 records (origin + tag,
// direction + t_max) that the traversal kernels read with coalesced 128-bit loads; the
// tag holds the path's pool index and its segment, so a ray finds its scene with one
// lookup. The shade kernel takes every queue entry -- surface hit, light hit or miss
// (shade_surface + shade_miss of the reference) -- and pushes surviving paths' next rays
// and shadow rays into compact queues with one atomic per warp. Queue sizes never leave
// the device: every kernel is a persistent grid-stride loop over the count its producer
// left.
//
// Every path's arithmetic depends only on its member, pixel and sample, and a pixel gets
// its samples in order, one per pass at most, so an image comes out bit for bit the same
// whichever members share the wave with it and however the pool splits its pixels.
//
// lr_renderer (Renderer of the reference) is a wave with one member whose segments are
// the reference's bands; lr_batch is a wave of many members that come and go.
#include <algorithm>
#include <cstddef>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <vector>

#include "device.hpp"
#include "loading.hpp"
#include <cuda_fp16.h>

#include "paths.cuh"
#include "shading.cuh"
#include "traverse.cuh"
#include "wave.cuh"

namespace lr {
namespace {

// camera.comp:14-50 and light_emit.comp:21-130: every camera segment's paths start a
// jittered primary ray, every light segment's a light path. Block 0 also starts the
// pass's queue counters.
__global__ void __launch_bounds__(kShadeBlock) camera_kernel(Wave w) {
    const Plan *plan = w.plan;
    const uint32_t paths = plan->head.paths;
    if (blockIdx.x == 0) {
        const uint32_t light_base = kLightCounters * w.rounds + 2;
        for (uint32_t i = threadIdx.x; i < counter_slots(w.rounds); i += blockDim.x)
            w.counters[i] = i == 0 ? plan->head.camera_paths : (i == light_base ? paths - plan->head.camera_paths : 0u);
    }
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t path = blockIdx.x * blockDim.x + threadIdx.x; path < paths; path += stride) {
        const uint32_t si = segment_of(plan, path);
        const Segment &sg = plan->seg[si];
        const Member &m = w.members[sg.member];
        if (sg.kind == kLightSegment) {
            const uint32_t slot = w.pool - 1u - (sg.kind_base + (path - sg.path_base));
            if (m.spectral) start_light_path<true>(w, m, sg, si, path, slot);
            else start_light_path<false>(w, m, sg, si, path, slot);
        } else {
            start_camera_path(w, m, sg, si, path, sg.kind_base + (path - sg.path_base));
        }
    }
}

// The bodies every pass variant shares, compiled once per spectral mode (out of line):
// the compiler fuses multiply-adds by the code around a body, so one body keeps a
// member's image the same bits alone and in any mix of members. All-diffuse camera paths
// take the lean body inlined instead (its registers decide the kernel's occupancy).
template <bool kSpectral>
__device__ __noinline__ void camera_layered(const Wave &w, const Member &m, uint32_t sample, uint32_t round, uint32_t i,
                                            float4 ro, ShadeOut &out) {
    shade_camera_path<kSpectral, true, LayeredOps>(w, m, sample, round, i, ro, out);
}
template <bool kSpectral>
__device__ __noinline__ void light_layered(const Wave &w, const Member &m, uint32_t sample, uint32_t round, uint32_t i,
                                           float4 ro, ShadeOut &out) {
    shade_light_path<kSpectral, LayeredLightOps>(w, m, sample, round, i, ro, out);
}
template <bool kSpectral>
__device__ __noinline__ void light_diffuse(const Wave &w, const Member &m, uint32_t sample, uint32_t round, uint32_t i,
                                           float4 ro, ShadeOut &out) {
    shade_light_path<kSpectral, DiffuseLightOps>(w, m, sample, round, i, ro, out);
}

// The octant of a direction (sign bits of x, y, z).
__device__ __forceinline__ uint32_t octant_of(float4 d) {
    return (d.x < 0.0f ? 1u : 0u) | (d.y < 0.0f ? 2u : 0u) | (d.z < 0.0f ? 4u : 0u);
}

// A block-wide push of the threads that `want`, grouped by `key` (0..7): one atomic on
// `counter` for the block, each key's rays contiguous in key order; returns this
// thread's slot. Every thread of the block calls it; `bins` is shared scratch (9 words).
__device__ __forceinline__ uint32_t block_push(uint32_t *counter, bool want, uint32_t key, uint32_t *bins) {
    if (threadIdx.x < 9u) bins[threadIdx.x] = 0u;
    __syncthreads();
    const uint32_t rank = want ? atomicAdd(&bins[key], 1u) : 0u;
    __syncthreads();
    if (threadIdx.x == 0u) {
        uint32_t total = 0;
        for (uint32_t b = 0; b < 8u; b++) {
            const uint32_t n = bins[b];
            bins[b] = total;
            total += n;
        }
        bins[8] = total ? atomicAdd(counter, total) : 0u;
    }
    __syncthreads();
    const uint32_t slot = bins[8] + bins[key] + rank;
    __syncthreads();  // the next push rewrites the bins
    return slot;
}

// Sorting keys of a shading tile: 0 for misses and light hits, 1 .. kSortBins - 2 for
// surface hits by member and material, kSortBins - 1 past the queue's end.
constexpr uint32_t kSortBins = 64;

// A block's tile of queue entries [tile, tile + blockDim.x) ordered by key, counting-sort
// style in shared memory; returns the tile position this thread shades. Every thread of
// the block calls it.
__device__ __forceinline__ uint32_t tile_order(const Wave &w, uint32_t q, uint32_t tile, uint32_t count, bool light,
                                               uint32_t *bins, uint32_t *order) {
    const uint32_t t = threadIdx.x, k = tile + t;
    uint32_t key = kSortBins - 1u;
    if (k < count) {
        const uint32_t i = light ? w.pool - 1u - k : k;
        const uint32_t what = __float_as_uint(w.hits[q][i].y);
        if (what == kNone || (what & kLightHit)) {
            key = 0u;
        } else {
            const uint32_t member = w.plan->seg[__float_as_uint(w.ray_o[q][i].w) >> kPathBits].member;
            const uint32_t material = __ldg(&w.members[member].scene.shading[what]).w;
            key = 1u + (material * 7u + member * 5u) % (kSortBins - 2u);
        }
    }
    for (uint32_t b = t; b < kSortBins; b += blockDim.x) bins[b] = 0u;
    __syncthreads();
    const uint32_t rank = atomicAdd(&bins[key], 1u);
    __syncthreads();
    if (t < 32u) {  // exclusive scan of the bins, two a lane
        const uint32_t a = bins[2u * t], b = bins[2u * t + 1u];
        uint32_t sum = a + b;
        for (uint32_t d = 1; d < 32u; d <<= 1) {
            const uint32_t up = __shfl_up_sync(0xffffffffu, sum, d);
            if (t >= d) sum += up;
        }
        const uint32_t before = sum - a - b;
        bins[2u * t] = before;
        bins[2u * t + 1u] = before + a;
    }
    __syncthreads();
    order[bins[key] + rank] = t;
    __syncthreads();
    const uint32_t mine = order[t];
    __syncthreads();  // the next tile rewrites the bins and the order
    return mine;
}

// 1,024 threads an SM (64 registers): the diffuse camera-path shading wants 128, which
// leaves 16 warps an SM to hide its memory latency; capped, it spills a little and runs
// 17 % faster (1.21 -> 1.01 ms a 1080p pass on the 1M-triangle scene; 48 registers: 0.99 ms
// with twice the spills).
// kTracing: the pass holds light paths or camera paths that weigh against them; passes
// without take the kernel without that code (it cost camera-only passes 16 %). kGlossy:
// the pass holds a member with glossy materials, whose entries take the layered OpenPBR
// shading (out of line, 4 blocks an SM for its registers); the rest shade as without it.
// kLight: the launch shades the light paths' rays (the queue's back) rather than the
// camera paths' (its front). Camera and light paths shade in launches of their own: mixed
// in one launch, their two large bodies fought over the instruction cache (the glossy box
// with light tracing: 4.2 -> 1.8 ms of shading a 512^2 sample).
template <bool kTracing, bool kGlossy, bool kLight>
__global__ void __launch_bounds__(kShadeBlock, (kGlossy ? 512 : 1024) / kShadeBlock) shade_kernel(Wave w, uint32_t round) {
    const uint32_t count = kLight ? *light_counter(w, round) : w.counters[round];
    const uint32_t q = round & 1u, nq = q ^ 1u;
    uint32_t *next_counter = kLight ? light_counter(w, round + 1) : &w.counters[round + 1];
    uint32_t *shadow_counter = &w.counters[w.rounds + 1 + round];
    // Outgoing rays are binned by octant in the rounds the plan's interval names (0: never).
    const uint32_t interval = w.plan->head.bin_interval;
    const bool binned = interval != 0u && round % interval == 0u;
    __shared__ uint32_t bins[kSortBins];
    // Shades queue entry k (all threads of the block call it: the pushes are warp- or
    // block-wide).
    auto shade = [&](uint32_t k) {
        const uint32_t i = kLight ? w.pool - 1u - k : k;
        ShadeOut out;
        if (k < count) {
            const float4 ro = w.ray_o[q][i];
            const Segment &sg = w.plan->seg[__float_as_uint(ro.w) >> kPathBits];
            const Member &m = w.members[sg.member];
            if (kLight) {
                if (kGlossy && m.glossy) {
                    if (m.spectral) light_layered<true>(w, m, sg.sample, round, i, ro, out);
                    else light_layered<false>(w, m, sg.sample, round, i, ro, out);
                } else if (m.spectral) {
                    light_diffuse<true>(w, m, sg.sample, round, i, ro, out);
                } else {
                    light_diffuse<false>(w, m, sg.sample, round, i, ro, out);
                }
            } else if (kGlossy && m.glossy) {
                if (m.spectral) camera_layered<true>(w, m, sg.sample, round, i, ro, out);
                else camera_layered<false>(w, m, sg.sample, round, i, ro, out);
            } else if (m.spectral) {
                shade_camera_path<true, kTracing, DiffuseOps>(w, m, sg.sample, round, i, ro, out);
            } else {
                shade_camera_path<false, kTracing, DiffuseOps>(w, m, sg.sample, round, i, ro, out);
            }
            // Past the member's last round (cut-outs passed at its last bounces) a ray is
            // not traced, as the reference's pass loop ends there.
            if (round + 1u >= m.rounds) out.next = false;
        }
        uint32_t at, sat;
        if (binned) {
            // The block's rays, grouped by direction octant in the queue: the traversal's
            // warps then take rays that order every node's children alike.
            at = block_push(next_counter, out.next, octant_of(out.d), bins);
            sat = block_push(shadow_counter, out.shadow, octant_of(out.sd), bins);
        } else {
            at = warp_push(next_counter, out.next);
            sat = warp_push(shadow_counter, out.shadow);
        }
        if (out.next) {
            const uint32_t slot = kLight ? w.pool - 1u - at : at;
            w.ray_o[nq][slot] = out.o;
            w.ray_d[nq][slot] = out.d;
        }
        if (out.shadow) {
            w.shadow_o[sat] = out.so;
            w.shadow_d[sat] = out.sd;
            w.shadow_c[sat] = out.sc;
        }
    };
    // Every block takes tiles of blockDim.x queue entries (block-uniform, so a block may
    // sort them, or its outgoing rays, in shared memory), the next one from the round's
    // cursor when it is done with the last, so blocks that drew slow paths take fewer.
    __shared__ uint32_t next_tile;
    uint32_t *cursor = shade_cursor(w, round, kLight);
    for (;;) {
        if (threadIdx.x == 0) next_tile = atomicAdd(cursor, blockDim.x);
        __syncthreads();
        const uint32_t tile = next_tile;
        __syncthreads();
        if (tile >= count) break;
        if constexpr (kGlossy) {
            // Layered surfaces branch by material: each tile is ordered by what its entries
            // shade before its warps take them, so a warp's lanes mostly follow one path
            // through the lobes.
            __shared__ uint32_t order[kShadeBlock];
            shade(tile + tile_order(w, q, tile, count, kLight, bins, order));
        } else {
            shade(tile + threadIdx.x);
        }
    }
}

// finish.comp:13-39: each path's radiance into its pixel (one sample per pixel a pass).
__global__ void __launch_bounds__(kShadeBlock) finish_kernel(Wave w) {
    const Plan *plan = w.plan;
    const uint32_t paths = plan->head.paths;
    const uint32_t stride = gridDim.x * blockDim.x;
    if (plan->head.dry) return;
    for (uint32_t path = blockIdx.x * blockDim.x + threadIdx.x; path < paths; path += stride) {
        const Segment &sg = plan->seg[segment_of(plan, path)];
        if (sg.kind == kLightSegment) continue;  // light paths reach the film by splats
        const Member &m = w.members[sg.member];
        const uint32_t pixel = w.path[path].x;
        if (pixel == kNone) continue;  // converged: no sample taken
        float3 value = m.spectral ? spec_to_film<true>(w.radiance[path], w.lambda[path], *m.k)
                                  : spec_to_film<false>(w.radiance[path], make_float4(0, 0, 0, 0), *m.k);
        if (!isfinite(value.x) || !isfinite(value.y) || !isfinite(value.z)) value = make_float3(0.0f, 0.0f, 0.0f);
        const float4 f = m.film[pixel];
        m.film[pixel] = make_float4(f.x + value.x, f.y + value.y, f.z + value.z, f.w + 1.0f);
        // Adaptive sampling's second estimate: every other sample, twice.
        if (m.half && (sg.sample & 1u)) {
            const float4 hs = m.half[pixel];
            m.half[pixel] = make_float4(hs.x + 2.0f * value.x, hs.y + 2.0f * value.y, hs.z + 2.0f * value.z, hs.w);
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        unsigned long long closest = 0, shadow = 0;
        for (uint32_t r = 0; r < w.rounds; r++) {
            closest += w.counters[r] + *light_counter(w, r);
            shadow += w.counters[w.rounds + 1 + r];
        }
        w.stats[0] += closest;
        w.stats[1] += shadow;
        w.stats[2] += plan->head.camera_paths;
        w.stats[3] += 1;
    }
}

// adaptive.comp (after Dammertz et al. and Cycles' film_adaptive_sampling), for the members
// the pass checks: phase 0 judges each pixel by how far its full and half estimates differ
// against the square root of its brightness; phase 1 marks a pixel converged (the half
// estimate's w) when its whole 3 x 3 neighbourhood is, so noise at a converged pixel's
// edge keeps it sampling.
__global__ void __launch_bounds__(kShadeBlock) adaptive_kernel(Wave w, uint32_t phase) {
    const Plan *plan = w.plan;
    if (plan->head.dry) return;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint32_t a = 0; a < plan->head.adapts; a++) {
        const Member &m = w.members[plan->adapt[a]];
        const float threshold = m.k->noise_threshold;
        for (uint64_t pixel = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; pixel < m.pixels; pixel += stride) {
            if (phase == 0u) {
                const float4 sum = m.film[pixel], half_sum = m.half[pixel];
                const float scale = 1.0f / fmaxf(sum.w, 1.0f);
                const float difference =
                    (fabsf(sum.x - half_sum.x) + fabsf(sum.y - half_sum.y) + fabsf(sum.z - half_sum.z)) * scale;
                const float brightness = fmaxf(0.0f, (sum.x + sum.y + sum.z) * scale);
                const float error = difference / (0.0001f + sqrtf(brightness));
                m.scratch[pixel] = error < threshold ? 1.0f : 0.0f;
                continue;
            }
            const int x = (int)(pixel % m.width), y = (int)(pixel / m.width);
            float converged = 1.0f;
            for (int dy = -1; dy <= 1; dy++)
                for (int dx = -1; dx <= 1; dx++) {
                    const int nx = x + dx, ny = y + dy;
                    if (nx < 0 || ny < 0 || nx >= (int)m.width || ny >= (int)m.height) continue;
                    converged = fminf(converged, m.scratch[(uint64_t)ny * m.width + nx]);
                }
            m.half[pixel].w = converged;
        }
    }
}

// The splats this lane's light paths left for the members traced in this pass, added into
// their films' splat accumulators (in pass order: the finish stages run one after another)
// and cleared for the lane's next pass.
__global__ void __launch_bounds__(kShadeBlock) fold_kernel(Wave w) {
    const Plan *plan = w.plan;
    if (plan->head.dry) return;
    const uint32_t folds = plan->head.folds;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint32_t f = 0; f < folds; f++) {
        const Member &m = w.members[plan->fold[f]];
        unsigned long long *lane = m.splat_lane[w.lane];
        for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m.pixels * 3; i += stride) {
            const unsigned long long v = lane[i];
            if (v) {
                m.splat[i] += v;
                lane[i] = 0ull;
            }
        }
    }
}

// film_convert.comp:36-53: the film's average, and the light paths' splats over the
// samples taken, into the rgba32f ACEScg image, for every member whose sample ended in
// this pass.
// Khronos PBR Neutral tone mapping (film_convert.comp:20-34): linear below 0.76, with
// hue-preserving compression above.
__device__ __forceinline__ float3 pbr_neutral(float3 c) {
    const float start = 0.8f - 0.04f, desaturation = 0.15f;
    const float x = fminf(c.x, fminf(c.y, c.z));
    const float offset = x < 0.08f ? x - 6.25f * x * x : 0.04f;
    c = make_float3(c.x - offset, c.y - offset, c.z - offset);
    const float peak = fmaxf(c.x, fmaxf(c.y, c.z));
    if (peak < start) return c;
    const float d = 1.0f - start;
    const float new_peak = 1.0f - d * d / (peak + d - start);
    c = c * (new_peak / peak);
    const float g = 1.0f - 1.0f / (desaturation * (peak - new_peak) + 1.0f);
    return make_float3(c.x * (1.0f - g) + new_peak * g, c.y * (1.0f - g) + new_peak * g, c.z * (1.0f - g) + new_peak * g);
}

__global__ void __launch_bounds__(kShadeBlock) convert_kernel(Wave w) {
    const Plan *plan = w.plan;
    const uint32_t converts = plan->head.converts;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint32_t c = 0; c < converts; c++) {
        const Member &m = w.members[plan->convert[c]];
        const Constants &k = *m.k;
        const double per_sample = m.light_paths ? 1.0 / (kSplatScale * (double)plan->convert_samples[c]) : 0.0;
        for (uint64_t pixel = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; pixel < m.pixels; pixel += stride) {
            const float4 sum = m.film[pixel];
            const float wsum = fmaxf(sum.w, 1.0f);
            float3 value = make_float3(sum.x / wsum, sum.y / wsum, sum.z / wsum);
            if (m.light_paths) {
                const unsigned long long *sp = m.splat + pixel * 3;
                value = value + make_float3((float)((double)(long long)sp[0] * per_sample),
                                            (float)((double)(long long)sp[1] * per_sample),
                                            (float)((double)(long long)sp[2] * per_sample));
            }
            if (m.spectral)
                value = make_float3(k.film[0] * value.x + k.film[1] * value.y + k.film[2] * value.z,
                                    k.film[3] * value.x + k.film[4] * value.y + k.film[5] * value.z,
                                    k.film[6] * value.x + k.film[7] * value.y + k.film[8] * value.z);
            m.image[pixel] = make_float4(value.x, value.y, value.z, 1.0f);
            if (c == 0 && plan->display.image) {
                // Exposed, in linear Rec.709 (ACEScg Bradford-adapted to D65), through the view.
                const float e = plan->display.scale;
                float3 shown = make_float3(fmaxf(0.0f, e * (1.70505f * value.x - 0.62179f * value.y - 0.08326f * value.z)),
                                           fmaxf(0.0f, e * (-0.13026f * value.x + 1.14080f * value.y - 0.01055f * value.z)),
                                           fmaxf(0.0f, e * (-0.02400f * value.x - 0.12897f * value.y + 1.15297f * value.z)));
                if (plan->display.view == 1u) shown = pbr_neutral(shown);
                __half *out = (__half *)plan->display.image + pixel * 4;
                out[0] = __float2half_rn(fminf(shown.x, 1.0f));
                out[1] = __float2half_rn(fminf(shown.y, 1.0f));
                out[2] = __float2half_rn(fminf(shown.z, 1.0f));
                out[3] = __float2half_rn(1.0f);
            }
        }
    }
}

// Kernel kinds for profiling (integrator.lucb:105-115).
enum Kind { kCamera = 0, kClosest = 1, kSurface = 2, kMiss = 3, kShadow = 4, kLightEmit = 5, kFinish = 6, kConvert = 7,
            kAdaptive = 8, kRest = 9 };

template <typename K>
int grid_of(K kernel, int block, int sm_count) {
    int per_sm = 0;
    LR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, 0));
    return std::max(1, per_sm) * sm_count;
}

size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

// Device memory carved into 256-byte aligned parts: add the parts, then allocate once.
struct Layout {
    struct Part {
        const void *src;
        size_t bytes, offset;
    };
    std::vector<Part> parts;
    size_t add(const void *src, size_t bytes) {
        parts.push_back({src, bytes, 0});
        return parts.size() - 1;
    }
    // One allocation, zeroed, with the host parts copied in; waits for the copies.
    void *allocate(cudaStream_t stream, size_t &total) {
        total = 0;
        for (auto &p : parts) {
            p.offset = total;
            total += align256(std::max<size_t>(p.bytes, 64));
        }
        void *block = nullptr;
        LR_CUDA(cudaMalloc(&block, total));
        char *base = (char *)block;
        LR_CUDA(cudaMemsetAsync(base, 0, total, stream));
        for (auto &p : parts)
            if (p.src && p.bytes) LR_CUDA(cudaMemcpyAsync(base + p.offset, p.src, p.bytes, cudaMemcpyHostToDevice, stream));
        LR_CUDA(cudaStreamSynchronize(stream));
        return block;
    }
};

// Pinned host memory that stages uploads, so that they queue on a stream without
// waiting for the work ahead of them: a ring of up to kChunks buffers, each reused once
// its own copies have run, so that a new upload waits only when every buffer is still
// being copied from. `copied` follows the latest upload queued (a lane waits on it).
struct Staging {
    static constexpr int kChunks = 8;
    struct Chunk {
        char *ptr = nullptr;
        size_t capacity = 0;
        cudaEvent_t done = nullptr;  // after the copies from it
        uint64_t queued_at = 0;      // 0: never queued
    };
    Chunk chunks[kChunks];
    int count = 0, current = -1;
    uint64_t uploads = 0;
    cudaEvent_t copied = nullptr;

    static bool idle(const Chunk &c) {
        if (!c.queued_at) return true;
        const cudaError_t e = cudaEventQuery(c.done);
        if (e == cudaErrorNotReady) return false;
        LR_CUDA(e);
        return true;
    }

    char *take(size_t bytes) {
        int pick = -1;
        // An idle buffer large enough; else an idle one to grow; else a new one; else the
        // one queued longest ago, once its copies have run.
        for (int i = 0; i < count && pick < 0; i++)
            if (chunks[i].capacity >= bytes && idle(chunks[i])) pick = i;
        for (int i = 0; i < count && pick < 0; i++)
            if (idle(chunks[i])) pick = i;
        if (pick < 0 && count < kChunks) pick = count++;
        if (pick < 0) {
            pick = 0;
            for (int i = 1; i < count; i++)
                if (chunks[i].queued_at < chunks[pick].queued_at) pick = i;
            LR_CUDA(cudaEventSynchronize(chunks[pick].done));
        }
        Chunk &c = chunks[pick];
        if (bytes > c.capacity) {
            if (c.ptr) LR_CUDA(cudaFreeHost(c.ptr));
            c.ptr = nullptr;
            c.capacity = std::max<size_t>(bytes, 1u << 20);
            LR_CUDA(cudaMallocHost((void **)&c.ptr, c.capacity));
        }
        current = pick;
        return c.ptr;
    }
    void queued(cudaStream_t stream) {
        if (!copied) LR_CUDA(cudaEventCreateWithFlags(&copied, cudaEventDisableTiming));
        LR_CUDA(cudaEventRecord(copied, stream));
        if (current < 0) return;
        Chunk &c = chunks[current];
        if (!c.done) LR_CUDA(cudaEventCreateWithFlags(&c.done, cudaEventDisableTiming));
        LR_CUDA(cudaEventRecord(c.done, stream));
        c.queued_at = ++uploads;
        current = -1;
    }
    void release() {
        for (int i = 0; i < count; i++) {
            Chunk &c = chunks[i];
            if (c.done) {
                cudaEventSynchronize(c.done);
                cudaEventDestroy(c.done);
            }
            if (c.ptr) cudaFreeHost(c.ptr);
        }
        if (copied) cudaEventDestroy(copied);
        *this = Staging{};
    }
};

// The Owen-scrambled Sobol sampler's byte tables (dimensions 1-3), set once per process
// and device.
void upload_sobol_tables(cudaStream_t stream) {
    static std::vector<uint32_t> sobol_bytes;
    if (sobol_bytes.empty()) {
        const uint32_t *dirs = sobol_table();
        sobol_bytes.assign(3 * 4 * 256, 0u);
        for (int d = 1; d < 4; d++)
            for (int b = 0; b < 4; b++)
                for (int value = 0; value < 256; value++) {
                    uint32_t x = 0;
                    for (int bit = 0; bit < 8; bit++)
                        if (value & (1 << bit)) x ^= dirs[d * 32 + b * 8 + bit];
                    sobol_bytes[(d - 1) * 1024 + b * 256 + value] = x;
                }
    }
    LR_CUDA(cudaMemcpyToSymbolAsync(g_sobol_bytes, sobol_bytes.data(), sobol_bytes.size() * sizeof(uint32_t), 0,
                                    cudaMemcpyHostToDevice, stream));
}

}  // namespace

// ---- Host side ------------------------------------------------------------------------

// A member as the host keeps it: its device record and block, and where its sampling
// stands (`sample`, `next_pixel`: the next segment to plan; `done`: samples whose last
// pass has finished).
struct MemberHost {
    bool used = false, leaving = false;
    Member dev{};
    void *block = nullptr;  // loaded records: lights, light tree, materials, constants
    void *view = nullptr;   // the view's memory: film, image, splat accumulators
    uint64_t view_pixels = 0;  // pixels the view memory holds
    bool view_traced = false;  // it holds splat accumulators
    bool view_adaptive = false;  // it holds the half estimate and verdicts
    lr_gpu_scene *owned = nullptr;  // a renderer's own upload (null when borrowed)
    // The upload the member traces and the refits of it its record has seen: a refit
    // (refit.cu) moves the root box, which the record holds by value.
    const lr_gpu_scene *source = nullptr;
    uint64_t source_refits = 0;
    uint32_t samples = 0, sample = 0, next_pixel = 0, done = 0;
    uint32_t light_next = 0;  // light paths of the current sample planned so far
    uint32_t max_bounces = 0;
    uint64_t last_pass = 0;  // the last pass (plus one) that traced it; 0: none
    // Passes recorded when its memory and records were last queued (add, restart): a
    // read before a later pass orders itself after those uploads.
    uint64_t placed_at = 0;
    uint64_t read_ticket = 0;  // its latest image read (member_read_async), 0: none
    // Restarts so far (integrator.lucb:572-582): passes of an older generation finish
    // uncounted; and what a restart needs again without reloading.
    uint32_t generation = 0;
    lr_settings settings{};
    size_t emitters = 0;
    double emit_share = 0.0;
};


// Scene-size classes the autotuner keeps a BVH width for: under 16k triangles, under
// 128k, and larger.
constexpr int kSizeClasses = 3;
inline int size_class(uint64_t triangles) { return triangles < 16384 ? 0 : (triangles < 131072 ? 1 : 2); }

struct PassRecord {
    uint64_t number;
    std::vector<std::pair<uint32_t, bool>> members;  // member, sample ended
    std::vector<uint32_t> generations;               // each member's generation at launch
    std::vector<std::pair<cudaEvent_t, int>> marks;  // profiling
    int display_slot = -1;                           // the display image it writes
    uint32_t width = 0, height = 0;                  // the view it shows
};

struct Graph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

// The default first round on the compressed 8-wide tree (WaveHost::thin_from).
constexpr int kThinRound = 3;

// A scene's compressed 8-wide tree as a pass variant's thin code: 1 or 2 for 16 or 32
// group entries, 0 when it has none (a device-built scene, or one too deep or large).
int thin_code(const DeviceScene &s) {
    const TraversalChoice c = choose_traversal(s, 8);
    return c.width != 8 ? 0 : (c.stack <= 16 ? 1 : 2);
}

// One of a wave's two lanes: a path pool with its queues, counters and plan, and the
// stream its passes run on. Consecutive passes take turns on the lanes, so a pass's
// last, thinly populated rounds run while the next pass's first rounds fill the GPU;
// only their film accumulation (finish and convert) is ordered, by an event chain, so
// every pixel still takes its samples in order.
struct Lane {
    void *block = nullptr;
    Wave w{};
    Plan *d_plan = nullptr;
    Plan *h_plan = nullptr;  // pinned staging of the plan
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::map<int, Graph> trace;  // camera and rounds, by variant: width * 1000 + stack
    Graph finish;                // finish and convert
    cudaEvent_t finished = nullptr;  // after its latest pass's convert
    uint64_t members_seen = 0;       // the member uploads its stream has waited for
    uint64_t reads_seen = 0;         // the image reads its film stage has waited for
};

struct WaveHost {
    lr_context *ctx = nullptr;
    uint32_t pool = 0, rounds = 0, capacity = 0;
    int profile = 0;
    void *block = nullptr;  // the member table and stats, shared by the lanes
    Lane lanes[2];
    int lane_count = 2;     // 1 when profiling: kernel times are taken one pass at a time
    // The first round traced on the compressed 8-wide tree when the pass walks the BVH2 and
    // its members have one (-1: every round on the BVH2). The first rounds hold most of a
    // pass's rays and the BVH2 traces them fastest; later rounds hold few, and each is as
    // long as its slowest rays' chains of dependent node fetches, which the 8-wide tree
    // shortens (measured: from round 3, 1,313 against 1,284-1,291 Mrays/s on the headline
    // pass; from round 2 1,294, from round 4 1,298-1,303).
    int thin_from = kThinRound;
    // Whether thin rounds switch for any mix of members (the tuner measured it on the mix)
    // or only when every member is a large scene (the default: measured faster there, and
    // slower for small scenes such as the Cornell box).
    bool thin_any = false;
    Member *d_members = nullptr;
    unsigned long long *d_stats = nullptr;
    std::vector<MemberHost> members;
    uint64_t member_uploads = 0;  // member records queued on the context's stream so far
    int grid_shade = 0, grid_shade_glossy = 0;
    std::map<int, int> grid_trace;  // by variant
    uint64_t recorded = 0, retired = 0;
    cudaEvent_t mark_start[2] = {nullptr, nullptr};
    std::deque<PassRecord> in_flight;
    double kernel_ms[10] = {0};
    uint32_t rotate = 0;  // the member the next plan starts from
    // Tunables (lr_batch_tune): the BVH width asked for each scene-size class (0: the
    // default) and the most paths a pass takes.
    int class_width[kSizeClasses] = {0, 0, 0};
    // ... the traversal kernels' block size (0: kTraceBlock) and the stack entries (0: the
    // members' bound; a larger choice only when the tuner found it faster) per class.
    int class_block[kSizeClasses] = {0, 0, 0};
    int class_stack[kSizeClasses] = {0, 0, 0};
    // Rounds whose outgoing rays the shade kernels group by direction octant: multiples of
    // this (0: none). The wavefront compacts every round (warp- or block-aggregated
    // pushes); this is how often it also sorts.
    uint32_t bin_interval = 0;
    // Idle lanes at which a traversal warp takes new queue entries (0: grid-stride walks).
    uint32_t refill_at = 0;
    uint32_t fill = 0;
    // The most camera paths a pass takes (0: as many as fit): a renderer's band, so that
    // its passes are the reference's bands, light paths riding along in a sample's first.
    uint32_t camera_cap = 0;
    Staging staging;  // member uploads
    // Image reads that overlap the passes after them (member_read_async): copies on their
    // own stream, each after the pass launched last; a film stage launched later waits
    // for them before it rewrites an image.
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t read_done = nullptr;
    uint64_t reads = 0;
    // Ticketed reads (member_read_ticket) in flight, oldest first, with the event each
    // copy records; the newest ticket seen landed; events to reuse.
    std::deque<std::pair<uint64_t, cudaEvent_t>> read_marks;
    uint64_t reads_landed = 0;
    std::vector<cudaEvent_t> spare_marks;
    // A renderer's display images (integrator.lucb:695-713): three rgba16f images of
    // `display_pixels`, the one shown (`front`, -1 none yet) and its size; a pass that ends
    // a sample writes one that is neither shown nor written by a pass in flight, and it
    // is shown once that pass retires in the current generation.
    void *display_block = nullptr;
    uint64_t display_pixels = 0;
    int front = -1;
    uint32_t shown_width = 0, shown_height = 0;
    float display_scale = 1.0f;  // exp2(exposure)
    uint32_t display_view = 0;
    bool display_stale = false;  // set_display since the last conversion
    // Scenes a reload or replacement let go, destroyed once the passes launched before
    // (the number) have retired.
    std::vector<std::pair<uint64_t, lr_gpu_scene *>> retiring_scenes;
};

namespace {

using Marks = std::vector<std::pair<cudaEvent_t, int>>;

void mark(cudaStream_t stream, Marks *marks, int kind) {
    if (!marks) return;
    cudaEvent_t e;
    LR_CUDA(cudaEventCreate(&e));
    LR_CUDA(cudaEventRecord(e, stream));
    marks->push_back({e, kind});
}

// Records a pass's tracing on `stream` with traversal (width, stack entries) in blocks of
// `block` threads: camera, then (closest, shade, shadow) for every round. With `marks`,
// an event follows each kernel (profiling); `count` takes the counting traversals.
void record_trace(const WaveHost *h, const Wave &w, int width, int stack, int block, bool count, bool refill,
                  int grid_trace, bool tracing, bool glossy, bool cutouts, cudaStream_t stream, Marks *marks,
                  int thin_stack, int thin_grid) {
    camera_kernel<<<h->grid_shade, kShadeBlock, 0, stream>>>(w);
    mark(stream, marks, kCamera);
    for (uint32_t round = 0; round < w.rounds; round++) {
        // From round thin_from on (thin queues, latency-bound) the compressed 8-wide tree.
        const bool thin = thin_stack && (int)round >= h->thin_from;
        const int rw = thin ? 8 : width, rs = thin ? thin_stack : stack, rg = thin ? thin_grid : grid_trace;
        launch_closest(rw, rs, block, count, refill, rg, stream, w, round);
        mark(stream, marks, kClosest);
        if (glossy) {
            if (tracing) {
                shade_kernel<true, true, false><<<h->grid_shade_glossy, kShadeBlock, 0, stream>>>(w, round);
                shade_kernel<true, true, true><<<h->grid_shade_glossy, kShadeBlock, 0, stream>>>(w, round);
            } else {
                shade_kernel<false, true, false><<<h->grid_shade_glossy, kShadeBlock, 0, stream>>>(w, round);
            }
        } else if (tracing) {
            shade_kernel<true, false, false><<<h->grid_shade, kShadeBlock, 0, stream>>>(w, round);
            shade_kernel<true, false, true><<<h->grid_shade, kShadeBlock, 0, stream>>>(w, round);
        } else {
            shade_kernel<false, false, false><<<h->grid_shade, kShadeBlock, 0, stream>>>(w, round);
        }
        mark(stream, marks, kSurface);
        launch_shadow(rw, rs, block, count, cutouts, refill, rg, stream, w, round);
        mark(stream, marks, kShadow);
    }
    LR_CUDA(cudaGetLastError());
}

// Records a pass's film accumulation: finish, then convert.
void record_finish(const WaveHost *h, const Wave &w, cudaStream_t stream, Marks *marks) {
    finish_kernel<<<h->grid_shade, kShadeBlock, 0, stream>>>(w);
    mark(stream, marks, kFinish);
    fold_kernel<<<h->grid_shade, kShadeBlock, 0, stream>>>(w);
    mark(stream, marks, kFinish);
    adaptive_kernel<<<h->grid_shade, kShadeBlock, 0, stream>>>(w, 0u);
    adaptive_kernel<<<h->grid_shade, kShadeBlock, 0, stream>>>(w, 1u);
    mark(stream, marks, kAdaptive);
    convert_kernel<<<h->grid_shade, kShadeBlock, 0, stream>>>(w);
    mark(stream, marks, kConvert);
    LR_CUDA(cudaGetLastError());
}

// The traversal kernels' block sizes the autotuner tries; a variant names one by index.
constexpr int kTraceBlocks[3] = {kTraceBlock, 64, 256};

// A pass's variant: its traversal (BVH width * 1000 + stack entries), plus kTracingVariant
// when it holds light tracing, kGlossyVariant when it holds glossy materials,
// kCutoutVariant when it holds cut-outs, kBlockVariant times the index of the traversal
// kernels' block size in kTraceBlocks, kRefillVariant when its traversal warps refill
// idle lanes from the queue, and kThinVariant times 1 or 2 when its later rounds walk the
// compressed 8-wide tree with 16 or 32 group entries.
constexpr int kTracingVariant = 100000, kGlossyVariant = 200000, kCutoutVariant = 400000, kBlockVariant = 800000,
              kRefillVariant = 3 * kBlockVariant, kThinVariant = 2 * kRefillVariant;

int variant_block(int variant) { return kTraceBlocks[(variant / kBlockVariant) % 3]; }

bool traversal_exists(int width, int stack) {
    switch (width * 1000 + stack) {
#define LR_CASE(wd, k) case wd * 1000 + k:
        LR_TRAVERSALS(LR_CASE)
#undef LR_CASE
        return true;
        default: return false;
    }
}

int grid_for(WaveHost *h, int width, int stack, int block, bool refill) {
    const int key = width * 1000 + stack + block * 100000 + (refill ? 100000000 : 0);
    auto it = h->grid_trace.find(key);
    if (it != h->grid_trace.end()) return it->second;
    const int g = closest_grid(width, stack, block, refill, h->ctx->sm_count);
    h->grid_trace[key] = g;
    return g;
}

void record_trace_any(WaveHost *h, const Wave &w, int variant, cudaStream_t stream, Marks *marks) {
    const int flags = (variant / kTracingVariant) & 7;
    const int traversal = variant % kTracingVariant;
    const int width = traversal / 1000, stack = traversal % 1000, block = variant_block(variant);
    const bool count = h->profile >= 2, refill = ((variant / kRefillVariant) & 1) && !count;
    const int grid = grid_for(h, width, stack, block, refill);
    const int thin = variant / kThinVariant;  // 0: none; 1, 2: the 8-wide tree with 16, 32 groups
    const int thin_stack = thin == 1 ? 16 : (thin == 2 ? 32 : 0);
    const int thin_grid = thin_stack ? grid_for(h, 8, thin_stack, block, refill) : 0;
    record_trace(h, w, width, stack, block, count, refill, grid, flags & 1, flags & 2, flags & 4, stream, marks,
                 thin_stack, thin_grid);
}

// Captures whatever `body` queues on a private stream as a graph.
template <class Body>
Graph capture(Body body) {
    Graph g;
    cudaStream_t stream;
    LR_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    LR_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
    body(stream);
    LR_CUDA(cudaStreamEndCapture(stream, &g.graph));
    LR_CUDA(cudaStreamDestroy(stream));
    LR_CUDA(cudaGraphInstantiate(&g.exec, g.graph, 0));
    return g;
}

// The trace graph of `variant` on a lane, captured on first use.
Graph &trace_graph(WaveHost *h, Lane &lane, int variant) {
    auto it = lane.trace.find(variant);
    if (it != lane.trace.end()) return it->second;
    Graph g = capture([&](cudaStream_t s) { record_trace_any(h, lane.w, variant, s, nullptr); });
    return lane.trace.emplace(variant, g).first->second;
}

void destroy_graph(Graph &g) {
    if (g.exec) cudaGraphExecDestroy(g.exec);
    if (g.graph) cudaGraphDestroy(g.graph);
    g = Graph{};
}

// The albedo tables (tables.comp), made once a device on `stream` by its first wave; the
// caller synchronizes the stream before any pass reads them.
void make_albedo_tables(int device, cudaStream_t stream) {
    static std::mutex lock;
    static bool made[64] = {};
    std::lock_guard<std::mutex> guard(lock);
    if (device < 0 || device >= 64) fail(LR_INVALID, "no such CUDA device");
    if (made[device]) return;
    const uint32_t nodes = kTableMu * kTableRoughness * (1u + kTableEta);
    albedo_table_kernel<<<(nodes + 63u) / 64u, 64, 0, stream>>>(0u);
    albedo_table_kernel<<<1, 64, 0, stream>>>(1u);
    LR_CUDA(cudaGetLastError());
    LR_CUDA(cudaStreamSynchronize(stream));
    made[device] = true;
}

// Each lane's path state, ray queues, counters and plan, for the wave's pool and rounds.
void lanes_create(WaveHost *h) {
    lr_context *ctx = h->ctx;
    const uint32_t rounds = h->rounds;
    const uint64_t P = h->pool;
    for (int li = 0; li < h->lane_count; li++) {
        Lane &lane = h->lanes[li];
        Layout L;
        const size_t p_throughput = L.add(nullptr, P * 16), p_radiance = L.add(nullptr, P * 16);
        const size_t p_lambda = L.add(nullptr, P * 16), p_vertex = L.add(nullptr, P * 16);
        const size_t p_path = L.add(nullptr, P * 16), p_mis = L.add(nullptr, P * 16);
        size_t p_ray[2][3];
        for (int q = 0; q < 2; q++)
            for (int j = 0; j < 3; j++) p_ray[q][j] = L.add(nullptr, P * 16);
        const size_t p_shadow_o = L.add(nullptr, P * 16), p_shadow_d = L.add(nullptr, P * 16);
        const size_t p_shadow_c = L.add(nullptr, P * 16);
        const size_t p_counters = L.add(nullptr, (size_t)counter_slots(rounds) * 4);
        const size_t p_plan = L.add(nullptr, sizeof(Plan));
        // Ray records (settings.profile = 3): three float4 per queue entry and round, for
        // the closest-hit and the shadow queue.
        const bool recording = h->profile == kProfileRecord;
        const size_t record_bytes = recording ? (size_t)rounds * P * 48 : 0;
        const size_t p_rec_closest = L.add(nullptr, record_bytes), p_rec_shadow = L.add(nullptr, record_bytes);
        size_t total = 0;
        lane.block = L.allocate(ctx->stream, total);
        char *base = (char *)lane.block;
        auto at = [&](size_t i) { return (void *)(base + L.parts[i].offset); };
        Wave &w = lane.w;
        w.lane = (uint32_t)li;
        w.pool = h->pool;
        w.rounds = rounds;
        w.mis = (float4 *)at(p_mis);
        w.throughput = (float4 *)at(p_throughput);
        w.radiance = (float4 *)at(p_radiance);
        w.lambda = (float4 *)at(p_lambda);
        w.vertex = (float4 *)at(p_vertex);
        w.path = (uint4 *)at(p_path);
        for (int q = 0; q < 2; q++) {
            w.ray_o[q] = (float4 *)at(p_ray[q][0]);
            w.ray_d[q] = (float4 *)at(p_ray[q][1]);
            w.hits[q] = (float4 *)at(p_ray[q][2]);
        }
        w.shadow_o = (float4 *)at(p_shadow_o);
        w.shadow_d = (float4 *)at(p_shadow_d);
        w.shadow_c = (float4 *)at(p_shadow_c);
        w.counters = (uint32_t *)at(p_counters);
        w.stats = h->d_stats;
        w.status = ctx->status;
        w.members = h->d_members;
        lane.d_plan = (Plan *)at(p_plan);
        w.record_closest = recording ? (float4 *)at(p_rec_closest) : nullptr;
        w.record_shadow = recording ? (float4 *)at(p_rec_shadow) : nullptr;
        w.plan = lane.d_plan;
        LR_CUDA(cudaMallocHost((void **)&lane.h_plan, sizeof(Plan)));
        if (li == 0) {
            lane.stream = ctx->stream;
        } else {
            LR_CUDA(cudaStreamCreateWithFlags(&lane.stream, cudaStreamNonBlocking));
            lane.own_stream = true;
        }
        LR_CUDA(cudaEventCreateWithFlags(&lane.finished, cudaEventDisableTiming));
    }
}

// Each lane's film stage as a graph (finish, fold, convert).
void lanes_capture(WaveHost *h) {
    for (int li = 0; li < h->lane_count; li++) {
        Lane &lane = h->lanes[li];
        lane.finish = capture([&](cudaStream_t s) { record_finish(h, lane.w, s, nullptr); });
    }
}

void wave_create(WaveHost *h, lr_context *ctx, uint64_t pool, uint32_t rounds, uint32_t capacity, int profile) {
    if (pool == 0 || rounds == 0 || capacity == 0) fail(LR_INVALID, "a wave needs paths, rounds and members");
    h->ctx = ctx;
    h->pool = (uint32_t)std::min<uint64_t>(pool, kMaxPool);
    h->rounds = rounds;
    h->capacity = capacity;
    h->profile = profile;
    h->lane_count = profile ? 1 : 2;
    // The environment variable LUCE_RENDER_B200_REFILL (1 to 32) sets the idle lanes at
    // which traversal warps refill until a tuner chooses, for measurement.
    if (const char *env = std::getenv("LUCE_RENDER_B200_REFILL")) {
        const int v = std::atoi(env);
        if (v >= 1 && v <= 32) h->refill_at = (uint32_t)v;
    }
    // LUCE_RENDER_B200_THIN (-1 to 15) sets the first thin round on the 8-wide tree, for any
    // mix of members, for measurement.
    if (const char *env = std::getenv("LUCE_RENDER_B200_THIN")) {
        const int v = std::atoi(env);
        if (v >= -1 && v <= 15) {
            h->thin_from = v;
            h->thin_any = true;
        }
    }
    // LUCE_RENDER_B200_BIN (0, 1 or 2) sets the rounds between octant sorts of outgoing rays
    // until a tuner chooses, for measurement.
    if (const char *env = std::getenv("LUCE_RENDER_B200_BIN")) {
        const int v = std::atoi(env);
        if (v >= 0 && v <= 2) h->bin_interval = (uint32_t)v;
    }
    // LUCE_RENDER_B200_TRACE_BLOCK (64, 128 or 256) sets the traversal kernels' block size
    // of every size class until a tuner chooses, for measurement.
    if (const char *env = std::getenv("LUCE_RENDER_B200_TRACE_BLOCK")) {
        const int v = std::atoi(env);
        if (v == 64 || v == 128 || v == 256)
            for (int &b : h->class_block) b = v;
    }
    LR_CUDA(cudaSetDevice(ctx->device));
    {
        Layout L;
        const size_t p_stats = L.add(nullptr, 8 * 8);
        const size_t p_members = L.add(nullptr, (size_t)capacity * sizeof(Member));
        size_t total = 0;
        h->block = L.allocate(ctx->stream, total);
        h->d_stats = (unsigned long long *)((char *)h->block + L.parts[p_stats].offset);
        h->d_members = (Member *)((char *)h->block + L.parts[p_members].offset);
    }
    lanes_create(h);
    upload_sobol_tables(ctx->stream);
    make_albedo_tables(ctx->device, ctx->stream);
    LR_CUDA(cudaStreamSynchronize(ctx->stream));
    h->grid_shade = grid_of(shade_kernel<false, false, false>, kShadeBlock, ctx->sm_count);
    h->grid_shade_glossy = grid_of(shade_kernel<false, true, false>, kShadeBlock, ctx->sm_count);
    if (profile)
        for (auto &e : h->mark_start) LR_CUDA(cudaEventCreate(&e));
    else
        lanes_capture(h);
    h->members.resize(capacity);
}

void settle(WaveHost *h);

void validate(const lr_settings &s, const lr_frame &f) {
    if (f.width == 0 || f.height == 0 || f.width > 16384 || f.height > 16384)
        fail(LR_INVALID, "an image is 1 to 16384 pixels on a side");
    if (s.samples == 0 || s.max_bounces == 0 || s.max_bounces > 1024)
        fail(LR_INVALID, "a render needs samples and 1 to 1024 bounces");
    if (s.guiding) fail(LR_INVALID, "path guiding is not part of this build (guiding off)");
    if (s.max_bounces > 253) fail(LR_INVALID, "this build traces at most 253 bounces");
}

// Loaded.light_paths (loading.lucb:163-168): light tracing's share of a view's pixels (at
// least one), at most a band's (the pool setting, or every pixel when fewer), and the band
// their sampler numbers follow. None for an orthographic camera, or a scene with neither
// emitters of the light tree nor light paths from afar (loading.lucb:149).
struct LightPaths {
    uint32_t count = 0, band = 0;
    double pixel_area_inv = 0.0;
};

LightPaths light_paths_of(const lr_settings &settings, const lr_frame &frame, uint64_t pixels, size_t emitters,
                          bool afar) {
    LightPaths out;
    const uint64_t pool = settings.pool ? settings.pool : kDefaultPool;
    out.band = (uint32_t)std::min<uint64_t>(pool, pixels);
    if (!(settings.light_tracing > 0.0) || frame.orthographic || (emitters == 0 && !afar)) return out;
    const double wanted = std::max(1.0, std::floor(settings.light_tracing * (double)pixels + 0.5));
    out.count = (uint32_t)std::min<double>(wanted, (double)out.band);
    const double du = std::sqrt(frame.du[0] * frame.du[0] + frame.du[1] * frame.du[1] + frame.du[2] * frame.du[2]);
    const double dv = std::sqrt(frame.dv[0] * frame.dv[0] + frame.dv[1] * frame.dv[1] + frame.dv[2] * frame.dv[2]);
    out.pixel_area_inv = du * dv > 0.0 ? 1.0 / (du * dv) : 0.0;
    return out;
}

// Gives `lay`'s parts their offsets (256-byte aligned); returns the block's size.
size_t lay_out(Layout &lay) {
    size_t total = 0;
    for (auto &p : lay.parts) {
        p.offset = total;
        total += align256(std::max<size_t>(p.bytes, 64));
    }
    return total;
}

// Lays out `lay` as one zeroed stream-ordered block on `stream` and copies the parts
// that have a source through the pinned `stage`, from `stage_at` on.
void *place(Layout &lay, cudaStream_t stream, char *stage, size_t &stage_at) {
    const size_t total = lay_out(lay);
    void *block = nullptr;
    LR_CUDA(cudaMallocAsync(&block, total, stream));
    char *base = (char *)block;
    LR_CUDA(cudaMemsetAsync(base, 0, total, stream));
    for (auto &p : lay.parts) {
        if (!p.src || !p.bytes) continue;
        std::memcpy(stage + stage_at, p.src, p.bytes);
        LR_CUDA(cudaMemcpyAsync(base + p.offset, stage + stage_at, p.bytes, cudaMemcpyHostToDevice, stream));
        stage_at += align256(p.bytes);
    }
    return block;
}

size_t staged_bytes(const Layout &lay) {
    size_t bytes = 0;
    for (const auto &p : lay.parts)
        if (p.src) bytes += align256(p.bytes);
    return bytes;
}

// A member's loaded records from `L`, in the layouts the kernels read: the emitter table
// (lights, the finite and from-afar index lists, the textured dome's image), the light
// tree's pair records, emitter records and triangle map, the per-material codes, the
// constants. The vectors hold the host copies until they are staged.
struct LoadedRecords {
    Constants k{};
    Layout lay;
    DeviceLights lights;
    DeviceTree tree;
    std::vector<float> codes;
    size_t p_lights = 0, p_finite = 0, p_afar = 0, p_texels = 0, p_cdf = 0, p_pairs = 0, p_records = 0, p_map = 0,
           p_codes = 0, p_constants = 0;
};

void loaded_records(const Loaded &L, const lr_settings &settings, double emit_share, LoadedRecords &r) {
    Constants &k = r.k;
    for (int i = 0; i < 9; i++) k.film[i] = (float)L.film.m[i];
    k.cmf_integrals[0] = (float)L.cmf_integrals.x;
    k.cmf_integrals[1] = (float)L.cmf_integrals.y;
    k.cmf_integrals[2] = (float)L.cmf_integrals.z;
    k.limits[0] = (float)settings.diffuse_bounces;
    k.limits[1] = (float)settings.glossy_bounces;
    k.limits[2] = (float)settings.transmission_bounces;
    k.clamp_indirect = (float)settings.clamp_indirect;
    k.background_fit = make_float4((float)L.background_fit[0], (float)L.background_fit[1], (float)L.background_fit[2],
                                   (float)L.background_fit[3]);
    k.background_rgb = make_float3((float)settings.background[0], (float)settings.background[1], (float)settings.background[2]);
    k.p_distant = (float)L.p_distant;
    k.max_bounces = settings.max_bounces;
    k.light_count = (uint32_t)L.lights.count;
    k.tree_nodes = (uint32_t)L.tree.node_count;
    k.seed = settings.seed;
    k.emit_share = (float)emit_share;
    k.emit_radius = (float)L.emit_radius;
    k.emit_center = make_float3((float)L.emit_center.x, (float)L.emit_center.y, (float)L.emit_center.z);
    k.noise_threshold = (float)std::max(0.0, settings.noise_threshold);
    r.lights = device_lights(L.lights);
    r.tree = device_tree(L.tree);
    for (const lr_openpbr &material : L.library) material_code(material, r.codes);
    static_assert(sizeof(DeviceLight) == 32 * 4 && sizeof(TreePair) == 24 * 4 && sizeof(MaterialCode) == 64 * 4,
                  "device record sizes");
    r.p_lights = r.lay.add(r.lights.records.data(), r.lights.records.size() * 4);
    r.p_finite = r.lay.add(r.lights.finite.data(), r.lights.finite.size() * 4);
    r.p_afar = r.lay.add(r.lights.afar.data(), r.lights.afar.size() * 4);
    r.p_texels = r.lay.add(r.lights.dome_texels.data(), r.lights.dome_texels.size() * 4);
    r.p_cdf = r.lay.add(r.lights.dome_cdf.data(), r.lights.dome_cdf.size() * 4);
    r.p_pairs = r.lay.add(r.tree.pairs.data(), r.tree.pairs.size() * 4);
    r.p_records = r.lay.add(L.tree.records.data(), L.tree.records.size() * 4);
    r.p_map = r.lay.add(L.tree.triangle_map.data(), L.tree.triangle_map.size() * 4);
    r.p_codes = r.lay.add(r.codes.data(), r.codes.size() * 4);
    r.p_constants = r.lay.add(&k, sizeof k);
}

// Points `m` at its loaded records in `block`.
void set_loaded(Member &m, const LoadedRecords &r, const Loaded &L, void *block, const lr_settings &settings,
                uint32_t rounds) {
    auto at = [&](size_t i) { return (void *)((char *)block + r.lay.parts[i].offset); };
    LightTable &T = m.lights;
    T = LightTable{};
    T.light = (const DeviceLight *)at(r.p_lights);
    T.count = (uint32_t)L.lights.count;
    T.finite = (const uint32_t *)at(r.p_finite);
    T.finite_count = (uint32_t)r.lights.finite.size();
    T.afar = (const uint32_t *)at(r.p_afar);
    T.afar_count = (uint32_t)r.lights.afar.size();
    if (r.lights.dome_light != kNone) {
        T.dome.texels = (const float4 *)at(r.p_texels);
        T.dome.cdf = (const float *)at(r.p_cdf);
        T.dome.width = r.lights.dome_width;
        T.dome.height = r.lights.dome_height;
        T.dome.light = r.lights.dome_light;
        T.dome.weight_sum = r.lights.dome_weight_sum;
    }
    m.spectral = settings.spectral ? 1u : 0u;
    m.tree = TreeTable{};
    m.tree.pairs = (const TreePair *)at(r.p_pairs);
    m.tree.records = (const uint4 *)at(r.p_records);
    m.tree.triangle_map = L.tree.triangle_map.empty() ? nullptr : (const uint32_t *)at(r.p_map);
    m.tree.root = r.tree.root;
    m.materials = (const MaterialCode *)at(r.p_codes);
    m.k = (const Constants *)at(r.p_constants);
    m.glossy = L.glossy ? 1u : 0u;
    m.cutouts = L.cutouts ? 1u : 0u;
    m.rounds = rounds;
}

// The view's memory for `pixels`: film, image and, for light tracing, the splat
// accumulators (the film's and one per lane); for adaptive sampling, the half estimate
// and the verdicts.
constexpr int kViewParts = 7;
Layout view_layout(uint64_t pixels, bool traced, bool adaptive, size_t parts[kViewParts]) {
    Layout lay;
    parts[0] = lay.add(nullptr, pixels * 16);
    parts[1] = lay.add(nullptr, pixels * 16);
    const size_t splat_bytes = traced ? pixels * 24 : 0;
    for (int i = 2; i < 5; i++) parts[i] = lay.add(nullptr, splat_bytes);
    parts[5] = lay.add(nullptr, adaptive ? pixels * 16 : 0);
    parts[6] = lay.add(nullptr, adaptive ? pixels * 4 : 0);
    return lay;
}

void set_view_memory(Member &m, const Layout &lay, const size_t parts[kViewParts], void *view, bool traced,
                     bool adaptive) {
    auto at = [&](size_t i) { return (void *)((char *)view + lay.parts[i].offset); };
    m.film = (float4 *)at(parts[0]);
    m.image = (float4 *)at(parts[1]);
    m.splat = traced ? (unsigned long long *)at(parts[2]) : nullptr;
    m.splat_lane[0] = traced ? (unsigned long long *)at(parts[3]) : nullptr;
    m.splat_lane[1] = traced ? (unsigned long long *)at(parts[4]) : nullptr;
    m.half = adaptive ? (float4 *)at(parts[5]) : nullptr;
    m.scratch = adaptive ? (float *)at(parts[6]) : nullptr;
}

// The view `m` renders: its frame, size and light paths.
void set_view(Member &m, const lr_frame &frame, const LightPaths &traced) {
    pack_frame(frame, m.frame);
    m.lens_radius = (float)frame.lens_radius;
    m.focus_distance = (float)frame.focus_distance;
    for (int i = 0; i < 3; i++) m.forward[i] = (float)frame.forward[i];
    m.width = frame.width;
    m.height = frame.height;
    m.pixels = (uint64_t)frame.width * frame.height;
    m.light_paths = traced.count;
    m.light_band = traced.band;
    m.pixel_area_inv = (float)traced.pixel_area_inv;
}

uint32_t rounds_of(const lr_scene &scene, const lr_settings &settings) {
    return settings.max_bounces + 1 + (has_cutouts(scene, settings) ? kCutoutRounds : 0);
}

void check_rounds(const WaveHost *h, uint32_t rounds) {
    if (rounds > h->rounds)
        fail(LR_LIMIT, "this wave traces " + std::to_string(h->rounds) + " rounds a pass; the render needs " +
                           std::to_string(rounds) + " (its bounces + 1, + " + std::to_string(kCutoutRounds) +
                           " with cut-outs)");
}

// Makes `scene` (uploaded as `gs`) seen through `frame` a member; returns its index.
uint32_t member_add(WaveHost *h, const lr_gpu_scene *gs, lr_gpu_scene *owned, const lr_scene *scene,
                    const lr_settings &settings, const lr_frame &frame) {
    validate(settings, frame);
    const uint32_t rounds = rounds_of(*scene, settings);
    check_rounds(h, rounds);
    if (!gs->ctx || gs->ctx->device != h->ctx->device) fail(LR_INVALID, "the scene was uploaded to another device");
    auto free_slot = [&] {
        for (uint32_t i = 0; i < h->capacity; i++)
            if (!h->members[i].used) return i;
        return h->capacity;
    };
    uint32_t index = free_slot();
    if (index == h->capacity && std::any_of(h->members.begin(), h->members.end(),
                                            [](const MemberHost &m) { return m.used && m.leaving; })) {
        // A member that left holds its slot until its passes finish: wait for them.
        settle(h);
        index = free_slot();
    }
    if (index == h->capacity) fail(LR_LIMIT, "the wave holds " + std::to_string(h->capacity) + " members");
    const Loaded L = load(*scene, settings);
    const uint64_t pixels = (uint64_t)frame.width * frame.height;
    const double emit_share = frame.orthographic ? 0.0 : L.emit_share;
    const LightPaths traced = light_paths_of(settings, frame, pixels, L.tree.emitter_count, emit_share > 0.0);
    LoadedRecords records;
    loaded_records(L, settings, emit_share, records);
    const bool adaptive = settings.noise_threshold > 0.0;
    size_t view_parts[kViewParts];
    Layout view = view_layout(pixels, traced.count > 0, adaptive, view_parts);
    MemberHost &mh = h->members[index];
    // Stream-ordered: the member's memory and data arrive ahead of the next pass without
    // waiting for the passes in flight.
    cudaStream_t stream = h->ctx->stream;
    char *stage = h->staging.take(sizeof(Member) + staged_bytes(records.lay) + staged_bytes(view));
    size_t stage_at = sizeof(Member);
    mh.block = place(records.lay, stream, stage, stage_at);
    mh.view = place(view, stream, stage, stage_at);
    Member &m = mh.dev;
    m = Member{};
    m.scene = gs->scene;
    mh.source = gs;
    mh.source_refits = gs->refits;
    set_loaded(m, records, L, mh.block, settings, rounds);
    set_view_memory(m, view, view_parts, mh.view, traced.count > 0, adaptive);
    set_view(m, frame, traced);
    std::memcpy(stage, &m, sizeof m);
    LR_CUDA(cudaMemcpyAsync(h->d_members + index, stage, sizeof m, cudaMemcpyHostToDevice, stream));
    h->staging.queued(stream);
    h->member_uploads++;
    mh.used = true;
    mh.leaving = false;
    mh.owned = owned;
    mh.samples = settings.samples;
    mh.sample = mh.next_pixel = mh.done = mh.light_next = 0;
    mh.max_bounces = settings.max_bounces;
    mh.last_pass = 0;
    mh.placed_at = h->recorded;
    mh.read_ticket = 0;
    mh.view_pixels = pixels;
    mh.view_traced = traced.count > 0;
    mh.view_adaptive = adaptive;
    mh.settings = settings;
    mh.emitters = L.tree.emitter_count;
    mh.emit_share = L.emit_share;
    return index;
}

MemberHost &member_at(WaveHost *h, uint32_t member);

// Orders the context's stream after every pass launched so far: what it does next (frees,
// record uploads, clears) does not overtake them.
void after_passes(WaveHost *h) {
    if (h->recorded == 0) return;
    for (int li = 0; li < h->lane_count; li++) {
        Lane &lane = h->lanes[li];
        if (lane.stream != h->ctx->stream) LR_CUDA(cudaStreamWaitEvent(h->ctx->stream, lane.finished, 0));
    }
}

// A view memory a restarted or reloaded view can grow into: a quarter more pixels each
// way than asked (integrator.lucb:478-482), so that a window resized a few pixels at a
// time makes it again seldom.
uint64_t roomy_pixels(const lr_frame &frame) {
    const uint64_t w = frame.width + frame.width / 4, h = frame.height + frame.height / 4;
    return w * h;
}

// Renderer.restart / reload / replace_scene (integrator.lucb:463-582) for member `index`:
// the view through `frame`, and when `scene` is given its records loaded again from it
// and `settings` (the geometry `gs`, its upload when `owned`). Passes in flight finish
// uncounted (a new generation), the film starts over, and nothing waits for the device:
// the member's new records, its cleared or new memory and the release of the old follow
// the passes launched so far on the context's stream.
void member_renew(WaveHost *h, uint32_t index, const lr_frame &frame, const lr_scene *scene, const lr_settings *settings,
                  const lr_gpu_scene *gs, lr_gpu_scene *owned) {
    MemberHost &mh = member_at(h, index);
    const lr_settings &chosen = settings ? *settings : mh.settings;
    validate(chosen, frame);
    cudaStream_t stream = h->ctx->stream;
    std::unique_ptr<Loaded> L;
    LoadedRecords records;
    uint32_t rounds = mh.dev.rounds;
    size_t emitters = mh.emitters;
    double emit_share = mh.emit_share;
    if (scene) {
        rounds = rounds_of(*scene, chosen);
        check_rounds(h, rounds);
        L = std::make_unique<Loaded>(load(*scene, chosen));
        emitters = L->tree.emitter_count;
        emit_share = L->emit_share;
        loaded_records(*L, chosen, frame.orthographic ? 0.0 : emit_share, records);
    }
    const uint64_t pixels = (uint64_t)frame.width * frame.height;
    const LightPaths traced = light_paths_of(chosen, frame, pixels, emitters, !frame.orthographic && emit_share > 0.0);
    const bool adaptive = chosen.noise_threshold > 0.0;
    const bool new_view = pixels > mh.view_pixels || (traced.count > 0 && !mh.view_traced) || (adaptive && !mh.view_adaptive);
    size_t view_parts[kViewParts];
    const uint64_t capacity = new_view ? roomy_pixels(frame) : mh.view_pixels;
    const bool view_traced = new_view ? traced.count > 0 : mh.view_traced;
    const bool view_adaptive = new_view ? adaptive : mh.view_adaptive;
    Layout view = view_layout(capacity, view_traced, view_adaptive, view_parts);
    lay_out(view);
    char *stage = h->staging.take(sizeof(Member) + (scene ? staged_bytes(records.lay) : 0));
    size_t stage_at = sizeof(Member);
    after_passes(h);
    Member m = mh.dev;
    if (scene) {
        void *block = place(records.lay, stream, stage, stage_at);
        LR_CUDA(cudaFreeAsync(mh.block, stream));
        mh.block = block;
        m.scene = gs->scene;
        mh.source = gs;
        mh.source_refits = gs->refits;
        set_loaded(m, records, *L, block, chosen, rounds);
    }
    if (new_view) {
        if (h->read_done) LR_CUDA(cudaStreamWaitEvent(stream, h->read_done, 0));
        void *fresh = place(view, stream, stage, stage_at);
        LR_CUDA(cudaFreeAsync(mh.view, stream));
        mh.view = fresh;
        mh.view_pixels = capacity;
        mh.view_traced = view_traced;
        mh.view_adaptive = view_adaptive;
    } else {
        // The film starts over; the image keeps the last one until a sample replaces it.
        LR_CUDA(cudaMemsetAsync((char *)mh.view + view.parts[view_parts[0]].offset, 0, pixels * 16, stream));
        if (view_traced)
            LR_CUDA(cudaMemsetAsync((char *)mh.view + view.parts[view_parts[2]].offset, 0, pixels * 24, stream));
        if (view_adaptive)
            LR_CUDA(cudaMemsetAsync((char *)mh.view + view.parts[view_parts[5]].offset, 0, pixels * 16, stream));
    }
    set_view_memory(m, view, view_parts, mh.view, view_traced, view_adaptive);
    set_view(m, frame, traced);
    if (!traced.count) m.splat = m.splat_lane[0] = m.splat_lane[1] = nullptr;
    if (!adaptive) m.half = nullptr, m.scratch = nullptr;
    mh.dev = m;
    std::memcpy(stage, &m, sizeof m);
    LR_CUDA(cudaMemcpyAsync(h->d_members + index, stage, sizeof m, cudaMemcpyHostToDevice, stream));
    h->staging.queued(stream);
    h->member_uploads++;
    if (owned && owned != mh.owned) {
        if (mh.owned) h->retiring_scenes.push_back({h->recorded, mh.owned});
        mh.owned = owned;
    }
    mh.generation++;
    mh.placed_at = h->recorded;
    mh.sample = mh.next_pixel = mh.done = mh.light_next = 0;
    mh.settings = chosen;
    mh.samples = chosen.samples;
    mh.max_bounces = chosen.max_bounces;
    mh.emitters = emitters;
    mh.emit_share = emit_share;
}

// The event of read `ticket` while it may still be in flight, else null.
cudaEvent_t read_in_flight(WaveHost *h, uint64_t ticket);

void member_free(WaveHost *h, MemberHost &mh, cudaStream_t stream) {
    // A read of the member's image still in flight finishes first.
    if (h && mh.read_ticket)
        if (cudaEvent_t e = read_in_flight(h, mh.read_ticket)) cudaStreamWaitEvent(stream, e, 0);
    if (mh.block) cudaFreeAsync(mh.block, stream);
    if (mh.view) cudaFreeAsync(mh.view, stream);
    if (mh.owned) lr_gpu_scene_destroy(mh.owned);
    mh = MemberHost{};
}

// Frees members that asked to leave once no pass in flight traces them.
void collect(WaveHost *h) {
    for (auto &mh : h->members)
        if (mh.used && mh.leaving && mh.last_pass <= h->retired) member_free(h, mh, h->ctx->stream);
}

bool has_work(const MemberHost &mh) { return mh.used && !mh.leaving && mh.sample < mh.samples; }

Lane &lane_of(WaveHost *h, uint64_t pass) { return h->lanes[pass % (uint64_t)h->lane_count]; }

// Paths in the plan of the pass launched last.
uint64_t h_plan_paths(WaveHost *h) { return lane_of(h, h->recorded - 1).h_plan->head.paths; }

// Retires the oldest pass in flight if it has finished (integrator.lucb:622-645).
bool retire_one(WaveHost *h, bool wait) {
    if (h->in_flight.empty()) return false;
    PassRecord &p = h->in_flight.front();
    cudaEvent_t e = lane_of(h, p.number).finished;
    if (wait) {
        LR_CUDA(cudaEventSynchronize(e));
    } else {
        cudaError_t q = cudaEventQuery(e);
        if (q == cudaErrorNotReady) return false;
        LR_CUDA(q);
    }
    if (h->profile && !p.marks.empty()) {
        cudaEvent_t prev = h->mark_start[p.number & 1];
        for (auto &[ev, kind] : p.marks) {
            float t = 0.0f;
            LR_CUDA(cudaEventElapsedTime(&t, prev, ev));
            h->kernel_ms[kind] += t;
            prev = ev;
        }
        for (auto &[ev, kind] : p.marks) cudaEventDestroy(ev);
    }
    bool current = true;
    for (size_t i = 0; i < p.members.size(); i++) {
        const auto &[m, ended] = p.members[i];
        if (h->members[m].generation != p.generations[i]) {
            current = false;  // launched before a restart: counts for nothing
            continue;
        }
        if (ended) h->members[m].done++;
    }
    if (p.display_slot >= 0 && current) {
        h->front = p.display_slot;
        h->shown_width = p.width;
        h->shown_height = p.height;
    }
    h->retired = p.number + 1;
    h->in_flight.pop_front();
    collect(h);
    for (size_t i = 0; i < h->retiring_scenes.size();) {
        if (h->retiring_scenes[i].first <= h->retired) {
            lr_gpu_scene_destroy(h->retiring_scenes[i].second);
            h->retiring_scenes.erase(h->retiring_scenes.begin() + (long)i);
        } else {
            i++;
        }
    }
    return true;
}

void settle(WaveHost *h) {
    while (!h->in_flight.empty()) retire_one(h, true);
}

// A renderer's display image `slot`.
void *display_image(WaveHost *h, int slot) {
    return (char *)h->display_block + (size_t)slot * align256(h->display_pixels * 8);
}

// A display image neither shown nor written by a pass in flight (of three, with at most
// two passes in flight, one is always free).
int free_display_slot(WaveHost *h) {
    for (int slot = 0; slot < 3; slot++) {
        if (slot == h->front) continue;
        bool busy = false;
        for (const PassRecord &p : h->in_flight) busy = busy || p.display_slot == slot;
        if (!busy) return slot;
    }
    return h->front;
}

// Plans and launches one pass: each member with work left adds its next segment, in
// turn from `rotate`, until the pass holds `fill` paths. A member takes one segment a
// pass at most, so a pixel never gets two samples in one pass. A dry pass (autotuning)
// plans the same way, from the members of size class `only` when it is not -1, but
// moves no member on and leaves the films alone. Returns false with no work.
// Members whose upload was refit since their record was made take its new scene record
// (root boxes) ahead of the next pass, stream-ordered like any member upload. Their
// loaded records (light tree, scene radius) stay as they were loaded: still an unbiased
// estimator, as each pdf comes from the same records that sample it.
void follow_refits(WaveHost *h) {
    for (size_t i = 0; i < h->members.size(); i++) {
        MemberHost &mh = h->members[i];
        if (!mh.used || !mh.source || mh.source->refits == mh.source_refits) continue;
        mh.dev.scene = mh.source->scene;
        mh.source_refits = mh.source->refits;
        const size_t at = (size_t)((const char *)&mh.dev.scene - (const char *)&mh.dev);
        char *stage = h->staging.take(sizeof(DeviceScene));
        std::memcpy(stage, &mh.dev.scene, sizeof(DeviceScene));
        LR_CUDA(cudaMemcpyAsync((char *)(h->d_members + i) + at, stage, sizeof(DeviceScene), cudaMemcpyHostToDevice,
                                h->ctx->stream));
        h->staging.queued(h->ctx->stream);
        h->member_uploads++;
    }
}

bool launch_pass(WaveHost *h, bool dry = false, int only = -1) {
    follow_refits(h);
    Lane &lane = lane_of(h, h->recorded);
    Plan *staging = lane.h_plan;
    Segment *seg = staging->seg;
    uint32_t n = 0, used = 0, converts = 0, camera_paths = 0, folds = 0, adapts = 0;
    uint64_t class_paths[kSizeClasses] = {0, 0, 0};
    PassRecord rec;
    rec.number = h->recorded;
    const uint32_t cap = h->capacity;
    const uint32_t fill = h->fill ? std::min(h->fill, h->pool) : h->pool;
    uint32_t last = h->rotate;
    for (uint32_t step = 0; step < cap && used < fill && n + 2 <= kMaxSegments; step++) {
        const uint32_t index = (h->rotate + step) % cap;
        MemberHost &mh = h->members[index];
        if (!has_work(mh)) continue;
        const int cls = size_class(mh.dev.scene.triangle_count);
        if (only >= 0 && cls != only) continue;
        // The light paths of the member's current sample come first, and its camera paths
        // end the sample only in a pass that plans the last of them: the pass that ends a
        // sample folds every splat of it before it converts the image.
        const uint32_t lights = mh.dev.light_paths;
        uint32_t light_next = mh.light_next;
        if (light_next < lights) {
            const uint32_t count = std::min(lights - light_next, fill - used);
            seg[n++] = Segment{index, light_next, count, mh.sample, used, 0u, kLightSegment, used - camera_paths};
            staging->fold[folds++] = index;
            used += count;
            light_next += count;
            class_paths[cls] += count;
        }
        const uint64_t left = mh.dev.pixels - mh.next_pixel;
        uint32_t count = (uint32_t)std::min<uint64_t>(left, fill - used);
        if (h->camera_cap) count = std::min(count, h->camera_cap);
        if (count == left && light_next < lights) count = (uint32_t)left - 1;
        const bool ends = count > 0 && count == left && !dry;
        rec.members.push_back({index, ends});
        rec.generations.push_back(mh.generation);
        if (count > 0) {
            seg[n++] = Segment{index, mh.next_pixel, count, mh.sample, used, ends ? 1u : 0u, kCameraSegment, camera_paths};
            if (ends) {
                staging->convert[converts] = index;
                staging->convert_samples[converts++] = mh.sample + 1;
                // After every 4th sample past the minimum, check which pixels converged
                // (integrator.lucb:819-826).
                const uint32_t taken = mh.sample + 1;
                if (mh.dev.half && taken >= mh.settings.adaptive_minimum && taken % 4u == 0u) staging->adapt[adapts++] = index;
            }
            used += count;
            camera_paths += count;
            class_paths[cls] += count;
        }
        if (!dry) {
            mh.light_next = light_next;
            if (count > 0 && count == left) {
                mh.sample++;
                mh.next_pixel = 0;
                mh.light_next = 0;
            } else {
                mh.next_pixel += count;
            }
        }
        mh.last_pass = h->recorded + 1;
        last = index;
    }
    if (n == 0) return false;
    if (!dry) h->rotate = (last + 1) % cap;
    // One traversal variant serves the pass: the width tuned for the size class holding
    // most of its paths, with the deepest stack among its members -- or the BVH2 when a
    // member's stack bound does not fit that width.
    const int dominant = (int)(std::max_element(class_paths, class_paths + kSizeClasses) - class_paths);
    int width = choose_traversal(h->members[rec.members[0].first].dev.scene, h->class_width[dominant]).width;
    int stack = 32;
    for (int attempt = 0; attempt < 2; attempt++) {
        bool fits = true;
        stack = 32;
        for (auto &[m, ended] : rec.members) {
            const TraversalChoice c = choose_traversal(h->members[m].dev.scene, width);
            if (c.width != width) fits = false;
            stack = std::max(stack, c.stack);
        }
        if (fits || width == 2) break;
        width = 2;
    }
    const bool tracing = std::any_of(rec.members.begin(), rec.members.end(),
                                     [&](const std::pair<uint32_t, bool> &e) { return h->members[e.first].dev.light_paths != 0u; });
    const bool glossy = std::any_of(rec.members.begin(), rec.members.end(),
                                    [&](const std::pair<uint32_t, bool> &e) { return h->members[e.first].dev.glossy != 0u; });
    const bool cutouts = std::any_of(rec.members.begin(), rec.members.end(),
                                     [&](const std::pair<uint32_t, bool> &e) { return h->members[e.first].dev.cutouts != 0u; });
    // The class's tuned stack, where the width's variants offer it and it holds the bound.
    const int tuned_stack = h->class_stack[dominant];
    if (tuned_stack > stack && traversal_exists(width, tuned_stack)) stack = tuned_stack;
    const int block = h->class_block[dominant] ? h->class_block[dominant] : kTraceBlock;
    const int block_index = block == kTraceBlocks[1] ? 1 : (block == kTraceBlocks[2] ? 2 : 0);
    // Thin rounds on the compressed 8-wide tree, where every member has one -- except in
    // counting passes (settings.profile 2), whose visits and tests are the BVH2's work.
    int thin = 0;
    const bool all_large = std::all_of(rec.members.begin(), rec.members.end(), [&](const std::pair<uint32_t, bool> &e) {
        return size_class(h->members[e.first].dev.scene.triangle_count) == kSizeClasses - 1;
    });
    if (h->thin_from >= 0 && width == 2 && h->profile < 2 && (h->thin_any || all_large)) {
        // The deepest stack any member needs; none when a member has no such tree.
        for (auto &[m, ended] : rec.members) {
            const int code = thin_code(h->members[m].dev.scene);
            if (code == 0) {
                thin = 0;
                break;
            }
            thin = std::max(thin, code);
        }
    }
    const int variant = width * 1000 + stack + (tracing ? kTracingVariant : 0) + (glossy ? kGlossyVariant : 0) +
                        (cutouts ? kCutoutVariant : 0) + block_index * kBlockVariant +
                        (h->refill_at ? kRefillVariant : 0) + thin * kThinVariant;
    staging->head = PlanHeader{n, used, converts, dry ? 1u : 0u, camera_paths, folds, adapts, h->bin_interval,
                               h->refill_at, {0u, 0u, 0u}};
    staging->display = PlanDisplay{0ull, h->display_scale, h->display_view, 0u, 0u};
    if (h->display_block && converts > 0) {
        rec.display_slot = free_display_slot(h);
        staging->display.image = (unsigned long long)display_image(h, rec.display_slot);
        const MemberHost &shown = h->members[staging->convert[0]];
        rec.width = shown.dev.width;
        rec.height = shown.dev.height;
        h->display_stale = false;
    }
    cudaStream_t stream = lane.stream;
    // Member records queued on the context's stream reach this lane first.
    if (stream != h->ctx->stream && lane.members_seen != h->member_uploads && h->staging.copied) {
        LR_CUDA(cudaStreamWaitEvent(stream, h->staging.copied, 0));
        lane.members_seen = h->member_uploads;
    }
    // The header and convert list, then the segments in use.
    LR_CUDA(cudaMemcpyAsync(lane.d_plan, staging, offsetof(Plan, seg) + n * sizeof(Segment), cudaMemcpyHostToDevice,
                            stream));
    // Film accumulation waits for the previous pass's, which ran on the other lane.
    Lane *before = rec.number > 0 && h->lane_count > 1 ? &lane_of(h, rec.number - 1) : nullptr;
    // The film stage rewrites images: it waits for the reads queued since this lane's last.
    auto after_reads = [&] {
        if (lane.reads_seen != h->reads) {
            LR_CUDA(cudaStreamWaitEvent(stream, h->read_done, 0));
            lane.reads_seen = h->reads;
        }
    };
    if (h->profile) {
        LR_CUDA(cudaEventRecord(h->mark_start[rec.number & 1], stream));
        record_trace_any(h, lane.w, variant, stream, &rec.marks);
        if (before) LR_CUDA(cudaStreamWaitEvent(stream, before->finished, 0));
        after_reads();
        record_finish(h, lane.w, stream, &rec.marks);
    } else {
        LR_CUDA(cudaGraphLaunch(trace_graph(h, lane, variant).exec, stream));
        if (before) LR_CUDA(cudaStreamWaitEvent(stream, before->finished, 0));
        after_reads();
        LR_CUDA(cudaGraphLaunch(lane.finish.exec, stream));
    }
    LR_CUDA(cudaEventRecord(lane.finished, stream));
    h->in_flight.push_back(std::move(rec));
    h->recorded++;
    return true;
}

// Orders the context's stream after every pass launched so far (their films and images).
void join_lanes(WaveHost *h) {
    if (h->recorded == 0) return;
    Lane &last = lane_of(h, h->recorded - 1);
    if (last.stream != h->ctx->stream) LR_CUDA(cudaStreamWaitEvent(h->ctx->stream, last.finished, 0));
}

// Renderer.advance (integrator.lucb:649-693): never waits; two passes in flight.
// A film stage alone for a renderer whose display settings changed after its last sample
// (integrator.lucb:663-675): its image and a display image converted again.
void launch_convert(WaveHost *h) {
    Lane &lane = lane_of(h, h->recorded);
    Plan *staging = lane.h_plan;
    MemberHost &mh = h->members[0];
    PassRecord rec;
    rec.number = h->recorded;
    rec.members.push_back({0u, false});
    rec.generations.push_back(mh.generation);
    staging->head = PlanHeader{0u, 0u, 1u, 0u, 0u, 0u, 0u, 0u, 0u, {0u, 0u, 0u}};
    staging->convert[0] = 0u;
    staging->convert_samples[0] = mh.sample;
    rec.display_slot = free_display_slot(h);
    staging->display = PlanDisplay{(unsigned long long)display_image(h, rec.display_slot), h->display_scale,
                                   h->display_view, 0u, 0u};
    rec.width = mh.dev.width;
    rec.height = mh.dev.height;
    h->display_stale = false;
    cudaStream_t stream = lane.stream;
    if (stream != h->ctx->stream && lane.members_seen != h->member_uploads && h->staging.copied) {
        LR_CUDA(cudaStreamWaitEvent(stream, h->staging.copied, 0));
        lane.members_seen = h->member_uploads;
    }
    LR_CUDA(cudaMemcpyAsync(lane.d_plan, staging, offsetof(Plan, seg), cudaMemcpyHostToDevice, stream));
    Lane *before = rec.number > 0 && h->lane_count > 1 ? &lane_of(h, rec.number - 1) : nullptr;
    if (before) LR_CUDA(cudaStreamWaitEvent(stream, before->finished, 0));
    if (lane.reads_seen != h->reads) {
        LR_CUDA(cudaStreamWaitEvent(stream, h->read_done, 0));
        lane.reads_seen = h->reads;
    }
    if (h->profile) {
        LR_CUDA(cudaEventRecord(h->mark_start[rec.number & 1], stream));
        record_finish(h, lane.w, stream, &rec.marks);
    } else {
        LR_CUDA(cudaGraphLaunch(lane.finish.exec, stream));
    }
    LR_CUDA(cudaEventRecord(lane.finished, stream));
    h->recorded++;
    h->in_flight.push_back(std::move(rec));
}

bool wave_advance(WaveHost *h) {
    while (retire_one(h, false)) {
    }
    if (h->in_flight.size() >= 2) return true;
    if (launch_pass(h)) return true;
    if (h->display_block && h->display_stale && h->members[0].used) {
        launch_convert(h);
        return true;
    }
    return !h->in_flight.empty();
}

// Times two dry passes from the current plan settings (members of size class `only`, or
// all) and returns their paths a millisecond.
double time_dry(WaveHost *h, int only, cudaEvent_t a, cudaEvent_t b) {
    launch_pass(h, true, only);  // warm: builds the variant's graph
    settle(h);
    uint64_t paths = 0;
    LR_CUDA(cudaEventRecord(a, h->ctx->stream));
    for (int i = 0; i < 2; i++) {
        if (!launch_pass(h, true, only)) break;
        paths += h_plan_paths(h);
    }
    join_lanes(h);
    LR_CUDA(cudaEventRecord(b, h->ctx->stream));
    LR_CUDA(cudaEventSynchronize(b));
    settle(h);
    float ms = 0.0f;
    LR_CUDA(cudaEventElapsedTime(&ms, a, b));
    return (double)paths / std::max(1e-3f, ms);
}

// The autotuner, on dry passes over the members as they stand: for each scene-size class
// present, the BVH width (2, 4, 8; a width all its members fall back from is skipped)
// whose passes of that class alone run fastest; then, with those widths, the pool fill
// (a quarter, half or all of the pool) of the mixed passes.
// The stacks of width `width`'s traversal variants that hold `bound` entries, smallest
// first.
std::vector<int> stacks_for(int width, int bound) {
    std::vector<int> out;
#define LR_CASE(wd, k) \
    if (wd == width && k >= bound) out.push_back(k);
    LR_TRAVERSALS(LR_CASE)
#undef LR_CASE
    std::sort(out.begin(), out.end());
    return out;
}

// lr_batch_tune: per scene-size class, dry passes of that class's members alone at every
// BVH width, every stack depth its variants offer above the members' bound, and the
// traversal kernels at 64, 128 and 256 threads a block -- the fastest kept; then the
// mixed passes at pool fill 1/4, 1/2 and all, and the interval at which the shade kernels
// group outgoing rays by octant (never, every round, every second round).
void wave_tune(WaveHost *h, lr_batch_tuning *out) {
    settle(h);
    if (!std::any_of(h->members.begin(), h->members.end(), has_work))
        fail(LR_INVALID, "tuning needs members with samples to come");
    if (out) *out = lr_batch_tuning{};
    cudaEvent_t a, b;
    LR_CUDA(cudaEventCreate(&a));
    LR_CUDA(cudaEventCreate(&b));
    uint32_t tried = 0;
    h->fill = h->pool;
    h->bin_interval = 0;
    for (int cls = 0; cls < kSizeClasses; cls++) {
        uint32_t members = 0;
        for (auto &mh : h->members)
            if (has_work(mh) && size_class(mh.dev.scene.triangle_count) == cls) members++;
        if (out) out->class_members[cls] = members;
        if (!members) continue;
        double best = -1.0;
        int best_width = 2, best_stack = 0, best_block = 0;
        std::vector<std::vector<int>> seen;
        for (int width : {2, 4, 8}) {
            std::vector<int> got;
            int effective = 2, bound = 0;
            for (auto &mh : h->members)
                if (has_work(mh) && size_class(mh.dev.scene.triangle_count) == cls) {
                    const TraversalChoice c = choose_traversal(mh.dev.scene, width);
                    got.push_back(c.width * 1000 + c.stack);
                    effective = c.width;
                    bound = std::max(bound, c.stack);
                }
            if (std::find(seen.begin(), seen.end(), got) != seen.end()) continue;
            seen.push_back(got);
            h->class_width[cls] = width;
            for (int stack : stacks_for(effective, bound)) {
                for (int block : kTraceBlocks) {
                    h->class_stack[cls] = stack;
                    h->class_block[cls] = block;
                    const double rate = time_dry(h, cls, a, b);
                    tried++;
                    if (rate > best) {
                        best = rate;
                        best_width = width;
                        best_stack = stack;
                        best_block = block;
                    }
                }
            }
        }
        h->class_width[cls] = best_width;
        h->class_stack[cls] = best_stack;
        h->class_block[cls] = best_block;
        if (out) {
            out->class_width[cls] = (uint32_t)best_width;
            out->class_stack[cls] = (uint32_t)best_stack;
            out->class_block[cls] = (uint32_t)best_block;
        }
    }
    double best = -1.0;
    uint32_t best_fill = h->pool;
    for (uint32_t fill : {h->pool / 4, h->pool / 2, h->pool}) {
        if (fill == 0) continue;
        h->fill = fill;
        const double rate = time_dry(h, -1, a, b);
        tried++;
        if (rate > best) {
            best = rate;
            best_fill = fill;
        }
    }
    h->fill = best_fill;
    uint32_t best_interval = 0;
    for (uint32_t interval : {1u, 2u}) {
        h->bin_interval = interval;
        const double rate = time_dry(h, -1, a, b);
        tried++;
        if (rate > best) {
            best = rate;
            best_interval = interval;
        }
    }
    h->bin_interval = best_interval;
    // Persistent warps that refill their idle lanes from the queue, at 32 (a whole warp at
    // a time), 16 or 8 idle lanes, against the grid-stride walks.
    uint32_t best_refill = h->refill_at;
    for (uint32_t refill : {0u, 32u, 16u, 8u}) {
        if (refill == h->refill_at) continue;
        const uint32_t kept = h->refill_at;
        h->refill_at = refill;
        const double rate = time_dry(h, -1, a, b);
        tried++;
        if (rate > best) {
            best = rate;
            best_refill = refill;
        }
        h->refill_at = kept;
    }
    h->refill_at = best_refill;
    // Where passes that walk the BVH2 switch to the compressed 8-wide tree for their thin
    // later rounds: from round 2, 3 or 4, or never.
    // Every candidate timed on this mix (the choice then holds for any mix of members).
    h->thin_any = true;
    int best_thin = -1;
    double best_thin_rate = -1.0;
    for (int from : {-1, 2, 3, 4}) {
        h->thin_from = from;
        const double rate = time_dry(h, -1, a, b);
        tried++;
        if (rate > best_thin_rate) {
            best_thin_rate = rate;
            best_thin = from;
        }
    }
    h->thin_from = best_thin;
    best = std::max(best, best_thin_rate);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (out) {
        out->fill = best_fill;
        out->paths_per_ms = best;
        out->candidates = tried;
        out->bin_interval = best_interval;
        out->refill_at = best_refill;
        out->thin_from = best_thin;
        int widest = 0;
        for (int cls = 0; cls < kSizeClasses; cls++) widest = std::max(widest, h->class_width[cls]);
        out->width = (uint32_t)(widest ? widest : 2);
    }
}

void wave_finish(WaveHost *h) {
    for (;;) {
        if (!wave_advance(h)) break;
        if (h->in_flight.size() >= 2) retire_one(h, true);
        else if (!h->in_flight.empty() && !std::any_of(h->members.begin(), h->members.end(), has_work))
            retire_one(h, true);
    }
    check_status(h->ctx);
}

void lanes_destroy(WaveHost *h) {
    for (auto &lane : h->lanes) {
        for (auto &[v, g] : lane.trace) destroy_graph(g);
        destroy_graph(lane.finish);
        if (lane.finished) cudaEventDestroy(lane.finished);
        if (lane.h_plan) cudaFreeHost(lane.h_plan);
        if (lane.own_stream && lane.stream) cudaStreamDestroy(lane.stream);
        if (lane.block) cudaFree(lane.block);
        lane = Lane{};
    }
}

// The wave's lanes made again for `pool` paths and `rounds` rounds, after the passes in
// flight; its members stay.
void wave_resize(WaveHost *h, uint64_t pool, uint32_t rounds) {
    settle(h);
    for (auto &lane : h->lanes)
        if (lane.stream) LR_CUDA(cudaStreamSynchronize(lane.stream));
    LR_CUDA(cudaStreamSynchronize(h->ctx->stream));
    lanes_destroy(h);
    h->pool = (uint32_t)std::min<uint64_t>(pool, kMaxPool);
    h->rounds = rounds;
    lanes_create(h);
    LR_CUDA(cudaStreamSynchronize(h->ctx->stream));
    if (!h->profile) lanes_capture(h);
}

void wave_destroy(WaveHost *h) {
    if (!h->ctx) return;
    cudaSetDevice(h->ctx->device);
    for (auto &lane : h->lanes)
        if (lane.stream) cudaStreamSynchronize(lane.stream);
    cudaStreamSynchronize(h->ctx->stream);
    for (auto &p : h->in_flight)
        for (auto &[e, k] : p.marks) cudaEventDestroy(e);
    for (auto e : h->mark_start)
        if (e) cudaEventDestroy(e);
    if (h->copy_stream) cudaStreamSynchronize(h->copy_stream);
    for (auto &mh : h->members)
        if (mh.used) member_free(nullptr, mh, h->ctx->stream);
    cudaStreamSynchronize(h->ctx->stream);
    h->staging.release();
    if (h->read_done) cudaEventDestroy(h->read_done);
    for (auto &mark : h->read_marks) cudaEventDestroy(mark.second);
    for (cudaEvent_t mark : h->spare_marks) cudaEventDestroy(mark);
    h->read_marks.clear();
    h->spare_marks.clear();
    if (h->copy_stream) cudaStreamDestroy(h->copy_stream);
    for (auto &[pass, gs] : h->retiring_scenes) lr_gpu_scene_destroy(gs);
    h->retiring_scenes.clear();
    if (h->display_block) cudaFree(h->display_block);
    h->display_block = nullptr;
    lanes_destroy(h);
    if (h->block) cudaFree(h->block);
}

// The last pass's ray records of round `round` (settings.profile = kProfileRecord): the
// camera paths' rays, then the light paths', of the closest-hit queue, or the shadow
// queue; 12 floats a ray (origin + tag, direction + reach, the traversal's answer).
uint64_t wave_records(WaveHost *h, uint32_t round, bool shadow, float *out, uint64_t capacity) {
    if (h->profile != kProfileRecord) fail(LR_INVALID, "ray records need settings.profile = 3");
    if (round >= h->rounds) fail(LR_INVALID, "no such round");
    settle(h);
    join_lanes(h);
    const Lane &lane = h->lanes[0];
    std::vector<uint32_t> counters(4 * (size_t)h->rounds + 2);
    LR_CUDA(cudaMemcpyAsync(counters.data(), lane.w.counters, counters.size() * 4, cudaMemcpyDeviceToHost,
                            h->ctx->stream));
    LR_CUDA(cudaStreamSynchronize(h->ctx->stream));
    const uint64_t front = shadow ? counters[h->rounds + 1 + round] : counters[round];
    const uint64_t back = shadow ? 0 : counters[kLightCounters * h->rounds + 2 + round];
    const uint64_t total = front + back;
    if (!out) return total;
    if (capacity < total * 12) fail(LR_LIMIT, "the output holds fewer rays than the round traced");
    const float4 *rec = (shadow ? lane.w.record_shadow : lane.w.record_closest) + (size_t)round * h->pool * 3;
    if (front) LR_CUDA(cudaMemcpyAsync(out, rec, front * 48, cudaMemcpyDeviceToHost, h->ctx->stream));
    // Light paths' rays fill the queue from its back: entry pool - 1 - k holds ray k.
    if (back)
        LR_CUDA(cudaMemcpyAsync(out + front * 12, rec + (h->pool - back) * 3, back * 48, cudaMemcpyDeviceToHost,
                                h->ctx->stream));
    LR_CUDA(cudaStreamSynchronize(h->ctx->stream));
    return total;
}

void wave_stats(WaveHost *h, lr_render_stats *out) {
    settle(h);
    unsigned long long s[8];
    join_lanes(h);
    LR_CUDA(cudaMemcpyAsync(s, h->d_stats, sizeof s, cudaMemcpyDeviceToHost, h->ctx->stream));
    LR_CUDA(cudaStreamSynchronize(h->ctx->stream));
    out->closest_rays = s[0];
    out->shadow_rays = s[1];
    out->shaded = s[2];
    out->passes = s[3];
    out->closest_nodes = s[4];
    out->closest_tests = s[5];
    out->shadow_nodes = s[6];
    out->shadow_tests = s[7];
}

void wave_kernel_times(WaveHost *h, double out[10]) {
    // Finished passes count: wait for those in flight and retire them.
    settle(h);
    for (int i = 0; i < 10; i++) out[i] = h->kernel_ms[i];
}

MemberHost &member_at(WaveHost *h, uint32_t member) {
    if (member >= h->capacity || !h->members[member].used || h->members[member].leaving)
        fail(LR_INVALID, "no such member");
    return h->members[member];
}

void member_read(WaveHost *h, uint32_t member, float *rgba, uint64_t count) {
    MemberHost &mh = member_at(h, member);
    if (count != mh.dev.pixels * 4) fail(LR_INVALID, "reading the image needs four floats a pixel");
    join_lanes(h);
    LR_CUDA(cudaMemcpyAsync(rgba, mh.dev.image, count * 4, cudaMemcpyDeviceToHost, h->ctx->stream));
    LR_CUDA(cudaStreamSynchronize(h->ctx->stream));
}

// Whether the copy with `ticket` (and so every copy queued before it, on the one copy
// stream) has arrived; never waits.
bool member_read_landed(WaveHost *h, uint64_t ticket) {
    while (!h->read_marks.empty()) {
        const cudaError_t e = cudaEventQuery(h->read_marks.front().second);
        if (e == cudaErrorNotReady) break;
        LR_CUDA(e);
        h->reads_landed = h->read_marks.front().first;
        h->spare_marks.push_back(h->read_marks.front().second);
        h->read_marks.pop_front();
    }
    return ticket <= h->reads_landed;
}

cudaEvent_t read_in_flight(WaveHost *h, uint64_t ticket) {
    if (member_read_landed(h, ticket)) return nullptr;
    for (auto &mark : h->read_marks)
        if (mark.first >= ticket) return mark.second;
    return h->read_done;
}

// Queues a copy of the member's image as the passes launched so far leave it into
// `rgba` (pinned host memory, so that the copy runs beside the passes after it) and
// returns its ticket without waiting; member_read_wait waits for every copy queued,
// member_read_landed says whether one has arrived. The copy waits only for what last
// wrote the image: the member's last pass while it may still run, or the uploads of
// its memory when no pass has traced it since.
uint64_t member_read_async(WaveHost *h, uint32_t member, float *rgba, uint64_t count) {
    MemberHost &mh = member_at(h, member);
    if (count != mh.dev.pixels * 4) fail(LR_INVALID, "reading the image needs four floats a pixel");
    if (!h->copy_stream) {
        LR_CUDA(cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking));
        LR_CUDA(cudaEventCreateWithFlags(&h->read_done, cudaEventDisableTiming));
    }
    if (mh.last_pass <= mh.placed_at) {
        // No pass since its memory was queued on the context's stream.
        cudaEvent_t ready;
        LR_CUDA(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
        LR_CUDA(cudaEventRecord(ready, h->ctx->stream));
        LR_CUDA(cudaStreamWaitEvent(h->copy_stream, ready, 0));
        LR_CUDA(cudaEventDestroy(ready));
    } else if (mh.last_pass > h->retired) {
        // Its lane's event stands for that pass or a later one on the lane.
        LR_CUDA(cudaStreamWaitEvent(h->copy_stream, lane_of(h, mh.last_pass - 1).finished, 0));
    }
    LR_CUDA(cudaMemcpyAsync(rgba, mh.dev.image, count * 4, cudaMemcpyDeviceToHost, h->copy_stream));
    LR_CUDA(cudaEventRecord(h->read_done, h->copy_stream));
    h->reads++;
    cudaEvent_t mark;
    if (!h->spare_marks.empty()) {
        mark = h->spare_marks.back();
        h->spare_marks.pop_back();
    } else {
        LR_CUDA(cudaEventCreateWithFlags(&mark, cudaEventDisableTiming));
    }
    LR_CUDA(cudaEventRecord(mark, h->copy_stream));
    h->read_marks.push_back({h->reads, mark});
    mh.read_ticket = h->reads;
    return h->reads;
}

void member_read_wait(WaveHost *h) {
    if (h->read_done) LR_CUDA(cudaEventSynchronize(h->read_done));
}

uint64_t member_read_ticket(WaveHost *h, uint32_t member, float *rgba, uint64_t count) {
    return member_read_async(h, member, rgba, count);
}

}  // namespace
}  // namespace lr

using namespace lr;

struct lr_renderer {
    WaveHost wave;
    uint32_t bands = 1;
    // The view it renders, and what a reload compares a scene with: a hash of the
    // geometry (points and triangles, leaf order) and the triangles' shading as uploaded
    // (normals and materials), staged for a reload's upload through `shading_stage`.
    lr_frame frame{};
    uint64_t geometry = 0;
    std::vector<uint32_t> shading;
    uint32_t *shading_stage = nullptr;
    cudaEvent_t shading_copied = nullptr;
};

struct lr_batch {
    WaveHost wave;
};

namespace lr {
namespace {

// FNV-1a over a scene's geometry: its points and triangles in leaf order (same_geometry,
// scene.lucb:168-181, asks the same of the geometry sets a compile starts from).
uint64_t geometry_hash(const lr_scene &scene) {
    uint64_t key = 14695981039346656037ull;
    auto mix = [&](const void *data, size_t bytes) {
        const unsigned char *p = (const unsigned char *)data;
        for (size_t i = 0; i < bytes; i++) key = (key ^ p[i]) * 1099511628211ull;
    };
    const uint64_t counts[2] = {scene.point_count(), scene.triangle_count()};
    mix(counts, sizeof counts);
    mix(scene.positions.data(), scene.positions.size() * sizeof(float));
    mix(scene.indices.data(), scene.indices.size() * sizeof(uint32_t));
    return key;
}

// A renderer's three display images, for views of up to `pixels` (made again, none shown,
// when a view outgrows them).
void display_images(WaveHost *h, uint64_t pixels) {
    if (h->display_block && pixels <= h->display_pixels) return;
    if (h->display_block) {
        settle(h);
        LR_CUDA(cudaStreamSynchronize(h->ctx->stream));
        LR_CUDA(cudaFree(h->display_block));
        h->display_block = nullptr;
    }
    h->display_pixels = pixels;
    LR_CUDA(cudaMalloc(&h->display_block, 3 * align256(pixels * 8)));
    LR_CUDA(cudaMemsetAsync(h->display_block, 0, 3 * align256(pixels * 8), h->ctx->stream));
    h->front = -1;
    h->shown_width = h->shown_height = 0;
}

// The band a renderer's passes take for `pixels` (integrator.lucb:419-423).
uint64_t band_of(const lr_settings &settings, uint64_t pixels) {
    return std::min<uint64_t>(std::min<uint64_t>(settings.pool ? settings.pool : kDefaultPool, kMaxPool), pixels);
}

// Renderer.restart / reload / replace_scene: the member renewed through `frame`, its
// bands and pass fill set for the new view. A view or scene that needs a larger path pool
// or more rounds than the renderer's wave has waits for the passes in flight and makes
// the wave again.
void renderer_renew(lr_renderer *r, const lr_frame &frame, const lr_scene *scene, const lr_settings *settings,
                    lr_gpu_scene *gs) {
    WaveHost *h = &r->wave;
    MemberHost &mh = member_at(h, 0);
    const lr_settings &chosen = settings ? *settings : mh.settings;
    validate(chosen, frame);
    if ((bool)frame.orthographic != (mh.dev.frame[3] > 0.5f)) fail(LR_INVALID, "a restart keeps the view's projection");
    const uint64_t pixels = (uint64_t)frame.width * frame.height;
    const uint64_t band = band_of(chosen, pixels);
    const uint64_t most_lights = light_paths_of(chosen, frame, pixels, 1, false).count;
    const uint32_t rounds = scene ? rounds_of(*scene, chosen) : mh.dev.rounds;
    // A view or scene that needs a larger path pool or more rounds than the wave has makes
    // the lanes again after the passes in flight (the reference makes its view's buffers
    // again in the same case).
    if (band + most_lights > h->pool || rounds > h->rounds)
        wave_resize(h, std::max<uint64_t>(band + most_lights, h->pool), std::max(rounds, h->rounds));
    member_renew(h, 0, frame, scene, settings, gs, gs);
    r->bands = (uint32_t)((pixels + band - 1) / band);
    h->fill = (uint32_t)std::min<uint64_t>(band + h->members[0].dev.light_paths, h->pool);
    h->camera_cap = (uint32_t)band;
    display_images(h, pixels);
}

void create(lr_context *ctx, const lr_scene *scene, const lr_settings &settings, const lr_frame &frame, lr_renderer **out) {
    validate(settings, frame);
    auto r = std::make_unique<lr_renderer>();
    LR_CUDA(cudaSetDevice(ctx->device));
    const uint64_t pixels = (uint64_t)frame.width * frame.height;
    const uint64_t band = std::min<uint64_t>(std::min<uint64_t>(settings.pool ? settings.pool : kDefaultPool, kMaxPool), pixels);
    r->bands = (uint32_t)((pixels + band - 1) / band);
    // A pass holds a band and, in a sample's first, its light paths (integrator.lucb:419-423);
    // room for them at most, until the scene says whether it has emitters.
    const uint64_t most_lights = light_paths_of(settings, frame, pixels, 1, false).count;
    lr_gpu_scene *gs = nullptr;
    int status = lr_gpu_scene_upload(ctx, scene, &gs);
    if (status != LR_OK) fail(status, lr_last_error());
    try {
        const uint32_t rounds = settings.max_bounces + 1 + (has_cutouts(*scene, settings) ? kCutoutRounds : 0);
        wave_create(&r->wave, ctx, band + most_lights, rounds, 1, settings.profile);
        member_add(&r->wave, gs, gs, scene, settings, frame);
        r->wave.fill = (uint32_t)std::min<uint64_t>(band + r->wave.members[0].dev.light_paths, r->wave.pool);
        r->wave.camera_cap = (uint32_t)band;
        display_images(&r->wave, pixels);
        r->frame = frame;
        r->geometry = geometry_hash(*scene);
        r->shading = scene->shading;
        // The graphs for the scene's traversal variant, made now rather than at the first pass.
        const TraversalChoice c = choose_traversal(gs->scene, 0);
        if (!settings.profile)
            for (int li = 0; li < r->wave.lane_count; li++)
                trace_graph(&r->wave, r->wave.lanes[li],
                            c.width * 1000 + c.stack + (r->wave.members[0].dev.light_paths ? kTracingVariant : 0) +
                                (r->wave.members[0].dev.glossy ? kGlossyVariant : 0) +
                                (r->wave.members[0].dev.cutouts ? kCutoutVariant : 0) +
                                (r->wave.refill_at ? kRefillVariant : 0) +
                                (r->wave.thin_from >= 0 && c.width == 2 && r->wave.profile < 2 &&
                                         size_class(gs->scene.triangle_count) == kSizeClasses - 1
                                     ? thin_code(gs->scene) * kThinVariant
                                     : 0));
    } catch (...) {
        const bool owned = !r->wave.members.empty() && r->wave.members[0].used;
        wave_destroy(&r->wave);
        if (!owned) lr_gpu_scene_destroy(gs);
        throw;
    }
    *out = r.release();
}

}  // namespace
}  // namespace lr

extern "C" {

void lr_settings_default(lr_settings *s, uint32_t width, uint32_t height, uint32_t samples) {
    if (!s) return;
    *s = lr_settings{};
    s->width = width;
    s->height = height;
    s->samples = samples;
    s->max_bounces = 12;
    s->spectral = 1;
    s->camera = -1;
    lr_openpbr_standard(&s->material);
    s->pool = 0;
    s->seed = 1;
    s->software_bvh = 0;
    s->diffuse_bounces = s->glossy_bounces = s->transmission_bounces = 1024;
    s->clamp_indirect = 0.0;
    s->noise_threshold = 0.0;
    s->adaptive_minimum = 16;
    s->profile = 0;
    s->guiding = 0;
    s->light_tracing = 0.5;
}

static void camera_of(const lr_scene *scene, const lr_settings *settings, lr_frame &frame) {
    if (settings->width == 0 || settings->height == 0 || settings->width > 16384 || settings->height > 16384)
        fail(LR_INVALID, "an image is 1 to 16384 pixels on a side");
    lr_camera cam;
    if (settings->camera >= 0) {
        if ((size_t)settings->camera >= scene->cameras.size()) fail(LR_INVALID, "the scene object is not a camera");
        cam = scene->cameras[(size_t)settings->camera];
    } else {
        if (scene->cameras.empty()) fail(LR_INVALID, "the scene has no camera");
        cam = scene->cameras[0];
    }
    camera_frame(cam, settings->width, settings->height, frame);
}

int lr_renderer_create(lr_context *ctx, const lr_scene *scene, const lr_settings *settings, lr_renderer **out) {
    return guarded([&] {
        if (!ctx || !scene || !settings || !out) fail(LR_INVALID, "a renderer needs a context, a scene and settings");
        *out = nullptr;
        lr_frame frame;
        camera_of(scene, settings, frame);
        create(ctx, scene, *settings, frame, out);
    });
}

int lr_renderer_create_viewed(lr_context *ctx, const lr_scene *scene, const lr_settings *settings, const lr_frame *frame,
                              lr_renderer **out) {
    return guarded([&] {
        if (!ctx || !scene || !settings || !frame || !out) fail(LR_INVALID, "a renderer needs a context, a scene and settings");
        *out = nullptr;
        create(ctx, scene, *settings, *frame, out);
    });
}

int lr_renderer_advance(lr_renderer *r, int32_t *more) {
    return guarded([&] {
        if (!r || !more) fail(LR_INVALID, "no renderer");
        *more = wave_advance(&r->wave) ? 1 : 0;
    });
}

int lr_renderer_finish(lr_renderer *r) {
    return guarded([&] {
        if (!r) fail(LR_INVALID, "no renderer");
        wave_finish(&r->wave);
    });
}

uint32_t lr_renderer_samples_done(const lr_renderer *r) { return r ? r->wave.members[0].done : 0u; }

int lr_renderer_passes(const lr_renderer *r, uint64_t *recorded, uint64_t *finished, uint32_t *bands) {
    return guarded([&] {
        if (!r) fail(LR_INVALID, "no renderer");
        if (recorded) *recorded = r->wave.recorded;
        if (finished) *finished = r->wave.retired;
        if (bands) *bands = r->bands;
    });
}

int lr_renderer_image(lr_renderer *r, void **device_rgba) {
    return guarded([&] {
        if (!r || !device_rgba) fail(LR_INVALID, "no renderer");
        *device_rgba = r->wave.members[0].dev.image;
    });
}

int lr_renderer_restart(lr_renderer *r, const lr_frame *frame) {
    return guarded([&] {
        if (!r || !frame) fail(LR_INVALID, "restart needs a renderer and a frame");
        LR_CUDA(cudaSetDevice(r->wave.ctx->device));
        renderer_renew(r, *frame, nullptr, nullptr, nullptr);
        r->frame = *frame;
    });
}

int lr_renderer_reload(lr_renderer *r, const lr_scene *scene, const lr_settings *settings, const lr_frame *frame) {
    return guarded([&] {
        if (!r || !scene || !settings) fail(LR_INVALID, "reload needs a renderer, a scene and settings");
        LR_CUDA(cudaSetDevice(r->wave.ctx->device));
        if (geometry_hash(*scene) != r->geometry) fail(LR_INVALID, "a reload keeps the scene's geometry");
        WaveHost *h = &r->wave;
        MemberHost &mh = member_at(h, 0);
        const lr_frame f = frame ? *frame : r->frame;
        lr_settings chosen = *settings;
        chosen.width = f.width;
        chosen.height = f.height;
        chosen.pool = mh.settings.pool;
        chosen.software_bvh = mh.settings.software_bvh;
        if (scene->shading != r->shading) {
            // The triangles' normals and materials again, into the upload, after the passes in
            // flight (the reference uploads the per-triangle shading again).
            const size_t bytes = scene->shading.size() * sizeof(uint32_t);
            if (r->shading_copied) LR_CUDA(cudaEventSynchronize(r->shading_copied));
            else LR_CUDA(cudaEventCreateWithFlags(&r->shading_copied, cudaEventDisableTiming));
            if (!r->shading_stage) LR_CUDA(cudaMallocHost((void **)&r->shading_stage, std::max<size_t>(bytes, 16)));
            std::memcpy(r->shading_stage, scene->shading.data(), bytes);
            after_passes(h);
            LR_CUDA(cudaMemcpyAsync((void *)mh.dev.scene.shading, r->shading_stage, bytes, cudaMemcpyHostToDevice,
                                    h->ctx->stream));
            LR_CUDA(cudaEventRecord(r->shading_copied, h->ctx->stream));
            r->shading = scene->shading;
        }
        renderer_renew(r, f, scene, &chosen, mh.owned);
        r->frame = f;
    });
}

int lr_renderer_replace_scene(lr_renderer *r, const lr_scene *scene, const lr_settings *settings, const lr_frame *frame) {
    return guarded([&] {
        if (!r || !scene || !settings || !frame) fail(LR_INVALID, "replace_scene needs a renderer, a scene, settings and a frame");
        WaveHost *h = &r->wave;
        MemberHost &mh = member_at(h, 0);
        if (settings->pool != mh.settings.pool || settings->software_bvh != mh.settings.software_bvh)
            fail(LR_INVALID, "a scene replaced keeps the pool and BVH choice");
        LR_CUDA(cudaSetDevice(h->ctx->device));
        lr_settings chosen = *settings;
        chosen.width = frame->width;
        chosen.height = frame->height;
        lr_gpu_scene *gs = nullptr;
        const int status = lr_gpu_scene_upload(h->ctx, scene, &gs);
        if (status != LR_OK) fail(status, lr_last_error());
        try {
            renderer_renew(r, *frame, scene, &chosen, gs);
        } catch (...) {
            if (member_at(h, 0).owned != gs) lr_gpu_scene_destroy(gs);
            throw;
        }
        r->frame = *frame;
        r->geometry = geometry_hash(*scene);
        r->shading = scene->shading;
    });
}

int lr_renderer_refit(lr_renderer *r, const lr_scene *scene, const lr_frame *frame) {
    return guarded([&] {
        if (!r || !scene) fail(LR_INVALID, "a refit needs a renderer and its scene with the points moved");
        WaveHost *h = &r->wave;
        MemberHost &mh = member_at(h, 0);
        lr_gpu_scene *gs = mh.owned;
        if (!gs || topology_hash(*scene) != gs->topology) fail(LR_INVALID, "a refit keeps the renderer's triangles");
        LR_CUDA(cudaSetDevice(h->ctx->device));
        const lr_frame f = frame ? *frame : r->frame;
        lr_settings chosen = mh.settings;
        chosen.width = f.width;
        chosen.height = f.height;
        // The passes in flight read the geometry: the new points and the refit follow them.
        after_passes(h);
        if (scene->point_count())
            LR_CUDA(cudaMemcpyAsync(const_cast<float *>(gs->scene.positions), scene->positions.data(),
                                    scene->positions.size() * sizeof(float), cudaMemcpyHostToDevice, h->ctx->stream));
        refit_scene(gs, h->ctx->stream);
        renderer_renew(r, f, scene, &chosen, gs);
        r->frame = f;
        r->geometry = geometry_hash(*scene);
        r->shading = scene->shading;
    });
}

int lr_renderer_display(lr_renderer *r, void **device_rgba16f) {
    return guarded([&] {
        if (!r || !device_rgba16f) fail(LR_INVALID, "no renderer");
        WaveHost *h = &r->wave;
        while (retire_one(h, false)) {
        }
        *device_rgba16f = display_image(h, h->front >= 0 ? h->front : 0);
    });
}

int lr_renderer_shown_size(lr_renderer *r, uint32_t out[2]) {
    return guarded([&] {
        if (!r || !out) fail(LR_INVALID, "no renderer");
        WaveHost *h = &r->wave;
        while (retire_one(h, false)) {
        }
        out[0] = h->front >= 0 ? h->shown_width : 0u;
        out[1] = h->front >= 0 ? h->shown_height : 0u;
    });
}

int lr_renderer_converged_pixels(lr_renderer *r, uint64_t *out) {
    return guarded([&] {
        if (!r || !out) fail(LR_INVALID, "no renderer");
        WaveHost *h = &r->wave;
        MemberHost &mh = member_at(h, 0);
        *out = 0;
        if (!mh.dev.half) return;
        std::vector<float4> half(mh.dev.pixels);
        join_lanes(h);
        LR_CUDA(cudaMemcpyAsync(half.data(), mh.dev.half, half.size() * sizeof(float4), cudaMemcpyDeviceToHost,
                                h->ctx->stream));
        LR_CUDA(cudaStreamSynchronize(h->ctx->stream));
        for (const float4 &v : half) *out += v.w > 0.5f ? 1u : 0u;
    });
}

int lr_renderer_set_display(lr_renderer *r, double exposure, int view) {
    return guarded([&] {
        if (!r) fail(LR_INVALID, "no renderer");
        if (view != 0 && view != 1) fail(LR_INVALID, "a display view is 0 (standard) or 1 (neutral)");
        r->wave.display_scale = (float)std::exp2(exposure);
        r->wave.display_view = (uint32_t)view;
        r->wave.display_stale = true;
    });
}

int lr_renderer_read(lr_renderer *r, float *rgba, uint64_t count) {
    return guarded([&] {
        if (!r || !rgba) fail(LR_INVALID, "no renderer");
        member_read(&r->wave, 0, rgba, count);
    });
}

int lr_renderer_read_async(lr_renderer *r, float *rgba, uint64_t count) {
    return guarded([&] {
        if (!r || !rgba) fail(LR_INVALID, "no renderer");
        member_read_async(&r->wave, 0, rgba, count);
    });
}

int lr_renderer_read_wait(lr_renderer *r) {
    return guarded([&] {
        if (!r) fail(LR_INVALID, "no renderer");
        member_read_wait(&r->wave);
    });
}

int lr_renderer_read_ticket(lr_renderer *r, float *rgba, uint64_t count, uint64_t *ticket) {
    return guarded([&] {
        if (!r || !rgba || !ticket) fail(LR_INVALID, "no renderer");
        *ticket = member_read_ticket(&r->wave, 0, rgba, count);
    });
}

int lr_renderer_read_landed(lr_renderer *r, uint64_t ticket, int32_t *landed) {
    return guarded([&] {
        if (!r || !landed) fail(LR_INVALID, "no renderer");
        *landed = member_read_landed(&r->wave, ticket) ? 1 : 0;
    });
}

int lr_renderer_join(lr_renderer *r) {
    return guarded([&] {
        if (!r) fail(LR_INVALID, "no renderer");
        join_lanes(&r->wave);
    });
}

int lr_renderer_set_samples(lr_renderer *r, uint32_t samples) {
    return guarded([&] {
        if (!r) fail(LR_INVALID, "no renderer");
        if (samples == 0) fail(LR_INVALID, "a render needs samples");
        r->wave.members[0].samples = samples;
    });
}

int lr_albedo_tables(lr_context *ctx, float *out, size_t count) {
    return guarded([&] {
        if (!ctx || !out) fail(LR_INVALID, "no context or buffer");
        static_assert(kTableSize == LR_ALBEDO_TABLE_SIZE, "the table layout is the header's");
        if (count < kTableSize) fail(LR_INVALID, "the tables hold " + std::to_string(kTableSize) + " floats");
        LR_CUDA(cudaSetDevice(ctx->device));
        make_albedo_tables(ctx->device, ctx->stream);
        LR_CUDA(cudaMemcpyFromSymbol(out, g_albedo_tables, kTableSize * sizeof(float)));
    });
}

int lr_renderer_kernel_times(lr_renderer *r, double out[10]) {
    return guarded([&] {
        if (!r || !out) fail(LR_INVALID, "kernel times need ten numbers");
        wave_kernel_times(&r->wave, out);
    });
}

int lr_renderer_recorded_rays(lr_renderer *r, uint32_t round, int32_t shadow, float *out, uint64_t capacity,
                              uint64_t *count) {
    return guarded([&] {
        if (!r || !count) fail(LR_INVALID, "no renderer");
        *count = wave_records(&r->wave, round, shadow != 0, out, capacity);
    });
}

int lr_renderer_stats(lr_renderer *r, lr_render_stats *out) {
    return guarded([&] {
        if (!r || !out) fail(LR_INVALID, "no renderer");
        wave_stats(&r->wave, out);
    });
}

void lr_renderer_destroy(lr_renderer *r) {
    if (!r) return;
    wave_destroy(&r->wave);
    if (r->shading_copied) cudaEventDestroy(r->shading_copied);
    if (r->shading_stage) cudaFreeHost(r->shading_stage);
    delete r;
}

// ---- Batches ------------------------------------------------------------------------

void lr_batch_settings_default(lr_batch_settings *s) {
    if (!s) return;
    *s = lr_batch_settings{};
    s->pool = (uint32_t)kDefaultPool;
    s->max_bounces = 12;
    s->capacity = 256;
    s->profile = 0;
}

int lr_batch_create(lr_context *ctx, const lr_batch_settings *settings, lr_batch **out) {
    return guarded([&] {
        if (!ctx || !settings || !out) fail(LR_INVALID, "a batch needs a context and settings");
        *out = nullptr;
        if (settings->max_bounces == 0 || settings->max_bounces > 253) fail(LR_INVALID, "a batch traces 1 to 253 bounces");
        if (settings->capacity == 0 || settings->capacity > 65536) fail(LR_INVALID, "a batch holds 1 to 65536 members");
        if (settings->pool == 0) fail(LR_INVALID, "a batch needs a pool of paths");
        auto b = std::make_unique<lr_batch>();
        try {
            wave_create(&b->wave, ctx, settings->pool, settings->max_bounces + 1, settings->capacity, settings->profile);
        } catch (...) {
            wave_destroy(&b->wave);
            throw;
        }
        *out = b.release();
    });
}

int lr_batch_add(lr_batch *b, const lr_gpu_scene *gs, const lr_scene *scene, const lr_settings *settings,
                 const lr_frame *frame, uint32_t *member) {
    return guarded([&] {
        if (!b || !gs || !scene || !settings || !member) fail(LR_INVALID, "a member needs a scene and settings");
        if (gs->device_built)
            fail(LR_INVALID, "a member renders an upload of its compiled scene (lr_gpu_scene_upload), not a device build");
        lr_frame f;
        if (frame) f = *frame;
        else camera_of(scene, settings, f);
        *member = member_add(&b->wave, gs, nullptr, scene, *settings, f);
    });
}

int lr_batch_remove(lr_batch *b, uint32_t member) {
    return guarded([&] {
        if (!b) fail(LR_INVALID, "no batch");
        MemberHost &mh = member_at(&b->wave, member);
        mh.leaving = true;
        collect(&b->wave);
    });
}

int lr_batch_advance(lr_batch *b, int32_t *more) {
    return guarded([&] {
        if (!b || !more) fail(LR_INVALID, "no batch");
        *more = wave_advance(&b->wave) ? 1 : 0;
    });
}

int lr_batch_finish(lr_batch *b) {
    return guarded([&] {
        if (!b) fail(LR_INVALID, "no batch");
        wave_finish(&b->wave);
    });
}

int lr_batch_join(lr_batch *b) {
    return guarded([&] {
        if (!b) fail(LR_INVALID, "no batch");
        join_lanes(&b->wave);
    });
}

int lr_batch_wait(lr_batch *b, int32_t *in_flight) {
    return guarded([&] {
        if (!b) fail(LR_INVALID, "no batch");
        retire_one(&b->wave, true);
        if (in_flight) *in_flight = (int32_t)b->wave.in_flight.size();
    });
}

int lr_batch_member_info(const lr_batch *b, uint32_t member, uint32_t *samples_done, uint32_t *samples_planned,
                         uint32_t *samples) {
    return guarded([&] {
        if (!b) fail(LR_INVALID, "no batch");
        const MemberHost &mh = member_at(const_cast<WaveHost *>(&b->wave), member);
        if (samples_done) *samples_done = mh.done;
        if (samples_planned) *samples_planned = mh.sample;
        if (samples) *samples = mh.samples;
    });
}

int lr_batch_set_samples(lr_batch *b, uint32_t member, uint32_t samples) {
    return guarded([&] {
        if (!b) fail(LR_INVALID, "no batch");
        if (samples == 0) fail(LR_INVALID, "a render needs samples");
        member_at(&b->wave, member).samples = samples;
    });
}

int lr_batch_image(lr_batch *b, uint32_t member, void **device_rgba) {
    return guarded([&] {
        if (!b || !device_rgba) fail(LR_INVALID, "no batch");
        *device_rgba = member_at(&b->wave, member).dev.image;
    });
}

int lr_batch_read(lr_batch *b, uint32_t member, float *rgba, uint64_t count) {
    return guarded([&] {
        if (!b || !rgba) fail(LR_INVALID, "no batch");
        member_read(&b->wave, member, rgba, count);
    });
}

int lr_batch_read_async(lr_batch *b, uint32_t member, float *rgba, uint64_t count) {
    return guarded([&] {
        if (!b || !rgba) fail(LR_INVALID, "no batch");
        member_read_async(&b->wave, member, rgba, count);
    });
}

int lr_batch_read_wait(lr_batch *b) {
    return guarded([&] {
        if (!b) fail(LR_INVALID, "no batch");
        member_read_wait(&b->wave);
    });
}

int lr_batch_read_ticket(lr_batch *b, uint32_t member, float *rgba, uint64_t count, uint64_t *ticket) {
    return guarded([&] {
        if (!b || !rgba || !ticket) fail(LR_INVALID, "no batch");
        *ticket = member_read_ticket(&b->wave, member, rgba, count);
    });
}

int lr_batch_read_landed(lr_batch *b, uint64_t ticket, int32_t *landed) {
    return guarded([&] {
        if (!b || !landed) fail(LR_INVALID, "no batch");
        *landed = member_read_landed(&b->wave, ticket) ? 1 : 0;
    });
}

int lr_batch_tune(lr_batch *b, lr_batch_tuning *out) {
    return guarded([&] {
        if (!b) fail(LR_INVALID, "no batch");
        wave_tune(&b->wave, out);
    });
}

int lr_batch_passes(const lr_batch *b, uint64_t *recorded, uint64_t *finished) {
    return guarded([&] {
        if (!b) fail(LR_INVALID, "no batch");
        if (recorded) *recorded = b->wave.recorded;
        if (finished) *finished = b->wave.retired;
    });
}

int lr_batch_kernel_times(lr_batch *b, double out[10]) {
    return guarded([&] {
        if (!b || !out) fail(LR_INVALID, "kernel times need ten numbers");
        wave_kernel_times(&b->wave, out);
    });
}

int lr_batch_stats(lr_batch *b, lr_render_stats *out) {
    return guarded([&] {
        if (!b || !out) fail(LR_INVALID, "no batch");
        wave_stats(&b->wave, out);
    });
}

void lr_batch_destroy(lr_batch *b) {
    if (!b) return;
    wave_destroy(&b->wave);
    delete b;
}

}  // extern "C"
