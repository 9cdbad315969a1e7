// The integrator's traversal kernels: intersect_closest.comp and intersect_shadow.comp of
// the reference, over the wave's ray queues (wave.cuh).
//
// This translation unit is compiled at IEEE single precision -- denormals kept, division
// and square root correctly rounded -- so the watertight triangle test here decides every
// hit exactly as the ray queries of device.cu (lr_trace_rays, lr_probe) do, and as the FP32
// brute force of the oracle does: an edge function that is a denormal stays a nonzero
// number of its sign instead of turning "outside" into "on the edge". The shading kernels
// (integrator.cu) take approximate division and flush denormals; nothing here depends on
// them.
#include "device.hpp"
#include "emitters.cuh"
#include "traverse.cuh"
#include "wave.cuh"

namespace lr {
namespace {

// The queue walk of the traversal kernels: each warp takes the next 32 consecutive entries
// (neighbouring primary rays, or rays a shading warp pushed together, so its lanes walk
// similar nodes) with one atomic on `next` (zeroed by the pass's camera kernel) whenever
// all its lanes are done, so warps that drew long rays take fewer batches and no warp
// waits at the end for a fixed share. `body(j)` handles entry j.
template <class Body>
__device__ __forceinline__ void warp_batches(uint32_t count, uint32_t *next, Body body) {
    const uint32_t lane = threadIdx.x & 31u;
    for (;;) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(next, 32u);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= count) break;
        if (base + lane < count) body(base + lane);
    }
}

// intersect_closest.comp:45-76: the nearest triangle, then the analytic lights
// before it (camera rays skip lights invisible to the camera). Two ways through the queue,
// chosen by the plan: warp batches (warp_batches: 32 neighbouring entries a warp at a
// time), which keep a warp's lanes on similar nodes; with plan refill_at > 0 persistent
// warps hand finished lanes new entries one by one instead (trace_refilling), which keeps
// more lanes busy on incoherent rays.
template <int W, int kStack, bool kCount, bool kRefill>
__device__ __forceinline__ void closest_body(const Wave &w, uint32_t round) {
    extern __shared__ int stack[];  // kInts entries a thread, strided by the block's size
    const uint32_t q = round & 1u;
    const uint32_t cameras = w.counters[round], count = cameras + *light_counter(w, round);
    bool overflow = false;
    Visits visits;
    const float4 *ray_o = w.ray_o[q], *ray_d = w.ray_d[q];
    float4 *hits = w.hits[q];
    typename TracerOf<W, false, kStack, kCount>::type tr(stack + threadIdx.x, blockDim.x);
    // The camera paths' rays, then the light paths' from the queue's back.
    auto entry = [&](uint32_t j) { return j < cameras ? j : w.pool - 1u - (j - cameras); };
    auto begin = [&](uint32_t j, DeviceScene &s) {
        const uint32_t i = entry(j);
        const float4 o = ray_o[i], d = ray_d[i];
        s = w.members[w.plan->seg[__float_as_uint(o.w) >> kPathBits].member].scene;
        return tr.start(s, Ray{xyz(o), 0.0f, xyz(d), d.w});
    };
    auto end = [&](uint32_t j) {
        const uint32_t i = entry(j);
        // The ray and its lights, read again past the traversal rather than held through it.
        const float4 o = ray_o[i], d = ray_d[i];
        if (w.record_closest) {
            float4 *rec = w.record_closest + ((size_t)round * w.pool + i) * 3u;
            rec[0] = o;
            rec[1] = d;
            rec[2] = make_float4(tr.h.t, __int_as_float(tr.h.id), tr.h.u, tr.h.v);
        }
        const Segment &sg = w.plan->seg[__float_as_uint(o.w) >> kPathBits];
        const Member &m = w.members[sg.member];
        const bool flow = sg.kind == kLightSegment;  // light paths follow light
        uint32_t what = tr.h.slot >= 0 ? (uint32_t)tr.h.slot : kNone;
        float t = tr.h.t;
        const uint32_t light = nearest_light(m.lights, xyz(o), xyz(d), t, round == 0, flow);
        if (light != kNone) what = kLightHit | light;
        hits[i] = make_float4(t, __uint_as_float(what), tr.h.u, tr.h.v);
    };
    if (kRefill) {
        auto begin_or_end = [&](uint32_t j, DeviceScene &s) {
            if (begin(j, s)) return true;
            end(j);
            return false;
        };
        trace_refilling(tr, count, fetch_counter(w, round, false), w.plan->head.refill_at, begin_or_end, end, overflow,
                        visits);
    } else {
        warp_batches(count, fetch_counter(w, round, false), [&](uint32_t j) {
            {
                DeviceScene s;
                if (begin(j, s)) {
                    while (!tr.step(s, overflow, visits)) {
                    }
                }
            }
            end(j);
        });
    }
    if (overflow) atomicAdd(&w.status[0], 1);
    if (kCount) add_visits(&w.stats[4], visits);
}

template <int W, int kStack, bool kCount, bool kRefill>
__global__ void __launch_bounds__(kTraceBlockMax, kTraceMinBlocks) closest_kernel(Wave w, uint32_t round) {
    closest_body<W, kStack, kCount, kRefill>(w, round);
}

// The BVH2's grid-stride walk, the renderer's default, at 56 registers: nine blocks of 128
// threads an SM instead of eight, for the latency of its dependent node fetches (8 bytes
// spilled outside the walk). Measured on the headline pass over several boxes: 1,225-1,237
// Mrays/s against 1,214-1,225 at 64 registers -- about 1 %, within what boxes differ by.
template <int kStack>
__global__ void __maxnreg__(56) closest_bvh2_kernel(Wave w, uint32_t round) {
    closest_body<2, kStack, false, false>(w, round);
}

// intersect_shadow.comp:28-92: unblocked light samples join their path's radiance; a light
// path's camera connection, unless a light the camera sees stands in it, splats its value
// (in the film's terms) on its pixel in the lane's accumulator.
template <int W, int kStack, bool kCount, bool kCutouts, bool kRefill>
__global__ void __launch_bounds__(kTraceBlockMax, kCutouts ? 1 : kTraceMinBlocks) shadow_kernel(Wave w, uint32_t round) {
    extern __shared__ int stack[];
    const uint32_t count = w.counters[w.rounds + 1 + round];
    bool overflow = false;
    Visits visits;
    typename TracerOf<W, true, kStack, kCount>::type tr(stack + threadIdx.x, blockDim.x);
    auto member_of = [&](uint32_t tag) -> const Member & { return w.members[w.plan->seg[tag >> kPathBits].member]; };
    auto record = [&](uint32_t i, float state) {
        if (w.record_shadow) w.record_shadow[((size_t)round * w.pool + i) * 3u + 2u] = make_float4(state, 0.0f, 0.0f, 0.0f);
    };
    // Light that reached the ray's end, `kept` of it past cut-outs (`cut`: the member has
    // some): a camera path's light sample joins its radiance; a light path's connection
    // splats on its pixel.
    auto deliver = [&](uint32_t i, float kept, bool cut) {
        const uint32_t tag = __float_as_uint(w.shadow_o[i].w);
        const Segment &sg = w.plan->seg[tag >> kPathBits];
        const Member &m = w.members[sg.member];
        const bool light_path = sg.kind == kLightSegment;
        float4 c = w.shadow_c[i];
        if (cut) c = make_float4(c.x * kept, c.y * kept, c.z * kept, light_path ? c.w : c.w * kept);
        if (!light_path) {
            const uint32_t path = tag & kPathMask;
            w.radiance[path] = w.radiance[path] + c;
        } else if (!w.plan->head.dry && isfinite(c.x) && isfinite(c.y) && isfinite(c.z)) {
            unsigned long long *at = m.splat_lane[w.lane] + (size_t)__float_as_uint(c.w) * 3;
            const float v[3] = {c.x, c.y, c.z};
            for (int k = 0; k < 3; k++) {
                const float clamped_v = fminf(fmaxf(v[k], -kSplatLimit), kSplatLimit);
                atomicAdd(at + k, (unsigned long long)llrint((double)clamped_v * kSplatScale));
            }
        }
    };
    // The ray's record (-1: not traced by the any-hit query -- a light the camera sees
    // stands in the connection, or the walk through cut-outs decides it); false when such
    // a light ends the connection and there is nothing to trace.
    auto prologue = [&](uint32_t i) {
        const float4 o = w.shadow_o[i], d = w.shadow_d[i];
        if (w.record_shadow) {
            float4 *rec = w.record_shadow + ((size_t)round * w.pool + i) * 3u;
            rec[0] = o;
            rec[1] = d;
            rec[2] = make_float4(-1.0f, 0.0f, 0.0f, 0.0f);
        }
        const uint32_t tag = __float_as_uint(o.w);
        const Member &m = member_of(tag);
        return !(w.plan->seg[tag >> kPathBits].kind == kLightSegment && seen_light_between(m.lights, xyz(o), xyz(d), d.w));
    };
    auto end = [&](uint32_t i) {
        const bool blocked = tr.h.id >= 0;
        record(i, blocked ? 1.0f : 0.0f);
        if (!blocked) deliver(i, 1.0f, false);
    };
    // Starts the any-hit walk: true when there is one to take, else the ray is finished.
    auto begin = [&](uint32_t i, DeviceScene &s) {
        if (!prologue(i)) return false;
        const float4 o = w.shadow_o[i], d = w.shadow_d[i];
        s = member_of(__float_as_uint(o.w)).scene;
        if (tr.start(s, Ray{xyz(o), 0.0f, xyz(d), d.w})) return true;
        end(i);
        return false;
    };
    // intersect_shadow.comp:70-91: on through the cut-outs it meets, keeping (1 - opacity)
    // of the light at each; anything opaque blocks. Closest hits, on the same stack (a
    // variant of its own: passes without cut-outs keep the leaner kernel).
    auto through_cutouts = [&](uint32_t i, const Member &m) {
        if (!prologue(i)) return;
        const float4 o = w.shadow_o[i], d = w.shadow_d[i];
        const DeviceScene s = m.scene;
        typename TracerOf<W, false, kStack, kCount>::type walk(stack + threadIdx.x, blockDim.x);
        float3 from = xyz(o);
        float remaining = d.w, kept = 1.0f;
        bool through = false;
        for (int hop = 0; hop < 16 && kept > 0.0f; hop++) {
            if (walk.start(s, Ray{from, 0.0f, xyz(d), remaining})) {
                while (!walk.step(s, overflow, visits)) {
                }
            }
            if (walk.h.slot < 0) {
                through = true;
                break;
            }
            const uint32_t material = __ldg(&s.shading[walk.h.slot]).w;
            kept *= 1.0f - fminf(fmaxf(__ldg(&m.materials[material].extra).x, 0.0f), 1.0f);
            if (kept < 1e-4f) kept = 0.0f;
            const float3 p = from + xyz(d) * walk.h.t;
            const float margin = 1e-4f * fmaxf(1.0f, fmaxf(fabsf(p.x), fmaxf(fabsf(p.y), fabsf(p.z))));
            from = p + xyz(d) * margin;
            remaining -= walk.h.t + margin;
            if (remaining <= 0.0f) {
                through = kept > 0.0f;
                break;
            }
        }
        if (through) deliver(i, kept, true);
    };
    if (kRefill && !kCutouts) {
        trace_refilling(tr, count, fetch_counter(w, round, true), w.plan->head.refill_at, begin, end, overflow, visits);
    } else {
        warp_batches(count, fetch_counter(w, round, true), [&](uint32_t i) {
            if (kCutouts) {
                const Member &m = member_of(__float_as_uint(w.shadow_o[i].w));
                if (m.cutouts) {
                    through_cutouts(i, m);
                    return;
                }
            }
            DeviceScene s;
            if (begin(i, s)) {
                while (!tr.step(s, overflow, visits)) {
                }
                end(i);
            }
        });
    }
    if (overflow) atomicAdd(&w.status[0], 1);
    if (kCount) add_visits(&w.stats[6], visits);
}

}  // namespace

// Shared memory a block of `block` threads needs for the stacks of variant (W, kStack):
// the shadow kernel's cut-out walk takes the closest-hit tracer's, the larger.
template <int W, int kStack>
size_t stack_bytes(int block) {
    return (size_t)TracerOf<W, false, kStack, false>::kInts * (size_t)block * sizeof(int);
}

void launch_closest(int width, int stack, int block, bool count, bool refill, int grid, cudaStream_t stream,
                    const Wave &w, uint32_t round) {
    switch (width * 1000 + stack) {
#define LR_CASE(wd, k)                                                                              \
    case wd * 1000 + k: {                                                                           \
        const size_t bytes = stack_bytes<wd, k>(block);                                             \
        if (count) closest_kernel<wd, k, true, false><<<grid, block, bytes, stream>>>(w, round);    \
        else if (refill) closest_kernel<wd, k, false, true><<<grid, block, bytes, stream>>>(w, round); \
        else if constexpr (wd == 2) closest_bvh2_kernel<k><<<grid, block, bytes, stream>>>(w, round); \
        else closest_kernel<wd, k, false, false><<<grid, block, bytes, stream>>>(w, round);         \
        return;                                                                                     \
    }
        LR_TRAVERSALS(LR_CASE)
#undef LR_CASE
        default: fail(LR_LIMIT, "no traversal variant for this scene");
    }
}

void launch_shadow(int width, int stack, int block, bool count, bool cutouts, bool refill, int grid,
                   cudaStream_t stream, const Wave &w, uint32_t round) {
    switch (width * 1000 + stack) {
#define LR_CASE(wd, k)                                                                                        \
    case wd * 1000 + k: {                                                                                     \
        const size_t bytes = stack_bytes<wd, k>(block);                                                       \
        if (count && cutouts) shadow_kernel<wd, k, true, true, false><<<grid, block, bytes, stream>>>(w, round);   \
        else if (count) shadow_kernel<wd, k, true, false, false><<<grid, block, bytes, stream>>>(w, round);        \
        else if (cutouts) shadow_kernel<wd, k, false, true, false><<<grid, block, bytes, stream>>>(w, round);      \
        else if (refill) shadow_kernel<wd, k, false, false, true><<<grid, block, bytes, stream>>>(w, round);       \
        else shadow_kernel<wd, k, false, false, false><<<grid, block, bytes, stream>>>(w, round);                  \
        return;                                                                                               \
    }
        LR_TRAVERSALS(LR_CASE)
#undef LR_CASE
        default: fail(LR_LIMIT, "no traversal variant for this scene");
    }
}

// Lets every kernel of variant (W, kStack) take `bytes` of dynamic shared memory (above
// the default 48 KB for deep stacks in large blocks).
template <int W, int kStack>
void allow_stacks(size_t bytes) {
    const int b = (int)bytes;
    const cudaFuncAttribute a = cudaFuncAttributeMaxDynamicSharedMemorySize;
    if constexpr (W == 2) LR_CUDA(cudaFuncSetAttribute(closest_bvh2_kernel<kStack>, a, b));
    else LR_CUDA(cudaFuncSetAttribute(closest_kernel<W, kStack, false, false>, a, b));
    LR_CUDA(cudaFuncSetAttribute(closest_kernel<W, kStack, false, true>, a, b));
    LR_CUDA(cudaFuncSetAttribute(closest_kernel<W, kStack, true, false>, a, b));
    LR_CUDA(cudaFuncSetAttribute(shadow_kernel<W, kStack, false, false, false>, a, b));
    LR_CUDA(cudaFuncSetAttribute(shadow_kernel<W, kStack, false, false, true>, a, b));
    LR_CUDA(cudaFuncSetAttribute(shadow_kernel<W, kStack, false, true, false>, a, b));
    LR_CUDA(cudaFuncSetAttribute(shadow_kernel<W, kStack, true, false, false>, a, b));
    LR_CUDA(cudaFuncSetAttribute(shadow_kernel<W, kStack, true, true, false>, a, b));
}

// Called (by the host, outside any stream capture) before a variant's first launch at a
// block size: sets the kernels' shared-memory allowance and returns the resident grid of
// the grid-stride or (`refill`) the refilling closest-hit kernel.
int closest_grid(int width, int stack, int block, bool refill, int sm_count) {
    int per_sm = 0;
    switch (width * 1000 + stack) {
#define LR_CASE(wd, k)                                                                                        \
    case wd * 1000 + k: {                                                                                     \
        const size_t bytes = stack_bytes<wd, k>(block);                                                       \
        allow_stacks<wd, k>(bytes);                                                                           \
        if (refill)                                                                                           \
            LR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, closest_kernel<wd, k, false, true>, block, \
                                                                  bytes));                                    \
        else if constexpr (wd == 2)                                                                           \
            LR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, closest_bvh2_kernel<k>, block, bytes)); \
        else                                                                                                  \
            LR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, closest_kernel<wd, k, false, false>, block, \
                                                                  bytes));                                    \
        break;                                                                                                \
    }
        LR_TRAVERSALS(LR_CASE)
#undef LR_CASE
        default: fail(LR_LIMIT, "no traversal variant for this scene");
    }
    return (per_sm > 0 ? per_sm : 1) * sm_count;
}

}  // namespace lr
