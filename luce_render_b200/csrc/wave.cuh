// What the wavefront's kernels share across translation units: the wave (one lane's path
// pool, ray queues, counters and plan), its members (a scene seen through one camera into
// one film), the pass plan's segments, and the launchers of the traversal kernels, which
// live in trace.cu so that they compile at IEEE single precision (no flush of denormals to
// zero, no approximate division) whatever flags the shading code takes.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "device.hpp"
#include "emitters.cuh"
#include "lighttree.cuh"
#include "shading.cuh"
#include "surface.cuh"

namespace lr {

constexpr int kTraceBlock = 128;     // the traversal kernels' block size unless tuned
constexpr int kTraceBlockMax = 256;  // the largest the autotuner tries (64, 128, 256)
// Resident blocks of kTraceBlockMax the traversal kernels are built for: at most 64
// registers a thread, so that 32 warps of an SM hide the node and triangle fetches (the
// walk through cut-outs, a kernel of its own, takes what it needs).
constexpr int kTraceMinBlocks = 4;
constexpr int kShadeBlock = 128;
constexpr size_t kDefaultPool = 2097152;  // 2^21 paths (integrator.lucb:98)
// A ray's tag: the path's pool index in the low bits, its segment in the high bits.
constexpr uint32_t kPathBits = 23;
constexpr uint32_t kPathMask = (1u << kPathBits) - 1u;
constexpr uint32_t kMaxPool = 1u << kPathBits;             // 8,388,608 paths
constexpr uint32_t kMaxSegments = 1u << (32 - kPathBits);  // 512 segments a pass
// Rounds a pass traces beyond the bounces when the scene has cut-outs (loading.lucb:161).
constexpr uint32_t kCutoutRounds = 8;
// settings.profile: 1 per-kernel times (one lane), 2 also traversal work counts, 3 also
// ray records (each round's rays and the traversal's answers, lr_renderer_recorded_rays).
constexpr int kProfileRecord = 3;

// One member of a wave: everything its paths read, fixed while it is a member.
struct Member {
    DeviceScene scene;
    LightTable lights;
    uint32_t spectral;
    TreeTable tree;
    const MaterialCode *materials;
    const Constants *k;
    float frame[16];
    float lens_radius, focus_distance;
    float forward[3];
    uint32_t width, height;
    uint64_t pixels;
    float4 *film, *image;
    // Light tracing (connect.glsl): light paths a sample (0: none), the band their
    // sampler numbers follow, 1 / a pixel's area on the image plane at unit distance, and
    // the splat accumulators (3 fixed-point words a pixel: kSplatScale units of the
    // film's terms): the film's, and one per lane that a pass's connections land in until
    // the pass's finish stage folds them into the film's, in pass order.
    uint32_t light_paths, light_band;
    float pixel_area_inv;
    unsigned long long *splat;
    unsigned long long *splat_lane[2];
    // A material of the member's has a specular, metal, coat or transmission lobe: its
    // surfaces take the layered OpenPBR shading (surface.cuh, paths.cuh).
    uint32_t glossy;
    // A material of the member's is a cut-out (geometry_opacity below 1), and the rounds
    // its passes trace: its bounces + 1, + 8 for rays passing through cut-outs at the same
    // bounce (integrator.lucb:806-808); a ray for a later round is not traced.
    uint32_t cutouts, rounds;
    // Adaptive sampling (adaptive.comp, finish.comp:22-23): the second estimate (odd
    // samples, twice; w: converged) and the convergence verdicts, or null when off.
    float4 *half;
    float *scratch;
};

// Splats add as 64-bit integers (units of 2^-32 of the film's terms), so their sum does
// not depend on the order the connections arrive in.
constexpr double kSplatScale = 4294967296.0;
constexpr float kSplatLimit = 1e9f;

// `count` pixels of member `member` from `first_pixel`, at sample `sample`, in pool
// paths path_base .. path_base + count -- or, of kind kLightSegment, `count` of the
// sample's light paths from number `first_pixel`. `convert`: this segment ends the
// member's sample, so its image is brought up to date after the pass. `kind_base`: the
// pass's paths of the segment's kind before it (its rays' place in the queues).
constexpr uint32_t kCameraSegment = 0, kLightSegment = 1;
struct Segment {
    uint32_t member, first_pixel, count, sample;
    uint32_t path_base, convert, kind, kind_base;
};

// `dry`: a trial pass (autotuning) that traces its segments but leaves films alone.
// `camera_paths`: the pass's camera paths; `folds`: members whose light paths it traces.
struct PlanHeader {
    uint32_t segments, paths, converts, dry;
    // bin_interval: the shade kernels group outgoing rays by direction octant in rounds
    // that are multiples of it (0: never; an autotuner choice).
    uint32_t camera_paths, folds, adapts, bin_interval;
    // refill_at: the traversal kernels' persistent warps take new queue entries once this
    // many of their lanes are idle (1 to 32; 0: grid-stride walks; an autotuner choice).
    uint32_t refill_at, reserved[3];
};

// A renderer's display image for the pass (film_convert.comp:50-52): where the pass that
// ends a sample writes the image ready to show (rgba16f, or none), its exposure scale and
// view (0 clipped, 1 PBR Neutral tone mapping).
struct PlanDisplay {
    unsigned long long image;
    float scale;
    uint32_t view, reserved0, reserved1;
};

// A pass's plan: its segments, the members whose images it brings up to date (and the
// samples they will then hold), and the members whose splats it folds into their films.
struct Plan {
    PlanHeader head;
    PlanDisplay display;  // for the first member converted (a renderer's own)
    uint32_t convert[kMaxSegments];
    uint32_t convert_samples[kMaxSegments];
    uint32_t fold[kMaxSegments];
    uint32_t adapt[kMaxSegments];  // members whose convergence the pass checks
    Segment seg[kMaxSegments];
};

// What a pass's kernels read besides the members: passed by value, fixed for the wave.
struct Wave {
    const Member *members;
    const Plan *plan;
    uint32_t pool, rounds;
    uint32_t lane;  // which of the wave's two lanes this is
    // path state, one slot per pool path
    float4 *throughput, *radiance, *lambda, *vertex;  // vertex: last scattering point, w survival scale
    float4 *mis;                                      // light tracing's MIS state (connect.glsl)
    uint4 *path;  // pixel (a light path's emitter), bounces, previous normal, ray pdf bits
    // ray queues (ping-pong by round) and their hits
    float4 *ray_o[2], *ray_d[2], *hits[2];
    float4 *shadow_o, *shadow_d, *shadow_c;
    // Ray queues hold camera paths' rays from the front and light paths' from the back
    // (index pool - 1 - k), so that each kind shades in a launch of its own.
    // counters[r]: camera paths' rays of round r; counters[rounds + 1 + r]: shadow rays of
    // round r; counters[kLightCounters * rounds + 2 + r] (light_counter): light paths' rays;
    // counters[4 * rounds + 2 + 4r] .. + 3: the next closest and shadow queue entry of
    // round r a traversal warp takes (fetch_counter), and the next entry of the camera and
    // the light paths' queues a shade block takes (shade_cursor). counter_slots(rounds) in
    // all, zeroed by each pass's camera kernel.
    uint32_t *counters;
    unsigned long long *stats;  // closest rays, shadow rays, paths, passes, then traversal work
    int *status;
    // Ray records (settings.profile = 3; null otherwise): per round and queue entry the ray
    // and the triangle traversal's answer -- closest: (t, source id, u, v) before the
    // analytic lights; shadow: (1 blocked / 0 clear, 0, 0, 0) -- three float4 each.
    float4 *record_closest, *record_shadow;
};

// Where the light paths' ray counts start in a wave's counters.
constexpr uint32_t kLightCounters = 2;
__device__ __forceinline__ uint32_t *light_counter(const Wave &w, uint32_t round) {
    return &w.counters[kLightCounters * w.rounds + 2 + round];
}
__device__ __forceinline__ uint32_t *fetch_counter(const Wave &w, uint32_t round, bool shadow) {
    return &w.counters[4 * w.rounds + 2 + 4 * round + (shadow ? 1u : 0u)];
}
// The next queue entry a shade kernel's block takes in round `round` (camera paths'
// queue, or with `light` the light paths').
__device__ __forceinline__ uint32_t *shade_cursor(const Wave &w, uint32_t round, bool light) {
    return &w.counters[4 * w.rounds + 2 + 4 * round + (light ? 3u : 2u)];
}
constexpr uint32_t counter_slots(uint32_t rounds) { return 8 * rounds + 6; }

__device__ __forceinline__ uint32_t warp_push(uint32_t *counter, bool want) {
    const unsigned mask = __ballot_sync(0xffffffffu, want);
    if (mask == 0u) return 0u;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(mask) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(counter, (uint32_t)__popc(mask));
    base = __shfl_sync(0xffffffffu, base, leader);
    return base + (uint32_t)__popc(mask & ((1u << lane) - 1u));
}

// The segment holding pool path `path` (segments lie end to end from path 0).
__device__ __forceinline__ uint32_t segment_of(const Plan *plan, uint32_t path) {
    uint32_t lo = 0, hi = plan->head.segments;
    while (hi - lo > 1u) {
        const uint32_t mid = (lo + hi) >> 1;
        if (plan->seg[mid].path_base <= path) lo = mid;
        else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ const Member &member_of_tag(const Wave &w, uint32_t tag) {
    return w.members[w.plan->seg[tag >> kPathBits].member];
}

// A light path's number among its sample's light paths.
__device__ __forceinline__ uint32_t tag_light_index(const Wave &w, uint32_t tag) {
    const Segment &sg = w.plan->seg[tag >> kPathBits];
    return sg.first_pixel + ((tag & kPathMask) - sg.path_base);
}

// The traversal variants a pass can take: (BVH width, stack entries).
#define LR_TRAVERSALS(X) X(8, 16) X(8, 32) X(4, 32) X(4, 48) X(2, 32) X(2, 64) X(2, 96)

// trace.cu: the closest-hit and shadow kernels of round `round` on `stream`, traversal
// variant (width, stack) in blocks of `block` threads (kTraceBlocks); `count`
// instantiates the counting traversals, `cutouts` the shadow walk through cut-outs,
// `refill` the persistent warps that refill idle lanes (trace_refilling; not with the
// other two). closest_grid: the resident grid of a variant at a block size.
void launch_closest(int width, int stack, int block, bool count, bool refill, int grid, cudaStream_t stream,
                    const Wave &w, uint32_t round);
void launch_shadow(int width, int stack, int block, bool count, bool cutouts, bool refill, int grid,
                   cudaStream_t stream, const Wave &w, uint32_t round);
int closest_grid(int width, int stack, int block, bool refill, int sm_count);

}  // namespace lr
