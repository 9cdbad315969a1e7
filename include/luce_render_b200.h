/*
 * luce_render_b200 — the C ABI of a B200-native (sm_100a) implementation of
 * luce-render's wavefront path-tracing hot path.
 *
 * Every entry point mirrors one of luce-render's `render` package API for this path
 * (package.prisma:13, public = ["render"]); each declaration cites the reference
 * interface it replaces. Conventions:
 *   - Status codes: 0 success; 400 invalid input, 401 past a limit, 402 stopped
 *     (src/render/module.lucb:60-63); 500 a CUDA call failed; 504 a bounded device
 *     wait gave up. The message of the last failing call on this thread is
 *     lr_last_error().
 *   - Handles are opaque. One host thread drives a context and the objects made on
 *     it (the reference's rule: device calls from the main thread, device.lucb:12).
 *   - Plain pointers and sizes only; "device" in a name means CUDA device memory.
 */
#ifndef LUCE_RENDER_B200_H
#define LUCE_RENDER_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Every declaration below is exported from the shared library. */
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

#define LR_OK 0
#define LR_INVALID 400 /* render.invalid (src/render/module.lucb:60) */
#define LR_LIMIT 401   /* render.limit (module.lucb:61) */
#define LR_STOPPED 402 /* render.stopped (module.lucb:63) */
#define LR_DEVICE 500  /* a CUDA runtime call failed */
#define LR_TIMEOUT 504 /* a device-side bounded wait gave up */

/* The message of the last failing call on this thread ("" when none). */
const char *lr_last_error(void);
/* The library version string. */
const char *lr_version(void);

/* ---- Context: one device and one stream (replaces luce-gpu's gpu.Device) --------- */

typedef struct lr_context lr_context;

/* gpu.Device.open (used at tests/gpu/main.lucb:18): a context on CUDA device `device`. */
int lr_context_create(int device, lr_context **out);
/* The same with a stream priority: 0 normal, 1 the device's highest (work queued on a
 * high-priority stream starts ahead of normal work waiting for the GPU; a serving loop
 * runs its probes there). */
int lr_context_create_ex(int device, int priority, lr_context **out);
void lr_context_destroy(lr_context *ctx);
/* Wait for all work queued on the context's stream. */
int lr_context_synchronize(lr_context *ctx);
/* The context's CUDA stream (a cudaStream_t), for callers that order their own work. */
void *lr_context_stream(lr_context *ctx);

/* Device memory for callers without an allocator of their own (tests, benches). */
int lr_device_alloc(lr_context *ctx, size_t bytes, void **out);
int lr_device_free(lr_context *ctx, void *ptr);
int lr_memcpy_htod(lr_context *ctx, void *dst, const void *src, size_t bytes);
int lr_memcpy_dtoh(lr_context *ctx, void *dst, const void *src, size_t bytes);
int lr_memset_device(lr_context *ctx, void *dst, int value, size_t bytes);
int lr_host_alloc_pinned(size_t bytes, void **out);
int lr_host_free_pinned(void *ptr);
/* CUDA-event timing on the context's stream: lr_timer_stop synchronizes and gives
 * the milliseconds since lr_timer_start. */
int lr_timer_start(lr_context *ctx);
int lr_timer_stop(lr_context *ctx, float *ms);

/* ---- Scene compile (src/render/scene.lucb:31-129, bvh.lucb:66-217) --------------- */

/* One mesh: the flat-array stand-in for a luce-geocore Mesh component placed in a
 * GeometrySet (scene.lucb:246-295). */
typedef struct {
    const float *positions;          /* xyz per point, in the mesh's space */
    uint64_t point_count;
    const uint32_t *indices;         /* 3 point indices per triangle (counter-clockwise) */
    uint64_t triangle_count;
    const uint32_t *triangle_faces;  /* the polygon of each triangle (NULL: its own index) */
    uint32_t face_count;             /* polygons in the mesh (0: triangle_count) */
    const float *normals;            /* shading normals xyz (NULL: each triangle's flat normal) */
    int32_t normals_per_corner;      /* 0: one normal per point; 1: three per triangle */
    const uint32_t *face_materials;  /* per polygon: 0 the default, k the library's k-th (NULL: 0) */
    double transform[12];            /* columns x, y, z, translation; all zeros: identity */
} lr_mesh;

/* A camera scene object (luce-geocore Camera as ray_frame reads it, camera.lucb:57-76). */
typedef struct {
    double matrix[12];        /* columns x (right), y (up), z (back), translation */
    int32_t projection;       /* 0 perspective, 1 orthographic */
    double focal_length;      /* mm */
    double horizontal_aperture; /* mm (orthographic: tenths of a scene unit) */
    double f_stop;            /* 0: a pinhole */
    double focus_distance;
} lr_camera;

/* A UsdLux light (lights.lucb:29-131). */
#define LR_LIGHT_RECT 0
#define LR_LIGHT_DISK 1
#define LR_LIGHT_SPHERE 2
#define LR_LIGHT_DISTANT 3
#define LR_LIGHT_DOME 4
typedef struct {
    double matrix[12];  /* columns x, y, z (the light shines down its -Z), translation */
    int32_t shape;      /* LR_LIGHT_* */
    double color[3];    /* linear ACEScg */
    double intensity, exposure, temperature; /* temperature in kelvin, 0: none */
    double width, height, radius, angle;     /* rect size, disk/sphere radius, distant angle (deg) */
    int32_t normalize, visible;              /* UsdLux normalize; visible to the camera */
    /* A dome's lat-long image (the pixels environment.lucb:102-156 reads from the dome's
     * OpenEXR file, which this ABI takes decoded): linear Rec.709 RGB, 3 floats a pixel,
     * image_width x image_height, rows from the top; its centre looks down the dome's -Z,
     * its top is +Y. NULL: the dome shines its colour evenly. As in the reference
     * (loading.lucb:55-61), only the first dome with an image lights by it. The compiled
     * scene keeps a copy. Ignored for other shapes. */
    const float *image;
    uint32_t image_width, image_height;
} lr_light;

/* OpenPBR Surface parameters (src/render/materials.lucb:17-53), shaded as
 * shaders/openpbr.glsl does: EON diffuse, GGX specular, F82-tint metal, coat, rough
 * transmission with dispersion (spectral build), emission, cut-out opacity.
 * base_diffuse_roughness outside 0..1 is rejected with 400; thin_walled is accepted and,
 * as in the reference's kernels, changes nothing. */
typedef struct {
    double base_weight, base_color[3], base_metalness, base_diffuse_roughness;
    double specular_weight, specular_color[3], specular_roughness, specular_roughness_anisotropy,
        specular_ior;
    double transmission_weight, transmission_color[3];
    double coat_weight, coat_color[3], coat_roughness, coat_roughness_anisotropy, coat_ior,
        coat_darkening;
    double emission_luminance, emission_color[3];
    double geometry_opacity;
    int32_t geometry_thin_walled;
    double transmission_dispersion_scale, transmission_dispersion_abbe_number;
} lr_openpbr;

/* OpenPbr.standard (materials.lucb:46-53). */
void lr_openpbr_standard(lr_openpbr *out);

/* The reference's 32-byte BVH node (bvh.lucb:23-27). */
typedef struct {
    float lo[3];
    uint32_t first; /* interior: first child of the pair; leaf: first triangle (leaf order) */
    float hi[3];
    uint32_t count; /* 0: interior; else triangles in the leaf */
} lr_bvh_node;

typedef struct lr_scene lr_scene;

/* render.compile_scene (scene.lucb:111): world-space triangles in BVH leaf order,
 * their polygons and shading attributes, the binned-SAH BVH2, cameras, lights and
 * the material library. The caller owns the result (CompiledScene.close ->
 * lr_scene_free). */
int lr_scene_compile(const lr_mesh *meshes, size_t mesh_count, const lr_camera *cameras,
                     size_t camera_count, const lr_light *lights, size_t light_count,
                     const lr_openpbr *materials, size_t material_count, lr_scene **out);
/* compile_scene(..., trees = false) (scene.lucb:111-129): with LR_COMPILE_NO_TREES the
 * host builds no BVH2 and the triangles stay in the meshes' order (order is the identity);
 * such a scene is for lr_gpu_scene_build, which builds its tree on the device. flags 0 is
 * lr_scene_compile. */
#define LR_COMPILE_NO_TREES 1u
int lr_scene_compile_ex(const lr_mesh *meshes, size_t mesh_count, const lr_camera *cameras,
                        size_t camera_count, const lr_light *lights, size_t light_count,
                        const lr_openpbr *materials, size_t material_count, uint32_t flags,
                        lr_scene **out);
/* CompiledScene.close (scene.lucb:87-98). */
void lr_scene_free(lr_scene *scene);
/* (No counterpart: the reference compiles a moved mesh again, rebuilding its BVH2,
 * bvh.lucb:66-82.) Moves a compiled scene's points to `positions` (3 floats a point, world
 * space, in the scene's point order: the meshes' points in the order they were passed)
 * with the triangles kept, and refits the BVH2 in place: every node's box again from its
 * triangles or children, the topology and leaf order unchanged; triangles compiled
 * without authored normals get their new flat normals. What lr_gpu_scene_refit does on
 * the device, on the host. */
int lr_scene_move_points(lr_scene *scene, const float *positions, uint64_t point_count);

typedef struct {
    uint64_t point_count, triangle_count, node_count;
    uint32_t face_count, camera_count, light_count, material_count, bvh_depth;
} lr_scene_info;
/* CompiledScene.triangle_count / point_count (scene.lucb:81-85) and the BVH's size. */
int lr_scene_info_get(const lr_scene *scene, lr_scene_info *out);
/* The compiled arrays (CompiledScene fields, scene.lucb:31-63), owned by the scene:
 * positions (3 floats a point), indices (3 a triangle, leaf order), faces (1 a
 * triangle), shading (4 a triangle: three octahedral normals, material), nodes and
 * order (the source triangle at each leaf slot). Any output may be NULL. */
int lr_scene_arrays(const lr_scene *scene, const float **positions, const uint32_t **indices,
                    const uint32_t **faces, const uint32_t **shading, const lr_bvh_node **nodes,
                    const uint32_t **order);

/* ---- Ray frames (src/render/camera.lucb) ------------------------------------------- */

/* RayFrame (camera.lucb:26-54). */
typedef struct {
    double position[3], corner[3], du[3], dv[3], forward[3];
    int32_t orthographic;
    uint32_t width, height;
    double lens_radius, focus_distance;
} lr_frame;

/* render.ray_frame (camera.lucb:57): the frame of camera `camera` for width x height. */
int lr_ray_frame(const lr_camera *camera, uint32_t width, uint32_t height, lr_frame *out);
/* render.look_frame (camera.lucb:84). */
int lr_look_frame(const double position[3], const double forward[3], const double up[3],
                  double tan_half_height, uint32_t width, uint32_t height, int32_t orthographic,
                  lr_frame *out);
/* RayFrame.pack (camera.lucb:41-47): the 16-float block the kernels read. */
int lr_frame_pack(const lr_frame *frame, float out[16]);
/* The scene's camera `index` (-1: the first camera; Renderer's find_camera,
 * integrator.lucb:955-961). */
int lr_scene_camera(const lr_scene *scene, int32_t index, lr_camera *out);

/* ---- The scene on the device (src/render/device.lucb) ----------------------------- */

typedef struct lr_gpu_scene lr_gpu_scene;

/* GpuScene.upload (device.lucb:41): the scene's traversal and shading buffers in HBM.
 * The scene may be freed afterwards. */
int lr_gpu_scene_upload(lr_context *ctx, const lr_scene *scene, lr_gpu_scene **out);
/* GpuScene.upload(accelerate = true) (device.lucb:41-89), where a ray-tracing device builds
 * its own acceleration structure: uploads the scene's triangles and builds a linear BVH2 on
 * the device (Morton codes of the centroids, a radix sort, the Karras hierarchy, boxes by
 * the refit climb), ignoring any host tree; a scene compiled with LR_COMPILE_NO_TREES skips
 * the host build entirely. Probes and ray queries on it (the BVH2 path only) return the same
 * exact closest hits as an upload; renders (lr_batch_add) refuse it, since its leaf order
 * is its own. Runs on ctx's stream and waits; LR_LIMIT past 2^27 triangles or 94 levels. */
int lr_gpu_scene_build(lr_context *ctx, const lr_scene *scene, lr_gpu_scene **out);
/* GpuScene.destroy (device.lucb:108-121). */
void lr_gpu_scene_destroy(lr_gpu_scene *scene);

/* (No counterpart: the reference rebuilds its BVH2 on the host when geometry changes,
 * bvh.lucb:66-82.) Moves an uploaded scene's points to `positions` (3 floats a point, in
 * the compiled scene's point order; host memory, or device memory of the scene's device
 * with LR_REFIT_DEVICE, e.g. a simulation's output) and refits it on the device: the
 * triangle records, flat normals, and the BVH2's boxes bottom-up in one launch, then the
 * watertight path's widened boxes and the 4- and 8-wide collapses' boxes; topology and leaf
 * order are kept, so traversal stays exact but slows as the tree fits the moved points
 * worse. The boxes equal lr_scene_move_points' bit for bit. Runs on `ctx`'s stream and
 * waits. Work that reads the scene must not be in flight: ray queries queued earlier on
 * other streams, or the passes of a batch with members tracing it (lr_batch_wait first).
 * Such members trace the moved geometry from their next pass on; their lights and light
 * tree stay as they were loaded (remove and add a member to load them again). A renderer
 * refits its own upload through lr_renderer_refit. */
#define LR_REFIT_DEVICE 1u
int lr_gpu_scene_refit(lr_context *ctx, lr_gpu_scene *scene, const void *positions, uint64_t point_count,
                       uint32_t flags);

/* What a scene holds on the device (no reference counterpart: the wide BVHs are this
 * build's): bytes, the BVH2's depth, the 4- and 8-wide collapses' node counts and
 * traversal stack bounds, and the width the watertight path takes by default. */
typedef struct {
    uint64_t bytes;
    uint32_t bvh2_depth;
    uint64_t wide4_nodes, wide8_nodes;
    uint32_t wide4_stack, wide8_stack;
    uint32_t width, stack;
} lr_gpu_scene_info;
int lr_gpu_scene_info_get(const lr_gpu_scene *scene, lr_gpu_scene_info *out);

/* Query flags. LR_TRACE_ANY: any-hit (trace_any, bvh.glsl:93-122) instead of the
 * closest hit. LR_TRACE_REFERENCE: the reference's own traversal and Moller-Trumbore
 * test (bvh.glsl:17-90, box order and tie rule included) instead of the default
 * watertight test with ties going to the smaller triangle id. LR_TRACE_COUNT: also add
 * the traversal's work (interior nodes visited, triangle tests) to the context's
 * counters, read by lr_trace_counts. */
#define LR_TRACE_ANY 1u
#define LR_TRACE_REFERENCE 2u
#define LR_TRACE_COUNT 4u
/* The watertight path's BVH width (at most one): the reference's BVH2, or its 4- or 8-wide
 * collapse (a wide request whose traversal stack does not fit falls back to 4, then 2).
 * None: the BVH2, the fastest on sm_100a. Results are the same bit for bit; only speed
 * differs. */
#define LR_TRACE_BVH2 8u
#define LR_TRACE_BVH4 16u
#define LR_TRACE_BVH8 32u

/* render.probe (device.lucb:138-160): the pixel-centre ray of every pixel of
 * `frame` (probe.comp:21-34), row by row from the top; per pixel the polygon hit
 * (0xffffffff: none) and its distance along the frame's unnormalized direction
 * (3e38 on a miss). Host buffers of width*height entries; waits for the result. */
int lr_probe(lr_context *ctx, const lr_gpu_scene *scene, const lr_frame *frame, uint32_t flags,
             uint32_t *faces, float *distances);

/* lr_probe without device allocation: the same results, bit for bit, staged through a
 * static device array of LR_PROBE_STATIC_PIXELS pixels (16 MiB, reserved when the
 * library's module loads on a device) instead of stream-ordered scratch. No counterpart
 * in the reference, whose probe allocates its result buffers per call; this one is for
 * callers that must not allocate device memory, such as a serving loop whose scene cache
 * holds the GPU at its memory budget. Larger frames are refused with LR_LIMIT. The
 * first call on a device does set-up (looks up the array's address, which may load the
 * module), so make it before any stream capture. All calls on one device share the
 * array, and two calls whose kernels overlapped on the GPU would race on it; so a call
 * holds a per-device lock of this library from its launch until its results are on the
 * host (on a failure too), and calls from several threads or contexts of one process
 * take turns. The array's address is kept for the process: do not use the library
 * across a cudaDeviceReset. */
#define LR_PROBE_STATIC_PIXELS 2097152u
int lr_probe_static(lr_context *ctx, const lr_gpu_scene *scene, const lr_frame *frame,
                    uint32_t flags, uint32_t *faces, float *distances);
/* (A diagnostic; the analogue of the reference's tests/gpu/overhead.lucb:9-39, which
 * times chains of dependent empty dispatches.) `count` dependent launches of an empty
 * kernel on the context's stream -- one after another, or with `graph` nonzero as one
 * captured CUDA graph -- best of five: out[0] microseconds a launch on the device (CUDA
 * events), out[1] microseconds a launch on the host's clock (launch calls and wait). */
int lr_launch_overhead(lr_context *ctx, uint32_t count, int32_t graph, double out[2]);
/* (No counterpart in the reference: a diagnostic.) The context's device memory: out[0]
 * free and out[1] total bytes (cudaMemGetInfo), out[2] the bytes the device's default
 * stream-ordered pool has handed out now, out[3] the most it has handed out at once since
 * the last reset; `reset_high` nonzero resets that high-water mark to the current use
 * first. lr_probe, lr_trace_rays and batch members allocate from that pool. */
int lr_context_memory(lr_context *ctx, int32_t reset_high, uint64_t out[4]);

/* Ray queries, the ray-list form of the probe. A ray is 8 floats (origin xyz, tmin,
 * direction xyz, tmax; hits have tmin < t < tmax); a hit is 4 words (t, triangle id as
 * int32 -- the caller's triangle numbering, -1 none --, barycentrics u and v of the
 * second and third vertices). lr_trace_rays copies host rays in and hits out and
 * waits; lr_trace_rays_device works on device buffers, queued on the context's
 * stream without waiting. */
int lr_trace_rays(lr_context *ctx, const lr_gpu_scene *scene, const float *rays, uint64_t count,
                  float *hits, uint32_t flags);
int lr_trace_rays_device(lr_context *ctx, const lr_gpu_scene *scene, const void *rays,
                         uint64_t count, void *hits, uint32_t flags);
/* The interior visits and triangle tests of LR_TRACE_COUNT queries since the last
 * call (the work shaders/bvh.glsl's trace_closest / trace_any do: 64 bytes of child
 * boxes per visit, 48 bytes of triangle per test); resets them. */
int lr_trace_counts(lr_context *ctx, uint64_t out[2]);

/* ---- The renderer (src/render/integrator.lucb) -------------------------------------- */

/* RenderSettings (integrator.lucb:42-82). */
typedef struct {
    uint32_t width, height, samples, max_bounces;
    int32_t spectral;
    int32_t camera; /* -1: the first camera */
    double background[3];
    lr_openpbr material;
    uint32_t pool, seed;
    int32_t software_bvh;
    uint32_t diffuse_bounces, glossy_bounces, transmission_bounces;
    double clamp_indirect, noise_threshold;
    uint32_t adaptive_minimum;
    int32_t profile, guiding;
    double light_tracing;
} lr_settings;

/* RenderSettings.of (integrator.lucb:84-85), with the reference's defaults. */
void lr_settings_default(lr_settings *out, uint32_t width, uint32_t height, uint32_t samples);

typedef struct lr_renderer lr_renderer;

/* Renderer.create (integrator.lucb:343): a renderer of `scene` through its camera.
 * The scene's buffers are uploaded; the scene may be freed afterwards. */
int lr_renderer_create(lr_context *ctx, const lr_scene *scene, const lr_settings *settings,
                       lr_renderer **out);
/* Renderer.create_viewed (integrator.lucb:375): through a caller's frame. */
int lr_renderer_create_viewed(lr_context *ctx, const lr_scene *scene, const lr_settings *settings,
                              const lr_frame *frame, lr_renderer **out);
/* Renderer.advance (integrator.lucb:649-693): queue the next pass (one sample of
 * one band) without waiting; *more is 1 while passes are running or to come. At most
 * two passes are in flight; they take turns on two path pools and streams, so the
 * second's first rounds overlap the first's last ones, and their film accumulation runs
 * in order. */
int lr_renderer_advance(lr_renderer *renderer, int32_t *more);
/* Renderer.finish (integrator.lucb:724-729): run every remaining pass and wait. */
int lr_renderer_finish(lr_renderer *renderer);
/* Renderer.samples_done (integrator.lucb:732-733). */
uint32_t lr_renderer_samples_done(const lr_renderer *renderer);
/* The pass bookkeeping behind advance (integrator.lucb:297-313, 622-645): passes
 * recorded so far, passes finished and retired, and bands a sample (passes per sample).
 * Any output may be NULL. */
int lr_renderer_passes(const lr_renderer *renderer, uint64_t *recorded, uint64_t *finished, uint32_t *bands);
/* Renderer.image (integrator.lucb:737-738): the rgba32f ACEScg image in device
 * memory, width*height*16 bytes, row by row from the top. */
int lr_renderer_image(lr_renderer *renderer, void **device_rgba);
/* Renderer.read (integrator.lucb:778-782): the image copied to `rgba` (4 floats a
 * pixel); waits for work in flight. */
int lr_renderer_read(lr_renderer *renderer, float *rgba, uint64_t float_count);
/* (No counterpart: the reference's read waits for the render.) Renderer.read without the
 * wait: queues a copy of the image as the pass launched last leaves it into `rgba` (4
 * floats a pixel; pinned host memory, e.g. lr_host_alloc_pinned, lets the copy run beside
 * the passes launched after it) and returns at once. The buffer must stay untouched until
 * lr_renderer_read_wait returns, which waits for every copy queued. Passes launched
 * later never change a copy in flight. */
int lr_renderer_read_async(lr_renderer *renderer, float *rgba, uint64_t count);
int lr_renderer_read_wait(lr_renderer *renderer);
/* As lr_renderer_read_async, and *ticket names the copy; lr_renderer_read_landed sets
 * *landed to 1 once the copy with `ticket` (and every copy queued before it) has arrived,
 * else 0, without waiting -- so a caller that cycles through a few buffers waits for the
 * copy that last filled the buffer it reuses, not for the newest. */
int lr_renderer_read_ticket(lr_renderer *renderer, float *rgba, uint64_t count, uint64_t *ticket);
int lr_renderer_read_landed(lr_renderer *renderer, uint64_t ticket, int32_t *landed);
/* Orders the context's stream after every pass queued so far, without waiting: work
 * the caller queues there afterwards (reading the device image, an event for timing)
 * sees their results. Passes run on two streams, taking turns; see lr_renderer_advance. */
int lr_renderer_join(lr_renderer *renderer);
/* Renderer.set_samples (integrator.lucb:609-611). */
int lr_renderer_set_samples(lr_renderer *renderer, uint32_t samples);
/* Renderer.restart (integrator.lucb:455-466): start over through `frame` (a moved camera, a
 * resized view; the projection kept). The film clears before the next pass; passes in
 * flight finish uncounted and never show (a new generation); the display keeps the last
 * whole image until the new view's first whole sample replaces it. Waits for nothing
 * unless the view outgrows the renderer's buffers (then the passes in flight are waited
 * for and the buffers made again, a quarter larger each way). */
int lr_renderer_restart(lr_renderer *renderer, const lr_frame *frame);
/* Renderer.reload (integrator.lucb:483-541): the same geometry with other lights,
 * materials or settings (the size and pool kept): `scene` must hold the renderer's points
 * and triangles (400 otherwise); the triangles' normals and materials are uploaded again
 * when they changed. The film starts over, through `frame` (NULL: the current view). */
int lr_renderer_reload(lr_renderer *renderer, const lr_scene *scene, const lr_settings *settings,
                       const lr_frame *frame);
/* Renderer.replace_scene (integrator.lucb:543-574): new geometry in the same renderer (the
 * pool and BVH choice kept, 400 otherwise); the display keeps the last image until the new
 * scene's first whole sample; the old upload is released once the passes that read it
 * have finished. */
int lr_renderer_replace_scene(lr_renderer *renderer, const lr_scene *scene, const lr_settings *settings,
                              const lr_frame *frame);
/* (No counterpart: the reference's replace_scene uploads geometry rebuilt on the host,
 * integrator.lucb:543-574.) The renderer's geometry with its points moved: `scene` is the
 * renderer's compiled scene after lr_scene_move_points (the same triangles, 400
 * otherwise). The renderer's upload is refit on the device after the passes in flight
 * (they finish uncounted, a new generation), the lights, light tree and materials are
 * loaded again from `scene`, and the film starts over through `frame` (NULL: the current
 * view); the display keeps the last whole image until the first new one. Waits for the
 * passes in flight. */
int lr_renderer_refit(lr_renderer *renderer, const lr_scene *scene, const lr_frame *frame);
/* Renderer.display (integrator.lucb:741-746): the render ready to show, rgba16f (4 halves a
 * pixel, row by row at the shown view's width): exposed, in linear Rec.709, through the
 * view; always one whole image of one view (no pass in flight writes it). */
int lr_renderer_display(lr_renderer *renderer, void **device_rgba16f);
/* Renderer.shown_size (integrator.lucb:748-751): the size of the image in the display,
 * (0, 0) before the first whole sample. */
int lr_renderer_shown_size(lr_renderer *renderer, uint32_t out[2]);
/* Renderer.set_display (integrator.lucb:753-757): `exposure` stops through `view` (0
 * standard: clipped; 1 Khronos PBR Neutral tone mapping); the next pass, or a conversion
 * of its own once every sample is taken, applies it. */
int lr_renderer_set_display(lr_renderer *renderer, double exposure, int view);
/* Renderer.converged_pixels (integrator.lucb:759-768): how many pixels adaptive sampling
 * (settings.noise_threshold > 0, checked every 4 samples from adaptive_minimum on) has
 * stopped; waits for work in flight. */
int lr_renderer_converged_pixels(lr_renderer *renderer, uint64_t *out);
/* Renderer.kernel_times (integrator.lucb:873-875): milliseconds per kernel kind
 * over finished passes with settings.profile on, in the order camera, intersect
 * closest, shade surface, shade miss, intersect shadow, light emission, finish,
 * film convert, adaptive, later rounds. */
int lr_renderer_kernel_times(lr_renderer *renderer, double out[10]);

/* Counters of the work finished passes did: rays traced for closest hits and for
 * shadows, paths started, and passes; with settings.profile = 2 also the traversal's
 * interior visits and triangle tests for closest and shadow rays. Waits for work in
 * flight. */
typedef struct {
    uint64_t closest_rays, shadow_rays, shaded, passes;
    uint64_t closest_nodes, closest_tests, shadow_nodes, shadow_tests;
} lr_render_stats;
int lr_renderer_stats(lr_renderer *renderer, lr_render_stats *out);
/* (No counterpart in the reference: a test hook.) With settings.profile = 3 every pass
 * records the rays its traversal kernels traced, round by round; this copies the last
 * pass's records of round `round` -- the closest-hit queue, or with `shadow` the shadow
 * queue -- after waiting for work in flight. 12 floats a ray: origin and the path's tag
 * bits, direction and reach (t_max; the query's t_min is 0), then the triangle
 * traversal's answer: closest (t, source triangle id as int32 bits or -1, u, v), before
 * the analytic lights are tested; shadow (1 blocked, 0 clear, -1 not traced by the
 * any-hit query, 0, 0). *count: the rays of that round; `out` may be NULL to ask for it,
 * else it holds at least 12 * count floats (`capacity`, in floats). */
int lr_renderer_recorded_rays(lr_renderer *renderer, uint32_t round, int32_t shadow, float *out,
                              uint64_t capacity, uint64_t *count);
/* Renderer.destroy (integrator.lucb:887-900). */
void lr_renderer_destroy(lr_renderer *renderer);

/* (No counterpart in the reference, whose tables stay inside its kernels.) The albedo
 * tables the glossy lobes' energy compensation reads (tables.comp:38-61,
 * microfacet.glsl:67-84): LR_ALBEDO_TABLE_SIZE floats -- E_ggx[roughness][mu] (32 x 32),
 * its average over mu (32), E_dielectric[z][roughness][mu] (16 x 32 x 32) -- made on the
 * device once; copied to `out` (count at least LR_ALBEDO_TABLE_SIZE). */
#define LR_ALBEDO_TABLE_SIZE 17440u
int lr_albedo_tables(lr_context *ctx, float *out, size_t count);

/* ---- Batches: many renders in one wavefront ------------------------------------------
 * No counterpart in the reference, which renders one scene per Renderer. A batch is a
 * pool of paths shared by its members (a member: an uploaded scene seen through one
 * camera into its own film, with its own RenderSettings). Every pass traces one sample
 * for as many members' pixels as the pool holds, all in the same kernel launches; each
 * member's image is bit for bit the image an lr_renderer of the same scene, frame and
 * settings makes, whatever else shares the batch. Members may join and leave between
 * passes. All calls on one batch from one host thread. */
typedef struct {
    uint32_t pool;        /* paths per pass (at most 8,388,608) */
    uint32_t max_bounces; /* the most bounces any member may ask for */
    uint32_t capacity;    /* the most members at once */
    int32_t profile;      /* as lr_settings.profile */
} lr_batch_settings;
typedef struct lr_batch lr_batch;

/* pool 2^21, max_bounces 12, capacity 256, profile 0. */
void lr_batch_settings_default(lr_batch_settings *out);
int lr_batch_create(lr_context *ctx, const lr_batch_settings *settings, lr_batch **out);
/* Adds `scene` (uploaded as `gpu_scene` to the batch's device; both stay the caller's
 * and must outlive the member) with `settings`, seen through `frame` or, when
 * it is NULL, through the camera settings name. *member: its index. */
int lr_batch_add(lr_batch *batch, const lr_gpu_scene *gpu_scene, const lr_scene *scene,
                 const lr_settings *settings, const lr_frame *frame, uint32_t *member);
/* The member plans no more passes; its memory goes when its passes in flight finish. */
int lr_batch_remove(lr_batch *batch, uint32_t member);
/* Queues the next pass without waiting (two in flight at most); *more is 1 while
 * passes are running or any member has samples to come. */
int lr_batch_advance(lr_batch *batch, int32_t *more);
/* Runs every remaining pass and waits. */
int lr_batch_finish(lr_batch *batch);
/* As lr_renderer_join, for a batch. */
int lr_batch_join(lr_batch *batch);
/* Waits for the oldest pass in flight, if any, and retires it; *in_flight: passes still
 * in flight after. */
int lr_batch_wait(lr_batch *batch, int32_t *in_flight);
/* Samples finished, samples planned so far and samples asked for. Any may be NULL. */
int lr_batch_member_info(const lr_batch *batch, uint32_t member, uint32_t *samples_done,
                         uint32_t *samples_planned, uint32_t *samples);
int lr_batch_set_samples(lr_batch *batch, uint32_t member, uint32_t samples);
/* As lr_renderer_image / lr_renderer_read, for one member. */
int lr_batch_image(lr_batch *batch, uint32_t member, void **device_rgba);
int lr_batch_read(lr_batch *batch, uint32_t member, float *rgba, uint64_t float_count);
/* lr_renderer_read_async / _wait for a member of a batch. */
int lr_batch_read_async(lr_batch *batch, uint32_t member, float *rgba, uint64_t count);
int lr_batch_read_wait(lr_batch *batch);
/* As lr_batch_read_async, and *ticket names the copy. lr_batch_read_landed sets *landed to
 * 1 once the copy with `ticket` (and every copy queued before it) has arrived in host
 * memory, else 0, without waiting. A member whose image is being read stays in the batch
 * (lr_batch_remove after it landed). */
int lr_batch_read_ticket(lr_batch *batch, uint32_t member, float *rgba, uint64_t count, uint64_t *ticket);
int lr_batch_read_landed(lr_batch *batch, uint64_t ticket, int32_t *landed);
/* The autotuner: times trial passes (which trace but change no film and move no member
 * on) on the members as they stand. For each scene-size class present (under 16k
 * triangles, under 128k, larger) it keeps the BVH width (2, 4, 8; a width all of the
 * class's members fall back from is skipped), the traversal stack depth (each depth the
 * width's kernels offer that holds the members' bound) and the traversal kernels' block
 * size (64, 128, 256 threads) whose passes of that class alone run fastest; a pass then
 * takes the choices of the class holding most of its paths. Then it keeps the fastest
 * pool fill (a quarter, half or all of the pool) for the mixed passes, and the fastest
 * interval at which the shade kernels group outgoing rays by direction octant (never,
 * every round, every second round; the queues are compacted every round regardless),
 * whether the traversal kernels walk their queues in warp batches or as persistent warps
 * that refill idle lanes from the queue (at 32, 16 or 8 idle lanes), and from which round
 * (2, 3, 4 or never) passes on the BVH2 trace their thin later rounds on the compressed
 * 8-wide tree. Images do not change, only speed. */
typedef struct {
    uint32_t width;            /* the widest BVH width chosen for any class */
    uint32_t fill;             /* paths a pass */
    double paths_per_ms;       /* the chosen candidate's measured rate */
    uint32_t candidates;       /* candidates timed */
    uint32_t class_width[3];   /* the width chosen per size class (0: class absent) */
    uint32_t class_members[3]; /* members with samples to come, per size class */
    uint32_t class_stack[3];   /* traversal stack entries chosen per size class */
    uint32_t class_block[3];   /* traversal kernels' threads a block chosen per size class */
    uint32_t bin_interval;     /* rounds between sorts of outgoing rays by octant (0: none) */
    uint32_t refill_at;        /* idle lanes at which traversal warps refill (0: warp batches) */
    int32_t thin_from;         /* first round of a BVH2 pass on the compressed 8-wide tree (-1: none) */
} lr_batch_tuning;
int lr_batch_tune(lr_batch *batch, lr_batch_tuning *out);
int lr_batch_passes(const lr_batch *batch, uint64_t *recorded, uint64_t *finished);
int lr_batch_kernel_times(lr_batch *batch, double out[10]);
int lr_batch_stats(lr_batch *batch, lr_render_stats *out);
void lr_batch_destroy(lr_batch *batch);

/* ---- Serving: sessions and probes as they arrive ----------------------------------
 * No counterpart in the reference. A server owns a batch on one device and two host
 * threads: a render thread that admits queued render sessions, in arrival order, while
 * a live slot is free and the device memory budget holds the session's scene (uploaded
 * on first use, kept resident, evicted least recently used when idle and room is
 * needed) and its film, and advances every live session in shared passes; and a probe
 * thread that runs probe queries on a high-priority stream (without device allocation
 * up to LR_PROBE_STATIC_PIXELS pixels: through lr_probe_static, whose one array a device
 * shares with every other lr_probe_static call of the process -- other servers' probe
 * threads included -- the calls taking turns on the library's per-device lock; its
 * 16 MiB count against budget_bytes, and lr_server_create does its set-up before the
 * threads start). Submitting never waits. A session's image is,
 * bit for bit, what an lr_renderer of the same scene and settings makes; a probe's
 * result is lr_probe's. Times are seconds on the host's steady clock since the server
 * started. */
typedef struct {
    int32_t device;
    uint64_t budget_bytes; /* device memory for resident scenes, live sessions and the pool */
    uint32_t capacity;     /* live sessions at once (1 to 512) */
    uint32_t pool;         /* paths a pass */
    uint32_t max_bounces;  /* the most bounces a session may ask for */
    int32_t probe_priority; /* 1: probes on the device's highest-priority stream */
} lr_server_settings;
typedef struct lr_server lr_server;

#define LR_REQUEST_RENDER 0
#define LR_REQUEST_PROBE 1
#define LR_REQUEST_QUEUED 0
#define LR_REQUEST_RUNNING 1
#define LR_REQUEST_DONE 2
#define LR_REQUEST_FAILED 3

typedef struct {
    int32_t kind, state, status;
    uint32_t scene;
    uint64_t pixels;
    uint32_t samples, samples_done;
    /* submitted; admitted (a live slot, or the probe thread took it); first image (the
     * first sample of every pixel finished); finished. -1: not yet. */
    double submitted, admitted, first, finished;
} lr_request_info;

typedef struct {
    uint64_t sessions_done, probes_done, failed;
    uint64_t pixel_samples; /* pixel-samples finished by render sessions */
    uint64_t probe_rays;
    uint64_t uploads, evictions;
    uint64_t queued, live, scenes_resident;
    uint64_t bytes_in_use;  /* resident scenes, live sessions and the pool */
    double seconds;         /* since the server started */
    uint64_t tunings;       /* autotuner runs on the live mix (from 32 live sessions, every 20 s) */
    /* The render thread: passes it queued, and host seconds spent queueing them, waiting
     * for the oldest in flight, noting progress (images out included), admitting, and
     * tuning. */
    uint64_t passes;
    double seconds_advance, seconds_wait, seconds_progress, seconds_admit, seconds_tune;
} lr_server_stats;

/* device 0, budget 150 GB, capacity 128, pool 2^22, max_bounces 12, probe_priority 1. */
void lr_server_settings_default(lr_server_settings *out);
int lr_server_create(const lr_server_settings *settings, lr_server **out);
/* Registers a compiled scene (the caller's; it must outlive the server). */
int lr_server_add_scene(lr_server *server, const lr_scene *scene, uint32_t *scene_id);
/* Uploads the scene now (on the caller's thread) rather than at its first request, if
 * the budget has room (LR_LIMIT otherwise); it stays resident until evicted. */
int lr_server_preload(lr_server *server, uint32_t scene_id);
/* A progressive render of `settings.samples` samples through `frame` (NULL: the camera
 * the settings name); when `rgba` is not NULL the finished image is copied there
 * (width*height*4 floats). The session leaves the GPU when it finishes. */
int lr_server_submit_render(lr_server *server, uint32_t scene_id, const lr_settings *settings,
                            const lr_frame *frame, float *rgba, uint64_t *request);
/* A probe (as lr_probe) into the caller's buffers, which must stay valid until it is
 * finished; pinned host memory keeps the copy short. */
int lr_server_submit_probe(lr_server *server, uint32_t scene_id, const lr_frame *frame,
                           uint32_t flags, uint32_t *faces, float *distances, uint64_t *request);
int lr_server_request_info(lr_server *server, uint64_t request, lr_request_info *out);
/* Waits up to `timeout_seconds` for the request: LR_OK when it finished, LR_TIMEOUT, or
 * the request's own failure. */
int lr_server_wait(lr_server *server, uint64_t request, double timeout_seconds);
int lr_server_stats_get(lr_server *server, lr_server_stats *out);
/* Stops both threads (requests not finished end with LR_STOPPED) and frees everything. */
void lr_server_destroy(lr_server *server);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif
#endif
