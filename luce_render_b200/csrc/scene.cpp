// Scene compile (src/render/scene.lucb:111-295) and ray frames (src/render/camera.lucb):
// meshes placed into one world-space triangle list with their polygons, octahedral
// shading normals and materials, then the BVH; cameras and lights carried through.
#include <algorithm>
#include <memory>

#include "common.hpp"

namespace lr {
namespace {

struct Placement {
    V3 x{1, 0, 0}, y{0, 1, 0}, z{0, 0, 1}, t{0, 0, 0};
    explicit Placement(const double m[12]) {
        bool zero = true;
        for (int k = 0; k < 12; k++) zero = zero && m[k] == 0.0;
        if (zero) return;
        x = {m[0], m[1], m[2]};
        y = {m[3], m[4], m[5]};
        z = {m[6], m[7], m[8]};
        t = {m[9], m[10], m[11]};
    }
    // Matrix4.transform_point
    V3 point(const V3 &p) const { return x * p.x + y * p.y + z * p.z + t; }
};

// The mesh's shading normals placed by its matrix's inverse transpose (the cofactors
// with the determinant's sign, scene.lucb:365-396) and encoded.
struct NormalPlacer {
    V3 c0, c1, c2;
    bool singular;
    explicit NormalPlacer(const Placement &m) {
        double det = m.x.dot(m.y.cross(m.z));
        double sign = det >= 0.0 ? 1.0 : -1.0;
        singular = det == 0.0 || !std::isfinite(det);
        c0 = m.y.cross(m.z) * sign;
        c1 = m.z.cross(m.x) * sign;
        c2 = m.x.cross(m.y) * sign;
    }
    uint32_t encode(const V3 &n) const {
        V3 placed = singular ? V3(0.0, 1.0, 0.0) : c0 * n.x + c1 * n.y + c2 * n.z;
        return octahedral(placed);
    }
};

void add_mesh(Scene &scene, const lr_mesh &mesh, uint32_t &face_base, size_t library) {
    if (mesh.triangle_count > 0 && (!mesh.indices || !mesh.positions))
        fail(LR_INVALID, "a mesh with triangles needs positions and indices");
    if (mesh.point_count > 0 && !mesh.positions) fail(LR_INVALID, "a mesh's points need positions");
    Placement m(mesh.transform);
    NormalPlacer normals(m);
    const uint64_t base = scene.point_count();
    if (base + mesh.point_count > 0xffffffffull) fail(LR_LIMIT, "a scene holds at most 2^32 points");
    for (uint64_t i = 0; i < mesh.point_count; i++) {
        V3 p = m.point({mesh.positions[i * 3], mesh.positions[i * 3 + 1], mesh.positions[i * 3 + 2]});
        scene.positions.push_back((float)p.x);
        scene.positions.push_back((float)p.y);
        scene.positions.push_back((float)p.z);
    }
    const uint32_t faces = mesh.face_count ? mesh.face_count : (uint32_t)mesh.triangle_count;
    if ((uint64_t)face_base + faces > 0xffffffffull) fail(LR_LIMIT, "a scene holds at most 2^32 polygons");
    for (uint64_t t = 0; t < mesh.triangle_count; t++) {
        uint32_t corner[3];
        for (int k = 0; k < 3; k++) {
            corner[k] = mesh.indices[t * 3 + k];
            if (corner[k] >= mesh.point_count) fail(LR_INVALID, "a triangle names a point the mesh lacks");
            scene.indices.push_back((uint32_t)(base + corner[k]));
        }
        uint32_t face = mesh.triangle_faces ? mesh.triangle_faces[t] : (uint32_t)t;
        if (face >= faces) fail(LR_INVALID, "a triangle names a polygon the mesh lacks");
        // A polygon's material: its library index + 1, or 0 (the render's default)
        // for none or an unknown one (scene.lucb:297-317).
        uint32_t material = mesh.face_materials ? mesh.face_materials[face] : 0u;
        if (material > library) material = 0;
        scene.used[material] = 1;
        uint32_t encoded[3];
        if (mesh.normals && mesh.normals_per_corner) {
            for (int k = 0; k < 3; k++) {
                const float *n = &mesh.normals[(t * 3 + k) * 3];
                encoded[k] = normals.encode({n[0], n[1], n[2]});
            }
        } else if (mesh.normals) {
            for (int k = 0; k < 3; k++) {
                const float *n = &mesh.normals[(size_t)corner[k] * 3];
                encoded[k] = normals.encode({n[0], n[1], n[2]});
            }
        } else {
            // No authored normals: the triangle's own (flat) normal, in world space.
            const float *p = scene.positions.data();
            const uint32_t flat =
                flat_normal(&p[(base + corner[0]) * 3], &p[(base + corner[1]) * 3], &p[(base + corner[2]) * 3]);
            encoded[0] = encoded[1] = encoded[2] = flat;
        }
        scene.flat.push_back(mesh.normals ? 0 : 1);
        scene.shading.push_back(encoded[0]);
        scene.shading.push_back(encoded[1]);
        scene.shading.push_back(encoded[2]);
        scene.shading.push_back(material);
        scene.faces.push_back(face_base + face);
    }
    face_base += faces;
}

}  // namespace

uint32_t flat_normal(const float *a, const float *b, const float *c) {
    const V3 pa(a[0], a[1], a[2]), pb(b[0], b[1], b[2]), pc(c[0], c[1], c[2]);
    return octahedral((pb - pa).cross(pc - pa));
}

// Moves the points and refits the BVH2 in place: every node's box again from its
// triangles (a leaf) or its children (an interior node; children follow their parent in
// the numbering, so one pass from the last node back reaches every child first), the
// topology and leaf order kept.
void move_points(Scene &scene, const float *positions) {
    std::copy(positions, positions + scene.positions.size(), scene.positions.begin());
    const float *p = scene.positions.data();
    const size_t T = scene.triangle_count();
    for (size_t t = 0; t < T; t++) {
        if (!scene.flat[t]) continue;
        const uint32_t n = flat_normal(&p[(size_t)scene.indices[t * 3] * 3], &p[(size_t)scene.indices[t * 3 + 1] * 3],
                                       &p[(size_t)scene.indices[t * 3 + 2] * 3]);
        scene.shading[t * 4] = scene.shading[t * 4 + 1] = scene.shading[t * 4 + 2] = n;
    }
    if (T == 0) return;
    for (size_t n = scene.nodes.size(); n-- > 0;) {
        lr_bvh_node &node = scene.nodes[n];
        float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        if (node.count > 0) {
            for (uint32_t t = node.first; t < node.first + node.count; t++)
                for (int c = 0; c < 3; c++) {
                    const float *v = &p[(size_t)scene.indices[(size_t)t * 3 + c] * 3];
                    for (int k = 0; k < 3; k++) {
                        lo[k] = std::min(lo[k], v[k]);
                        hi[k] = std::max(hi[k], v[k]);
                    }
                }
        } else {
            for (uint32_t c = node.first; c < node.first + 2; c++)
                for (int k = 0; k < 3; k++) {
                    lo[k] = std::min(lo[k], scene.nodes[c].lo[k]);
                    hi[k] = std::max(hi[k], scene.nodes[c].hi[k]);
                }
        }
        for (int k = 0; k < 3; k++) {
            node.lo[k] = lo[k];
            node.hi[k] = hi[k];
        }
    }
}

// ray_frame (camera.lucb:57-76)
void camera_frame(const lr_camera &camera, uint32_t width, uint32_t height, lr_frame &out) {
    if (width == 0 || height == 0) fail(LR_INVALID, "an image needs pixels");
    const double *m = camera.matrix;
    V3 right = unit({m[0], m[1], m[2]}, "the camera's x axis");
    V3 up = unit({m[3], m[4], m[5]}, "the camera's y axis");
    V3 back = unit({m[6], m[7], m[8]}, "the camera's z axis");
    V3 forward = back * -1.0;
    double aspect = (double)height / (double)width;
    bool ortho = camera.projection == 1;
    if (!ortho && !(camera.focal_length > 0.0)) fail(LR_INVALID, "a perspective camera needs a focal length");
    double half_width = ortho ? 0.05 * camera.horizontal_aperture : 0.5 * camera.horizontal_aperture / camera.focal_length;
    double half_height = half_width * aspect;
    V3 corner = right * -half_width + up * half_height + (ortho ? V3() : forward);
    V3 du = right * (2.0 * half_width / (double)width);
    V3 dv = up * (-2.0 * half_height / (double)height);
    out = lr_frame{};
    for (int k = 0; k < 3; k++) {
        out.position[k] = m[9 + k];
        out.corner[k] = corner[k];
        out.du[k] = du[k];
        out.dv[k] = dv[k];
        out.forward[k] = forward[k];
    }
    out.orthographic = ortho ? 1 : 0;
    out.width = width;
    out.height = height;
    out.lens_radius = camera.f_stop > 0.0 && !ortho ? 0.0005 * camera.focal_length / camera.f_stop : 0.0;
    out.focus_distance = camera.focus_distance;
}

// look_frame (camera.lucb:84-95)
void look_frame(const double position[3], const double forward[3], const double up[3],
                double tan_half_height, uint32_t width, uint32_t height, bool orthographic,
                lr_frame &out) {
    if (width == 0 || height == 0) fail(LR_INVALID, "an image needs pixels");
    if (!(tan_half_height > 0.0 && tan_half_height < 1e6))
        fail(LR_INVALID, "a view needs a field of view between 0 and 180 degrees, or a height");
    V3 ahead = unit({forward[0], forward[1], forward[2]}, "the view's forward");
    V3 right = unit(ahead.cross({up[0], up[1], up[2]}), "the view's right");
    V3 above = right.cross(ahead);
    double half_height = tan_half_height;
    double half_width = half_height * (double)width / (double)height;
    V3 corner = right * -half_width + above * half_height + (orthographic ? V3() : ahead);
    V3 du = right * (2.0 * half_width / (double)width);
    V3 dv = above * (-2.0 * half_height / (double)height);
    out = lr_frame{};
    for (int k = 0; k < 3; k++) {
        out.position[k] = position[k];
        out.corner[k] = corner[k];
        out.du[k] = du[k];
        out.dv[k] = dv[k];
        out.forward[k] = ahead[k];
    }
    out.orthographic = orthographic ? 1 : 0;
    out.width = width;
    out.height = height;
    out.lens_radius = 0.0;
    out.focus_distance = 1.0;
}

// RayFrame.pack (camera.lucb:41-47)
void pack_frame(const lr_frame &f, float out[16]) {
    const double v[16] = {f.position[0], f.position[1], f.position[2], f.orthographic ? 1.0 : 0.0,
                          f.corner[0],   f.corner[1],   f.corner[2],   0.0,
                          f.du[0],       f.du[1],       f.du[2],       (double)f.width,
                          f.dv[0],       f.dv[1],       f.dv[2],       (double)f.height};
    for (int k = 0; k < 16; k++) out[k] = (float)v[k];
}

}  // namespace lr

using namespace lr;

extern "C" {

void lr_openpbr_standard(lr_openpbr *m) {
    if (!m) return;
    *m = lr_openpbr{};
    m->base_weight = 1.0;
    for (int k = 0; k < 3; k++) {
        m->base_color[k] = 0.8;
        m->specular_color[k] = 1.0;
        m->transmission_color[k] = 1.0;
        m->coat_color[k] = 1.0;
        m->emission_color[k] = 1.0;
    }
    m->specular_weight = 1.0;
    m->specular_roughness = 0.3;
    m->specular_ior = 1.5;
    m->coat_ior = 1.6;
    m->coat_darkening = 1.0;
    m->geometry_opacity = 1.0;
    m->transmission_dispersion_abbe_number = 20.0;
}

int lr_scene_compile(const lr_mesh *meshes, size_t mesh_count, const lr_camera *cameras,
                     size_t camera_count, const lr_light *lights, size_t light_count,
                     const lr_openpbr *materials, size_t material_count, lr_scene **out) {
    return lr_scene_compile_ex(meshes, mesh_count, cameras, camera_count, lights, light_count, materials,
                               material_count, 0u, out);
}

int lr_scene_compile_ex(const lr_mesh *meshes, size_t mesh_count, const lr_camera *cameras,
                        size_t camera_count, const lr_light *lights, size_t light_count,
                        const lr_openpbr *materials, size_t material_count, uint32_t flags, lr_scene **out) {
    return guarded([&] {
        if (flags & ~LR_COMPILE_NO_TREES) fail(LR_INVALID, "unknown compile flags");
        if (!out) fail(LR_INVALID, "compile_scene needs somewhere to put the scene");
        *out = nullptr;
        if ((mesh_count && !meshes) || (camera_count && !cameras) || (light_count && !lights) ||
            (material_count && !materials))
            fail(LR_INVALID, "a count without its array");
        auto scene = std::make_unique<lr_scene>();
        scene->materials.assign(materials, materials + material_count);
        scene->used.assign(material_count + 1, 0);
        uint32_t face_base = 0;
        for (size_t i = 0; i < mesh_count; i++) add_mesh(*scene, meshes[i], face_base, material_count);
        scene->face_count = face_base;
        scene->cameras.assign(cameras, cameras + camera_count);
        scene->light_images.resize(light_count);
        for (size_t i = 0; i < light_count; i++) {
            const lr_light &l = lights[i];
            if (l.shape < 0 || l.shape > LR_LIGHT_DOME) fail(LR_INVALID, "a light is rect, disk, sphere, distant or dome");
            if (l.shape != LR_LIGHT_DOME || !l.image) continue;
            // A dome's image (environment.lucb:102-156; the reference caps images at 2^26 pixels).
            const uint64_t pixels = (uint64_t)l.image_width * l.image_height;
            if (pixels == 0) fail(LR_INVALID, "a dome's image has no pixels");
            if (pixels > (1ull << 26)) fail(LR_LIMIT, "a dome's image is larger than 67,108,864 pixels");
            scene->light_images[i].assign(l.image, l.image + pixels * 3);
        }
        scene->lights.assign(lights, lights + light_count);
        for (lr_light &l : scene->lights) l.image = nullptr;
        if (flags & LR_COMPILE_NO_TREES) {
            // Without trees (scene.lucb:127-128): the triangles in the meshes' order.
            if (scene->triangle_count() > 0x7fffffffull) fail(LR_LIMIT, "a scene holds at most 2^31 triangles");
            scene->nodes.clear();
            scene->order.resize(scene->triangle_count());
            for (size_t t = 0; t < scene->order.size(); t++) scene->order[t] = (uint32_t)t;
            scene->bvh_depth = 0;
        } else {
            build_bvh(*scene);
        }
        *out = scene.release();
    });
}

void lr_scene_free(lr_scene *scene) { delete scene; }

int lr_scene_move_points(lr_scene *scene, const float *positions, uint64_t point_count) {
    return guarded([&] {
        if (!scene || (point_count && !positions)) fail(LR_INVALID, "moving points needs a scene and its points");
        if (point_count != scene->point_count()) fail(LR_INVALID, "a move keeps the scene's point count");
        for (uint64_t i = 0; i < point_count * 3; i++)
            if (!std::isfinite(positions[i])) fail(LR_INVALID, "a moved point is not finite");
        move_points(*scene, positions);
    });
}

int lr_scene_info_get(const lr_scene *scene, lr_scene_info *out) {
    return guarded([&] {
        if (!scene || !out) fail(LR_INVALID, "no scene");
        out->point_count = scene->point_count();
        out->triangle_count = scene->triangle_count();
        out->node_count = scene->nodes.size();
        out->face_count = scene->face_count;
        out->camera_count = (uint32_t)scene->cameras.size();
        out->light_count = (uint32_t)scene->lights.size();
        out->material_count = (uint32_t)scene->materials.size();
        out->bvh_depth = scene->bvh_depth;
    });
}

int lr_scene_arrays(const lr_scene *scene, const float **positions, const uint32_t **indices,
                    const uint32_t **faces, const uint32_t **shading, const lr_bvh_node **nodes,
                    const uint32_t **order) {
    return guarded([&] {
        if (!scene) fail(LR_INVALID, "no scene");
        if (positions) *positions = scene->positions.data();
        if (indices) *indices = scene->indices.data();
        if (faces) *faces = scene->faces.data();
        if (shading) *shading = scene->shading.data();
        if (nodes) *nodes = scene->nodes.data();
        if (order) *order = scene->order.data();
    });
}

int lr_ray_frame(const lr_camera *camera, uint32_t width, uint32_t height, lr_frame *out) {
    return guarded([&] {
        if (!camera || !out) fail(LR_INVALID, "a ray frame needs a camera");
        camera_frame(*camera, width, height, *out);
    });
}

int lr_look_frame(const double position[3], const double forward[3], const double up[3],
                  double tan_half_height, uint32_t width, uint32_t height, int32_t orthographic,
                  lr_frame *out) {
    return guarded([&] {
        if (!position || !forward || !up || !out) fail(LR_INVALID, "a view needs a place");
        look_frame(position, forward, up, tan_half_height, width, height, orthographic != 0, *out);
    });
}

int lr_frame_pack(const lr_frame *frame, float out[16]) {
    return guarded([&] {
        if (!frame || !out) fail(LR_INVALID, "a ray frame packs into 16 floats");
        pack_frame(*frame, out);
    });
}

int lr_scene_camera(const lr_scene *scene, int32_t index, lr_camera *out) {
    return guarded([&] {
        if (!scene || !out) fail(LR_INVALID, "no scene");
        if (index >= 0) {
            if ((size_t)index >= scene->cameras.size()) fail(LR_INVALID, "the scene object is not a camera");
            *out = scene->cameras[(size_t)index];
            return;
        }
        if (scene->cameras.empty()) fail(LR_INVALID, "the scene has no camera");
        *out = scene->cameras[0];
    });
}

}  // extern "C"
