/*
 * Scene compile for the oracle (TEST INFRASTRUCTURE): meshes placed into one world-space
 * triangle list with polygons, octahedral shading normals and materials, then the BVH
 * and the leaf order (src/render/scene.lucb:111-129 compile_scene, 253-294 add_mesh,
 * 364-398 shading_normals / encode_all, bvh.lucb:66-82 build_bvh, 198-217 reorder).
 *
 * The reference reads meshes from a luce-geocore GeometrySet, which is not available
 * here; the boundary takes flat arrays instead, with the same meaning: per-point or
 * per-corner normals, else the triangle's own normal (the reference's smooth normals
 * come from luce-geocore and are not restated), a polygon per triangle and a material
 * index per polygon (0 the render's default, index + 1 a library material, an unknown
 * one 0: scene.lucb:297-317). Placement and the normals' cofactor matrix are f64, the
 * placed points f32, as in the reference.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

typedef struct {
    double x[3], y[3], z[3], t[3];
} placement;

static placement placement_of(const double m[12]) {
    placement p = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {0, 0, 0}};
    int zero = 1;
    for (int k = 0; k < 12; k++) zero = zero && m[k] == 0.0;
    if (zero) return p;
    for (int k = 0; k < 3; k++) {
        p.x[k] = m[k];
        p.y[k] = m[3 + k];
        p.z[k] = m[6 + k];
        p.t[k] = m[9 + k];
    }
    return p;
}

static void cross3(const double a[3], const double b[3], double out[3]) {
    out[0] = a[1] * b[2] - a[2] * b[1];
    out[1] = a[2] * b[0] - a[0] * b[2];
    out[2] = a[0] * b[1] - a[1] * b[0];
}

/* The normal placer of shading_normals (scene.lucb:364-398): the cofactors of the
 * placement scaled by its determinant's sign; a singular placement gives +Y. */
typedef struct {
    double c0[3], c1[3], c2[3];
    int singular;
} normal_placer;

static normal_placer placer_of(const placement *m) {
    normal_placer np;
    double yz[3], zx[3], xy[3];
    cross3(m->y, m->z, yz);
    cross3(m->z, m->x, zx);
    cross3(m->x, m->y, xy);
    double det = m->x[0] * yz[0] + m->x[1] * yz[1] + m->x[2] * yz[2];
    double sign = det >= 0.0 ? 1.0 : -1.0;
    np.singular = det == 0.0 || !isfinite(det);
    for (int k = 0; k < 3; k++) {
        np.c0[k] = yz[k] * sign;
        np.c1[k] = zx[k] * sign;
        np.c2[k] = xy[k] * sign;
    }
    return np;
}

static uint32_t place_normal(const normal_placer *np, const float n[3]) {
    double placed[3] = {0.0, 1.0, 0.0};
    if (!np->singular)
        for (int k = 0; k < 3; k++) placed[k] = np->c0[k] * n[0] + np->c1[k] * n[1] + np->c2[k] * n[2];
    return or_octahedral(placed);
}

static uint32_t triangle_normal(const float *a, const float *b, const float *c) {
    double e1[3], e2[3], n[3];
    for (int k = 0; k < 3; k++) {
        e1[k] = (double)b[k] - (double)a[k];
        e2[k] = (double)c[k] - (double)a[k];
    }
    cross3(e1, e2, n);
    return or_octahedral(n);
}

int or_compile_meshes(const or_mesh *meshes, size_t mesh_count, size_t library, float *positions, uint32_t *indices,
                      uint32_t *shading, uint32_t *faces, or_node *nodes, uint32_t *order, size_t *node_count) {
    size_t points = 0, triangles = 0;
    uint32_t face_base = 0;
    for (size_t mi = 0; mi < mesh_count; mi++) {
        const or_mesh *mesh = &meshes[mi];
        placement m = placement_of(mesh->transform);
        normal_placer np = placer_of(&m);
        const uint32_t base = (uint32_t)points;
        for (uint64_t i = 0; i < mesh->point_count; i++) {
            const float *p = &mesh->positions[i * 3];
            for (int k = 0; k < 3; k++)
                positions[(points + i) * 3 + k] =
                    (float)(m.x[k] * p[0] + m.y[k] * p[1] + m.z[k] * p[2] + m.t[k]);
        }
        const uint32_t polygons = mesh->face_count ? mesh->face_count : (uint32_t)mesh->triangle_count;
        for (uint64_t t = 0; t < mesh->triangle_count; t++) {
            const size_t out = triangles + t;
            uint32_t corner[3];
            for (int k = 0; k < 3; k++) {
                corner[k] = mesh->indices[t * 3 + k];
                if (corner[k] >= mesh->point_count) return -1;
                indices[out * 3 + k] = base + corner[k];
            }
            const uint32_t face = mesh->faces ? mesh->faces[t] : (uint32_t)t;
            if (face >= polygons) return -1;
            uint32_t material = mesh->face_materials ? mesh->face_materials[face] : 0u;
            if (material > library) material = 0u;
            for (int k = 0; k < 3; k++) {
                if (mesh->normals)
                    shading[out * 4 + k] =
                        place_normal(&np, &mesh->normals[(mesh->normals_per_corner ? t * 3 + k : corner[k]) * 3]);
                else
                    shading[out * 4 + k] = triangle_normal(&positions[(size_t)(base + corner[0]) * 3],
                                                           &positions[(size_t)(base + corner[1]) * 3],
                                                           &positions[(size_t)(base + corner[2]) * 3]);
            }
            shading[out * 4 + 3] = material;
            faces[out] = face_base + face;
        }
        points += mesh->point_count;
        triangles += mesh->triangle_count;
        face_base += polygons;
    }
    *node_count = or_build_bvh(positions, indices, triangles, nodes, order);
    or_reorder(order, triangles, indices, faces, shading, NULL);
    return 0;
}
