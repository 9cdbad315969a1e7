/*
 * Oracle (test infrastructure): the reference's software traversal (shaders/bvh.glsl)
 * with visit counters, the reference's f64 brute force (tests/gpu/main.lucb:82-119),
 * and an FP32 brute force over the watertight test the CUDA kernels use.
 */
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include "oracle.h"

/* ---- shaders/bvh.glsl ------------------------------------------------------------ */

static void safe_inverse(const float d[3], float inv[3]) {
    /* bvh.glsl:55-56: components below 1e-20 in magnitude become +-1e-20 (+1e-20 for 0). */
    for (int k = 0; k < 3; k++) {
        float s = d[k];
        if (fabsf(d[k]) < 1e-20f) {
            float sign = d[k] > 0.0f ? 1.0f : (d[k] < 0.0f ? -1.0f : 0.0f);
            s = sign * 1e-20f + (d[k] == 0.0f ? 1.0f : 0.0f) * 1e-20f;
        }
        inv[k] = 1.0f / s;
    }
}

static float fmin32(float a, float b) { return a < b ? a : b; }
static float fmax32(float a, float b) { return a > b ? a : b; }

/* box_entry (bvh.glsl:17-25) */
static float box_entry(const float lo[3], const float hi[3], const float o[3], const float inv[3],
                       float t_max) {
    float near_[3], far_[3];
    for (int k = 0; k < 3; k++) {
        float a = (lo[k] - o[k]) * inv[k];
        float b = (hi[k] - o[k]) * inv[k];
        near_[k] = fmin32(a, b);
        far_[k] = fmax32(a, b);
    }
    float enter = fmax32(fmax32(near_[0], near_[1]), fmax32(near_[2], 0.0f));
    float leave = fmin32(fmin32(far_[0], far_[1]), fmin32(far_[2], t_max));
    return enter <= leave ? enter : -1.0f;
}

static void point_at(const float *positions, uint32_t index, float p[3]) {
    p[0] = positions[(size_t)index * 3];
    p[1] = positions[(size_t)index * 3 + 1];
    p[2] = positions[(size_t)index * 3 + 2];
}

static void cross3(const float a[3], const float b[3], float out[3]) {
    out[0] = a[1] * b[2] - a[2] * b[1];
    out[1] = a[2] * b[0] - a[0] * b[2];
    out[2] = a[0] * b[1] - a[1] * b[0];
}

static float dot3(const float a[3], const float b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

/* triangle_hit (bvh.glsl:27-47): Moller-Trumbore. */
static int triangle_hit(const float *positions, const uint32_t *indices, uint32_t triangle,
                        const float o[3], const float d[3], or_hit *hit) {
    float p0[3], p1[3], p2[3], e1[3], e2[3], p[3], s[3], q[3];
    point_at(positions, indices[(size_t)triangle * 3], p0);
    point_at(positions, indices[(size_t)triangle * 3 + 1], p1);
    point_at(positions, indices[(size_t)triangle * 3 + 2], p2);
    for (int k = 0; k < 3; k++) {
        e1[k] = p1[k] - p0[k];
        e2[k] = p2[k] - p0[k];
    }
    cross3(d, e2, p);
    float determinant = dot3(e1, p);
    if (fabsf(determinant) < 1e-20f) return 0;
    float inverse = 1.0f / determinant;
    for (int k = 0; k < 3; k++) s[k] = o[k] - p0[k];
    float u = dot3(s, p) * inverse;
    if (u < 0.0f || u > 1.0f) return 0;
    cross3(s, e1, q);
    float v = dot3(d, q) * inverse;
    if (v < 0.0f || u + v > 1.0f) return 0;
    float t = dot3(e2, q) * inverse;
    if (t <= 0.0f || t >= hit->t) return 0;
    hit->t = t;
    hit->triangle = triangle;
    hit->u = u;
    hit->v = v;
    return 1;
}

#define REF_STACK 32 /* bvh.glsl:49 */

typedef struct {
    uint32_t *items;
    size_t depth, cap;
    int limit;
} stack_t_;

static int push(stack_t_ *s, uint32_t v, or_counts *c) {
    if (s->limit > 0 && s->depth >= (size_t)s->limit) {
        if (c) c->dropped++;
        return 0;
    }
    if (s->depth == s->cap) {
        s->cap *= 2;
        s->items = realloc(s->items, s->cap * sizeof(uint32_t));
    }
    s->items[s->depth++] = v;
    return 1;
}

/* trace_closest (bvh.glsl:51-90) */
or_hit or_trace_closest(const or_node *nodes, const float *positions, const uint32_t *indices,
                        const float o[3], const float d[3], float t_max, int stack_limit,
                        or_counts *counts) {
    or_hit hit = {t_max, OR_NONE, 0.0f, 0.0f};
    float inv[3];
    safe_inverse(d, inv);
    uint32_t local[64];
    stack_t_ st = {local, 0, 64, stack_limit};
    uint32_t node = 0;
    if (nodes[0].lo[0] > nodes[0].hi[0] || box_entry(nodes[0].lo, nodes[0].hi, o, inv, hit.t) < 0.0f)
        return hit;
    for (;;) {
        const or_node *current = &nodes[node];
        if (current->count > 0) {
            for (uint32_t i = 0; i < current->count; i++) {
                if (counts) counts->triangles++;
                triangle_hit(positions, indices, current->first + i, o, d, &hit);
            }
        } else {
            if (counts) counts->interior++;
            uint32_t left = current->first, right = left + 1;
            float a = box_entry(nodes[left].lo, nodes[left].hi, o, inv, hit.t);
            float b = box_entry(nodes[right].lo, nodes[right].hi, o, inv, hit.t);
            int take_left = a >= 0.0f, take_right = b >= 0.0f;
            if (take_left && take_right) {
                uint32_t near_child = a <= b ? left : right;
                uint32_t far_child = a <= b ? right : left;
                push(&st, far_child, counts);
                node = near_child;
                continue;
            }
            if (take_left) {
                node = left;
                continue;
            }
            if (take_right) {
                node = right;
                continue;
            }
        }
        if (st.depth == 0) break;
        node = st.items[--st.depth];
    }
    if (st.items != local) free(st.items);
    return hit;
}

/* trace_any (bvh.glsl:93-122) */
int or_trace_any(const or_node *nodes, const float *positions, const uint32_t *indices,
                 const float o[3], const float d[3], float t_max, int stack_limit,
                 or_counts *counts) {
    or_hit hit = {t_max, OR_NONE, 0.0f, 0.0f};
    float inv[3];
    safe_inverse(d, inv);
    uint32_t local[64];
    stack_t_ st = {local, 0, 64, stack_limit};
    uint32_t node = 0;
    int found = 0;
    if (nodes[0].lo[0] > nodes[0].hi[0] || box_entry(nodes[0].lo, nodes[0].hi, o, inv, t_max) < 0.0f)
        return 0;
    for (;;) {
        const or_node *current = &nodes[node];
        if (current->count > 0) {
            for (uint32_t i = 0; i < current->count; i++) {
                if (counts) counts->triangles++;
                if (triangle_hit(positions, indices, current->first + i, o, d, &hit)) {
                    found = 1;
                    goto done;
                }
            }
        } else {
            if (counts) counts->interior++;
            uint32_t left = current->first;
            int take_left = box_entry(nodes[left].lo, nodes[left].hi, o, inv, t_max) >= 0.0f;
            int take_right = box_entry(nodes[left + 1].lo, nodes[left + 1].hi, o, inv, t_max) >= 0.0f;
            if (take_left && take_right) {
                push(&st, left + 1, counts);
                node = left;
                continue;
            }
            if (take_left) {
                node = left;
                continue;
            }
            if (take_right) {
                node = left + 1;
                continue;
            }
        }
        if (st.depth == 0) break;
        node = st.items[--st.depth];
    }
done:
    if (st.items != local) free(st.items);
    return found;
}

/* ---- A tiny thread pool over index ranges ---------------------------------------- */

typedef void (*range_fn)(void *ctx, size_t begin, size_t end, or_counts *counts);

typedef struct {
    range_fn fn;
    void *ctx;
    size_t n, next, chunk;
    pthread_mutex_t lock;
    or_counts total;
} pool_t;

static void *pool_worker(void *arg) {
    pool_t *p = arg;
    or_counts mine = {0, 0, 0};
    for (;;) {
        pthread_mutex_lock(&p->lock);
        size_t begin = p->next;
        p->next = begin + p->chunk < p->n ? begin + p->chunk : p->n;
        size_t end = p->next;
        pthread_mutex_unlock(&p->lock);
        if (begin >= end) break;
        p->fn(p->ctx, begin, end, &mine);
    }
    pthread_mutex_lock(&p->lock);
    p->total.interior += mine.interior;
    p->total.triangles += mine.triangles;
    p->total.dropped += mine.dropped;
    pthread_mutex_unlock(&p->lock);
    return NULL;
}

static void run_pool(range_fn fn, void *ctx, size_t n, int threads, size_t chunk, or_counts *counts) {
    if (threads <= 0) threads = (int)sysconf(_SC_NPROCESSORS_ONLN);
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    pool_t p;
    p.fn = fn;
    p.ctx = ctx;
    p.n = n;
    p.next = 0;
    p.chunk = chunk ? chunk : 64;
    memset(&p.total, 0, sizeof p.total);
    pthread_mutex_init(&p.lock, NULL);
    pthread_t ids[256];
    for (int i = 0; i < threads; i++) pthread_create(&ids[i], NULL, pool_worker, &p);
    for (int i = 0; i < threads; i++) pthread_join(ids[i], NULL);
    pthread_mutex_destroy(&p.lock);
    if (counts) *counts = p.total;
}

typedef struct {
    const or_node *nodes;
    const float *positions;
    const uint32_t *indices;
    const float *rays;
    int stack_limit;
    or_hit *hits;
    uint8_t *any;
} trace_ctx;

static void closest_range(void *c, size_t begin, size_t end, or_counts *counts) {
    trace_ctx *x = c;
    for (size_t i = begin; i < end; i++) {
        const float *r = &x->rays[i * 8];
        x->hits[i] = or_trace_closest(x->nodes, x->positions, x->indices, r, r + 4, r[7],
                                      x->stack_limit, counts);
    }
}

static void any_range(void *c, size_t begin, size_t end, or_counts *counts) {
    trace_ctx *x = c;
    for (size_t i = begin; i < end; i++) {
        const float *r = &x->rays[i * 8];
        x->any[i] = (uint8_t)or_trace_any(x->nodes, x->positions, x->indices, r, r + 4, r[7],
                                          x->stack_limit, counts);
    }
}

void or_trace_closest_batch(const or_node *nodes, const float *positions, const uint32_t *indices,
                            const float *rays, size_t n, int stack_limit, or_hit *out,
                            or_counts *counts, int threads) {
    trace_ctx x = {nodes, positions, indices, rays, stack_limit, out, NULL};
    run_pool(closest_range, &x, n, threads, 256, counts);
}

void or_trace_any_batch(const or_node *nodes, const float *positions, const uint32_t *indices,
                        const float *rays, size_t n, int stack_limit, uint8_t *out,
                        or_counts *counts, int threads) {
    trace_ctx x = {nodes, positions, indices, rays, stack_limit, NULL, out};
    run_pool(any_range, &x, n, threads, 256, counts);
}

/* ---- tests/gpu/main.lucb:82-119: the f64 brute force ------------------------------ */

typedef struct {
    const float *positions;
    const uint32_t *indices, *faces;
    size_t triangle_count;
    const float *rays;
    int64_t *face;
    double *distance, *margin;
} nearest_ctx;

/* hit (main.lucb:105-119): Moller-Trumbore in f64; -1 when the ray misses. */
static double hit_f64(const float *p, const uint32_t *corners, const double o[3], const double d[3]) {
    double a[3], e1[3], e2[3], q[3], s[3], r[3];
    for (int k = 0; k < 3; k++) {
        a[k] = p[(size_t)corners[0] * 3 + k];
        e1[k] = (double)p[(size_t)corners[1] * 3 + k] - a[k];
        e2[k] = (double)p[(size_t)corners[2] * 3 + k] - a[k];
    }
    q[0] = d[1] * e2[2] - d[2] * e2[1];
    q[1] = d[2] * e2[0] - d[0] * e2[2];
    q[2] = d[0] * e2[1] - d[1] * e2[0];
    double determinant = e1[0] * q[0] + e1[1] * q[1] + e1[2] * q[2];
    if (fabs(determinant) < 1e-30) return -1.0;
    for (int k = 0; k < 3; k++) s[k] = o[k] - a[k];
    double u = (s[0] * q[0] + s[1] * q[1] + s[2] * q[2]) / determinant;
    if (u < 0.0 || u > 1.0) return -1.0;
    r[0] = s[1] * e1[2] - s[2] * e1[1];
    r[1] = s[2] * e1[0] - s[0] * e1[2];
    r[2] = s[0] * e1[1] - s[1] * e1[0];
    double v = (d[0] * r[0] + d[1] * r[1] + d[2] * r[2]) / determinant;
    if (v < 0.0 || u + v > 1.0) return -1.0;
    double t = (e2[0] * r[0] + e2[1] * r[1] + e2[2] * r[2]) / determinant;
    return t > 0.0 ? t : -1.0;
}

/* nearest (main.lucb:82-98) */
static void nearest_range(void *c, size_t begin, size_t end, or_counts *counts) {
    (void)counts;
    nearest_ctx *x = c;
    for (size_t i = begin; i < end; i++) {
        const float *ray = &x->rays[i * 8];
        double o[3] = {ray[0], ray[1], ray[2]}, d[3] = {ray[4], ray[5], ray[6]};
        double best = 1.0e300, second = 1.0e300;
        int64_t face = -1;
        for (size_t at = 0; at < x->triangle_count; at++) {
            double t = hit_f64(x->positions, &x->indices[at * 3], o, d);
            if (t < 0.0) continue;
            int64_t polygon = x->faces ? (int64_t)x->faces[at] : (int64_t)at;
            if (t < best) {
                if (polygon != face) second = best;
                best = t;
                face = polygon;
            } else if (t < second && polygon != face) {
                second = t;
            }
        }
        x->face[i] = face;
        x->distance[i] = best;
        x->margin[i] = face >= 0 ? (second - best) / best : 1.0;
    }
}

void or_nearest_f64(const float *positions, const uint32_t *indices, const uint32_t *faces,
                    size_t triangle_count, const float *rays, size_t n, int64_t *face,
                    double *distance, double *margin, int threads) {
    nearest_ctx x = {positions, indices, faces, triangle_count, rays, face, distance, margin};
    run_pool(nearest_range, &x, n, threads, 16, NULL);
}

/* ---- The watertight FP32 test (Woop, Benthin and Wald 2013) ---------------------- */

int or_watertight(const float o[3], const float d[3], float tmin, float tmax, const float a[3],
                  const float b[3], const float c[3], float *t_out, float *u_out, float *v_out) {
    /* The ray's shear: kz its largest direction component (first on ties), kx and ky
     * the next two, swapped when d[kz] < 0 to keep the winding. */
    int kz = 0;
    if (fabsf(d[1]) > fabsf(d[kz])) kz = 1;
    if (fabsf(d[2]) > fabsf(d[kz])) kz = 2;
    int kx = kz + 1 == 3 ? 0 : kz + 1;
    int ky = kx + 1 == 3 ? 0 : kx + 1;
    if (d[kz] < 0.0f) {
        int s = kx;
        kx = ky;
        ky = s;
    }
    float sx = d[kx] / d[kz], sy = d[ky] / d[kz], sz = 1.0f / d[kz];
    float A[3], B[3], C[3];
    for (int k = 0; k < 3; k++) {
        A[k] = a[k] - o[k];
        B[k] = b[k] - o[k];
        C[k] = c[k] - o[k];
    }
    float ax = A[kx] - sx * A[kz], ay = A[ky] - sy * A[kz];
    float bx = B[kx] - sx * B[kz], by = B[ky] - sy * B[kz];
    float cx = C[kx] - sx * C[kz], cy = C[ky] - sy * C[kz];
    float U = cx * by - cy * bx;
    float V = ax * cy - ay * cx;
    float W = bx * ay - by * ax;
    if (U == 0.0f || V == 0.0f || W == 0.0f) {
        U = (float)((double)cx * (double)by - (double)cy * (double)bx);
        V = (float)((double)ax * (double)cy - (double)ay * (double)cx);
        W = (float)((double)bx * (double)ay - (double)by * (double)ax);
    }
    if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return 0;
    float det = U + V + W;
    if (det == 0.0f) return 0;
    float az = sz * A[kz], bz = sz * B[kz], cz = sz * C[kz];
    float T = U * az + V * bz + W * cz;
    float rcp = 1.0f / det;
    float t = T * rcp;
    if (!(t > tmin && t < tmax)) return 0;
    *t_out = t;
    *u_out = V * rcp;
    *v_out = W * rcp;
    return 1;
}

typedef struct {
    const float *positions;
    const uint32_t *indices, *ids;
    size_t triangle_count;
    const float *rays;
    int any_hit;
    int32_t *prim;
    float *t, *u, *v;
} brute_ctx;

static void brute_range(void *c, size_t begin, size_t end, or_counts *counts) {
    (void)counts;
    brute_ctx *x = c;
    for (size_t i = begin; i < end; i++) {
        const float *ray = &x->rays[i * 8];
        float best_t = ray[7], best_u = 0.0f, best_v = 0.0f;
        int64_t best = -1;
        for (size_t at = 0; at < x->triangle_count; at++) {
            float a[3], b[3], cc[3], t, u, v;
            point_at(x->positions, x->indices[at * 3], a);
            point_at(x->positions, x->indices[at * 3 + 1], b);
            point_at(x->positions, x->indices[at * 3 + 2], cc);
            int64_t id = x->ids ? (int64_t)x->ids[at] : (int64_t)at;
            /* Accept t up to and including the best so far: equal t goes to the
             * smaller id. */
            float limit = best >= 0 ? nextafterf(best_t, 3.0e38f) : ray[7];
            if (!or_watertight(ray, ray + 4, ray[3], limit, a, b, cc, &t, &u, &v)) continue;
            if (best >= 0 && t == best_t && id > best) continue;
            best = id;
            best_t = t;
            best_u = u;
            best_v = v;
            if (x->any_hit) break;
        }
        x->prim[i] = (int32_t)best;
        x->t[i] = best >= 0 ? best_t : ray[7];
        if (x->u) x->u[i] = best_u;
        if (x->v) x->v[i] = best_v;
    }
}

void or_brute_watertight(const float *positions, const uint32_t *indices, const uint32_t *ids,
                         size_t triangle_count, const float *rays, size_t n, int any_hit,
                         int32_t *prim, float *t, float *u, float *v, int threads) {
    brute_ctx x = {positions, indices, ids, triangle_count, rays, any_hit, prim, t, u, v};
    run_pool(brute_range, &x, n, threads, 16, NULL);
}
