// Ray traversal of the BVH2 on sm_100a: the device half of probe, the ray queries and
// the integrator's closest-hit and shadow kernels.
//
// Two triangle tests share one traversal loop:
//   - the default, watertight FP32 test (Woop, Benthin and Wald, JCGT 2013) over
//     48-byte triangle records, with boxes widened outward and slab exits scaled up
//     so the box test never culls a hit the triangle test would report; ties in t
//     go to the smaller source triangle id, so the closest hit does not depend on
//     the visiting order and equals an FP32 brute force over all triangles;
//   - the reference's own Moller-Trumbore test and box test (shaders/bvh.glsl:17-90)
//     over exact boxes, visiting nearer children first and keeping the first tested
//     on equal t, for bit-level parity with the reference's traversal.
// All arithmetic that decides a hit or a distance uses explicitly rounded intrinsics,
// so no multiply-add contraction changes a result between this code and its CPU
// restatement.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "device.hpp"
#include "quantize.hpp"

namespace lr {

constexpr float kNoHitT = 3.0e38f;

struct Ray {
    float3 o;
    float tmin;
    float3 d;
    float tmax;
};

struct Hit {
    float t;
    int id;    // source triangle id, -1 none
    int slot;  // leaf slot, -1 none
    float u, v;
};

__device__ __forceinline__ float fmul_(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fadd_(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub_(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float comp(const float3 &v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }

// bvh.glsl:55-56: components below 1e-20 in magnitude become +-1e-20 (+ for zero).
__device__ __forceinline__ float3 safe_inverse(float3 d) {
    auto one = [](float x) {
        if (fabsf(x) < 1e-20f) x = x > 0.0f ? 1e-20f : (x < 0.0f ? -1e-20f : 1e-20f);
        return __frcp_rn(x);
    };
    return make_float3(one(d.x), one(d.y), one(d.z));
}

// The ray's shear for the watertight test: kz the largest |d| component (the first on
// ties), kx and ky the next two (swapped when d[kz] < 0).
struct Shear {
    int kx, ky, kz;
    float sx, sy, sz;
    float ox, oy, oz;  // the origin's permuted components
};

__device__ __forceinline__ Shear make_shear(float3 o, float3 d) {
    Shear s;
    int kz = 0;
    if (fabsf(d.y) > fabsf(comp(d, kz))) kz = 1;
    if (fabsf(d.z) > fabsf(comp(d, kz))) kz = 2;
    int kx = kz == 2 ? 0 : kz + 1;
    int ky = kx == 2 ? 0 : kx + 1;
    if (comp(d, kz) < 0.0f) {
        int t = kx;
        kx = ky;
        ky = t;
    }
    float dz = comp(d, kz);
    s.kx = kx;
    s.ky = ky;
    s.kz = kz;
    s.sx = __fdiv_rn(comp(d, kx), dz);
    s.sy = __fdiv_rn(comp(d, ky), dz);
    s.sz = __frcp_rn(dz);
    s.ox = comp(o, kx);
    s.oy = comp(o, ky);
    s.oz = comp(o, kz);
    return s;
}

// One triangle, watertight; true with t in (tmin, tmax).
__device__ __forceinline__ bool watertight(const Shear &s, float tmin, float tmax, float4 a4, float4 b4,
                                           float4 c4, float &t_out, float &u_out, float &v_out) {
    float3 a = make_float3(a4.x, a4.y, a4.z), b = make_float3(b4.x, b4.y, b4.z),
           c = make_float3(c4.x, c4.y, c4.z);
    float Ax = fsub_(comp(a, s.kx), s.ox), Ay = fsub_(comp(a, s.ky), s.oy), Az = fsub_(comp(a, s.kz), s.oz);
    float Bx = fsub_(comp(b, s.kx), s.ox), By = fsub_(comp(b, s.ky), s.oy), Bz = fsub_(comp(b, s.kz), s.oz);
    float Cx = fsub_(comp(c, s.kx), s.ox), Cy = fsub_(comp(c, s.ky), s.oy), Cz = fsub_(comp(c, s.kz), s.oz);
    float ax = fsub_(Ax, fmul_(s.sx, Az)), ay = fsub_(Ay, fmul_(s.sy, Az));
    float bx = fsub_(Bx, fmul_(s.sx, Bz)), by = fsub_(By, fmul_(s.sy, Bz));
    float cx = fsub_(Cx, fmul_(s.sx, Cz)), cy = fsub_(Cy, fmul_(s.sy, Cz));
    float U = fsub_(fmul_(cx, by), fmul_(cy, bx));
    float V = fsub_(fmul_(ax, cy), fmul_(ay, cx));
    float W = fsub_(fmul_(bx, ay), fmul_(by, ax));
    if (U == 0.0f || V == 0.0f || W == 0.0f) {
        // Edge functions at exactly zero: settle them in double (the products of two
        // floats are exact there), as Woop et al. prescribe.
        U = __double2float_rn(__dsub_rn(__dmul_rn(cx, by), __dmul_rn(cy, bx)));
        V = __double2float_rn(__dsub_rn(__dmul_rn(ax, cy), __dmul_rn(ay, cx)));
        W = __double2float_rn(__dsub_rn(__dmul_rn(bx, ay), __dmul_rn(by, ax)));
    }
    if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
    float det = fadd_(fadd_(U, V), W);
    if (det == 0.0f) return false;
    float az = fmul_(s.sz, Az), bz = fmul_(s.sz, Bz), cz = fmul_(s.sz, Cz);
    float T = fadd_(fadd_(fmul_(U, az), fmul_(V, bz)), fmul_(W, cz));
    float rcp = __frcp_rn(det);
    float t = fmul_(T, rcp);
    if (!(t > tmin && t < tmax)) return false;
    t_out = t;
    u_out = fmul_(V, rcp);
    v_out = fmul_(W, rcp);
    return true;
}

// The slab test of the watertight path, one fused multiply-add per plane:
// t = lo * inv + (-o * inv). The boxes are widened at upload by 2^-16 of the scene's
// coordinate scale, which covers the rounding of this form (it moves a plane by at most
// 4 ulps of the largest coordinate involved) and the watertight test's own (a hit lies
// within a few ulps of |v - o| of its triangle) for origins within 64 scene scales;
// exits are also scaled by 1 + 2*gamma(3) (Ize 2013). True when [tmin, tmax] meets the
// box; `enter` is the entry distance.
__device__ __forceinline__ bool box_exact(float lox, float hix, float loy, float hiy, float loz, float hiz,
                                          const float3 &inv, const float3 &oinv, float tmin, float tmax,
                                          float &enter) {
    const float kScale = 1.0000003576f;
    const float x0 = fmaf(lox, inv.x, oinv.x), x1 = fmaf(hix, inv.x, oinv.x);
    const float y0 = fmaf(loy, inv.y, oinv.y), y1 = fmaf(hiy, inv.y, oinv.y);
    const float z0 = fmaf(loz, inv.z, oinv.z), z1 = fmaf(hiz, inv.z, oinv.z);
    const float e = fmaxf(fmaxf(fminf(x0, x1), fminf(y0, y1)), fmaxf(fminf(z0, z1), tmin));
    const float l = fminf(fminf(fmaxf(x0, x1), fmaxf(y0, y1)), fminf(fmaxf(z0, z1), tmax)) * kScale;
    enter = e;
    return e <= l;
}

__device__ __forceinline__ float3 neg_origin_times(const float3 &o, const float3 &inv) {
    return make_float3(-fmul_(o.x, inv.x), -fmul_(o.y, inv.y), -fmul_(o.z, inv.z));
}

// box_entry (bvh.glsl:17-25), exactly: the entry (0 when inside) or -1.
__device__ __forceinline__ float box_reference(float lox, float hix, float loy, float hiy, float loz, float hiz,
                                               const float3 &o, const float3 &inv, float t_max) {
    float x0 = fmul_(fsub_(lox, o.x), inv.x), x1 = fmul_(fsub_(hix, o.x), inv.x);
    float y0 = fmul_(fsub_(loy, o.y), inv.y), y1 = fmul_(fsub_(hiy, o.y), inv.y);
    float z0 = fmul_(fsub_(loz, o.z), inv.z), z1 = fmul_(fsub_(hiz, o.z), inv.z);
    float enter = fmaxf(fmaxf(fminf(x0, x1), fminf(y0, y1)), fmaxf(fminf(z0, z1), 0.0f));
    float leave = fminf(fminf(fmaxf(x0, x1), fmaxf(y0, y1)), fminf(fmaxf(z0, z1), t_max));
    return enter <= leave ? enter : -1.0f;
}

__device__ __forceinline__ float3 point_at(const float *p, uint32_t i) {
    return make_float3(__ldg(&p[i * 3]), __ldg(&p[i * 3 + 1]), __ldg(&p[i * 3 + 2]));
}

__device__ __forceinline__ float3 sub3(float3 a, float3 b) { return make_float3(fsub_(a.x, b.x), fsub_(a.y, b.y), fsub_(a.z, b.z)); }
__device__ __forceinline__ float3 cross3(float3 a, float3 b) {
    return make_float3(fsub_(fmul_(a.y, b.z), fmul_(a.z, b.y)), fsub_(fmul_(a.z, b.x), fmul_(a.x, b.z)),
                       fsub_(fmul_(a.x, b.y), fmul_(a.y, b.x)));
}
__device__ __forceinline__ float dot3(float3 a, float3 b) {
    return fadd_(fadd_(fmul_(a.x, b.x), fmul_(a.y, b.y)), fmul_(a.z, b.z));
}

// triangle_hit (bvh.glsl:27-47), exactly.
__device__ __forceinline__ bool triangle_reference(const DeviceScene &s, uint32_t slot, const float3 &o,
                                                   const float3 &d, Hit &hit) {
    float3 p0 = point_at(s.positions, __ldg(&s.indices[slot * 3]));
    float3 e1 = sub3(point_at(s.positions, __ldg(&s.indices[slot * 3 + 1])), p0);
    float3 e2 = sub3(point_at(s.positions, __ldg(&s.indices[slot * 3 + 2])), p0);
    float3 p = cross3(d, e2);
    float determinant = dot3(e1, p);
    if (fabsf(determinant) < 1e-20f) return false;
    float inverse = __frcp_rn(determinant);
    float3 sv = sub3(o, p0);
    float u = fmul_(dot3(sv, p), inverse);
    if (u < 0.0f || u > 1.0f) return false;
    float3 q = cross3(sv, e1);
    float v = fmul_(dot3(d, q), inverse);
    if (v < 0.0f || fadd_(u, v) > 1.0f) return false;
    float t = fmul_(dot3(e2, q), inverse);
    if (t <= 0.0f || t >= hit.t) return false;
    hit.t = t;
    hit.slot = (int)slot;
    hit.u = u;
    hit.v = v;
    return true;
}

__device__ __forceinline__ void leaf_range(int link, uint32_t &first, uint32_t &count) {
    uint32_t code = (uint32_t)(-1 - link);
    first = code >> kLeafShift;
    count = (code & ((1u << kLeafShift) - 1)) + 1;
}

// The stack lives in shared memory, one column per thread: element k of thread i at
// stack[k * stride + i]. `overflow` counts pushes past kStack (never expected: the host
// picks kStack above the tree's depth).
template <int kStack>
struct SharedStack {
    int *base;
    int stride;
    int sp = 0;
    __device__ __forceinline__ SharedStack(int *b, int s) : base(b), stride(s) {}
    __device__ __forceinline__ bool push(int v) {
        if (sp >= kStack) return false;
        base[sp * stride] = v;
        sp++;
        return true;
    }
    __device__ __forceinline__ int pop() { return base[--sp * stride]; }
    __device__ __forceinline__ bool empty() const { return sp == 0; }
};

// Work a traversal did: interior nodes visited (both children's boxes read) and
// triangle tests. Counted only when the traversal is instantiated with kCount.
struct Visits {
    uint32_t nodes = 0, tests = 0;
};

// One ray's watertight traversal as resumable state: `start` tests the root, `step` runs
// interior visits down to a leaf and tests that leaf's triangles, and reports whether
// the ray is done. The closest hit keeps ties in t for the smaller source id, so the
// result is independent of the visiting order.
template <bool kAny, int kStack, bool kCount>
struct ExactTracer {
    Ray r;
    float3 inv, oinv;
    Shear sh;
    Hit h;
    int node;
    SharedStack<kStack> st;

    __device__ __forceinline__ ExactTracer(int *stack_base, int stride) : st(stack_base, stride) {}

    // False when the ray misses the scene's root box (h is then the miss).
    __device__ __forceinline__ bool start(const DeviceScene &s, const Ray &ray) {
        const DeviceBvh &b = s.bvh;
        r = ray;
        h = Hit{r.tmax, -1, -1, 0.0f, 0.0f};
        st.sp = 0;
        if (b.empty) return false;
        inv = safe_inverse(r.d);
        oinv = neg_origin_times(r.o, inv);
        sh = make_shear(r.o, r.d);
        float enter;
        node = b.root;
        return box_exact(b.root_lo[0], b.root_hi[0], b.root_lo[1], b.root_hi[1], b.root_lo[2], b.root_hi[2], inv, oinv,
                         r.tmin, r.tmax, enter);
    }

    // Interior visits until a leaf, then that leaf. True when the ray is done.
    __device__ __forceinline__ bool step(const DeviceScene &s, bool &overflow, Visits &visits) {
        const DeviceBvh &b = s.bvh;
        while (node >= 0) {
            if (kCount) visits.nodes++;
            const float4 *e = b.entries + (size_t)node * 4;
            const float4 n0 = __ldg(e), n1 = __ldg(e + 1), n2 = __ldg(e + 2), n3 = __ldg(e + 3);
            float ea, eb;
            const bool ha = box_exact(n0.x, n0.y, n0.z, n0.w, n2.x, n2.y, inv, oinv, r.tmin, h.t, ea);
            const bool hb = box_exact(n1.x, n1.y, n1.z, n1.w, n2.z, n2.w, inv, oinv, r.tmin, h.t, eb);
            const int l0 = __float_as_int(n3.x), l1 = __float_as_int(n3.y);
            if (ha && hb) {
                const bool left_first = ea <= eb;
                if (!st.push(left_first ? l1 : l0)) overflow = true;
                node = left_first ? l0 : l1;
            } else if (ha) {
                node = l0;
            } else if (hb) {
                node = l1;
            } else {
                if (st.empty()) return true;
                node = st.pop();
            }
        }
        uint32_t first, count;
        leaf_range(node, first, count);
        if (kCount) visits.tests += count;
        for (uint32_t i = 0; i < count; i++) {
            const float4 *tri = s.tris + (size_t)(first + i) * 3;
            const float4 a = __ldg(tri), bb = __ldg(tri + 1), c = __ldg(tri + 2);
            // Equal t may still win on a smaller id: test up to the next float above h.t.
            const float limit = h.id >= 0 ? __int_as_float(__float_as_int(h.t) + 1) : r.tmax;
            float t, u, v;
            if (!watertight(sh, r.tmin, limit, a, bb, c, t, u, v)) continue;
            const int id = __float_as_int(a.w);
            if (h.id >= 0 && t == h.t && id > h.id) continue;
            h.t = t;
            h.id = id;
            h.slot = (int)(first + i);
            h.u = u;
            h.v = v;
            if (kAny) return true;
        }
        if (st.empty()) return true;
        node = st.pop();
        return false;
    }
};

__device__ __forceinline__ float fmax3(float a, float b, float c) {
    float r;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

__device__ __forceinline__ float fmin3(float a, float b, float c) {
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

// A per-thread stack of (link, entry distance) pairs in local memory (L1-cached and
// interleaved across a warp's lanes, so same-depth accesses coalesce); unlike shared
// memory it does not cap how many blocks an SM holds.
template <int kStack>
struct PairStack {
    int2 items[kStack];
    int sp = 0;
    __device__ __forceinline__ PairStack(int *, int) {}
    __device__ __forceinline__ bool push(int link, float t) {
        if (sp >= kStack) return false;
        items[sp] = make_int2(link, __float_as_int(t));
        sp++;
        return true;
    }
    __device__ __forceinline__ void pop(int &link, float &t) {
        sp--;
        const int2 e = items[sp];
        link = e.x;
        t = __int_as_float(e.y);
    }
    __device__ __forceinline__ bool empty() const { return sp == 0; }
};

// The watertight traversal over a wide BVH (wide.cpp): each node's W child boxes are
// tested together (one fused multiply-add per plane, the near and far planes picked once
// per ray by the direction's signs), the nearest hit child is taken next and the others
// are pushed far to near with their entry distances, so a popped subtree that starts
// beyond the current hit is skipped without fetching it. Leaves and triangles are the
// BVH2's, with the same tie rule, so results equal the BVH2 path's bit for bit.
template <int W, bool kAny, int kStack, bool kCount>
struct WideTracer {
    Ray r;
    float3 inv, oinv;
    Shear sh;
    Hit h;
    int node;
    PairStack<kStack> st;

    __device__ __forceinline__ WideTracer(int *stack_base, int stride) : st(stack_base, stride) {}

    __device__ __forceinline__ bool start(const DeviceScene &s, const Ray &ray) {
        r = ray;
        h = Hit{r.tmax, -1, -1, 0.0f, 0.0f};
        st.sp = 0;
        const DeviceBvh &b = s.bvh;
        if (b.empty) return false;
        inv = safe_inverse(r.d);
        oinv = neg_origin_times(r.o, inv);
        sh = make_shear(r.o, r.d);
        node = 0;
        float enter;
        return box_exact(b.root_lo[0], b.root_hi[0], b.root_lo[1], b.root_hi[1], b.root_lo[2], b.root_hi[2], inv, oinv,
                         r.tmin, r.tmax, enter);
    }

    // Compare-and-swap of (entry, link) pairs in registers, for the sorting networks.
    static __device__ __forceinline__ void order(float &ka, int &la, float &kb, int &lb) {
        const bool swap = ka > kb;
        const float k = swap ? kb : ka;
        const int l = swap ? lb : la;
        kb = swap ? ka : kb;
        lb = swap ? la : lb;
        ka = k;
        la = l;
    }

    // Runs to the end of the ray's traversal (`step` keeps the two-phase interface of
    // ExactTracer: here one call finishes the ray).
    __device__ __forceinline__ bool step(const DeviceScene &s, bool &overflow, Visits &visits) {
        const DeviceWide &wide = W == 4 ? s.wide4 : s.wide8;
        constexpr int kPlanes = W / 4;
        constexpr int kFloat4s = 7 * kPlanes;
        const float kMiss = __int_as_float(0x7f800000);  // +infinity: a child not hit
        // The near and far plane of each axis for this ray's direction signs.
        const int nx = inv.x >= 0.0f ? 0 : kPlanes, fx = kPlanes - nx;
        const int ny = (inv.y >= 0.0f ? 2 : 3) * kPlanes, fy = 5 * kPlanes - ny;
        const int nz = (inv.z >= 0.0f ? 4 : 5) * kPlanes, fz = 9 * kPlanes - nz;
        for (;;) {
            if (node >= 0) {
                if (kCount) visits.nodes++;
                const float4 *n = wide.nodes + (size_t)node * kFloat4s;
                float key[W];
                int link[W];
#pragma unroll
                for (int p = 0; p < kPlanes; p++) {
                    const float4 Nx = __ldg(n + nx + p), Fx = __ldg(n + fx + p);
                    const float4 Ny = __ldg(n + ny + p), Fy = __ldg(n + fy + p);
                    const float4 Nz = __ldg(n + nz + p), Fz = __ldg(n + fz + p);
                    const int4 ln = __ldg(reinterpret_cast<const int4 *>(n + 6 * kPlanes + p));
                    const float nxs[4] = {Nx.x, Nx.y, Nx.z, Nx.w}, fxs[4] = {Fx.x, Fx.y, Fx.z, Fx.w};
                    const float nys[4] = {Ny.x, Ny.y, Ny.z, Ny.w}, fys[4] = {Fy.x, Fy.y, Fy.z, Fy.w};
                    const float nzs[4] = {Nz.x, Nz.y, Nz.z, Nz.w}, fzs[4] = {Fz.x, Fz.y, Fz.z, Fz.w};
                    const int ls[4] = {ln.x, ln.y, ln.z, ln.w};
#pragma unroll
                    for (int c = 0; c < 4; c++) {
                        const float e = fmax3(fmaf(nxs[c], inv.x, oinv.x), fmaf(nys[c], inv.y, oinv.y),
                                              fmaxf(fmaf(nzs[c], inv.z, oinv.z), r.tmin));
                        const float l = fmin3(fmaf(fxs[c], inv.x, oinv.x), fmaf(fys[c], inv.y, oinv.y),
                                              fminf(fmaf(fzs[c], inv.z, oinv.z), h.t)) * 1.0000003576f;
                        key[p * 4 + c] = e <= l ? e : kMiss;
                        link[p * 4 + c] = ls[c];
                    }
                }
                // Sort the children by entry (misses last), all in registers.
                if (W == 4) {
                    order(key[0], link[0], key[1], link[1]);
                    order(key[2], link[2], key[3], link[3]);
                    order(key[0], link[0], key[2], link[2]);
                    order(key[1], link[1], key[3], link[3]);
                    order(key[1], link[1], key[2], link[2]);
                } else {
                    constexpr int kNet[19][2] = {{0, 2}, {1, 3}, {4, 6}, {5, 7}, {0, 4}, {1, 5}, {2, 6},
                                                 {3, 7}, {0, 1}, {2, 3}, {4, 5}, {6, 7}, {2, 4}, {3, 5},
                                                 {1, 4}, {3, 6}, {1, 2}, {3, 4}, {5, 6}};
#pragma unroll
                    for (int i = 0; i < 19; i++)
                        order(key[kNet[i][0]], link[kNet[i][0]], key[kNet[i][1]], link[kNet[i][1]]);
                }
                if (key[0] != kMiss) {
                    // The rest onto the stack, farthest first; the nearest goes next.
#pragma unroll
                    for (int k = W - 1; k >= 1; k--)
                        if (key[k] != kMiss && !st.push(link[k], key[k])) overflow = true;
                    node = link[0];
                    continue;
                }
            } else {
                uint32_t first, count;
                leaf_range(node, first, count);
                if (kCount) visits.tests += count;
                for (uint32_t i = 0; i < count; i++) {
                    const float4 *tri = s.tris + (size_t)(first + i) * 3;
                    const float4 a = __ldg(tri), bb = __ldg(tri + 1), c = __ldg(tri + 2);
                    const float limit = h.id >= 0 ? __int_as_float(__float_as_int(h.t) + 1) : r.tmax;
                    float t, u, v;
                    if (!watertight(sh, r.tmin, limit, a, bb, c, t, u, v)) continue;
                    const int id = __float_as_int(a.w);
                    if (h.id >= 0 && t == h.t && id > h.id) continue;
                    h.t = t;
                    h.id = id;
                    h.slot = (int)(first + i);
                    h.u = u;
                    h.v = v;
                    if (kAny) return true;
                }
            }
            // Next from the stack, skipping subtrees that start beyond the hit so far.
            for (;;) {
                if (st.empty()) return true;
                float t;
                st.pop(node, t);
                if (!(t > h.t)) break;
            }
        }
    }
};

// The watertight traversal over the compressed 8-wide BVH (quantize.hpp): a visit loads
// one 96-byte node, decodes its children's planes from bytes (one fused multiply-add per
// plane: the step times the inverse direction and the origin's offset are set once a
// node), tests the eight boxes together and orders the children it hits by entry
// distance. The nearest is taken next; the rest stay behind as one *group* -- the node and
// its remaining children in order, four bits each -- so a visit pushes at most one stack
// entry (two ints in shared memory) however many children it hit, and the stack holds at
// most the tree's interior depth. Leaves and triangles are the BVH2's, with the same tie
// rule, so results equal the BVH2 path's bit for bit. Any-hit rays skip the ordering.
template <bool kAny, int kStack, bool kCount>
struct CompressedTracer {
    Ray r;
    float3 inv, oinv;
    Shear sh;
    Hit h;
    uint32_t oct;  // bit k: the direction's component k is negative (its inverse, here)
    int *base;
    int stride;
    int sp = 0;

    __device__ __forceinline__ CompressedTracer(int *stack_base, int s) : base(stack_base), stride(s) {}

    __device__ __forceinline__ bool start(const DeviceScene &s, const Ray &ray) {
        r = ray;
        h = Hit{r.tmax, -1, -1, 0.0f, 0.0f};
        sp = 0;
        const DeviceBvh &b = s.bvh;
        if (b.empty) return false;
        inv = safe_inverse(r.d);
        oinv = neg_origin_times(r.o, inv);
        sh = make_shear(r.o, r.d);
        oct = (inv.x < 0.0f ? 1u : 0u) | (inv.y < 0.0f ? 2u : 0u) | (inv.z < 0.0f ? 4u : 0u);
        float enter;
        return box_exact(b.root_lo[0], b.root_hi[0], b.root_lo[1], b.root_hi[1], b.root_lo[2], b.root_hi[2], inv, oinv,
                         r.tmin, r.tmax, enter);
    }

    // Byte k (0..3) of w as a float, exactly: placed under the exponent of 2^23, less 2^23.
    static __device__ __forceinline__ float byte_at(uint32_t w, int k) {
        return __uint_as_float(__byte_perm(w, 0x4B000000u, (uint32_t)k | 0x7540u)) - 8388608.0f;
    }

    // Tests node n's children. False when none is hit; else `next` is the link of the hit
    // child of lowest rank (rank = slot ^ the ray's octant: the builder's nearest-first
    // order for this direction) and `more` the ranks of the other hit children, one bit
    // each (0: none).
    __device__ __forceinline__ bool visit(const float4 *n, int &next, uint32_t &more) {
        const float4 head = __ldg(n), la = __ldg(n + 1), lb = __ldg(n + 2), px = __ldg(n + 3), py = __ldg(n + 4),
                     pz = __ldg(n + 5);
        const uint32_t meta = __float_as_uint(head.w);
        const float ax = q_step(meta & 0xffu) * inv.x, ay = q_step((meta >> 8) & 0xffu) * inv.y,
                    az = q_step((meta >> 16) & 0xffu) * inv.z;
        const float bx = fmaf(head.x, inv.x, oinv.x), by = fmaf(head.y, inv.y, oinv.y), bz = fmaf(head.z, inv.z, oinv.z);
        // The near and far plane bytes of each axis for this ray's direction signs.
        const bool px_up = !(oct & 1u), py_up = !(oct & 2u), pz_up = !(oct & 4u);
        const uint32_t nx0 = __float_as_uint(px_up ? px.x : px.z), nx1 = __float_as_uint(px_up ? px.y : px.w);
        const uint32_t fx0 = __float_as_uint(px_up ? px.z : px.x), fx1 = __float_as_uint(px_up ? px.w : px.y);
        const uint32_t ny0 = __float_as_uint(py_up ? py.x : py.z), ny1 = __float_as_uint(py_up ? py.y : py.w);
        const uint32_t fy0 = __float_as_uint(py_up ? py.z : py.x), fy1 = __float_as_uint(py_up ? py.w : py.y);
        const uint32_t nz0 = __float_as_uint(pz_up ? pz.x : pz.z), nz1 = __float_as_uint(pz_up ? pz.y : pz.w);
        const uint32_t fz0 = __float_as_uint(pz_up ? pz.z : pz.x), fz1 = __float_as_uint(pz_up ? pz.w : pz.y);
        uint32_t mask = 0;
#pragma unroll
        for (int c = 0; c < 8; c++) {
            const int k = c & 3;
            const uint32_t nx = c < 4 ? nx0 : nx1, fx = c < 4 ? fx0 : fx1;
            const uint32_t ny = c < 4 ? ny0 : ny1, fy = c < 4 ? fy0 : fy1;
            const uint32_t nz = c < 4 ? nz0 : nz1, fz = c < 4 ? fz0 : fz1;
            const float e = fmax3(fmaf(byte_at(nx, k), ax, bx), fmaf(byte_at(ny, k), ay, by),
                                  fmaxf(fmaf(byte_at(nz, k), az, bz), r.tmin));
            const float l = fmin3(fmaf(byte_at(fx, k), ax, bx), fmaf(byte_at(fy, k), ay, by),
                                  fminf(fmaf(byte_at(fz, k), az, bz), h.t)) * 1.0000003576f;
            mask |= e <= l ? 1u << c : 0u;
        }
        mask &= meta >> 24;  // occupied slots only
        if (!mask) return false;
        // From slots to ranks: bit s moves to bit s ^ oct.
        if (oct & 1u) mask = ((mask & 0x55u) << 1) | ((mask >> 1) & 0x55u);
        if (oct & 2u) mask = ((mask & 0x33u) << 2) | ((mask >> 2) & 0x33u);
        if (oct & 4u) mask = ((mask & 0x0fu) << 4) | ((mask >> 4) & 0x0fu);
        const uint32_t slot = (uint32_t)(__ffs(mask) - 1) ^ oct;
        more = mask & (mask - 1u);
        const int links[8] = {__float_as_int(la.x), __float_as_int(la.y), __float_as_int(la.z), __float_as_int(la.w),
                              __float_as_int(lb.x), __float_as_int(lb.y), __float_as_int(lb.z), __float_as_int(lb.w)};
        int chosen = links[0];
#pragma unroll
        for (int c = 1; c < 8; c++) chosen = slot == (uint32_t)c ? links[c] : chosen;
        next = chosen;
        return true;
    }

    // Runs to the end of the ray's traversal. A group is a node with the ranks of its hit
    // children not yet visited: (node << 8) | ranks, one int on the stack.
    __device__ __forceinline__ bool step(const DeviceScene &s, bool &overflow, Visits &visits) {
        const float4 *nodes = s.wide8.nodes;
        uint32_t group = 0;  // the group being walked (no ranks left: none)
        int link = 0;        // the wide root
        for (;;) {
            if (link >= 0) {
                if (kCount) visits.nodes++;
                const float4 *n = nodes + (size_t)link * kQNodeFloat4s;
                int next;
                uint32_t more;
                if (visit(n, next, more)) {
                    // The nearest hit child next; the group walked so far waits on the stack
                    // and this node's other hit children become the group in hand.
                    if (more) {
                        if (group & 0xffu) {
                            if (sp < kStack) {
                                base[sp * stride] = (int)group;
                                sp++;
                            } else {
                                overflow = true;
                            }
                        }
                        group = ((uint32_t)link << 8) | more;
                    }
                    link = next;
                    continue;
                }
            } else {
                uint32_t first, count;
                leaf_range(link, first, count);
                if (kCount) visits.tests += count;
                for (uint32_t i = 0; i < count; i++) {
                    const float4 *tri = s.tris + (size_t)(first + i) * 3;
                    const float4 a = __ldg(tri), bb = __ldg(tri + 1), c = __ldg(tri + 2);
                    const float limit = h.id >= 0 ? __int_as_float(__float_as_int(h.t) + 1) : r.tmax;
                    float t, u, v;
                    if (!watertight(sh, r.tmin, limit, a, bb, c, t, u, v)) continue;
                    const int id = __float_as_int(a.w);
                    if (h.id >= 0 && t == h.t && id > h.id) continue;
                    h.t = t;
                    h.id = id;
                    h.slot = (int)(first + i);
                    h.u = u;
                    h.v = v;
                    if (kAny) return true;
                }
            }
            // The next child: from the group in hand, else from the stack.
            if (!(group & 0xffu)) {
                if (sp == 0) return true;
                sp--;
                group = (uint32_t)base[sp * stride];
            }
            const uint32_t slot = (uint32_t)(__ffs(group & 0xffu) - 1) ^ oct;
            group &= group - 1u;  // the lowest rank: a bit of the low byte
            link = __ldg(reinterpret_cast<const int *>(nodes + (size_t)(group >> 8) * kQNodeFloat4s + 1) + slot);
        }
    }
};

// The closest (or any) hit along r, watertight. `overflow` is set when a push was lost.
template <bool kAny, int kStack, bool kCount = false>
__device__ __forceinline__ Hit trace_exact(const DeviceScene &s, const Ray &r, int *stack_base, int stride,
                                           bool &overflow, Visits &visits) {
    ExactTracer<kAny, kStack, kCount> tr(stack_base, stride);
    if (!tr.start(s, r)) return tr.h;
    while (!tr.step(s, overflow, visits)) {
    }
    return tr.h;
}

// The watertight tracer of a BVH width: 2 (the BVH2 itself), 4 or 8 (wide.cpp: 8 is the
// compressed layout), and the shared-memory ints per thread its stack takes.
template <int W, bool kAny, int kStack, bool kCount>
struct TracerOf {
    using type = WideTracer<W, kAny, kStack, kCount>;
    static constexpr int kInts = 1;  // the 4-wide tracer's stack is in local memory
};
template <bool kAny, int kStack, bool kCount>
struct TracerOf<8, kAny, kStack, kCount> {
    using type = CompressedTracer<kAny, kStack, kCount>;
    static constexpr int kInts = kStack;  // (node << 8) | ranks, a group
};
template <bool kAny, int kStack, bool kCount>
struct TracerOf<2, kAny, kStack, kCount> {
    using type = ExactTracer<kAny, kStack, kCount>;
    static constexpr int kInts = kStack;
};

// A resident grid over a queue of `count` rays in warp batches: each warp takes the next
// 32 consecutive entries (neighbouring primary rays keep its lanes on similar nodes) with
// one atomic on `next` (zero at launch) whenever its lanes are done, so warps that drew
// long rays take fewer batches. `load(i)` gives ray i and `store(i, hit, ray)` takes its
// result.
template <int W, bool kAny, int kStack, bool kCount, class Load, class Store>
__device__ __forceinline__ void trace_batched(const DeviceScene &s, uint32_t count, uint32_t *next, int *stack_base,
                                              int stride, Load load, Store store, bool &overflow, Visits &visits) {
    typename TracerOf<W, kAny, kStack, kCount>::type tr(stack_base, stride);
    const uint32_t lane = threadIdx.x & 31u;
    for (;;) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(next, 32u);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= count) break;
        const uint32_t i = base + lane;
        if (i >= count) continue;
        if (tr.start(s, load(i))) {
            while (!tr.step(s, overflow, visits)) {
            }
        }
        store(i, tr.h, tr.r);
    }
}

// Persistent warps that replace finished rays from a shared queue (Aila and Laine,
// "Understanding the Efficiency of Ray Traversal on GPUs", HPG 2009: dynamic fetch with
// replacement of terminated rays). Each lane keeps one ray; once `refill_at` lanes of
// the warp (1 to 32) have none, one lane takes that many consecutive queue entries with
// one atomic on `next` (zero when the launch starts) and the idle lanes share them in
// lane order. `begin(i, s)` loads ray i, its scene into `s` and starts the tracer: true
// when there is a walk to take, else it has finished ray i itself; `end(i)` finishes ray
// i after its walk. Finished walks wait for the refill to end, so that the lanes that
// finished run `end` together rather than one or two at a time. The warp stays converged
// around each ballot; a walk ends in a bounded number of steps, so every warp leaves once
// the queue is drained.
template <class Tracer, class Begin, class End>
__device__ __forceinline__ void trace_refilling(Tracer &tr, uint32_t count, uint32_t *next, uint32_t refill_at,
                                                Begin begin, End end, bool &overflow, Visits &visits) {
    const uint32_t lane = threadIdx.x & 31u;
    DeviceScene s;
    uint32_t i = 0;
    bool busy = false, ended = true, drained = false;
    for (;;) {
        const uint32_t idle = __ballot_sync(0xffffffffu, !busy);
        const uint32_t want = (uint32_t)__popc(idle);
        const bool last = drained && idle == 0xffffffffu;
        if (last || (!drained && want >= refill_at)) {
            if (!busy && !ended) {
                end(i);
                ended = true;
            }
            if (last) break;
            uint32_t base = 0;
            if (lane == 0) base = atomicAdd(next, want);
            base = __shfl_sync(0xffffffffu, base, 0);
            drained = base + want >= count;
            if (!busy) {
                i = base + (uint32_t)__popc(idle & ((1u << lane) - 1u));
                if (i < count) {
                    busy = begin(i, s);
                    ended = !busy;
                }
            }
        }
        if (busy && tr.step(s, overflow, visits)) busy = false;
    }
}

// trace_closest / trace_any (bvh.glsl:51-122) over the reference's exact boxes.
template <bool kAny, int kStack, bool kCount = false>
__device__ __forceinline__ Hit trace_reference(const DeviceScene &s, const Ray &r, int *stack_base, int stride,
                                               bool &overflow, Visits &visits) {
    Hit h{r.tmax, -1, -1, 0.0f, 0.0f};
    const DeviceBvh &b = s.ref_bvh;
    if (b.empty) return h;
    const float3 inv = safe_inverse(r.d);
    if (box_reference(b.root_lo[0], b.root_hi[0], b.root_lo[1], b.root_hi[1], b.root_lo[2], b.root_hi[2], r.o,
                      inv, h.t) < 0.0f)
        return h;
    SharedStack<kStack> st(stack_base, stride);
    int node = b.root;
    for (;;) {
        if (node < 0) {
            uint32_t first, count;
            leaf_range(node, first, count);
            for (uint32_t i = 0; i < count; i++) {
                if (kCount) visits.tests++;
                if (triangle_reference(s, first + i, r.o, r.d, h) && kAny) {
                    h.id = (int)__ldg(&s.ids[h.slot]);
                    return h;
                }
            }
        } else {
            if (kCount) visits.nodes++;
            const float4 *e = b.entries + (size_t)node * 4;
            const float4 n0 = __ldg(e), n1 = __ldg(e + 1), n2 = __ldg(e + 2), n3 = __ldg(e + 3);
            const float tl = kAny ? r.tmax : h.t;
            const float a = box_reference(n0.x, n0.y, n0.z, n0.w, n2.x, n2.y, r.o, inv, tl);
            const float bb = box_reference(n1.x, n1.y, n1.z, n1.w, n2.z, n2.w, r.o, inv, tl);
            const int l0 = __float_as_int(n3.x), l1 = __float_as_int(n3.y);
            const bool take_left = a >= 0.0f, take_right = bb >= 0.0f;
            if (take_left && take_right) {
                const bool left_near = kAny ? true : a <= bb;
                if (!st.push(left_near ? l1 : l0)) overflow = true;
                node = left_near ? l0 : l1;
                continue;
            }
            if (take_left) {
                node = l0;
                continue;
            }
            if (take_right) {
                node = l1;
                continue;
            }
        }
        if (st.empty()) break;
        node = st.pop();
    }
    if (h.slot >= 0) h.id = (int)__ldg(&s.ids[h.slot]);
    return h;
}

// Adds each lane's visits into two 64-bit counters with one atomic per warp. Every
// lane of the warp must call it.
__device__ __forceinline__ void add_visits(unsigned long long *counters, const Visits &v) {
    unsigned long long nodes = v.nodes, tests = v.tests;
#pragma unroll
    for (int offset = 16; offset > 0; offset >>= 1) {
        nodes += __shfl_down_sync(0xffffffffu, nodes, offset);
        tests += __shfl_down_sync(0xffffffffu, tests, offset);
    }
    if ((threadIdx.x & 31) == 0 && (nodes || tests)) {
        atomicAdd(&counters[0], nodes);
        atomicAdd(&counters[1], tests);
    }
}

}  // namespace lr
