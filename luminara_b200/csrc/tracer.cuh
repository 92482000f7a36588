// tracer.cuh -- device code of the path-tracing core (sm_100a).
//
// Restates the reference's hot path in f32 on the GPU:
//   primitive hits   src/sphere.rs:23-62, quad.rs:29-62, triangle.rs:21-64, obj.rs:259-313,
//                    disk.rs:31-58, plane.rs:42-69, constant_medium.rs:25-69, hit.rs:19-43
//   traversal        src/bvh.rs:52-68 + src/scene.rs:816-834 (closest hit: BVH then planes)
//   materials        src/material.rs:59-391, constant_medium.rs:81-89, texture.rs:9-50
//   NEE              src/render.rs:1333-1466
//   integrator       src/render.rs:1472-1537 (iterative form, see path_bounce)
//   camera           src/camera.rs:82-102
// Random numbers come from Philox4x32-10 keyed by (pixel, stratum, bounce, call).
#pragma once

#include <cuda_runtime.h>
#include <math_constants.h>
#include <stdint.h>

#include "device_scene.h"

namespace lum {

// ------------------------------------------------------------------------------- vectors
struct V {
    float x, y, z;
};
__device__ __forceinline__ V mk(float x, float y, float z) { return V{x, y, z}; }
__device__ __forceinline__ V mk(const float* p) { return V{p[0], p[1], p[2]}; }
__device__ __forceinline__ V operator+(V a, V b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V operator-(V a, V b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V operator-(V a) { return {-a.x, -a.y, -a.z}; }
__device__ __forceinline__ V operator*(V a, float t) { return {a.x * t, a.y * t, a.z * t}; }
__device__ __forceinline__ V operator*(float t, V a) { return a * t; }
__device__ __forceinline__ V mul(V a, V b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
__device__ __forceinline__ float dot(V a, V b) { return fmaf(a.x, b.x, fmaf(a.y, b.y, a.z * b.z)); }
__device__ __forceinline__ V cross(V a, V b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ float len2(V a) { return dot(a, a); }
__device__ __forceinline__ V unit(V a) { return a * rsqrtf(len2(a)); }
__device__ __forceinline__ V fma3(V a, float t, V b) { return {fmaf(a.x, t, b.x), fmaf(a.y, t, b.y), fmaf(a.z, t, b.z)}; }
__device__ __forceinline__ V xyz(float4 a) { return {a.x, a.y, a.z}; }
__device__ __forceinline__ bool near_zero(V a) {
    return fabsf(a.x) < 1e-8f && fabsf(a.y) < 1e-8f && fabsf(a.z) < 1e-8f;
}
__device__ __forceinline__ V reflect(V v, V n) { return v - n * (2.0f * dot(v, n)); }
__device__ __forceinline__ bool has_nan(V a) { return isnan(a.x) || isnan(a.y) || isnan(a.z); }

// -------------------------------------------------------------------------------- RNG
// Philox4x32-10 (Salmon et al., SC'11).  U: unroll factor of the ten rounds (philox_unroll).
__device__ __forceinline__ void philox_round(uint4& c, uint32_t k0, uint32_t k1) {
    uint32_t lo0 = 0xD2511F53u * c.x, hi0 = __umulhi(0xD2511F53u, c.x);
    uint32_t lo1 = 0xCD9E8D57u * c.z, hi1 = __umulhi(0xCD9E8D57u, c.z);
    c = make_uint4(hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0);
}
template <int U = 10>
__device__ __forceinline__ uint4 philox(uint4 c, uint32_t k0, uint32_t k1) {
    if constexpr (U >= 10) {
#pragma unroll
        for (int r = 0; r < 10; ++r) {
            if (r > 0) {
                k0 += 0x9E3779B9u;
                k1 += 0xBB67AE85u;
            }
            philox_round(c, k0, k1);
        }
    } else {
#pragma unroll U
        for (int r = 0; r < 10; ++r) {
            if (r > 0) {
                k0 += 0x9E3779B9u;
                k1 += 0xBB67AE85u;
            }
            philox_round(c, k0, k1);
        }
    }
    return c;
}
__device__ __forceinline__ float u24(uint32_t x) { return (float)(x >> 8) * (1.0f / 16777216.0f); }
template <int U = 10>
__device__ __forceinline__ float4 draw4(uint32_t k0, uint32_t k1, uint32_t pixel, uint32_t stratum, uint32_t bounce,
                                        uint32_t call) {
    uint4 o = philox<U>(make_uint4(pixel, stratum, bounce, call), k0, k1);
    return make_float4(u24(o.x), u24(o.y), u24(o.z), u24(o.w));
}
enum : uint32_t { CALL_CAMERA = 0, CALL_CAMERA2 = 1, CALL_SCATTER = 2, CALL_NEE = 3, CALL_EXTRA = 4, CALL_BLEND = 5 };

// Direct (rejection-free) samplers; same distributions as src/vec3.rs:96-122.
__device__ __forceinline__ V unit_vector(float a, float b) {
    float z = 1.0f - 2.0f * a;
    float r = sqrtf(fmaxf(0.0f, 1.0f - z * z));
    float s, c;
    sincospif(2.0f * b, &s, &c);
    return {r * c, r * s, z};
}
__device__ __forceinline__ V in_unit_sphere(float a, float b, float c) { return unit_vector(a, b) * cbrtf(c); }

// ------------------------------------------------------------------------------ ray/hit
struct Ray {
    V o, d;
    float time;
};

struct Hit {
    float t;
    int prim;     // index into the reordered primitive array; -1 none; <= -2 : plane (-2 - index)
    float b1, b2; // triangle barycentrics (u, v)
};

// Record k (0-3, a constant at every call site) of primitive i.
__device__ __forceinline__ float4 ldp(const SceneDev& S, int i, int k) {
    return k < 3 ? __ldg(reinterpret_cast<const float4*>(S.prims) + 3 * i + k)
                 : __ldg(reinterpret_cast<const float4*>(S.prims3) + i);
}

// Robust sphere roots (Haines et al., "Precision Improvements for Ray/Sphere Intersection",
// Ray Tracing Gems 2019): discriminant from the ray-to-centre distance, near root from c/q.
// Spheres of radius >= kBigSphere (ground spheres) evaluate o - c and |o - c|^2 - r^2 in
// f64: in f32 that difference loses ~r * 6e-8 absolutely, which near the surface of an
// r = 1000 sphere is a large relative error of the near root.
constexpr float kBigSphere = 32.0f;
// a = |d|^2 and ia = 1 / a are the ray's (the caller may compute them once per ray).
__device__ __forceinline__ bool sphere_roots(V c, float r, const Ray& ray, float a, float ia, float& t0, float& t1) {
    V oc;
    float cc;
    if (r >= kBigSphere) {
        double dx = (double)ray.o.x - (double)c.x, dy = (double)ray.o.y - (double)c.y, dz = (double)ray.o.z - (double)c.z;
        oc = mk((float)dx, (float)dy, (float)dz);
        cc = (float)fma(dx, dx, fma(dy, dy, fma(dz, dz, -(double)r * (double)r)));
    } else {
        oc = ray.o - c;
        cc = fmaf(-r, r, len2(oc));
    }
    float b = dot(oc, ray.d);
    V f = fma3(ray.d, -b * ia, oc);
    float disc = a * (r * r - len2(f));
    if (disc < 0.0f) return false;
    float q = -b - copysignf(sqrtf(disc), b);
    float ta = cc / q, tb = q * ia;
    if (q == 0.0f) ta = tb = -b * ia;
    t0 = fminf(ta, tb);
    t1 = fmaxf(ta, tb);
    return true;
}

__device__ __forceinline__ bool sphere_roots(V c, float r, const Ray& ray, float& t0, float& t1) {
    const float a = len2(ray.d);
    return sphere_roots(c, r, ray, a, 1.0f / a, t0, t1);
}

// sphere.rs:24-45: near root if in [tmin, tmax], else far root.  ia: 1 / |d|^2 of the ray, or 0
// to compute it here.
__device__ __forceinline__ bool hit_sphere(float4 a, float4 b, const Ray& ray, float tmin, float tmax, float& t,
                                           float ia = 0.0f) {
    V c = xyz(a);
    if (b.w != 0.0f) c = fma3(xyz(b) - c, ray.time, c);   // MovingSphere::center_at
    float t0, t1;
    const float aa = len2(ray.d);
    if (!sphere_roots(c, a.w, ray, aa, ia != 0.0f ? ia : 1.0f / aa, t0, t1)) return false;
    if (t0 >= tmin && t0 <= tmax) { t = t0; return true; }
    if (t1 >= tmin && t1 <= tmax) { t = t1; return true; }
    return false;
}

// quad.rs:29-62.  The record keeps w = (u x v)/|u x v|^2 and |u x v|, so the plane test,
// the parallel threshold on the unit normal and the planar coordinates are the reference's.
__device__ __forceinline__ bool hit_quad(float4 a, float4 b, float4 c, float4 d, const Ray& ray, float tmin,
                                         float tmax, float& t, float* uv = nullptr) {
    V w = xyz(d);
    float denom = dot(w, ray.d);
    if (fabsf(denom * b.w) < 1e-8f) return false;
    float tt = (a.w - dot(w, ray.o)) / denom;
    if (!(tt >= tmin && tt <= tmax)) return false;
    V p = fma3(ray.d, tt, ray.o);
    V ph = p - xyz(a);
    float alpha = dot(w, cross(ph, xyz(c)));
    float beta = dot(w, cross(xyz(b), ph));
    if (!(alpha >= 0.0f && alpha <= 1.0f && beta >= 0.0f && beta <= 1.0f)) return false;
    t = tt;
    if (uv) { uv[0] = alpha; uv[1] = beta; }
    return true;
}

// triangle.rs:21-64 (Moller-Trumbore)
// The barycentric bounds are tested on the numerators against the determinant (u = su / aa in
// [0, 1] <=> su between 0 and aa, and likewise v >= 0, u + v <= 1), so the division is done only
// for the few candidates that pass them; u, v and t are then the reference's f * numerator.
__device__ __forceinline__ bool hit_tri(float4 a, float4 b, float4 c, const Ray& ray, float tmin, float tmax,
                                        float& t, float& bu, float& bv) {
    V e1 = xyz(b), e2 = xyz(c);
    V h = cross(ray.d, e2);
    float aa = dot(e1, h);
    if (fabsf(aa) < 1e-8f) return false;
    V s = ray.o - xyz(a);
    const float su = dot(s, h);
    const float sg = aa > 0.0f ? 1.0f : -1.0f, da = fabsf(aa);   // numerators scaled to aa > 0
    if (!(su * sg >= 0.0f && su * sg <= da)) return false;
    V q = cross(s, e1);
    const float sv = dot(ray.d, q);
    if (sv * sg < 0.0f || (su + sv) * sg > da) return false;
    const float f = 1.0f / aa;
    const float u = f * su, v = f * sv;
    float tt = f * dot(e2, q);
    if (!(tt >= tmin && tt <= tmax)) return false;
    t = tt;
    bu = u;
    bv = v;
    return true;
}

// disk.rs:31-58
__device__ __forceinline__ bool hit_disk(float4 a, float4 b, const Ray& ray, float tmin, float tmax, float& t) {
    V n = xyz(b);
    float denom = dot(n, ray.d);
    if (fabsf(denom) < 1e-8f) return false;
    float tt = dot(xyz(a) - ray.o, n) / denom;
    if (!(tt >= tmin && tt <= tmax)) return false;
    V off = fma3(ray.d, tt, ray.o) - xyz(a);
    if (len2(off) > a.w * a.w) return false;
    t = tt;
    return true;
}

// constant_medium.rs:25-69.  Boundary entry/exit over the whole line (t_min = -inf), the
// second hit at least 1e-4 past the first; the free-flight distance is the reference's
// deterministic hash of the ray, evaluated in f64 without contraction.
__device__ __forceinline__ bool hit_fog(int type, float4 a, float4 b, float4 c, const Ray& ray, float tmin,
                                        float tmax, float& t) {
    float e0, e1;
    if (type == PT_FOG_SPHERE) {
        if (!sphere_roots(xyz(a), a.w, ray, e0, e1)) return false;
    } else {
        float lo = -CUDART_INF_F, hi = CUDART_INF_F;
        float o[3] = {ray.o.x, ray.o.y, ray.o.z}, d[3] = {ray.d.x, ray.d.y, ray.d.z};
        float mn[3] = {a.x, a.y, a.z}, mx[3] = {b.x, b.y, b.z};
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            float inv = 1.0f / d[k];
            float ta = (mn[k] - o[k]) * inv, tb = (mx[k] - o[k]) * inv;
            lo = fmaxf(lo, fminf(ta, tb));
            hi = fminf(hi, fmaxf(ta, tb));
        }
        if (!(lo <= hi)) return false;
        e0 = lo;
        e1 = hi;
    }
    if (!(e1 >= e0 + 0.0001f)) return false;
    float t1 = fmaxf(e0, tmin), t2 = fminf(e1, tmax);
    if (t1 >= t2) return false;
    if (t1 < 0.0f) t1 = 0.0f;
    float rl = sqrtf(len2(ray.d));
    float inside = (t2 - t1) * rl;
    double hv = __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn((double)ray.o.x, 73856093.0), __dmul_rn((double)ray.o.y, 19349663.0)),
                                    __dmul_rn((double)ray.o.z, 83492791.0)),
                          __dmul_rn((double)ray.d.x, 47392381.0));
    hv = fabs(hv - trunc(hv));
    double hd = (double)c.x * log(fmax(1.0 - hv, 1e-10));
    if (hd > (double)inside) return false;
    t = t1 + (float)hd / rl;
    return true;
}

// hit_fog out of line, for the mesh class's leaf loop (CLS_MESH): that build is bound by
// instruction fetch, and the fog test (two box or sphere roots and the f64 free-flight hash)
// runs for a handful of primitives only.  With the light sampler out of line as well the dense
// mesh ran 173.3 -> 169.8 ms on B200 (fog test alone: 172.1 ms); the other builds inline both.
static __device__ __noinline__ bool hit_fog_cold(int type, float4 a, float4 b, float4 c, const Ray& ray, float tmin,
                                                 float tmax, float& t) {
    return hit_fog(type, a, b, c, ray, tmin, tmax, t);
}

// Scene classes of the general megakernel build (CLS): the primitive types and NEE light kinds
// the kernel carries code for.  A scene runs the smallest class that holds all its primitives
// and lights (SceneDev::cls, chosen by lum_scene_create); code a scene cannot reach costs
// instruction-fetch time in the megakernel.
enum : int {
    CLS_ALL = 0,    // every primitive type and light kind
    CLS_QUAD = 1,   // quads (rects, boxes) with rect lights (box room, quad scenes)
    CLS_MESH = 2    // triangles, disks and media with disk and rect lights (meshes)
};

// Unroll factor of the Philox rounds in a scene-class build.  The mesh class's megakernel is
// bound by instruction fetch (no_instructions is a quarter of its stall samples), and each
// inlined draw site carries the ten rounds: rolled by two they shrink it, and the dense mesh
// ran 186.1 -> 173.3 ms on B200; the sphere field, bound by issue, ran 6% slower that way and
// keeps them unrolled, as do the other classes (box room 1% slower rolled).
template <int CLS>
constexpr int philox_unroll() { return CLS == CLS_MESH ? 2 : 10; }
template <int CLS>
__host__ __device__ constexpr bool cls_has_prim(int type) {
    return CLS == CLS_ALL || (CLS == CLS_QUAD && type == PT_QUAD) ||
           (CLS == CLS_MESH && (type == PT_TRIANGLE || type == PT_DISK || type == PT_FOG_SPHERE || type == PT_FOG_BOX));
}
template <int CLS>
__host__ __device__ constexpr bool cls_has_light(int kind) {   // 1 sphere, 2 rect, 3 disk
    return CLS == CLS_ALL || (CLS == CLS_QUAD && kind == 2) || (CLS == CLS_MESH && (kind == 2 || kind == 3));
}

// One primitive test; updates the closest hit when t is within [tmin, hit.t].
// SPH: the scene's primitives are all static spheres (SceneDev::spheres_basic), so the other
// primitive tests are left out of the kernel and a test reads only record 0 (centre, radius).
// ia_ray: 1 / |d|^2 of the ray, computed once per walk by the sphere-class build (0 elsewhere).
template <bool COUNT = false, bool SPH = false, int CLS = CLS_ALL>
__device__ __forceinline__ bool test_prim(const SceneDev& S, int i, const Ray& ray, float tmin, Hit& hit,
                                          TestTally* tl = nullptr, float ia_ray = 0.0f) {
    float4 a = ldp(S, i, 0);
    float t;
    if constexpr (SPH && !COUNT) {
        if (hit_sphere(a, make_float4(0.0f, 0.0f, 0.0f, 0.0f), ray, tmin, hit.t, t, ia_ray)) {
            hit.t = t;
            hit.prim = i;
            return true;
        }
        return false;
    }
    int type = __ldg(S.meta + i) & 15;
    if constexpr (COUNT) tl->prim[type]++;
    switch (type) {
        case PT_SPHERE: {
            if constexpr (!cls_has_prim<CLS>(PT_SPHERE)) return false;
            float4 b = ldp(S, i, 1);
            if (hit_sphere(a, b, ray, tmin, hit.t, t)) { hit.t = t; hit.prim = i; return true; }
            return false;
        }
        case PT_QUAD: {
            if constexpr (!cls_has_prim<CLS>(PT_QUAD)) return false;
            float4 b = ldp(S, i, 1), c = ldp(S, i, 2), d = ldp(S, i, 3);
            if (hit_quad(a, b, c, d, ray, tmin, hit.t, t)) { hit.t = t; hit.prim = i; return true; }
            return false;
        }
        case PT_TRIANGLE: {
            if constexpr (!cls_has_prim<CLS>(PT_TRIANGLE)) return false;
            float4 b = ldp(S, i, 1), c = ldp(S, i, 2);
            float bu, bv;
            if (hit_tri(a, b, c, ray, tmin, hit.t, t, bu, bv)) {
                hit.t = t; hit.prim = i; hit.b1 = bu; hit.b2 = bv;
                return true;
            }
            return false;
        }
        case PT_DISK: {
            if constexpr (!cls_has_prim<CLS>(PT_DISK)) return false;
            float4 b = ldp(S, i, 1);
            if (hit_disk(a, b, ray, tmin, hit.t, t)) { hit.t = t; hit.prim = i; return true; }
            return false;
        }
        default: {
            if constexpr (!cls_has_prim<CLS>(PT_FOG_BOX)) return false;
            float4 b = ldp(S, i, 1), c = ldp(S, i, 2);
            const bool fog_hit = CLS == CLS_MESH ? hit_fog_cold(type, a, b, c, ray, tmin, hit.t, t)
                                                 : hit_fog(type, a, b, c, ray, tmin, hit.t, t);
            if (fog_hit) { hit.t = t; hit.prim = i; return true; }
            return false;
        }
    }
}

// plane.rs:42-69
__device__ __forceinline__ bool hit_plane(const PlaneDev& P, const Ray& ray, float tmin, float tmax, float& t) {
    V n = mk(P.n);
    float denom = dot(n, ray.d);
    if (fabsf(denom) < 1e-8f) return false;
    float tt = dot(mk(P.p) - ray.o, n) / denom;
    if (!(tt >= tmin && tt <= tmax)) return false;
    t = tt;
    return true;
}

// ------------------------------------------------------------------------------ traversal
// BVH2 traversal with postponed leaves (the "while-while" organisation of Aila & Laine,
// "Understanding the Efficiency of Ray Traversal on GPUs", HPG 2009): a lane that reaches a
// leaf keeps it pending and goes on descending inner nodes until every active lane of the
// warp holds a leaf; then all lanes test their leaves together.  Inner nodes are visited
// near child first.  Stack entries (shared memory, entry k of thread j at
// stack[k * blockDim.x + j]) are inner-node indices (>= 0) or leaf ranges ~(first << 3 |
// count - 1); kSentinel marks the empty stack.
constexpr int kSentinel = 0x7fffffff;

// Place of a suspended BVH walk (trace_resume): the next node to visit (an inner node index, or
// kSentinel when the walk is over) and the stack depth; the stack entries stay in shared memory
// and the closest hit so far in the caller's Hit.
struct Trav {
    int node;
    int sp;
};

// The BVH walk of `trace`, resumable.  With SUSPEND > 0 the walk stops at the top of an outer
// iteration (no postponed leaf pending) once at most SUSPEND lanes of the warp are still
// walking: it saves its place in tv and returns false, so that the lanes which finished can
// shade and start new rays before the warp walks on (Aila & Laine 2009 replace terminated rays
// in the same spirit: a warp's traversal otherwise runs as long as its longest ray while the
// finished lanes idle).  Returns true when the walk is complete (planes tested, `found` final).
// SUSPEND == 0 never stops early.  tv starts as {0, 0} (or kSentinel for a scene without
// nodes), found as false.
template <bool COUNT = false, bool SPH = false, int SUSPEND = 0, int CLS = CLS_ALL>
__device__ __forceinline__ bool trace_resume(const SceneDev& S, const Ray& ray, float tmin, bool any, Hit& hit,
                                             bool& found, Trav& tv, int* stack, uint32_t& err,
                                             TestTally* tl = nullptr) {
    if (tv.node != kSentinel) {
        // Reciprocals of direction components clamped away from zero: the FMA slab form
        // lo*inv - o*inv would give inf - inf = NaN for an axis-parallel ray, while a finite
        // +-1e20 keeps the ordering of the reference's (lo - o) * (1/d) (aabb.rs:23-25).
        const float ix = 1.0f / (fabsf(ray.d.x) > 1e-20f ? ray.d.x : copysignf(1e-20f, ray.d.x));
        const float iy = 1.0f / (fabsf(ray.d.y) > 1e-20f ? ray.d.y : copysignf(1e-20f, ray.d.y));
        const float iz = 1.0f / (fabsf(ray.d.z) > 1e-20f ? ray.d.z : copysignf(1e-20f, ray.d.z));
        const float ox = -ray.o.x * ix, oy = -ray.o.y * iy, oz = -ray.o.z * iz;
        // the sphere class divides by |d|^2 once per walk instead of once per sphere test
        float ia_ray = 0.0f;
        if constexpr (SPH && !COUNT) ia_ray = 1.0f / len2(ray.d);
        const float4* nodes = reinterpret_cast<const float4*>(S.nodes);
        const int stride = blockDim.x;
        int sp = tv.sp;
        int node = tv.node;   // inner node index, leaf (< 0) or kSentinel
        int leaf = 0;         // postponed leaf (< 0) or 0
        for (;;) {
            while ((unsigned)node < (unsigned)kSentinel) {
                float4 n0 = __ldg(nodes + 4 * node + 0);
                float4 n1 = __ldg(nodes + 4 * node + 1);
                float4 n2 = __ldg(nodes + 4 * node + 2);
                const int2 n3 = __ldg(reinterpret_cast<const int2*>(nodes + 4 * node + 3));
                if constexpr (COUNT) tl->node++;
                // slab tests of both children (aabb.rs:18-56)
                float a0 = fmaf(n0.x, ix, ox), a1 = fmaf(n0.y, ix, ox);
                float b0 = fmaf(n0.z, iy, oy), b1 = fmaf(n0.w, iy, oy);
                float c0 = fmaf(n2.x, iz, oz), c1 = fmaf(n2.y, iz, oz);
                float en0 = fmaxf(fmaxf(fminf(a0, a1), fminf(b0, b1)), fmaxf(fminf(c0, c1), tmin));
                float ex0 = fminf(fminf(fmaxf(a0, a1), fmaxf(b0, b1)), fminf(fmaxf(c0, c1), hit.t));
                float d0 = fmaf(n1.x, ix, ox), d1 = fmaf(n1.y, ix, ox);
                float e0 = fmaf(n1.z, iy, oy), e1 = fmaf(n1.w, iy, oy);
                float f0 = fmaf(n2.z, iz, oz), f1 = fmaf(n2.w, iz, oz);
                float en1 = fmaxf(fmaxf(fminf(d0, d1), fminf(e0, e1)), fmaxf(fminf(f0, f1), tmin));
                float ex1 = fminf(fminf(fmaxf(d0, d1), fmaxf(e0, e1)), fminf(fmaxf(f0, f1), hit.t));
                const bool h0 = en0 < ex0, h1 = en1 < ex1;
                const int c0e = n3.x, c1e = n3.y;   // links: inner node or encoded leaf
                if (!h0 && !h1) {
                    node = sp > 0 ? stack[--sp * stride] : kSentinel;
                } else {
                    const bool first0 = h0 && (!h1 || en0 <= en1);
                    node = first0 ? c0e : c1e;
                    if (h0 && h1) {
                        if (sp < S.stack_depth) {
                            stack[sp++ * stride] = first0 ? c1e : c0e;
                        } else {
                            err |= LUM_KERR_STACK_OVERFLOW;
                        }
                    }
                }
                if (node < 0 && leaf == 0) {
                    leaf = node;
                    node = sp > 0 ? stack[--sp * stride] : kSentinel;
                }
                if (!__any_sync(__activemask(), leaf == 0)) break;
            }
            while (leaf < 0) {
                const int first = (~leaf) >> 3, cnt = ((~leaf) & 7) + 1;
                for (int k = 0; k < cnt; ++k) {
                    if (test_prim<COUNT, SPH, CLS>(S, first + k, ray, tmin, hit, tl, ia_ray)) {
                        found = true;
                        if (any) {
                            tv.node = kSentinel;
                            return true;
                        }
                    }
                }
                leaf = 0;
                if (node < 0) {
                    leaf = node;
                    node = sp > 0 ? stack[--sp * stride] : kSentinel;
                }
            }
            if (node == kSentinel) break;
            if constexpr (SUSPEND > 0) {
                if (__popc(__activemask()) <= SUSPEND) {
                    tv.node = node;
                    tv.sp = sp;
                    return false;
                }
            }
        }
        tv.node = kSentinel;
    }
    for (int k = 0; k < S.n_planes; ++k) {                             // scene.rs:826-831
        if constexpr (COUNT) tl->plane++;
        float t;
        if (hit_plane(S.planes[k], ray, tmin, hit.t, t)) {
            hit.t = t;
            hit.prim = -2 - k;
            found = true;
            if (any) return true;
        }
    }
    return true;
}

// LUM_SUSPEND_LANES, the SUSPEND of the persistent kernels' walks: lanes still walking the BVH
// when at most that many of the warp are left keep their place and let the finished lanes shade
// and start new rays first (trace_resume); 0 = every walk runs to its end before any lane
// shades.  Measured on B200 against 0 (kernel time per frame, images
// identical): 4 / 8 / 16 lanes gave the sphere field 101.7 -> 91.1 / 91.9 / 92.4 ms, the box room
// 2.57 -> 2.40 / 2.29 / 2.23 ms, the quad scene 13.6 -> 11.5 / 11.4 / 11.8 ms and the dense mesh
// 238.4 -> 200.6 / 198.3 / 199.7 ms.
#ifndef LUM_SUSPEND_LANES
#define LUM_SUSPEND_LANES 8
#endif

// Closest hit (any = false) keeps the nearest accepted t; any = true returns at the first
// accepted hit (the shadow query, render.rs:1457-1460).  Unbounded planes follow the BVH
// (scene.rs:826-831).
template <bool COUNT = false, bool SPH = false>
__device__ __forceinline__ bool trace(const SceneDev& S, const Ray& ray, float tmin, bool any, Hit& hit, int* stack,
                                      uint32_t& err, TestTally* tl = nullptr) {
    bool found = false;
    Trav tv{S.n_nodes > 0 ? 0 : kSentinel, 0};
    trace_resume<COUNT, SPH, 0>(S, ray, tmin, any, hit, found, tv, stack, err, tl);
    return found;
}

// ---------------------------------------------------------------------------- hit details
struct Surface {
    V p, n;          // point, normal facing the ray
    bool front;
    int mat;
};

// Point, outward normal, face orientation and material of a hit (hit.rs:19-43).
template <bool SPH = false, int CLS = CLS_ALL>
__device__ __forceinline__ Surface surface_of(const SceneDev& S, const Ray& ray, const Hit& h) {
    Surface s;
    s.p = fma3(ray.d, h.t, ray.o);
    V on;
    if (h.prim <= -2) {
        const PlaneDev& P = S.planes[-2 - h.prim];
        on = mk(P.n);
        s.mat = P.material;
    } else {
        int meta = __ldg(S.meta + h.prim);
        int type = SPH ? (int)PT_SPHERE : meta & 15;
        s.mat = meta >> 4;
        float4 a = ldp(S, h.prim, 0);
        switch (type) {
            case PT_SPHERE: {
                if constexpr (!cls_has_prim<CLS>(PT_SPHERE)) break;
                V c = xyz(a);
                if constexpr (!SPH) {
                    float4 b = ldp(S, h.prim, 1);
                    if (b.w != 0.0f) c = fma3(xyz(b) - c, ray.time, c);
                }
                on = (s.p - c) * (1.0f / a.w);
                break;
            }
            case PT_QUAD: {
                if constexpr (!cls_has_prim<CLS>(PT_QUAD)) break;
                float4 d = ldp(S, h.prim, 3);
                on = unit(xyz(d)) * d.w;
                break;
            }
            case PT_TRIANGLE: {
                if constexpr (!cls_has_prim<CLS>(PT_TRIANGLE)) break;
                float4 d = ldp(S, h.prim, 3);
                int si = __float_as_int(d.w);
                if (si >= 0) {
                    const float* sn = S.smooth_n + 9 * si;
                    float w0 = 1.0f - h.b1 - h.b2;
                    on = unit(mk(sn) * w0 + mk(sn + 3) * h.b1 + mk(sn + 6) * h.b2);
                } else {
                    on = xyz(d);
                }
                break;
            }
            case PT_DISK:
                if constexpr (cls_has_prim<CLS>(PT_DISK)) on = xyz(ldp(S, h.prim, 1));
                break;
            default: on = mk(1.0f, 0.0f, 0.0f); break;                 // constant_medium.rs:63
        }
    }
    s.front = dot(ray.d, on) < 0.0f;
    s.n = s.front ? on : -on;
    return s;
}

// ------------------------------------------------------------------------------ shading
__device__ __forceinline__ V tex_value(const MatDev& m, V p) {           // texture.rs:19-50
    if (m.tex == 0) return mk(m.color);
    float inv = 1.0f / m.tex_scale;
    long long x = (long long)floorf(p.x * inv), y = (long long)floorf(p.y * inv), z = (long long)floorf(p.z * inv);
    return ((x + y + z) % 2 == 0) ? mk(m.color) : mk(m.color2);
}

__device__ __forceinline__ V emitted(const MatDev& m, V p) {           // material.rs:241-243
    return m.kind == 4 ? tex_value(m, p) * m.intensity : mk(0.0f, 0.0f, 0.0f);
}

__device__ __forceinline__ float schlick(float cosine, float ref_idx) { // material.rs:138-141
    float r0 = (1.0f - ref_idx) / (1.0f + ref_idx);
    r0 = r0 * r0;
    float m = 1.0f - cosine;
    float m2 = m * m;
    return r0 + (1.0f - r0) * (m2 * m2 * m);
}

__device__ __forceinline__ V fresnel(float cos_t, V f0) {              // material.rs:291-294
    float m = fmaxf(1.0f - cos_t, 0.0f);
    float m2 = m * m;
    float t = m2 * m2 * m;
    return f0 * (1.0f - t) + mk(t, t, t);
}

// material.rs:297-319 with tan(theta) evaluated directly (same angle, no atan/sin/cos).
__device__ __forceinline__ V ggx_normal(V n, float alpha, float r1, float r2) {
    float tan2 = alpha * alpha * r1 / (1.0f - r1 + 1e-10f);
    float ct = rsqrtf(1.0f + tan2);
    float st = sqrtf(tan2) * ct;
    float sp, cp;
    sincospif(2.0f * r2, &sp, &cp);
    V up = fabsf(n.y) < 0.999f ? mk(0.f, 1.f, 0.f) : mk(1.f, 0.f, 0.f);
    V tg = unit(cross(up, n));
    V bt = cross(n, tg);
    return unit(tg * (st * cp) + bt * (st * sp) + n * ct);
}

struct Scatter {
    V dir;
    V att;
    V org;   // origin of the scattered ray: the hit point (set by the caller), or Subsurface's exit point
};

enum : int { MAT_BLEND = 7 };

// Blend::scatter's choice (material.rs:408-415): one draw per level, mat_a with probability
// ratio, down to a material that is not a Blend.
__device__ __forceinline__ const MatDev* blend_walk(const MatDev* mats, const MatDev* m, uint32_t key0,
                                                        uint32_t key1, uint32_t pixel, uint32_t stratum,
                                                        uint32_t bounce) {
    const float4 u = draw4(key0, key1, pixel, stratum, bounce, CALL_BLEND);
    const float uu[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
    for (int l = 0; l < kMaxBlendDepth; ++l) {
        if (m->kind != MAT_BLEND) break;
        m = &mats[uu[l] < m->extra[0] ? m->sub[0] : m->sub[1]];
    }
    return m;
}
__device__ __forceinline__ const MatDev& blend_leaf(const SceneDev& S, const MatDev& m, const RenderDev& R,
                                                    uint32_t pixel, uint32_t stratum, uint32_t bounce) {
    return m.kind == MAT_BLEND ? *blend_walk(S.mats, &m, R.key0, R.key1, pixel, stratum, bounce) : m;
}

// Blend::emitted (material.rs:417-420): ratio * emitted(a) + (1 - ratio) * emitted(b),
// evaluated from the blend's flattened list of emissive leaves (no recursion, no call).
__device__ __forceinline__ V emitted_at(const SceneDev& S, int idx, const MatDev& m, V p) {
    if (m.kind != MAT_BLEND) return emitted(m, p);
    V e = mk(0.f, 0.f, 0.f);
    for (int k = 0; k < m.n_emit; ++k) {
        const BlendEmit be = S.blend_emit[m.emit_first + k];
        e = e + emitted(S.mats[be.leaf], p) * be.weight;
    }
    return e;
}

// Iridescent::thin_film_color (material.rs:469-491): sin^2(phase / 2) at 650 / 532 / 450 nm
// with phase = 2 pi opd / lambda, i.e. sin^2(pi opd / lambda).
__device__ __forceinline__ V thin_film(float cos_t, float thickness, float film_ior) {
    float sin_t = sqrtf(fmaxf(1.0f - cos_t * cos_t, 0.0f));
    float sf = sin_t / film_ior;
    float cf = sqrtf(fmaxf(1.0f - sf * sf, 0.0f));
    float opd = 2.0f * thickness * film_ior * cf;
    float r = sinpif(opd / 650.0f), g = sinpif(opd / 532.0f), b = sinpif(opd / 450.0f);
    return mk(r * r, g * g, b * b);
}

// The other materials' scatter (material.rs:408-865).  Keyed draws: CALL_SCATTER slots as
// noted, Subsurface's exit direction from CALL_EXTRA.  Inlined like everything the megakernel
// calls: a device-function call makes every value live across it a spill candidate.
struct ScatterMore {
    V dir, att, org;
    bool ok;
};
__device__ __forceinline__ ScatterMore scatter_more(const MatDev* mp, V rd, V hp, V hn, float4 s, uint32_t key0,
                                                       uint32_t key1, uint32_t pixel, uint32_t stratum,
                                                       uint32_t bounce) {
    const MatDev& m = *mp;
    ScatterMore out;
    out.org = hp;
    out.ok = true;
    struct {
        V p, n;
    } sf{hp, hn};
    struct {
        V d;
    } ray{rd};
    switch (m.kind) {
        case 8: {                                                      // Transparent, material.rs:429-435
            out.dir = ray.d;
            out.att = mk(1.f, 1.f, 1.f);
            return out;
        }
        case 9: {                                                      // Iridescent, material.rs:499-527
            V ud = unit(ray.d);
            float ct = fminf(fabsf(dot(-ud, sf.n)), 1.0f);
            out.att = mul(mk(m.color), thin_film(ct, m.extra[0], m.ior));
            V d = reflect(ud, sf.n);
            if (m.roughness > 0.0f) {
                d = d + in_unit_sphere(s.x, s.y, s.z) * m.roughness;
                if (dot(d, sf.n) <= 0.0f) { out.ok = false; return out; }
            }
            out.dir = d;
            return out;
        }
        case 10: {                                                     // Toon, material.rs:549-577
            V d = sf.n + unit_vector(s.x, s.y);
            if (near_zero(d)) d = sf.n;
            V du = unit(d);
            float ndl = fmaxf(dot(du, sf.n), 0.0f);
            float band = fminf(fmaxf(floorf(ndl * m.extra[0]) / (m.extra[0] - 1.0f), 0.0f), 1.0f);
            V hv = unit(unit(-ray.d) + du);
            float spec = powf(fmaxf(dot(hv, sf.n), 0.0f), m.extra[1] * 100.0f);
            out.dir = d;
            out.att = mk(m.color) * (band + (spec > 0.5f ? 0.3f : 0.0f));
            return out;
        }
        case 11: {                                                     // Anisotropic, material.rs:607-641
            V refl = reflect(unit(ray.d), sf.n);
            const int ax = (int)m.extra[2];
            V wt = ax == 0 ? mk(1.f, 0.f, 0.f) : (ax == 1 ? mk(0.f, 1.f, 0.f) : mk(0.f, 0.f, 1.f));
            V t = unit(wt - sf.n * dot(wt, sf.n));
            V b = cross(sf.n, t);
            float sp, cp;
            sincospif(2.0f * s.x, &sp, &cp);
            float r2 = sqrtf(s.y);
            V sc = unit(refl + t * (cp * r2 * m.extra[0]) + b * (sp * r2 * m.extra[1]));
            if (!(dot(sc, sf.n) > 0.0f)) { out.ok = false; return out; }
            out.dir = sc;
            out.att = mk(m.color);
            return out;
        }
        case 12: {                                                     // Clearcoat, material.rs:664-707
            V ud = unit(ray.d);
            float ct = fminf(fabsf(dot(-ud, sf.n)), 1.0f);
            float r0 = (1.0f - m.ior) / (1.0f + m.ior);
            r0 = r0 * r0;
            float om = 1.0f - ct, om2 = om * om;
            float fr = r0 + (1.0f - r0) * (om2 * om2 * om);
            if (s.x < fr * m.extra[0]) {
                V refl = reflect(ud, sf.n);
                float rough = (1.0f - m.extra[0]) * 0.3f;
                V d = refl;
                if (rough > 0.001f) {
                    V fz = refl + in_unit_sphere(s.y, s.z, s.w) * rough;
                    if (dot(fz, sf.n) > 0.0f) d = fz;
                }
                out.dir = d;
                out.att = mk(1.f, 1.f, 1.f);
                return out;
            }
            V d = sf.n + unit_vector(s.y, s.z);
            if (near_zero(d)) d = sf.n;
            out.dir = d;
            out.att = mk(m.color);
            return out;
        }
        case 13: {                                                     // Velvet, material.rs:724-746
            V d = sf.n + unit_vector(s.x, s.y);
            if (near_zero(d)) d = sf.n;
            float ct = fabsf(dot(-unit(ray.d), sf.n));
            float st = sqrtf(fmaxf(1.0f - ct * ct, 0.0f));
            out.dir = d;
            out.att = mk(m.color) * (1.0f + st * sqrtf(st) * m.extra[0]);
            return out;
        }
        case 14: {                                                     // Translucent, material.rs:769-797
            V d;
            if (s.x < m.extra[0]) {
                V below = -sf.n + unit_vector(s.y, s.z);
                d = unit(ray.d) * (1.0f - m.extra[1]) + below * m.extra[1];
                if (near_zero(d)) d = -sf.n;
            } else {
                d = sf.n + unit_vector(s.y, s.z);
                if (near_zero(d)) d = sf.n;
            }
            out.dir = d;
            out.att = mk(m.color);
            return out;
        }
        case 15: {                                                     // Subsurface, material.rs:823-864
            float fr = schlick(fabsf(dot(unit(ray.d), sf.n)), 1.0f / 1.4f);
            if (s.x < fr) {
                V d = sf.n + unit_vector(s.y, s.z);
                if (near_zero(d)) d = sf.n;
                out.dir = d;
                out.att = mk(m.color);
                return out;
            }
            const float mfp = m.extra[0];
            float step = -mfp * logf(fmaxf(s.y, 1e-10f));
            out.org = sf.p + unit_vector(s.z, s.w) * step;
            float4 ex = draw4(key0, key1, pixel, stratum, bounce, CALL_EXTRA);
            V d = sf.n + unit_vector(ex.x, ex.y);
            out.dir = near_zero(d) ? sf.n : unit(d);
            const float k = -step / mfp;
            out.att = mul(mk(m.color), mk(__expf(k * (1.0f - m.color2[0])), __expf(k * (1.0f - m.color2[1])),
                                          __expf(k * (1.0f - m.color2[2]))));
            return out;
        }
        default:
            { out.ok = false; return out; }
    }
}

// Material::scatter; draws s = (s0..s3) of CALL_SCATTER, extra for dispersion.
// KIND >= 0 fixes the material kind at compile time (the material-sorted shading kernels of
// the wavefront tracer); KIND = -1 dispatches on m.kind.  Both run the same arithmetic.
// EXT = false leaves out the other materials (material.rs:396-865): kernels for scenes
// without them carry none of their code (the megakernel is sensitive to its code size).
// SPH: the scene's materials are Lambertian / Metal / Dielectric / Emissive only.
template <int KIND = -1, bool EXT = true, bool SPH = false, int U = 10>
__device__ __forceinline__ bool scatter(const MatDev& m, const Ray& ray, const Surface& sf, float hit_t, float4 s,
                                        const RenderDev& R, uint32_t pixel, uint32_t stratum, uint32_t bounce,
                                        Scatter& out) {
    if constexpr (SPH) {
        if (KIND < 0 && m.kind > 3) return false;                      // Emissive: no scatter
    }
    switch (KIND >= 0 ? KIND : m.kind) {
        case 1: {                                                      // material.rs:59-71
            V d = sf.n + unit_vector(s.x, s.y);
            if (near_zero(d)) d = sf.n;
            out.dir = d;
            out.att = tex_value(m, sf.p);
            return true;
        }
        case 2: {                                                      // material.rs:94-106
            V refl = reflect(unit(ray.d), sf.n);
            V sc = refl + in_unit_sphere(s.x, s.y, s.z) * m.fuzz;
            if (dot(sc, sf.n) > 0.0f) {
                out.dir = sc;
                out.att = mk(m.color);
                return true;
            }
            return false;
        }
        case 3: {                                                      // material.rs:149-213
            float ior = m.ior;
            V chan = mk(1.f, 1.f, 1.f);
            if (m.dispersion > 0.0f) {
                float4 ex = draw4<U>(R.key0, R.key1, pixel, stratum, bounce, CALL_EXTRA);
                uint32_t ch = (uint32_t)(ex.x * 3.0f);
                ior += ch == 0 ? -m.dispersion : (ch == 1 ? 0.0f : m.dispersion);
                chan = ch == 0 ? mk(3.f, 0.f, 0.f) : (ch == 1 ? mk(0.f, 3.f, 0.f) : mk(0.f, 0.f, 3.f));
            }
            float eta = sf.front ? 1.0f / ior : ior;
            V ud = unit(ray.d);
            float ct = fminf(dot(-ud, sf.n), 1.0f);
            float st = sqrtf(1.0f - ct * ct);
            V d;
            if (eta * st > 1.0f || schlick(ct, eta) > s.x) {
                d = reflect(ud, sf.n);
            } else {                                                   // vec3.rs:73-78
                V rp = (ud + sf.n * ct) * eta;
                d = rp + sf.n * -sqrtf(fabsf(1.0f - len2(rp)));
            }
            if (m.roughness > 0.0f) d = d + in_unit_sphere(s.y, s.z, s.w) * m.roughness;
            V att;
            if (!sf.front && !m.tint_white)
                att = mk(__expf(-(1.0f - m.tint[0]) * hit_t), __expf(-(1.0f - m.tint[1]) * hit_t),
                         __expf(-(1.0f - m.tint[2]) * hit_t));
            else
                att = mk(m.tint);
            if (m.dispersion > 0.0f) att = mul(att, chan);
            out.dir = d;
            out.att = att;
            return true;
        }
        case 5: {                                                      // material.rs:328-390
            float alpha = m.roughness * m.roughness;
            V v = unit(-ray.d);
            V n = sf.n;
            V alb = tex_value(m, sf.p);
            float ndv = fmaxf(dot(n, v), 0.001f);
            V f0 = mk(0.04f, 0.04f, 0.04f) * (1.0f - m.metallic) + alb * m.metallic;
            V fw = fresnel(ndv, f0);
            float sp = fminf(fmaxf((fw.x + fw.y + fw.z) * (1.0f / 3.0f), 0.1f), 0.9f);
            if (s.x < sp) {
                V h = ggx_normal(n, alpha, s.y, s.z);
                V l = h * (2.0f * dot(v, h)) - v;
                float ndl = dot(n, l);
                if (ndl <= 0.0f) return false;
                float ndh = fmaxf(dot(n, h), 0.0f);
                float vdh = fmaxf(dot(v, h), 0.0f);
                float k = (m.roughness + 1.0f) * (m.roughness + 1.0f) * 0.125f;
                float g = (ndv / (ndv * (1.0f - k) + k)) * (ndl / (ndl * (1.0f - k) + k));
                V f = fresnel(vdh, f0);
                V w = ndh > 0.001f ? f * (g * vdh / (ndv * ndh)) : mk(0.f, 0.f, 0.f);
                out.dir = l;
                out.att = w * (1.0f / sp);
                return true;
            }
            V d = n + unit_vector(s.y, s.z);
            if (near_zero(d)) d = n;
            V kd = (mk(1.f, 1.f, 1.f) - fw) * (1.0f - m.metallic);
            out.dir = d;
            out.att = mul(kd, alb) * (1.0f / (1.0f - sp));
            return true;
        }
        case 6: {                                                      // constant_medium.rs:81-89
            out.dir = in_unit_sphere(s.x, s.y, s.z);
            out.att = mk(m.color);
            return true;
        }
        case 8: case 9: case 10: case 11: case 12: case 13: case 14: case 15: {
            if constexpr (EXT) {
                const ScatterMore r = scatter_more(&m, ray.d, sf.p, sf.n, s, R.key0, R.key1, pixel, stratum, bounce);
                out.dir = r.dir;
                out.att = r.att;
                out.org = r.org;
                return r.ok;
            }
            return false;
        }
        default:                                                       // Emissive: no scatter
            return false;
    }
}

// render.rs:1333-1343 (Frisvad)
__device__ __forceinline__ void build_onb(V n, V& a, V& b) {
    if (n.z < -0.9999999f) {
        a = mk(0.f, -1.f, 0.f);
        b = mk(-1.f, 0.f, 0.f);
        return;
    }
    float aa = 1.0f / (1.0f + n.z);
    float bb = -n.x * n.y * aa;
    a = mk(1.0f - n.x * n.x * aa, bb, -n.x);
    b = mk(bb, 1.0f - n.y * n.y * aa, -n.y);
}

// Samples one light (render.rs:1346-1455).  Returns false when the sample contributes
// nothing before visibility; otherwise the shadow ray and unoccluded contribution.
template <int CLS = CLS_ALL>
__device__ __forceinline__ bool sample_light(const SceneDev& S, V hp, V normal, V albedo, float4 u, Ray& shadow,
                                             float& shadow_tmax, V& contrib) {
    int nl = S.n_lights;
    int idx = min((int)(u.y * (float)nl), nl - 1);
    const LightDev& L = S.lights[idx];
    V lp, ln;
    float area;
    if (!cls_has_light<CLS>(L.kind)) return false;                      // not in this build's class
    if (cls_has_light<CLS>(1) && L.kind == 1) {
        V to_c = mk(L.p0) - hp;
        float d2c = len2(to_c);
        if (d2c < L.radius * L.radius) return false;
        float dc = sqrtf(d2c);
        float stm = L.radius / dc;
        float ctm = sqrtf(fmaxf(1.0f - stm * stm, 0.0f));
        float ct = 1.0f - u.z * (1.0f - ctm);
        float st = sqrtf(fmaxf(1.0f - ct * ct, 0.0f));
        float sp, cp;
        sincospif(2.0f * u.w, &sp, &cp);
        V w = to_c * (1.0f / dc);
        V a, b;
        build_onb(w, a, b);
        V dir = unit(a * (st * cp) + b * (st * sp) + w * ct);
        V oc = hp - mk(L.p0);
        float bc = dot(oc, dir);
        float cc = len2(oc) - L.radius * L.radius;
        float disc = bc * bc - cc;
        float t;
        if (disc > 0.0f) {
            float sq = sqrtf(disc);
            float t1 = -bc - sq;
            t = t1 > 0.001f ? t1 : -bc + sq;
        } else {
            t = dc;
        }
        lp = fma3(dir, t, hp);
        ln = unit(lp - mk(L.p0));
        float solid = 2.0f * CUDART_PI_F * (1.0f - ctm);
        area = solid * t * t / fmaxf(fabsf(dot(-dir, ln)), 0.001f);
    } else if (cls_has_light<CLS>(2) && L.kind == 2) {
        lp = mk(L.p0) + mk(L.u) * u.z + mk(L.v) * u.w;
        area = L.area;
        ln = mk(L.n);
    } else if constexpr (cls_has_light<CLS>(3)) {
        float r = sqrtf(u.z) * L.radius;
        float sp, cp;
        sincospif(2.0f * u.w, &sp, &cp);
        V w = mk(L.n);
        V av = fabsf(w.x) > 0.9f ? mk(0.f, 1.f, 0.f) : mk(1.f, 0.f, 0.f);
        V ut = unit(cross(w, av));
        V vt = cross(w, ut);
        lp = mk(L.p0) + ut * (r * cp) + vt * (r * sp);
        area = L.area;
        ln = w;
    } else {
        return false;
    }
    V tl = lp - hp;
    float d2 = len2(tl);
    float dist = sqrtf(d2);
    V dir = tl * (1.0f / dist);
    float ct = dot(normal, dir);
    if (ct <= 0.0f) return false;
    float ctl = fabsf(dot(-dir, ln));
    if (ctl <= 0.001f) return false;
    shadow.o = hp;
    shadow.d = dir;
    shadow.time = 0.0f;                                                // Ray::new (render.rs:1457)
    shadow_tmax = dist - 0.001f;
    contrib = mul(mk(L.e), albedo) * (ct * ctl * area * (float)nl / (CUDART_PI_F * d2));
    return true;
}

// sample_light out of line for the mesh class (see hit_fog_cold).
template <int CLS>
__device__ __noinline__ bool sample_light_cold(const SceneDev& S, V hp, V normal, V albedo, float4 u, Ray& shadow,
                                               float& shadow_tmax, V& contrib) {
    return sample_light<CLS>(S, hp, normal, albedo, u, shadow, shadow_tmax, contrib);
}

// Background::Starfield (render.rs:86-112): dark blue space plus stars hashed from the
// direction quantised at 500 * density cells per unit.
__device__ __forceinline__ V starfield(float density, float brightness, V ud, float t) {
    V space = mk(0.0f, 0.0f, 0.02f) * (1.0f - t) + mk(0.02f, 0.0f, 0.05f) * t;
    const float scale = 500.0f * density;
    const long long ix = (long long)floorf(ud.x * scale), iy = (long long)floorf(ud.y * scale),
                    iz = (long long)floorf(ud.z * scale);
    const unsigned long long hash = ((unsigned long long)ix * 73856093ull) ^ ((unsigned long long)iy * 19349663ull) ^
                                    ((unsigned long long)iz * 83492791ull);
    const float star = (float)(hash % 10000ull) / 10000.0f;
    if (!(star > 0.997f)) return space;
    const float rh = (float)((hash >> 8) % 100ull) / 100.0f;
    const V c = rh < 0.3f ? mk(1.0f, 0.9f, 0.8f) : (rh < 0.6f ? mk(0.9f, 0.9f, 1.0f) : mk(1.f, 1.f, 1.f));
    return space + c * (star * brightness);
}

// Background::EnvMap (render.rs:113-151): equirectangular lookup, bilinear, times intensity.
__device__ __forceinline__ V envmap(const float* env, uint32_t env_w, uint32_t env_h, float intensity, V ud) {
    if (!env) return mk(0.f, 0.f, 0.f);
    const float theta = acosf(-ud.y);
    const float phi = atan2f(-ud.z, ud.x) + CUDART_PI_F;
    const float fx = phi * (0.5f / CUDART_PI_F) * (float)env_w - 0.5f;
    const float fy = theta * (1.0f / CUDART_PI_F) * (float)env_h - 0.5f;
    const float flx = floorf(fx), fly = floorf(fy);
    const int w = (int)env_w, h = (int)env_h;
    int x0 = (int)flx % w;
    if (x0 < 0) x0 += w;
    const int y0 = (int)fminf(fmaxf(fly, 0.0f), (float)(h - 1));
    const int x1 = (x0 + 1) % w, y1 = min(y0 + 1, h - 1);
    const float tx = fx - flx, ty = fy - fly;
    auto px = [&](int x, int y) { return mk(env + 3 * ((size_t)y * w + x)); };
    const V c = px(x0, y0) * ((1.0f - tx) * (1.0f - ty)) + px(x1, y0) * (tx * (1.0f - ty)) +
                px(x0, y1) * ((1.0f - tx) * ty) + px(x1, y1) * (tx * ty);
    return c * intensity;
}

template <bool EXT = true>
__device__ __forceinline__ V background(const SceneDev& S, const RenderDev& R, const Ray& r) {  // render.rs:73-171
    if (R.background == 1) return mk(R.bg_color);
    V ud = unit(r.d);
    float t = 0.5f * (ud.y + 1.0f);
    if (R.background == 2) return mk(R.bg_color) * (1.0f - t) + mk(R.bg_color2) * t;
    if (R.background == 3) {
        V sky = mk(1.f, 1.f, 1.f) * (1.0f - t) + mk(R.bg_color2) * t;
        float sd = dot(ud, unit(mk(R.bg_dir)));
        if (sd > 0.9995f) return mk(R.bg_color) * R.bg_intensity;
        if (sd > 0.995f) {
            float glow = (sd - 0.995f) / (0.9995f - 0.995f);
            return sky + mk(R.bg_color) * (R.bg_intensity * 0.3f * glow);
        }
        return sky;
    }
    if constexpr (EXT) {
        if (R.background == 4) return starfield(R.star_density, R.star_brightness, ud, t);
        if (R.background == 5) return envmap(S.env, S.env_w, S.env_h, R.bg_intensity, ud);
    }
    return mk(1.f, 1.f, 1.f) * (1.0f - t) + mk(0.5f, 0.7f, 1.0f) * t;
}

// The pixel filter is written with explicitly rounded operations (no FMA contraction): the
// compiler contracts a*b+c per call site, so the same expression could round differently in the
// megakernel and in the wavefront kernels, and the images of both must agree bit for bit.
__device__ __forceinline__ float mitchell_1d(float x) {                // render.rs:220-237
    x = fabsf(x);
    const float b = 1.0f / 3.0f, c = 1.0f / 3.0f;
    const float x2 = __fmul_rn(x, x), x3 = __fmul_rn(x2, x);
    if (x < 1.0f)
        return __fdiv_rn(__fadd_rn(__fadd_rn(__fmul_rn(12.f - 9.f * b - 6.f * c, x3),
                                             __fmul_rn(-18.f + 12.f * b + 6.f * c, x2)),
                                   6.f - 2.f * b), 6.f);
    if (x < 2.0f)
        return __fdiv_rn(__fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(-b - 6.f * c, x3), __fmul_rn(6.f * b + 30.f * c, x2)),
                                             __fmul_rn(-12.f * b - 48.f * c, x)),
                                   8.f * b + 24.f * c), 6.f);
    return 0.0f;
}
__device__ __forceinline__ float filter_weight(int f, float dx, float dy) {  // render.rs:201-216
    if (f == 1)
        return __fmul_rn(fmaxf(__fsub_rn(1.0f, __fmul_rn(fabsf(dx), 2.0f)), 0.0f),
                         fmaxf(__fsub_rn(1.0f, __fmul_rn(fabsf(dy), 2.0f)), 0.0f));
    if (f == 2) return __expf(__fdiv_rn(-__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), 2.0f * 0.35f * 0.35f));
    if (f == 3) return __fmul_rn(mitchell_1d(__fmul_rn(dx, 2.0f)), mitchell_1d(__fmul_rn(dy, 2.0f)));
    return 1.0f;
}

// A finished path's contribution to its pixel (render.rs:1692-1701): radiance clamped to
// luminance 100, times the filter weight, and the weight; explicitly rounded like the filter.
__device__ __forceinline__ float4 path_sample(const RenderDev& R, V L, float jx, float jy) {
    const float lum = __fadd_rn(__fadd_rn(__fmul_rn(0.2126f, L.x), __fmul_rn(0.7152f, L.y)), __fmul_rn(0.0722f, L.z));
    const float k = lum > 100.0f ? __fdiv_rn(100.0f, lum) : 1.0f;
    const float w = filter_weight(R.pixel_filter, __fsub_rn(jx, 0.5f), __fsub_rn(jy, 0.5f));
    if (lum > 100.0f) L = V{__fmul_rn(L.x, k), __fmul_rn(L.y, k), __fmul_rn(L.z, k)};
    return make_float4(__fmul_rn(L.x, w), __fmul_rn(L.y, w), __fmul_rn(L.z, w), w);
}

// ------------------------------------------------------------------------------ path state
struct Path {
    Ray ray;
    V beta;        // throughput B_j
    V L;           // accumulated radiance
    float jx, jy;  // stratum jitter (pixel filter)
    uint32_t stratum;
    uint32_t bounce;
    bool skip_emission;
};

__device__ __forceinline__ unsigned long long globaltimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Camera ray through sub-pixel position (jx, jy) of pixel (gi, gj) for stratum st; c holds
// the stratum's camera draws (z, w: lens) (render.rs:1683-1690, camera.rs:82-102).
template <int U = 10>
__device__ __forceinline__ void start_path_at(const SceneDev& S, const RenderDev& R, uint32_t gi, uint32_t gj,
                                              uint32_t pixel, uint32_t st, float4 c, float jx, float jy, Path& P) {
    P.jx = jx;
    P.jy = jy;
    float y = (float)(R.full_h - 1 - gj);
    float uc = ((float)gi + P.jx) / (float)(R.full_w - 1);
    float vc = (y + P.jy) / (float)(R.full_h - 1);
    const CameraDev& C = S.cam;
    if (C.panorama) {
        // equirectangular (camera.rs:83-90): latitude theta = pi (1 - t), longitude
        // phi = 2 pi s - pi, unit direction; no lens
        // (explicitly rounded: the compiler contracts a * b + c into an FMA per call site, and
        // every kernel must produce the same direction bit for bit)
        float st_, ct_, sp_, cp_;
        sincospif(1.0f - vc, &st_, &ct_);
        sincospif(fmaf(2.0f, uc, -1.0f), &sp_, &cp_);
        const float a_ = __fmul_rn(st_, cp_), b_ = __fmul_rn(st_, sp_);
        const V d = mk(fmaf(C.fwd[0], a_, fmaf(C.u[0], b_, __fmul_rn(C.v[0], ct_))),
                       fmaf(C.fwd[1], a_, fmaf(C.u[1], b_, __fmul_rn(C.v[1], ct_))),
                       fmaf(C.fwd[2], a_, fmaf(C.u[2], b_, __fmul_rn(C.v[2], ct_))));
        P.ray.o = mk(C.origin);
        P.ray.d = d * rsqrtf(len2(d));
    } else {
        V off = mk(0.f, 0.f, 0.f);
        if (C.lens_radius > 0.0f) {
            float r = sqrtf(c.z) * C.lens_radius, sp, cp;
            sincospif(2.0f * c.w, &sp, &cp);
            off = mk(C.u) * (r * cp) + mk(C.v) * (r * sp);
        }
        P.ray.o = mk(C.origin) + off;
        P.ray.d = mk(C.llc) + mk(C.hor) * uc + mk(C.ver) * vc - mk(C.origin) - off;
    }
    // time matters only to moving spheres; a static scene skips the draw (the keyed draws of
    // the other calls do not depend on it)
    P.ray.time = S.moving ? draw4<U>(R.key0, R.key1, pixel, st, 0, CALL_CAMERA2).x : 0.0f;
    P.beta = mk(1.f, 1.f, 1.f);
    P.L = mk(0.f, 0.f, 0.f);
    P.stratum = st;
    P.bounce = 0;
    P.skip_emission = false;
}

// Camera ray of stratum st: stratified jitter (render.rs:1683-1690).
template <int U = 10>
__device__ __forceinline__ void start_path(const SceneDev& S, const RenderDev& R, uint32_t gi, uint32_t gj,
                                           uint32_t pixel, uint32_t st, Path& P) {
    uint32_t sx = st % R.sqrt_spp, sy = st / R.sqrt_spp;
    float4 c = draw4<U>(R.key0, R.key1, pixel, st, 0, CALL_CAMERA);
    float inv_n = 1.0f / (float)R.sqrt_spp;
    start_path_at<U>(S, R, gi, gj, pixel, st, c, ((float)sx + c.x) * inv_n, ((float)sy + c.y) * inv_n, P);
}

// The one sample of a pixel after the time limit: stratum 0's draws, the pixel centre
// (render.rs:1612-1616).
__device__ __forceinline__ void start_path_centre(const SceneDev& S, const RenderDev& R, uint32_t gi, uint32_t gj,
                                                  uint32_t pixel, Path& P) {
    start_path_at(S, R, gi, gj, pixel, 0, draw4(R.key0, R.key1, pixel, 0, 0, CALL_CAMERA), 0.5f, 0.5f, P);
}

// Path states of the megakernel lanes.
enum : int { ST_IDLE = 0, ST_CLOSEST = 1, ST_SHADOW = 2, ST_DONE = 3 };

// NEE shadow query pending after a bounce: direction from the new hit point, its t range
// end, and the contribution B_j * (E albedo cos cos' A N / (pi d^2)) added if unoccluded.
// The shadow ray starts at the path's origin (P.ray.o), the hit point.  When Subsurface moves
// the next segment's origin to its exit point while a shadow query is pending, shade keeps the
// hit point in P.ray.o, writes the exit point to the caller's stash and negates tmax; the
// caller traces the shadow to |tmax| and then moves P.ray.o to the stashed point
// (shadow_done).
struct Pending {
    V dir;
    float tmax;
    V contrib;
};

// After a shadow query: the deferred Subsurface origin move, if any.
template <bool EXT>
__device__ __forceinline__ void shadow_done(Path& P, Pending& pend, const V* exit_stash) {
    if constexpr (EXT) {
        if (pend.tmax < 0.0f) {
            P.ray.o = *exit_stash;
            pend.tmax = -pend.tmax;
        }
    }
}

// Shading after the closest hit of segment j (ray_color, render.rs:1472-1537, iterative):
// L += B_j e_j now, B_{j+1} = B_j att_j rrw_j, the NEE term B_j d_j once its shadow ray is
// known to be unoccluded.  Returns the lane's next state.
// NEE = false builds the shading step of scenes without lights: no light-sampling code in the
// kernel (the megakernel runs ~11% faster on a light-free scene without it: instruction fetch).
template <int KIND = -1, bool EXT = true, bool NEE = true, bool SPH = false, int CLS = CLS_ALL>
__device__ __forceinline__ int shade(const SceneDev& S, const RenderDev& R, uint32_t pixel, Path& P, bool found,
                                     const Hit& h, Pending& pend, V* exit_stash = nullptr) {
    if (!found) {
        P.L = P.L + mul(P.beta, background<EXT>(S, R, P.ray));
        return ST_DONE;
    }
    const uint32_t depth = R.max_depth - P.bounce;
    Surface sf = surface_of<SPH, CLS>(S, P.ray, h);
    // A non-finite hit point (e.g. a fog hit at t = inf along a zero-length direction, where
    // the reference's distance test compares against NaN) makes this level's result NaN in
    // the reference, which its guard turns into zero for the level and everything deeper
    // (render.rs:1526-1531).  Ending the path here drops the same terms and keeps NaN rays
    // (whose slab tests pass every box) out of the traversal.
    if (!isfinite(sf.p.x) || !isfinite(sf.p.y) || !isfinite(sf.p.z)) return ST_DONE;
    const MatDev& m = S.mats[sf.mat];
    V e = P.skip_emission ? mk(0.f, 0.f, 0.f)
                          : (EXT && KIND < 0 ? emitted_at(S, sf.mat, m, sf.p) : emitted(m, sf.p));
    float4 su = draw4<philox_unroll<CLS>()>(R.key0, R.key1, pixel, P.stratum, P.bounce, CALL_SCATTER);
    Scatter sc;
    sc.org = sf.p;
    const MatDev& ms = EXT && KIND < 0 ? blend_leaf(S, m, R, pixel, P.stratum, P.bounce) : m;
    if (!scatter<KIND, EXT, SPH, philox_unroll<CLS>()>(ms, P.ray, sf, h.t, su, R, pixel, P.stratum, P.bounce, sc)) {
        P.L = P.L + mul(P.beta, e);
        return ST_DONE;
    }
    // A zero or non-finite scatter direction (in_unit_sphere at radius 0) would make the
    // next level NaN in the reference (its unit vectors divide by zero): end the path.
    const float dl2 = len2(sc.dir);
    if (!(dl2 > 0.0f) || !isfinite(dl2)) {
        P.L = P.L + mul(P.beta, e);
        return ST_DONE;
    }
    // the next segment (its origin and direction are dead past this point otherwise; a path
    // that ends below no longer reads its ray)
    P.ray.o = sc.org;
    P.ray.d = sc.dir;
    float4 nu = draw4<philox_unroll<CLS>()>(R.key0, R.key1, pixel, P.stratum, P.bounce, CALL_NEE);
    float surv = fminf(fmaxf(fmaxf(fmaxf(sc.att.x, sc.att.y), sc.att.z), 0.05f), 1.0f);
    if (depth < 47 && nu.x > surv) {                                   // Russian roulette
        P.L = P.L + mul(P.beta, e);
        return ST_DONE;
    }
    float rrw = depth < 47 ? 1.0f / surv : 1.0f;
    V nb = mul(P.beta, sc.att) * rrw;
    if (has_nan(e) || has_nan(nb)) return ST_DONE;                     // render.rs:1526-1531
    P.L = P.L + mul(P.beta, e);
    bool use_nee = NEE && !m.specular && S.n_lights > 0;
    bool shadow = false;
    if (use_nee) {
        Ray sr;
        V contrib;
        const bool lit = CLS == CLS_MESH ? sample_light_cold<CLS>(S, sf.p, sf.n, sc.att, nu, sr, pend.tmax, contrib)
                                         : sample_light<CLS>(S, sf.p, sf.n, sc.att, nu, sr, pend.tmax, contrib);
        if (lit) {
            pend.dir = sr.d;
            pend.contrib = mul(P.beta, contrib);
            shadow = !has_nan(pend.contrib);
        }
    }
    P.beta = nb;
    P.skip_emission = use_nee;
    ++P.bounce;
    if constexpr (EXT) {
        if (shadow && (P.ray.o.x != sf.p.x || P.ray.o.y != sf.p.y || P.ray.o.z != sf.p.z)) {
            *exit_stash = P.ray.o;                     // Subsurface: the shadow starts at the hit point
            P.ray.o = sf.p;
            pend.tmax = -pend.tmax;
        }
    }
    if (shadow) return ST_SHADOW;
    return P.bounce >= R.max_depth ? ST_DONE : ST_CLOSEST;             // depth == 0 -> black
}

}  // namespace lum
