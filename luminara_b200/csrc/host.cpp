// host.cpp -- C ABI of the path-tracing core (include/luminara_gpu.h): scene flattening,
// BVH build, device upload and the render / ray-set entry points.
//
// lum_scene_create restates the world construction of scene::load_scene and
// SceneWorld::from_list (src/scene.rs:846-1645, 786-808) for the description's objects:
// transform wrappers (src/transform.rs) are applied to the geometry once, in f64, so the
// device sees world-space primitives; rects and boxes become quads that keep the rects'
// outward normals (src/rect.rs) and planar coordinates.
#include <cuda_runtime.h>
#include <omp.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/luminara_gpu.h"
#include "bvh_build.h"
#include "device_scene.h"
#include "kernels.h"
#include "scene_access.h"

namespace {

thread_local std::string g_error;

lum_status fail(lum_status code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_error = buf;
    return code;
}

lum_status cuda_fail(cudaError_t e, const char* what) {
    cudaGetLastError();
    if (e == cudaErrorMemoryAllocation) return fail(LUM_ERR_OUT_OF_MEMORY, "%s: %s", what, cudaGetErrorString(e));
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver)
        return fail(LUM_ERR_NO_DEVICE, "%s: %s", what, cudaGetErrorString(e));
    return fail(LUM_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define CU(call, what)                              \
    do {                                            \
        cudaError_t e_ = (call);                    \
        if (e_ != cudaSuccess) return cuda_fail(e_, what); \
    } while (0)

// ----------------------------------------------------------------------------- f64 math
struct D3 {
    double x, y, z;
};
D3 d3(const double* p) { return {p[0], p[1], p[2]}; }
D3 operator+(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
D3 operator-(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
D3 operator*(D3 a, double t) { return {a.x * t, a.y * t, a.z * t}; }
double dot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
D3 cross(D3 a, D3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
double length(D3 a) { return std::sqrt(dot(a, a)); }
D3 unit(D3 a) { return a * (1.0 / length(a)); }
bool near_zero(D3 a) { return std::fabs(a.x) < 1e-8 && std::fabs(a.y) < 1e-8 && std::fabs(a.z) < 1e-8; }

// Input validation.  The device computes in f32, so a parameter must be finite after the
// conversion to float; a NaN or an infinity would reach the BVH builder's bin index (an
// out-of-range integer conversion) and every ray's arithmetic.  The reference has no such
// checks (its scene loader parses finite TOML numbers, scene.rs:846), so these rejections
// only turn undefined behaviour into LUM_ERR_INVALID_ARGUMENT.
bool finite32(double x) { return std::isfinite(x) && std::fabs(x) <= 3.0e38; }
int first_nonfinite(const double* p, int n) {
    for (int k = 0; k < n; ++k)
        if (!finite32(p[k])) return k;
    return -1;
}
// Parameters lum_object.p[] holds for each object kind (include/luminara_gpu.h).
int object_param_count(int kind) {
    switch (kind) {
        case LUM_OBJ_SPHERE: return 4;
        case LUM_OBJ_MOVING_SPHERE: return 7;
        case LUM_OBJ_QUAD: return 9;
        case LUM_OBJ_RECT_XY: case LUM_OBJ_RECT_XZ: case LUM_OBJ_RECT_YZ: return 5;
        case LUM_OBJ_TRIANGLE: return 9;
        case LUM_OBJ_DISK: return 7;
        case LUM_OBJ_PLANE: return 6;
        case LUM_OBJ_BOX: return 6;
        case LUM_OBJ_FOG_SPHERE: return 5;
        case LUM_OBJ_FOG_BOX: return 7;
        default: return 0;
    }
}

// Composite of the transform wrappers, object -> world: p' = M p + T.
struct Xf {
    double M[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    D3 T{0, 0, 0};
    double scale = 1.0;
    bool drops_time = false;   // Translate, RotateY and Scale rebuild the ray with time 0
    D3 point(D3 p) const {
        return {M[0][0] * p.x + M[0][1] * p.y + M[0][2] * p.z + T.x, M[1][0] * p.x + M[1][1] * p.y + M[1][2] * p.z + T.y,
                M[2][0] * p.x + M[2][1] * p.y + M[2][2] * p.z + T.z};
    }
    D3 vec(D3 v) const {
        return {M[0][0] * v.x + M[0][1] * v.y + M[0][2] * v.z, M[1][0] * v.x + M[1][1] * v.y + M[1][2] * v.z,
                M[2][0] * v.x + M[2][1] * v.y + M[2][2] * v.z};
    }
    void left(const double R[3][3]) {
        double N[3][3];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) N[i][j] = R[i][0] * M[0][j] + R[i][1] * M[1][j] + R[i][2] * M[2][j];
        std::memcpy(M, N, sizeof N);
        D3 t = T;
        T = {R[0][0] * t.x + R[0][1] * t.y + R[0][2] * t.z, R[1][0] * t.x + R[1][1] * t.y + R[1][2] * t.z,
             R[2][0] * t.x + R[2][1] * t.y + R[2][2] * t.z};
    }
};

lum_status make_xf(const lum_transform& t, Xf& xf) {
    if (t.n_ops < 0 || t.n_ops > LUM_MAX_XF_OPS) return fail(LUM_ERR_INVALID_ARGUMENT, "transform has %d ops", t.n_ops);
    for (int i = 0; i < t.n_ops; ++i) {
        const double* a = t.arg[i];
        if (first_nonfinite(a, t.op[i] == LUM_XF_TRANSLATE ? 3 : 1) >= 0)
            return fail(LUM_ERR_INVALID_ARGUMENT, "transform op %d: non-finite argument", i);
        switch (t.op[i]) {
            case LUM_XF_TRANSLATE:                                      // transform.rs:18-29
                xf.T = xf.T + d3(a);
                xf.drops_time = true;
                break;
            case LUM_XF_ROTATE_X:
            case LUM_XF_ROTATE_Y:
            case LUM_XF_ROTATE_Z: {                                     // transform.rs:71-256
                double rad = a[0] * (3.14159265358979323846 / 180.0);
                double s = std::sin(rad), c = std::cos(rad);
                double R[3][3];
                if (t.op[i] == LUM_XF_ROTATE_Y) {
                    double r[3][3] = {{c, 0, s}, {0, 1, 0}, {-s, 0, c}};
                    std::memcpy(R, r, sizeof r);
                    xf.drops_time = true;
                } else if (t.op[i] == LUM_XF_ROTATE_X) {
                    double r[3][3] = {{1, 0, 0}, {0, c, -s}, {0, s, c}};
                    std::memcpy(R, r, sizeof r);
                } else {
                    double r[3][3] = {{c, -s, 0}, {s, c, 0}, {0, 0, 1}};
                    std::memcpy(R, r, sizeof r);
                }
                xf.left(R);
                break;
            }
            case LUM_XF_SCALE: {                                        // transform.rs:258-284
                double f = std::fabs(a[0]) < 1e-10 ? 1.0 : a[0];
                double R[3][3] = {{f, 0, 0}, {0, f, 0}, {0, 0, f}};
                xf.left(R);
                xf.scale *= f;
                xf.drops_time = true;
                break;
            }
            default:
                return fail(LUM_ERR_INVALID_ARGUMENT, "unknown transform op %d", t.op[i]);
        }
    }
    return LUM_OK;
}

// ----------------------------------------------------------------------------- flattening
struct PrimH {
    int type;
    int material;
    int orig;
    float rec[16];
    lum::BuildBox box;
};

float pad_of(double m) { return (float)(1e-4 + 1e-6 * m); }

void box_of_points(const std::vector<D3>& pts, double pad_abs, lum::BuildBox& b) {
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300}, m = 0;
    for (const D3& p : pts) {
        double v[3] = {p.x, p.y, p.z};
        for (int k = 0; k < 3; ++k) {
            lo[k] = std::min(lo[k], v[k]);
            hi[k] = std::max(hi[k], v[k]);
            m = std::max(m, std::fabs(v[k]));
        }
    }
    float pad = (float)pad_abs + pad_of(m);
    for (int k = 0; k < 3; ++k) {
        b.lo[k] = std::nextafter((float)lo[k], -INFINITY) - pad;
        b.hi[k] = std::nextafter((float)hi[k], INFINITY) + pad;
    }
}

void set4(float* r, int k, D3 v, float w) {
    r[4 * k + 0] = (float)v.x;
    r[4 * k + 1] = (float)v.y;
    r[4 * k + 2] = (float)v.z;
    r[4 * k + 3] = w;
}

PrimH make_quad(D3 q, D3 u, D3 v, double sign, int mat, int orig) {
    PrimH p{};
    p.type = lum::PT_QUAD;
    p.material = mat;
    p.orig = orig;
    D3 nn = cross(u, v);
    double nl2 = dot(nn, nn);
    D3 w = nn * (1.0 / nl2);
    set4(p.rec, 0, q, (float)dot(w, q));
    set4(p.rec, 1, u, (float)std::sqrt(nl2));
    set4(p.rec, 2, v, 0.0f);
    set4(p.rec, 3, w, (float)sign);
    box_of_points({q, q + u, q + v, q + u + v}, 0.0, p.box);
    return p;
}

// A quad whose plane is undefined: u x v is zero, or so small that w = n / |n|^2 leaves the f32
// range.  No ray hits it in the reference (its normal and planar coordinates are NaN).
bool degenerate_quad(D3 u, D3 v) {
    const D3 n = cross(u, v);
    const double l2 = dot(n, n);
    return !(l2 > 0.0) || !finite32(std::sqrt(l2)) || !finite32(1.0 / std::sqrt(l2));
}

bool box_finite(const lum::BuildBox& b) {
    for (int k = 0; k < 3; ++k)
        if (!std::isfinite(b.lo[k]) || !std::isfinite(b.hi[k])) return false;
    return true;
}

struct Flat {
    std::vector<PrimH> prims;
    std::vector<lum::PlaneDev> planes;
    std::vector<float> smooth;
};

// rect (plane 0 XY, 1 XZ, 2 YZ) -> quad keeping the rect's +axis outward normal
// (src/rect.rs:36,76,116) and its (u, v) = first/second coordinate fractions.
void rect_quad(int plane, double a0, double a1, double b0, double b1, double k, D3& q, D3& u, D3& v, double& sign) {
    if (plane == 0) {
        q = {a0, b0, k}; u = {a1 - a0, 0, 0}; v = {0, b1 - b0, 0}; sign = 1.0;    // x cross y = +z
    } else if (plane == 1) {
        q = {a0, k, b0}; u = {a1 - a0, 0, 0}; v = {0, 0, b1 - b0}; sign = -1.0;   // x cross z = -y
    } else {
        q = {k, a0, b0}; u = {0, a1 - a0, 0}; v = {0, 0, b1 - b0}; sign = 1.0;    // y cross z = +x
    }
}

lum_status flatten(const lum_scene_desc& d, Flat& F) {
    int32_t id = 0;
    for (uint32_t i = 0; i < d.n_objects; ++i) {
        const lum_object& o = d.objects[i];
        if (o.material < 0 || (uint32_t)o.material >= d.n_materials)
            return fail(LUM_ERR_INVALID_ARGUMENT, "object %u: material %d out of range", i, o.material);
        const int n_par = object_param_count(o.kind);
        if (n_par == 0) return fail(LUM_ERR_INVALID_ARGUMENT, "object %u: unknown kind %d", i, o.kind);
        const int bad = first_nonfinite(o.p, n_par);
        if (bad >= 0) return fail(LUM_ERR_INVALID_ARGUMENT, "object %u: parameter p[%d] is not finite", i, bad);
        const size_t first_prim = F.prims.size();
        Xf xf;
        bool has_xf = o.transform >= 0;
        if (has_xf) {
            if ((uint32_t)o.transform >= d.n_transforms || !d.transforms)
                return fail(LUM_ERR_INVALID_ARGUMENT, "object %u: transform %d out of range", i, o.transform);
            lum_status st = make_xf(d.transforms[o.transform], xf);
            if (st != LUM_OK) return st;
        }
        const double* p = o.p;
        switch (o.kind) {
            case LUM_OBJ_SPHERE:
            case LUM_OBJ_MOVING_SPHERE: {
                PrimH s{};
                s.type = lum::PT_SPHERE;
                s.material = o.material;
                s.orig = id++;
                bool moving = o.kind == LUM_OBJ_MOVING_SPHERE;
                double r = (moving ? p[6] : p[3]) * std::fabs(xf.scale);
                D3 c0 = xf.point(d3(p));
                D3 c1 = moving ? xf.point(d3(p + 3)) : c0;
                if (moving && xf.drops_time) c1 = c0;     // inner ray sees time 0: static at center0
                bool mv = moving && !xf.drops_time;
                set4(s.rec, 0, c0, (float)r);
                set4(s.rec, 1, c1, mv ? 1.0f : 0.0f);
                D3 rr{r, r, r};
                box_of_points({c0 - rr, c0 + rr, c1 - rr, c1 + rr}, 0.0, s.box);
                F.prims.push_back(s);
                break;
            }
            case LUM_OBJ_QUAD: {
                D3 q = xf.point(d3(p)), u = xf.vec(d3(p + 3)), v = xf.vec(d3(p + 6));
                if (degenerate_quad(u, v)) return fail(LUM_ERR_INVALID_ARGUMENT, "object %u: degenerate quad (u x v = 0)", i);
                F.prims.push_back(make_quad(q, u, v, 1.0, o.material, id++));
                break;
            }
            case LUM_OBJ_RECT_XY:
            case LUM_OBJ_RECT_XZ:
            case LUM_OBJ_RECT_YZ: {
                D3 q, u, v;
                double sg;
                rect_quad(o.kind - LUM_OBJ_RECT_XY, p[0], p[1], p[2], p[3], p[4], q, u, v, sg);
                if (degenerate_quad(xf.vec(u), xf.vec(v)))
                    return fail(LUM_ERR_INVALID_ARGUMENT, "object %u: degenerate rect (zero extent)", i);
                F.prims.push_back(make_quad(xf.point(q), xf.vec(u), xf.vec(v), sg, o.material, id++));
                break;
            }
            case LUM_OBJ_BOX: {                                         // rect.rs:128-141 order
                D3 mn = d3(p), mx = d3(p + 3);
                struct R { int plane; double a0, a1, b0, b1, k; } sides[6] = {
                    {0, mn.x, mx.x, mn.y, mx.y, mx.z}, {0, mn.x, mx.x, mn.y, mx.y, mn.z},
                    {1, mn.x, mx.x, mn.z, mx.z, mx.y}, {1, mn.x, mx.x, mn.z, mx.z, mn.y},
                    {2, mn.y, mx.y, mn.z, mx.z, mx.x}, {2, mn.y, mx.y, mn.z, mx.z, mn.x}};
                for (const R& r : sides) {
                    D3 q, u, v;
                    double sg;
                    rect_quad(r.plane, r.a0, r.a1, r.b0, r.b1, r.k, q, u, v, sg);
                    // a box flat along one axis (a panel) has four zero-area sides, which no ray
                    // hits in the reference either: they keep their primitive ids but are left out
                    if (degenerate_quad(xf.vec(u), xf.vec(v))) {
                        ++id;
                        continue;
                    }
                    F.prims.push_back(make_quad(xf.point(q), xf.vec(u), xf.vec(v), sg, o.material, id++));
                }
                break;
            }
            case LUM_OBJ_TRIANGLE: {
                PrimH t{};
                t.type = lum::PT_TRIANGLE;
                t.material = o.material;
                t.orig = id++;
                D3 v0 = xf.point(d3(p)), v1 = xf.point(d3(p + 3)), v2 = xf.point(d3(p + 6));
                D3 e1 = v1 - v0, e2 = v2 - v0;
                set4(t.rec, 0, v0, 0.0f);
                set4(t.rec, 1, e1, 0.0f);
                set4(t.rec, 2, e2, 0.0f);
                D3 ng = cross(e1, e2);
                ng = length(ng) > 0 ? unit(ng) : D3{0, 0, 0};
                float m1;
                int32_t mi = -1;
                std::memcpy(&m1, &mi, 4);
                set4(t.rec, 3, ng, m1);
                box_of_points({v0, v1, v2}, 0.0, t.box);
                F.prims.push_back(t);
                break;
            }
            case LUM_OBJ_DISK: {                                        // disk.rs:16-29, 60-64
                PrimH k{};
                k.type = lum::PT_DISK;
                k.material = o.material;
                k.orig = id++;
                D3 n = d3(p + 3);
                n = near_zero(n) ? D3{0, 1, 0} : unit(n);
                n = unit(xf.vec(n));
                D3 c = xf.point(d3(p));
                double r = p[6] * std::fabs(xf.scale);
                if (r == 0.0) return fail(LUM_ERR_INVALID_ARGUMENT, "object %u: degenerate disk (radius 0)", i);
                set4(k.rec, 0, c, (float)r);
                set4(k.rec, 1, n, 0.0f);
                D3 rr{r, r, r};
                box_of_points({c - rr, c + rr}, 0.0, k.box);
                F.prims.push_back(k);
                break;
            }
            case LUM_OBJ_PLANE: {                                       // plane.rs:18-40
                lum::PlaneDev pl{};
                D3 n = d3(p + 3);
                n = near_zero(n) ? D3{0, 1, 0} : unit(n);
                n = unit(xf.vec(n));
                D3 pt = xf.point(d3(p));
                D3 up = std::fabs(n.y) > 0.999 ? D3{1, 0, 0} : D3{0, 1, 0};
                D3 ua = unit(cross(up, n));
                D3 va = cross(n, ua);
                pl.p[0] = (float)pt.x; pl.p[1] = (float)pt.y; pl.p[2] = (float)pt.z;
                pl.n[0] = (float)n.x; pl.n[1] = (float)n.y; pl.n[2] = (float)n.z;
                pl.ua[0] = (float)ua.x; pl.ua[1] = (float)ua.y; pl.ua[2] = (float)ua.z;
                pl.va[0] = (float)va.x; pl.va[1] = (float)va.y; pl.va[2] = (float)va.z;
                pl.material = o.material;
                pl.orig_id = id++;
                F.planes.push_back(pl);
                break;
            }
            case LUM_OBJ_FOG_SPHERE:
            case LUM_OBJ_FOG_BOX: {                                     // constant_medium.rs:15-22
                if (has_xf) return fail(LUM_ERR_UNSUPPORTED, "object %u: transformed constant medium", i);
                if (p[o.kind == LUM_OBJ_FOG_SPHERE ? 4 : 6] < 0.0)
                    return fail(LUM_ERR_INVALID_ARGUMENT, "object %u: negative medium density", i);
                PrimH f{};
                f.material = o.material;
                f.orig = id++;
                if (o.kind == LUM_OBJ_FOG_SPHERE) {
                    f.type = lum::PT_FOG_SPHERE;
                    D3 c = d3(p);
                    set4(f.rec, 0, c, (float)p[3]);
                    set4(f.rec, 2, D3{-1.0 / p[4], 0, 0}, 0.0f);
                    D3 rr{p[3], p[3], p[3]};
                    box_of_points({c - rr, c + rr}, 0.0, f.box);
                } else {
                    f.type = lum::PT_FOG_BOX;
                    D3 mn = d3(p), mx = d3(p + 3);
                    set4(f.rec, 0, mn, 0.0f);
                    set4(f.rec, 1, mx, 0.0f);
                    set4(f.rec, 2, D3{-1.0 / p[6], 0, 0}, 0.0f);
                    box_of_points({mn, mx}, 1e-4, f.box);
                }
                F.prims.push_back(f);
                break;
            }
            default:
                return fail(LUM_ERR_INVALID_ARGUMENT, "object %u: unknown kind %d", i, o.kind);
        }
        // a transform can take finite parameters out of the f32 range
        for (size_t k = first_prim; k < F.prims.size(); ++k)
            if (!box_finite(F.prims[k].box))
                return fail(LUM_ERR_INVALID_ARGUMENT, "object %u: geometry outside the f32 range", i);
        if (o.kind == LUM_OBJ_PLANE) {
            const lum::PlaneDev& pl = F.planes.back();
            for (int k = 0; k < 3; ++k)
                if (!std::isfinite(pl.p[k]) || !std::isfinite(pl.n[k]))
                    return fail(LUM_ERR_INVALID_ARGUMENT, "object %u: geometry outside the f32 range", i);
        }
    }
    for (uint32_t mi = 0; mi < d.n_meshes; ++mi) {
        const lum_mesh& m = d.meshes[mi];
        if (!m.positions || !m.indices) return fail(LUM_ERR_INVALID_ARGUMENT, "mesh %u: null arrays", mi);
        for (size_t k = 0; k < 3 * (size_t)m.n_vertices; ++k)
            if (!finite32(m.positions[k]) || (m.normals && !finite32(m.normals[k])))
                return fail(LUM_ERR_INVALID_ARGUMENT, "mesh %u vertex %zu: position or normal is not finite", mi, k / 3);
        for (uint32_t t = 0; t < m.n_triangles; ++t) {
            const uint32_t* ix = m.indices + 3 * (size_t)t;
            if (ix[0] >= m.n_vertices || ix[1] >= m.n_vertices || ix[2] >= m.n_vertices)
                return fail(LUM_ERR_INVALID_ARGUMENT, "mesh %u triangle %u: vertex index out of range", mi, t);
            int mat = m.tri_material ? m.tri_material[t] : m.material;
            if (mat < 0 || (uint32_t)mat >= d.n_materials)
                return fail(LUM_ERR_INVALID_ARGUMENT, "mesh %u triangle %u: material %d out of range", mi, t, mat);
            PrimH tr{};
            tr.type = lum::PT_TRIANGLE;
            tr.material = mat;
            tr.orig = id++;
            D3 v0 = d3(m.positions + 3 * (size_t)ix[0]), v1 = d3(m.positions + 3 * (size_t)ix[1]),
               v2 = d3(m.positions + 3 * (size_t)ix[2]);
            D3 e1 = v1 - v0, e2 = v2 - v0;
            set4(tr.rec, 0, v0, 0.0f);
            set4(tr.rec, 1, e1, 0.0f);
            set4(tr.rec, 2, e2, 0.0f);
            D3 ng = cross(e1, e2);
            ng = length(ng) > 0 ? unit(ng) : D3{0, 0, 0};
            int32_t si = -1;
            if (m.normals) {
                si = (int32_t)(F.smooth.size() / 9);
                for (int k = 0; k < 3; ++k)
                    for (int c = 0; c < 3; ++c) F.smooth.push_back((float)m.normals[3 * (size_t)ix[k] + c]);
            }
            float sf;
            std::memcpy(&sf, &si, 4);
            set4(tr.rec, 3, ng, sf);
            box_of_points({v0, v1, v2}, 0.0, tr.box);
            F.prims.push_back(tr);
        }
    }
    return LUM_OK;
}

lum::MatDev make_mat(const lum_material& m) {
    lum::MatDev o{};
    for (int k = 0; k < 3; ++k) {
        o.color[k] = (float)m.color[k];
        o.color2[k] = (float)m.color2[k];
        o.tint[k] = (float)m.tint[k];
    }
    o.kind = m.kind;
    o.tex = m.texture;
    o.tex_scale = (float)(std::fabs(m.tex_scale) < 1e-10 ? 1.0 : m.tex_scale);  // texture.rs:32-35
    o.fuzz = (float)std::fmin(m.fuzz, 1.0);                                     // material.rs:81-86
    o.ior = (float)m.ior;
    o.roughness = (float)m.roughness;
    o.metallic = (float)m.metallic;
    if (m.kind == LUM_MAT_MICROFACET) {                                         // material.rs:255-261
        o.roughness = (float)std::min(std::max(m.roughness, 0.01), 1.0);
        o.metallic = (float)std::min(std::max(m.metallic, 0.0), 1.0);
    }
    o.intensity = (float)m.intensity;
    o.dispersion = (float)m.dispersion;
    o.tint_white = (m.tint[0] == 1.0 && m.tint[1] == 1.0 && m.tint[2] == 1.0) ? 1 : 0;
    o.specular = m.kind == LUM_MAT_METAL || m.kind == LUM_MAT_DIELECTRIC ||
                 (m.kind == LUM_MAT_MICROFACET && o.metallic > 0.9f && o.roughness < 0.1f);
    // is_specular compares the clamped f64 values (material.rs:323-326)
    if (m.kind == LUM_MAT_MICROFACET) {
        double r = std::min(std::max(m.roughness, 0.01), 1.0), mt = std::min(std::max(m.metallic, 0.0), 1.0);
        o.specular = mt > 0.9 && r < 0.1;
    }
    // the other materials: their constructors' clamps (material.rs:396-865)
    auto clamp = [](double x, double lo, double hi) { return std::min(std::max(x, lo), hi); };
    const double* e = m.extra;
    switch (m.kind) {
        case LUM_MAT_BLEND:                                                     // :402-406
            o.extra[0] = (float)clamp(e[0], 0.0, 1.0);
            o.sub[0] = m.sub[0];
            o.sub[1] = m.sub[1];
            break;
        case LUM_MAT_TRANSPARENT: o.specular = 1; break;                        // :437-439
        case LUM_MAT_IRIDESCENT:                                                // :459-466
            o.extra[0] = (float)std::max(e[0], 100.0);
            o.ior = (float)std::max(m.ior, 1.0);
            o.roughness = (float)clamp(m.roughness, 0.0, 1.0);
            o.specular = 1;
            break;
        case LUM_MAT_TOON:                                                      // :538-545 (bands: u32)
            o.extra[0] = (float)std::max(std::floor(clamp(e[0], 0.0, 4294967295.0)), 2.0);
            o.extra[1] = (float)std::max(e[1], 0.0);
            break;
        case LUM_MAT_ANISOTROPIC:                                               // :592-599 (axis: usize)
            o.extra[0] = (float)clamp(e[0], 0.001, 1.0);
            o.extra[1] = (float)clamp(e[1], 0.001, 1.0);
            o.extra[2] = (float)std::min(std::floor(std::max(e[2], 0.0)), 2.0);
            o.specular = 1;
            break;
        case LUM_MAT_CLEARCOAT:                                                 // :655-661
            o.extra[0] = (float)clamp(e[0], 0.0, 1.0);
            o.ior = (float)std::max(m.ior, 1.0);
            break;
        case LUM_MAT_VELVET: o.extra[0] = (float)clamp(e[0], 0.0, 2.0); break;  // :718-720
        case LUM_MAT_TRANSLUCENT:                                               // :760-766
            o.extra[0] = (float)clamp(e[0], 0.0, 1.0);
            o.extra[1] = (float)clamp(e[1], 0.0, 1.0);
            break;
        case LUM_MAT_SUBSURFACE: o.extra[0] = (float)std::max(e[0], 0.001); break;   // :812-818
        default: break;
    }
    return o;
}

// Blend trees: children in range, nesting at most kMaxBlendDepth levels (which also rules out
// cycles); each Blend's emissive leaves with their weights go to `table` (Blend::emitted,
// material.rs:417-420, flattened).
lum_status check_blends(const lum_scene_desc& d, std::vector<lum::MatDev>& mats, std::vector<lum::BlendEmit>& table) {
    const int n = (int)d.n_materials;
    std::function<int(int, int, double, std::vector<lum::BlendEmit>&)> walk =
        [&](int i, int level, double w, std::vector<lum::BlendEmit>& out) -> int {
        const lum_material& m = d.materials[i];
        if (m.kind != LUM_MAT_BLEND) {
            if (m.kind == LUM_MAT_EMISSIVE) out.push_back({i, (float)w});
            return 0;
        }
        if (level > lum::kMaxBlendDepth) return -1;
        const double r = std::min(std::max(m.extra[0], 0.0), 1.0);
        for (int k = 0; k < 2; ++k) {
            if (m.sub[k] < 0 || m.sub[k] >= n) return -2;
            int c = walk(m.sub[k], level + 1, w * (k == 0 ? r : 1.0 - r), out);
            if (c < 0) return c;
        }
        return 0;
    };
    for (int i = 0; i < n; ++i) {
        if (d.materials[i].kind != LUM_MAT_BLEND) continue;
        std::vector<lum::BlendEmit> leaves;
        int r = walk(i, 1, 1.0, leaves);
        if (r == -2) return fail(LUM_ERR_INVALID_ARGUMENT, "material %d: blend child index out of range", i);
        if (r < 0) return fail(LUM_ERR_UNSUPPORTED, "material %d: blends nest more than %d deep", i, lum::kMaxBlendDepth);
        mats[i].n_emit = (int32_t)leaves.size();
        mats[i].emit_first = (int32_t)table.size();
        table.insert(table.end(), leaves.begin(), leaves.end());
    }
    return LUM_OK;
}

lum::CameraDev make_camera(const lum_camera& c) {                      // camera.rs:48-76
    double theta = c.vfov_degrees * (3.14159265358979323846 / 180.0);
    double h = std::tan(theta / 2.0);
    double vh = 2.0 * h, vw = c.aspect_ratio * vh;
    D3 w = unit(d3(c.look_from) - d3(c.look_at));
    D3 u = unit(cross(d3(c.vup), w));
    D3 v = cross(w, u);
    D3 hor = u * (vw * c.focus_dist), ver = v * (vh * c.focus_dist);
    D3 org = d3(c.look_from);
    D3 llc = org - hor * 0.5 - ver * 0.5 - w * c.focus_dist;
    lum::CameraDev o{};
    auto put = [](float* dst, D3 s) { dst[0] = (float)s.x; dst[1] = (float)s.y; dst[2] = (float)s.z; };
    put(o.origin, org);
    put(o.llc, llc);
    put(o.hor, hor);
    put(o.ver, ver);
    put(o.u, u);
    put(o.v, v);
    o.lens_radius = (float)(c.aperture / 2.0);
    put(o.fwd, w * -1.0);                                              // camera.rs:72-74
    o.panorama = c.panorama ? 1 : 0;
    return o;
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace

// ----------------------------------------------------------------------------- scene handle
struct lum_scene {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    void* d_buf = nullptr;
    size_t d_bytes = 0;
    lum::WorkCounters* d_work = nullptr;
    float* d_out = nullptr;
    size_t d_out_cap = 0;
    void* d_rays = nullptr;
    size_t d_rays_cap = 0;
    void* d_ldr = nullptr;      // RGBA8 image of lum_render_ldr
    size_t d_ldr_cap = 0;
    void* d_tone = nullptr;     // tone-map reduction scratch
    size_t d_tone_cap = 0;
    void* d_part = nullptr;     // sums of the split tiles of a render's task plan
    size_t d_part_cap = 0;
    void* d_env = nullptr;      // environment map (LUM_BG_ENVMAP)
    void* d_aov = nullptr;      // AOV outputs of lum_render_aov
    size_t d_aov_cap = 0;
    lum::SceneDev dev{};
    uint32_t n_prims = 0, n_nodes = 0, n_lights = 0, bvh_depth = 0;
    int max_mat_kind = 0;
    std::mutex mu;
};

namespace {

// Device memory of the scenes comes from one stream-ordered pool per device (cudaMemPool) that
// keeps up to kPoolKeepBytes of freed memory for reuse, so creating and destroying scenes and
// growing their render buffers does not go to the driver's allocator every time: on B200,
// cudaMalloc and cudaFree of a 1080p frame buffer took 0.35 and 0.7 ms, and cudaFree
// synchronises the device.
constexpr int kPoolDevices = 64;
constexpr uint64_t kPoolKeepBytes = 4ull << 30;

lum_status scene_pool(int dev, cudaMemPool_t* out) {
    static std::mutex mu;
    static cudaMemPool_t pools[kPoolDevices] = {};
    if (dev < 0 || dev >= kPoolDevices) return fail(LUM_ERR_TOO_LARGE, "device ordinal above 63");
    std::lock_guard<std::mutex> lk(mu);
    if (!pools[dev]) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        CU(cudaMemPoolCreate(&pools[dev], &props), "cudaMemPoolCreate");
        uint64_t keep = kPoolKeepBytes;
        CU(cudaMemPoolSetAttribute(pools[dev], cudaMemPoolAttrReleaseThreshold, &keep), "cudaMemPoolSetAttribute");
    }
    *out = pools[dev];
    return LUM_OK;
}

// Pool allocation ordered on the scene's stream; `sync` waits for it, so that the memory can be
// used from any stream.
lum_status pool_alloc(lum_scene* s, void** ptr, size_t bytes, bool sync = true) {
    cudaMemPool_t pool = nullptr;
    lum_status st = scene_pool(s->device, &pool);
    if (st != LUM_OK) return st;
    CU(cudaMallocFromPoolAsync(ptr, bytes, pool, s->stream), "cudaMallocFromPoolAsync");
    if (sync) CU(cudaStreamSynchronize(s->stream), "cudaStreamSynchronize");
    return LUM_OK;
}

// Grows a scene buffer.  The old buffer may still be read by work the caller enqueued on its own
// streams, so the device is synchronised before it goes back to the pool (as cudaFree would).
lum_status ensure(lum_scene* s, void** ptr, size_t* cap, size_t bytes) {
    if (*cap >= bytes) return LUM_OK;
    if (*ptr) {
        CU(cudaDeviceSynchronize(), "cudaDeviceSynchronize");
        CU(cudaFreeAsync(*ptr, s->stream), "cudaFreeAsync");
    }
    *ptr = nullptr;
    *cap = 0;
    lum_status st = pool_alloc(s, ptr, bytes);
    if (st != LUM_OK) return st;
    *cap = bytes;
    return LUM_OK;
}

// Readback of a device buffer into pageable host memory through two pinned staging chunks: the
// copy engine fills one chunk while host threads copy the other into place.  A direct
// cudaMemcpy into pageable memory took 1.4-6.3 ms for a 25 MB frame on the B200 box, a copy into
// pinned memory 0.46 ms.  The staging buffers are per device and shared; a readback that finds
// them busy (another thread's) copies directly.
constexpr size_t kStageChunk = 4u << 20;

struct Staging {
    std::mutex mu;
    unsigned char* buf[2] = {nullptr, nullptr};
    cudaEvent_t ev[2] = {nullptr, nullptr};
};

Staging* staging(int dev) {
    static Staging st[kPoolDevices];
    return dev >= 0 && dev < kPoolDevices ? &st[dev] : nullptr;
}

void host_copy(unsigned char* dst, const unsigned char* src, size_t n) {
    constexpr size_t kSlice = 256u << 10;
    const long slices = (long)((n + kSlice - 1) / kSlice);
    const int nt = std::max(1, std::min({8, omp_get_num_procs(), (int)slices}));
#pragma omp parallel for num_threads(nt) schedule(static)
    for (long k = 0; k < slices; ++k) {
        const size_t o = (size_t)k * kSlice;
        std::memcpy(dst + o, src + o, std::min(kSlice, n - o));
    }
}

lum_status readback(lum_scene* s, void* dst, const void* src, size_t bytes, cudaStream_t stream) {
    Staging* sg = staging(s->device);
    std::unique_lock<std::mutex> lk;
    if (sg) lk = std::unique_lock<std::mutex>(sg->mu, std::try_to_lock);
    if (bytes < 2 * kStageChunk || !sg || !lk.owns_lock()) {
        CU(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, stream), "cudaMemcpyAsync D2H");
        CU(cudaStreamSynchronize(stream), "D2H");
        return LUM_OK;
    }
    for (int b = 0; b < 2; ++b) {
        if (!sg->buf[b]) CU(cudaHostAlloc((void**)&sg->buf[b], kStageChunk, cudaHostAllocPortable), "cudaHostAlloc");
        if (!sg->ev[b]) CU(cudaEventCreateWithFlags(&sg->ev[b], cudaEventDisableTiming), "cudaEventCreate");
    }
    const size_t n_chunks = (bytes + kStageChunk - 1) / kStageChunk;
    auto* d = static_cast<unsigned char*>(dst);
    const auto* g = static_cast<const unsigned char*>(src);
    for (size_t i = 0; i <= n_chunks; ++i) {
        if (i < n_chunks) {   // chunk i into buffer i % 2, whose previous chunk the host has copied out
            const size_t o = i * kStageChunk, n = std::min(kStageChunk, bytes - o);
            CU(cudaMemcpyAsync(sg->buf[i & 1], g + o, n, cudaMemcpyDeviceToHost, stream), "cudaMemcpyAsync D2H");
            CU(cudaEventRecord(sg->ev[i & 1], stream), "cudaEventRecord");
        }
        if (i > 0) {          // chunk i - 1 to its place
            const size_t j = i - 1, o = j * kStageChunk, n = std::min(kStageChunk, bytes - o);
            CU(cudaEventSynchronize(sg->ev[j & 1]), "D2H");
            host_copy(d + o, sg->buf[j & 1], n);
        }
    }
    return LUM_OK;
}

lum_status make_render_dev(const lum_scene* s, const lum_render_params& p, lum::RenderDev& R) {
    R = lum::RenderDev{};
    R.full_w = std::max<uint32_t>(p.width, 1);
    R.full_h = std::max<uint32_t>(p.height, 1);
    if (p.has_crop) {                                                   // render.rs:1575-1583
        R.crop_x = std::min(p.crop[0], R.full_w);
        R.crop_y = std::min(p.crop[1], R.full_h);
        R.w = std::min(p.crop[2], R.full_w);
        R.h = std::min(p.crop[3], R.full_h);
    } else {
        R.w = R.full_w;
        R.h = R.full_h;
    }
    if ((uint64_t)R.full_w * R.full_h > 0xFFFFFFFFull) return fail(LUM_ERR_TOO_LARGE, "image has more than 2^32 pixels");
    R.sqrt_spp = (uint32_t)std::ceil(std::sqrt((double)p.samples_per_pixel));   // render.rs:1589
    uint32_t total = R.sqrt_spp * R.sqrt_spp;
    R.s_begin = std::min(p.sample_begin, total);
    R.s_end = p.sample_count ? std::min(total, R.s_begin + p.sample_count) : total;
    R.max_depth = p.max_depth;
    R.key0 = (uint32_t)p.seed;
    R.key1 = (uint32_t)(p.seed >> 32);
    R.background = p.background;
    R.pixel_filter = p.pixel_filter;
    for (int k = 0; k < 3; ++k) {
        R.bg_color[k] = (float)p.bg_color[k];
        R.bg_color2[k] = (float)p.bg_color2[k];
        R.bg_dir[k] = (float)p.bg_dir[k];
    }
    R.bg_intensity = (float)p.bg_intensity;
    R.exposure = (float)p.exposure;
    R.ext = (s->max_mat_kind > LUM_MAT_ISOTROPIC || p.background >= LUM_BG_STARFIELD) ? 1u : 0u;
    R.star_density = (float)p.bg_star_density;
    R.star_brightness = (float)p.bg_star_brightness;
    if (p.background == LUM_BG_ENVMAP && !s->dev.env)
        return fail(LUM_ERR_INVALID_ARGUMENT, "LUM_BG_ENVMAP without an environment map (lum_scene_set_envmap)");
    R.tiles_x = (R.w + 7) / 8;
    uint64_t tasks = (uint64_t)R.tiles_x * ((R.h + 3) / 4);
    if (tasks > 0x7FFFFFFFull) return fail(LUM_ERR_TOO_LARGE, "image too large");
    R.n_tasks = (uint32_t)tasks;
    (void)s;
    return LUM_OK;
}

// Adaptive sampling or a time limit: the sample loop's in-loop branches (render.rs:1592-1678).
bool sampled(const lum_render_params& p) { return p.adaptive != 0 || p.time_limit > 0.0; }

lum::SamplingDev sampling_of(const lum_render_params& p, const lum::RenderDev& R) {
    lum::SamplingDev A{};
    A.adaptive = p.adaptive ? 1u : 0u;
    A.min_samples = std::max<uint32_t>(R.sqrt_spp * R.sqrt_spp / 4, 16);   // render.rs:1592
    A.threshold = p.adaptive_threshold;
    if (p.time_limit > 0.0)
        A.limit_ns = (unsigned long long)std::max(1.0, std::min(p.time_limit * 1e9, 1.8e19));
    return A;
}

lum_status check_params(const lum_render_params* p) {
    if (!p) return fail(LUM_ERR_INVALID_ARGUMENT, "params is null");
    if (sampled(*p)) {
        const uint32_t sq = (uint32_t)std::ceil(std::sqrt((double)p->samples_per_pixel));
        if (p->sample_begin != 0 || (p->sample_count != 0 && p->sample_count < sq * sq))
            return fail(LUM_ERR_UNSUPPORTED, "adaptive sampling and the time limit need all strata "
                                             "(sample_begin 0, sample_count 0)");
    }
    if (p->background < LUM_BG_SKY || p->background > LUM_BG_ENVMAP)
        return fail(LUM_ERR_INVALID_ARGUMENT, "unknown background %d", p->background);
    if (p->pixel_filter < LUM_FILTER_BOX || p->pixel_filter > LUM_FILTER_MITCHELL)
        return fail(LUM_ERR_INVALID_ARGUMENT, "unknown pixel filter %d", p->pixel_filter);
    return LUM_OK;
}

// sync = false: enqueue only (no counter readback, no synchronisation, no error flags).
lum_status run_render(lum_scene* s, const lum_render_params* params, float* d_out, cudaStream_t stream,
                      lum_stats* stats, bool sync = true) {
    lum::RenderDev R;
    lum_status st = make_render_dev(s, *params, R);
    if (st != LUM_OK) return st;
    auto t0 = std::chrono::steady_clock::now();
    CU(cudaMemsetAsync(s->d_work, 0, sizeof(lum::WorkCounters), stream), "cudaMemsetAsync");
    CU(cudaEventRecord(s->ev0, stream), "cudaEventRecord");
    const bool smp = sampled(*params);
    if (smp && R.n_tasks > 0) {
        // adaptive sampling / time limit: one task per tile, all strata, no stratum groups
        CU(lum::launch_render_sampled(s->dev, R, sampling_of(*params, R), d_out, s->d_work, stream), "render launch");
    } else if (R.n_tasks > 0 && R.s_end > R.s_begin) {
        // frames with fewer tiles than resident warps split their strata into groups
        const lum::RenderGroups grp = lum::render_groups(R);
        const size_t scratch = lum::render_scratch_bytes(R, grp);
        if (scratch > 0) {
            st = ensure(s, &s->d_part, &s->d_part_cap, scratch);
            if (st != LUM_OK) return st;
        }
        CU(lum::launch_render_grouped(s->dev, R, d_out, s->d_work, stream, scratch ? s->d_part : nullptr, scratch,
                                      grp), "render launch");
    } else if (R.w > 0 && R.h > 0) {
        CU(cudaMemsetAsync(d_out, 0, sizeof(float) * 3 * (size_t)R.w * R.h, stream), "cudaMemsetAsync");
    }
    CU(cudaEventRecord(s->ev1, stream), "cudaEventRecord");
    if (!sync) return LUM_OK;
    lum::WorkCounters wc{};
    CU(cudaMemcpyAsync(&wc, s->d_work, sizeof wc, cudaMemcpyDeviceToHost, stream), "cudaMemcpyAsync");
    CU(cudaStreamSynchronize(stream), "render");
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, s->ev0, s->ev1);
    if (stats) {
        stats->paths = smp ? wc.samples : (uint64_t)R.w * R.h * (R.s_end - R.s_begin);
        stats->segments = wc.segments;
        stats->shadow_rays = wc.shadow_rays;
        stats->kernel_ms = ms;
        stats->total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        stats->error_flags = wc.error_flags;
    }
    if (wc.error_flags) return fail(LUM_ERR_KERNEL, "render kernel reported error flags 0x%x", wc.error_flags);
    return LUM_OK;
}

}  // namespace

extern "C" {

int32_t lum_abi_version(void) { return LUM_ABI_VERSION; }

const char* lum_last_error(void) { return g_error.c_str(); }

lum_status lum_scene_create(const lum_scene_desc* desc, lum_scene** out) {
    if (!desc || !out) return fail(LUM_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    if ((desc->n_objects && !desc->objects) || (desc->n_materials && !desc->materials) ||
        (desc->n_lights && !desc->lights) || (desc->n_meshes && !desc->meshes))
        return fail(LUM_ERR_INVALID_ARGUMENT, "null array with non-zero count");
    for (uint32_t i = 0; i < desc->n_materials; ++i) {
        int k = desc->materials[i].kind;
        if (k < LUM_MAT_LAMBERTIAN || k > LUM_MAT_SUBSURFACE)
            return fail(LUM_ERR_INVALID_ARGUMENT, "material %u: unknown kind %d", i, k);
        int t = desc->materials[i].texture;
        if (t != LUM_TEX_SOLID && t != LUM_TEX_CHECKER)
            return fail(LUM_ERR_INVALID_ARGUMENT, "material %u: unknown texture %d", i, t);
        const lum_material& m = desc->materials[i];
        const double scalars[] = {m.tex_scale, m.fuzz, m.ior, m.roughness, m.metallic, m.intensity, m.dispersion,
                                  m.extra[0], m.extra[1], m.extra[2], m.extra[3]};
        if (first_nonfinite(m.color, 3) >= 0 || first_nonfinite(m.color2, 3) >= 0 || first_nonfinite(m.tint, 3) >= 0 ||
            first_nonfinite(scalars, (int)(sizeof scalars / sizeof scalars[0])) >= 0)
            return fail(LUM_ERR_INVALID_ARGUMENT, "material %u: a parameter is not finite", i);
    }
    for (uint32_t i = 0; i < desc->n_lights; ++i) {
        const lum_light& l = desc->lights[i];
        int k = l.kind;
        if (k < LUM_LIGHT_SPHERE || k > LUM_LIGHT_DISK)
            return fail(LUM_ERR_INVALID_ARGUMENT, "light %u: unknown kind %d", i, k);
        if (first_nonfinite(l.p0, 3) >= 0 || first_nonfinite(l.u, 3) >= 0 || first_nonfinite(l.v, 3) >= 0 ||
            first_nonfinite(l.normal, 3) >= 0 || first_nonfinite(l.emission, 3) >= 0 || !finite32(l.radius))
            return fail(LUM_ERR_INVALID_ARGUMENT, "light %u: a parameter is not finite", i);
    }
    {
        const lum_camera& c = desc->camera;
        const double scalars[] = {c.vfov_degrees, c.aspect_ratio, c.aperture, c.focus_dist};
        if (first_nonfinite(c.look_from, 3) >= 0 || first_nonfinite(c.look_at, 3) >= 0 ||
            first_nonfinite(c.vup, 3) >= 0 || first_nonfinite(scalars, 4) >= 0)
            return fail(LUM_ERR_INVALID_ARGUMENT, "camera: a parameter is not finite");
    }
    Flat F;
    lum_status st = flatten(*desc, F);
    if (st != LUM_OK) return st;
    if (F.prims.size() >= (1u << 27)) return fail(LUM_ERR_TOO_LARGE, "too many primitives");

    std::vector<lum::BuildBox> boxes(F.prims.size());
    for (size_t i = 0; i < F.prims.size(); ++i) boxes[i] = F.prims[i].box;
    // relative test costs in the SAH: a quad test reads four 16-byte records against one to
    // three for the others; weighting quads 2 made the box-room frame 6% faster, while sphere
    // and triangle scenes measured best at the plain weight 1
    std::vector<float> weights(F.prims.size());
    for (size_t i = 0; i < F.prims.size(); ++i) weights[i] = F.prims[i].type == lum::PT_QUAD ? 2.0f : 1.0f;
    lum::BvhOptions opt;
    lum::BvhResult bvh = lum::build_bvh(boxes, opt, &weights);
    if (bvh.max_depth > (uint32_t)lum::kMaxBvhDepth)
        return fail(LUM_ERR_TOO_LARGE, "BVH depth %u exceeds the traversal stack", bvh.max_depth);

    const size_t np = F.prims.size();
    std::vector<float> prims(16 * np);
    std::vector<int32_t> meta(np), orig(np);
    for (size_t k = 0; k < np; ++k) {
        const PrimH& p = F.prims[bvh.order[k]];
        std::memcpy(&prims[16 * k], p.rec, sizeof p.rec);
        meta[k] = (p.material << 4) | p.type;
        orig[k] = p.orig;
    }
    std::vector<lum::MatDev> mats(desc->n_materials);
    for (uint32_t i = 0; i < desc->n_materials; ++i) mats[i] = make_mat(desc->materials[i]);
    std::vector<lum::BlendEmit> blend_emit;
    st = check_blends(*desc, mats, blend_emit);
    if (st != LUM_OK) return st;
    std::vector<lum::LightDev> lights(desc->n_lights);
    for (uint32_t i = 0; i < desc->n_lights; ++i) {
        const lum_light& l = desc->lights[i];
        lum::LightDev& o = lights[i];
        o = lum::LightDev{};
        o.kind = l.kind;
        for (int k = 0; k < 3; ++k) {
            o.p0[k] = (float)l.p0[k];
            o.u[k] = (float)l.u[k];
            o.v[k] = (float)l.v[k];
            o.n[k] = (float)l.normal[k];
            o.e[k] = (float)l.emission[k];
        }
        o.radius = (float)l.radius;
        if (l.kind == LUM_LIGHT_RECT) o.area = (float)length(cross(d3(l.u), d3(l.v)));   // render.rs:1419
        if (l.kind == LUM_LIGHT_DISK) o.area = (float)(3.14159265358979323846 * l.radius * l.radius);
    }

    auto* s = new lum_scene();
    auto cleanup = [&](lum_status code) {
        lum_scene_destroy(s);
        return code;
    };
    cudaError_t ce = cudaGetDevice(&s->device);
    if (ce != cudaSuccess) return cleanup(cuda_fail(ce, "cudaGetDevice"));
    if ((ce = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking)) != cudaSuccess)
        return cleanup(cuda_fail(ce, "cudaStreamCreate"));
    if ((ce = cudaEventCreate(&s->ev0)) != cudaSuccess || (ce = cudaEventCreate(&s->ev1)) != cudaSuccess)
        return cleanup(cuda_fail(ce, "cudaEventCreate"));

    size_t off_nodes = 0;
    // records 0-2 (the hit tests' 48 bytes) apart from record 3: the traversal's working set
    // of a large triangle mesh shrinks by a quarter
    std::vector<float> prims012(12 * np), prims3(4 * np);
    for (size_t k = 0; k < np; ++k) {
        std::memcpy(&prims012[12 * k], &prims[16 * k], 12 * sizeof(float));
        std::memcpy(&prims3[4 * k], &prims[16 * k + 12], 4 * sizeof(float));
    }
    size_t off_prims = align256(off_nodes + bvh.nodes.size() * sizeof(lum::NodeDev));
    size_t off_prims3 = align256(off_prims + prims012.size() * sizeof(float));
    size_t off_meta = align256(off_prims3 + prims3.size() * sizeof(float));
    size_t off_orig = align256(off_meta + meta.size() * 4);
    size_t off_smooth = align256(off_orig + orig.size() * 4);
    size_t off_mats = align256(off_smooth + F.smooth.size() * 4);
    size_t off_lights = align256(off_mats + mats.size() * sizeof(lum::MatDev));
    size_t off_planes = align256(off_lights + lights.size() * sizeof(lum::LightDev));
    size_t off_blend = align256(off_planes + F.planes.size() * sizeof(lum::PlaneDev));
    size_t total = align256(off_blend + blend_emit.size() * sizeof(lum::BlendEmit)) + 256;
    if ((st = pool_alloc(s, &s->d_buf, total, false)) != LUM_OK) return cleanup(st);
    s->d_bytes = total;
    if ((st = pool_alloc(s, (void**)&s->d_work, sizeof(lum::WorkCounters))) != LUM_OK) return cleanup(st);
    char* base = (char*)s->d_buf;
    auto up = [&](size_t off, const void* src, size_t bytes) -> cudaError_t {
        if (!bytes) return cudaSuccess;
        return cudaMemcpy(base + off, src, bytes, cudaMemcpyHostToDevice);
    };
    if ((ce = up(off_nodes, bvh.nodes.data(), bvh.nodes.size() * sizeof(lum::NodeDev))) != cudaSuccess ||
        (ce = up(off_prims, prims012.data(), prims012.size() * 4)) != cudaSuccess ||
        (ce = up(off_prims3, prims3.data(), prims3.size() * 4)) != cudaSuccess ||
        (ce = up(off_meta, meta.data(), meta.size() * 4)) != cudaSuccess ||
        (ce = up(off_orig, orig.data(), orig.size() * 4)) != cudaSuccess ||
        (ce = up(off_smooth, F.smooth.data(), F.smooth.size() * 4)) != cudaSuccess ||
        (ce = up(off_mats, mats.data(), mats.size() * sizeof(lum::MatDev))) != cudaSuccess ||
        (ce = up(off_lights, lights.data(), lights.size() * sizeof(lum::LightDev))) != cudaSuccess ||
        (ce = up(off_planes, F.planes.data(), F.planes.size() * sizeof(lum::PlaneDev))) != cudaSuccess ||
        (ce = up(off_blend, blend_emit.data(), blend_emit.size() * sizeof(lum::BlendEmit))) != cudaSuccess)
        return cleanup(cuda_fail(ce, "cudaMemcpy scene"));

    lum::SceneDev& D = s->dev;
    D.nodes = base + off_nodes;
    D.prims = base + off_prims;
    D.prims3 = base + off_prims3;
    D.meta = (const int32_t*)(base + off_meta);
    D.orig = (const int32_t*)(base + off_orig);
    D.smooth_n = (const float*)(base + off_smooth);
    D.mats = (const lum::MatDev*)(base + off_mats);
    D.lights = (const lum::LightDev*)(base + off_lights);
    D.planes = (const lum::PlaneDev*)(base + off_planes);
    D.blend_emit = (const lum::BlendEmit*)(base + off_blend);
    D.n_nodes = (int32_t)bvh.nodes.size();
    D.n_prims = (int32_t)np;
    D.n_lights = (int32_t)lights.size();
    D.n_planes = (int32_t)F.planes.size();
    D.n_mats = (int32_t)mats.size();
    // the sphere-and-basic-materials kernel class (planes are tested in the general way)
    bool sph = true;
    for (size_t k = 0; k < np && sph; ++k)   // static spheres: record 1's w (moving flag) is 0
        sph = (meta[k] & 15) == lum::PT_SPHERE && prims[16 * k + 7] == 0.0f;
    for (uint32_t i = 0; i < desc->n_materials && sph; ++i)
        sph = desc->materials[i].kind >= LUM_MAT_LAMBERTIAN && desc->materials[i].kind <= LUM_MAT_EMISSIVE;
    D.spheres_basic = sph ? 1 : 0;
    // the scene class of the general megakernel build: the primitive types and light kinds
    // present (planes are tested apart from the BVH in every class)
    {
        bool quad_only = true, mesh_only = true;
        for (size_t k = 0; k < np; ++k) {
            const int t = meta[k] & 15;
            quad_only = quad_only && t == lum::PT_QUAD;
            mesh_only = mesh_only && (t == lum::PT_TRIANGLE || t == lum::PT_DISK || t == lum::PT_FOG_SPHERE ||
                                      t == lum::PT_FOG_BOX);
        }
        for (uint32_t i = 0; i < desc->n_lights; ++i) {
            const int k = desc->lights[i].kind;
            quad_only = quad_only && k == LUM_LIGHT_RECT;
            mesh_only = mesh_only && (k == LUM_LIGHT_RECT || k == LUM_LIGHT_DISK);
        }
        D.cls = np == 0 ? 0 : quad_only ? 1 : mesh_only ? 2 : 0;   // CLS_QUAD, CLS_MESH, CLS_ALL
    }
    D.moving = 0;
    for (size_t k = 0; k < np && !D.moving; ++k)
        D.moving = (meta[k] & 15) == lum::PT_SPHERE && prims[16 * k + 7] != 0.0f ? 1 : 0;
    // a traversal holds at most one pushed entry per level above its node
    D.stack_depth = (int32_t)std::min<uint32_t>((uint32_t)lum::kStackDepth, bvh.max_depth + 1);
    // Diagnostic: LUM_STACK_BUDGET=n caps the traversal stack below what the tree needs, so the
    // overflow path (LUM_KERR_STACK_OVERFLOW, the far subtree skipped) can be exercised; the push
    // is bounds-checked against this value.
    if (const char* sb = std::getenv("LUM_STACK_BUDGET")) {
        const long b = std::strtol(sb, nullptr, 10);
        if (b >= 1 && b < D.stack_depth) D.stack_depth = (int32_t)b;
    }
    D.cam = make_camera(desc->camera);
    s->n_prims = (uint32_t)(np + F.planes.size());
    s->n_nodes = (uint32_t)bvh.nodes.size();
    s->n_lights = (uint32_t)lights.size();
    s->bvh_depth = bvh.max_depth;
    for (uint32_t i = 0; i < desc->n_materials; ++i) s->max_mat_kind = std::max(s->max_mat_kind, desc->materials[i].kind);
    // With lazy module loading the render kernels' module (and the allocation-free render's
    // fixed array in it) would load at the first render on this device; load it now, while the
    // caller evidently can still allocate.
    lum::noalloc_preload();
    *out = s;
    return LUM_OK;
}

lum_status lum_scene_destroy(lum_scene* s) {
    if (!s) return LUM_OK;
    cudaSetDevice(s->device);
    // work the caller enqueued on its own streams may still read the scene (cudaFree would wait
    // for it too); then the buffers go back to the pool in the scene stream's order
    cudaDeviceSynchronize();
    for (void* p : {s->d_buf, (void*)s->d_work, (void*)s->d_out, s->d_rays, s->d_ldr, s->d_tone, s->d_part, s->d_aov})
        if (p) cudaFreeAsync(p, s->stream);
    if (s->d_env) cudaFree(s->d_env);
    if (s->ev0) cudaEventDestroy(s->ev0);
    if (s->ev1) cudaEventDestroy(s->ev1);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
    return LUM_OK;
}

lum_status lum_scene_info(const lum_scene* s, uint32_t* n_prims, uint32_t* n_nodes, uint32_t* n_lights,
                          uint64_t* device_bytes) {
    if (!s) return fail(LUM_ERR_INVALID_ARGUMENT, "scene is null");
    if (n_prims) *n_prims = s->n_prims;
    if (n_nodes) *n_nodes = s->n_nodes;
    if (n_lights) *n_lights = s->n_lights;
    if (device_bytes) *device_bytes = s->d_bytes;
    return LUM_OK;
}

lum_status lum_render_device(lum_scene* s, const lum_render_params* params, float* d_out, void* stream,
                             lum_stats* stats) {
    if (!s || !d_out) return fail(LUM_ERR_INVALID_ARGUMENT, "null argument");
    lum_status st = check_params(params);
    if (st != LUM_OK) return st;
    std::lock_guard<std::mutex> lk(s->mu);
    CU(cudaSetDevice(s->device), "cudaSetDevice");
    cudaStream_t cs = stream ? (cudaStream_t)stream : s->stream;
    return run_render(s, params, d_out, cs, stats, stats != nullptr);
}

lum_status lum_render_sums_device(lum_scene* s, const lum_render_params* params, int64_t* d_sums, void* stream,
                                  lum_stats* stats) {
    if (!s || !d_sums) return fail(LUM_ERR_INVALID_ARGUMENT, "null argument");
    lum_status st = check_params(params);
    if (st != LUM_OK) return st;
    if (sampled(*params))
        return fail(LUM_ERR_UNSUPPORTED, "raw sums are not defined for adaptive sampling or the time limit");
    std::lock_guard<std::mutex> lk(s->mu);
    CU(cudaSetDevice(s->device), "cudaSetDevice");
    cudaStream_t cs = stream ? (cudaStream_t)stream : s->stream;
    lum::RenderDev R;
    st = make_render_dev(s, *params, R);
    if (st != LUM_OK) return st;
    auto t0 = std::chrono::steady_clock::now();
    auto* sums = reinterpret_cast<unsigned long long*>(d_sums);
    CU(cudaMemsetAsync(s->d_work, 0, sizeof(lum::WorkCounters), cs), "cudaMemsetAsync");
    CU(cudaEventRecord(s->ev0, cs), "cudaEventRecord");
    if (R.n_tasks > 0 && R.s_end > R.s_begin) {
        CU(lum::launch_render_sums(s->dev, R, sums, s->d_work, cs), "render launch");
    } else if (R.w > 0 && R.h > 0) {
        CU(cudaMemsetAsync(sums, 0, 32 * (size_t)R.w * R.h, cs), "cudaMemsetAsync");
    }
    CU(cudaEventRecord(s->ev1, cs), "cudaEventRecord");
    if (!stats) return LUM_OK;
    lum::WorkCounters wc{};
    CU(cudaMemcpyAsync(&wc, s->d_work, sizeof wc, cudaMemcpyDeviceToHost, cs), "cudaMemcpyAsync");
    CU(cudaStreamSynchronize(cs), "render");
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, s->ev0, s->ev1);
    stats->paths = (uint64_t)R.w * R.h * (R.s_end - R.s_begin);
    stats->segments = wc.segments;
    stats->shadow_rays = wc.shadow_rays;
    stats->kernel_ms = ms;
    stats->total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    stats->error_flags = wc.error_flags;
    if (wc.error_flags) return fail(LUM_ERR_KERNEL, "render kernel reported error flags 0x%x", wc.error_flags);
    return LUM_OK;
}

lum_status lum_sums_finalize_device(const int64_t* d_sums, uint32_t width, uint32_t height, double exposure,
                                    float* d_rgb, void* stream) {
    if ((!d_sums || !d_rgb) && (uint64_t)width * height > 0) return fail(LUM_ERR_INVALID_ARGUMENT, "null argument");
    if (!std::isfinite(exposure)) return fail(LUM_ERR_INVALID_ARGUMENT, "exposure is not finite");
    CU(lum::launch_fixed_finalize(reinterpret_cast<const unsigned long long*>(d_sums), (size_t)width * height,
                                  (float)exposure, d_rgb, (cudaStream_t)stream),
       "finalize launch");
    return LUM_OK;
}

lum_status lum_scene_set_envmap(lum_scene* s, const float* rgb, uint32_t width, uint32_t height) {
    if (!s) return fail(LUM_ERR_INVALID_ARGUMENT, "scene is null");
    if (rgb && (width == 0 || height == 0)) return fail(LUM_ERR_INVALID_ARGUMENT, "empty environment map");
    if (rgb && (uint64_t)width * height > (1ull << 31)) return fail(LUM_ERR_TOO_LARGE, "environment map too large");
    std::lock_guard<std::mutex> lk(s->mu);
    CU(cudaSetDevice(s->device), "cudaSetDevice");
    CU(cudaStreamSynchronize(s->stream), "cudaStreamSynchronize");
    if (s->d_env) cudaFree(s->d_env);
    s->d_env = nullptr;
    s->dev.env = nullptr;
    s->dev.env_w = s->dev.env_h = 0;
    if (!rgb) return LUM_OK;
    const size_t bytes = sizeof(float) * 3 * (size_t)width * height;
    CU(cudaMalloc(&s->d_env, bytes), "cudaMalloc");
    CU(cudaMemcpy(s->d_env, rgb, bytes, cudaMemcpyHostToDevice), "cudaMemcpy H2D");
    s->dev.env = (const float*)s->d_env;
    s->dev.env_w = width;
    s->dev.env_h = height;
    return LUM_OK;
}

lum_status lum_render_aov(lum_scene* s, const lum_render_params* params, float* depth, uint8_t* normals,
                          uint8_t* albedo) {
    if (!s) return fail(LUM_ERR_INVALID_ARGUMENT, "null argument");
    lum_status st = check_params(params);
    if (st != LUM_OK) return st;
    std::lock_guard<std::mutex> lk(s->mu);
    CU(cudaSetDevice(s->device), "cudaSetDevice");
    lum::RenderDev R;
    st = make_render_dev(s, *params, R);
    if (st != LUM_OK) return st;
    const size_t px = (size_t)R.w * R.h;
    if (px == 0 || (!depth && !normals && !albedo)) return LUM_OK;
    st = ensure(s, &s->d_aov, &s->d_aov_cap, 10 * px);
    if (st != LUM_OK) return st;
    float* d_depth = (float*)s->d_aov;
    uint8_t* d_norm = (uint8_t*)s->d_aov + 4 * px;
    uint8_t* d_alb = d_norm + 3 * px;
    CU(cudaMemsetAsync(s->d_work, 0, sizeof(lum::WorkCounters), s->stream), "cudaMemsetAsync");
    CU(lum::launch_aov(s->dev, R, depth ? d_depth : nullptr, normals ? d_norm : nullptr, albedo ? d_alb : nullptr,
                       s->d_work, s->stream), "aov launch");
    if (depth) CU(cudaMemcpyAsync(depth, d_depth, 4 * px, cudaMemcpyDeviceToHost, s->stream), "D2H");
    if (normals) CU(cudaMemcpyAsync(normals, d_norm, 3 * px, cudaMemcpyDeviceToHost, s->stream), "D2H");
    if (albedo) CU(cudaMemcpyAsync(albedo, d_alb, 3 * px, cudaMemcpyDeviceToHost, s->stream), "D2H");
    lum::WorkCounters wc{};
    CU(cudaMemcpyAsync(&wc, s->d_work, sizeof wc, cudaMemcpyDeviceToHost, s->stream), "D2H");
    CU(cudaStreamSynchronize(s->stream), "aov");
    if (wc.error_flags) return fail(LUM_ERR_KERNEL, "AOV kernel reported error flags 0x%x", wc.error_flags);
    return LUM_OK;
}

lum_status lum_render(lum_scene* s, const lum_render_params* params, float* out_rgb, lum_stats* stats) {
    if (!s || !out_rgb) return fail(LUM_ERR_INVALID_ARGUMENT, "null argument");
    lum_status st = check_params(params);
    if (st != LUM_OK) return st;
    std::lock_guard<std::mutex> lk(s->mu);
    CU(cudaSetDevice(s->device), "cudaSetDevice");
    auto t0 = std::chrono::steady_clock::now();
    lum::RenderDev R;
    st = make_render_dev(s, *params, R);
    if (st != LUM_OK) return st;
    size_t bytes = sizeof(float) * 3 * (size_t)R.w * R.h;
    if (bytes == 0) {
        if (stats) std::memset(stats, 0, sizeof *stats);
        return LUM_OK;
    }
    st = ensure(s, (void**)&s->d_out, &s->d_out_cap, bytes);
    if (st != LUM_OK) return st;
    lum_status rs = run_render(s, params, s->d_out, s->stream, stats);
    if (rs != LUM_OK && rs != LUM_ERR_KERNEL) return rs;
    st = readback(s, out_rgb, s->d_out, bytes, s->stream);
    if (st != LUM_OK) return st;
    if (stats) stats->total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return rs;
}

lum_status lum_render_ldr(lum_scene* s, const lum_render_params* params, const lum_tonemap_params* tm,
                          uint8_t* out_rgba, lum_stats* stats) {
    if (!s || !out_rgba || !tm) return fail(LUM_ERR_INVALID_ARGUMENT, "null argument");
    lum_status st = check_params(params);
    if (st != LUM_OK) return st;
    if (tm->tone_map < LUM_TONEMAP_ACES || tm->tone_map > LUM_TONEMAP_NONE)
        return fail(LUM_ERR_INVALID_ARGUMENT, "unknown tone_map");
    std::lock_guard<std::mutex> lk(s->mu);
    CU(cudaSetDevice(s->device), "cudaSetDevice");
    auto t0 = std::chrono::steady_clock::now();
    lum::RenderDev R;
    st = make_render_dev(s, *params, R);
    if (st != LUM_OK) return st;
    const size_t px = (size_t)R.w * R.h;
    if (px == 0) {
        if (stats) std::memset(stats, 0, sizeof *stats);
        return LUM_OK;
    }
    st = ensure(s, (void**)&s->d_out, &s->d_out_cap, sizeof(float) * 3 * px);
    if (st == LUM_OK) st = ensure(s, &s->d_ldr, &s->d_ldr_cap, 4 * px);
    if (st == LUM_OK) st = ensure(s, &s->d_tone, &s->d_tone_cap, LUM_TONEMAP_SCRATCH_BYTES);
    if (st != LUM_OK) return st;
    // the HDR stage at exposure 1: the chain applies the exposure (src/render.rs:2594-2608)
    lum_render_params hp = *params;
    hp.exposure = 1.0;
    lum_status rs = run_render(s, &hp, s->d_out, s->stream, stats);
    if (rs != LUM_OK && rs != LUM_ERR_KERNEL) return rs;
    CU(lum::launch_tonemap(s->d_out, R.w, R.h, *tm, params->exposure, (double*)s->d_tone, (uint8_t*)s->d_ldr,
                           s->stream),
       "tone map launch");
    st = readback(s, out_rgba, s->d_ldr, 4 * px, s->stream);
    if (st != LUM_OK) return st;
    if (stats) stats->total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return rs;
}

lum_status lum_count_tests(lum_scene* s, const lum_render_params* params, lum_test_counts* out) {
    if (!s || !out) return fail(LUM_ERR_INVALID_ARGUMENT, "null argument");
    lum_status st = check_params(params);
    if (st != LUM_OK) return st;
    std::lock_guard<std::mutex> lk(s->mu);
    CU(cudaSetDevice(s->device), "cudaSetDevice");
    lum::RenderDev R;
    st = make_render_dev(s, *params, R);
    if (st != LUM_OK) return st;
    std::memset(out, 0, sizeof *out);
    size_t bytes = sizeof(float) * 3 * (size_t)R.w * R.h;
    if (bytes == 0 || R.s_end <= R.s_begin) return LUM_OK;
    st = ensure(s, (void**)&s->d_out, &s->d_out_cap, bytes);
    if (st != LUM_OK) return st;
    CU(cudaMemsetAsync(s->d_work, 0, sizeof(lum::WorkCounters), s->stream), "cudaMemsetAsync");
    CU(lum::launch_render_counted(s->dev, R, s->d_out, s->d_work, s->stream), "counted render launch");
    lum::WorkCounters wc{};
    CU(cudaMemcpyAsync(&wc, s->d_work, sizeof wc, cudaMemcpyDeviceToHost, s->stream), "cudaMemcpyAsync");
    CU(cudaStreamSynchronize(s->stream), "counted render");
    out->node_visits = wc.tally.node;
    out->sphere_tests = wc.tally.prim[lum::PT_SPHERE];
    out->quad_tests = wc.tally.prim[lum::PT_QUAD];
    out->triangle_tests = wc.tally.prim[lum::PT_TRIANGLE];
    out->disk_tests = wc.tally.prim[lum::PT_DISK];
    out->fog_tests = wc.tally.prim[lum::PT_FOG_SPHERE] + wc.tally.prim[lum::PT_FOG_BOX];
    out->plane_tests = wc.tally.plane;
    out->segments = wc.segments;
    out->shadow_rays = wc.shadow_rays;
    out->paths = (uint64_t)R.w * R.h * (R.s_end - R.s_begin);
    if (wc.error_flags) return fail(LUM_ERR_KERNEL, "counted render reported error flags 0x%x", wc.error_flags);
    return LUM_OK;
}

lum_status lum_intersect(lum_scene* s, const lum_ray* rays, uint32_t n, lum_hit* hits) {
    if (!s || (n && (!rays || !hits))) return fail(LUM_ERR_INVALID_ARGUMENT, "null argument");
    if (n == 0) return LUM_OK;
    std::lock_guard<std::mutex> lk(s->mu);
    CU(cudaSetDevice(s->device), "cudaSetDevice");
    size_t rb = align256(sizeof(lum_ray) * (size_t)n), hb = sizeof(lum_hit) * (size_t)n;
    lum_status st = ensure(s, &s->d_rays, &s->d_rays_cap, rb + hb);
    if (st != LUM_OK) return st;
    lum_ray* d_r = (lum_ray*)s->d_rays;
    lum_hit* d_h = (lum_hit*)((char*)s->d_rays + rb);
    CU(cudaMemcpyAsync(d_r, rays, sizeof(lum_ray) * (size_t)n, cudaMemcpyHostToDevice, s->stream), "H2D rays");
    CU(cudaMemsetAsync(s->d_work, 0, sizeof(lum::WorkCounters), s->stream), "memset");
    CU(lum::launch_intersect(s->dev, d_r, n, d_h, s->d_work, s->stream), "intersect launch");
    lum::WorkCounters wc{};
    CU(cudaMemcpyAsync(hits, d_h, hb, cudaMemcpyDeviceToHost, s->stream), "D2H hits");
    CU(cudaMemcpyAsync(&wc, s->d_work, sizeof wc, cudaMemcpyDeviceToHost, s->stream), "D2H counters");
    CU(cudaStreamSynchronize(s->stream), "intersect");
    if (wc.error_flags) return fail(LUM_ERR_KERNEL, "intersect kernel reported error flags 0x%x", wc.error_flags);
    return LUM_OK;
}

lum_status lum_occluded(lum_scene* s, const lum_ray* rays, uint32_t n, int32_t* occluded) {
    if (!s || (n && (!rays || !occluded))) return fail(LUM_ERR_INVALID_ARGUMENT, "null argument");
    if (n == 0) return LUM_OK;
    std::lock_guard<std::mutex> lk(s->mu);
    CU(cudaSetDevice(s->device), "cudaSetDevice");
    size_t rb = align256(sizeof(lum_ray) * (size_t)n), ob = sizeof(int32_t) * (size_t)n;
    lum_status st = ensure(s, &s->d_rays, &s->d_rays_cap, rb + ob);
    if (st != LUM_OK) return st;
    lum_ray* d_r = (lum_ray*)s->d_rays;
    int32_t* d_o = (int32_t*)((char*)s->d_rays + rb);
    CU(cudaMemcpyAsync(d_r, rays, sizeof(lum_ray) * (size_t)n, cudaMemcpyHostToDevice, s->stream), "H2D rays");
    CU(cudaMemsetAsync(s->d_work, 0, sizeof(lum::WorkCounters), s->stream), "memset");
    CU(lum::launch_occluded(s->dev, d_r, n, d_o, s->d_work, s->stream), "occluded launch");
    lum::WorkCounters wc{};
    CU(cudaMemcpyAsync(occluded, d_o, ob, cudaMemcpyDeviceToHost, s->stream), "D2H occluded");
    CU(cudaMemcpyAsync(&wc, s->d_work, sizeof wc, cudaMemcpyDeviceToHost, s->stream), "D2H counters");
    CU(cudaStreamSynchronize(s->stream), "occluded");
    if (wc.error_flags) return fail(LUM_ERR_KERNEL, "occluded kernel reported error flags 0x%x", wc.error_flags);
    return LUM_OK;
}

}  // extern "C"

// ----------------------------------------------------------------------------- internal access
namespace lum {

lum_status set_error(lum_status code, const char* msg) { return fail(code, "%s", msg); }

lum_status prepare_render(lum_scene* s, const lum_render_params* params, SceneDev& dev, RenderDev& R,
                          cudaStream_t& stream) {
    if (!s) return fail(LUM_ERR_INVALID_ARGUMENT, "scene is null");
    lum_status st = check_params(params);
    if (st != LUM_OK) return st;
    if (sampled(*params))
        return fail(LUM_ERR_UNSUPPORTED, "adaptive sampling and the time limit are lum_render / lum_render_device "
                                         "/ lum_render_ldr features");
    st = make_render_dev(s, *params, R);
    if (st != LUM_OK) return st;
    CU(cudaSetDevice(s->device), "cudaSetDevice");
    dev = s->dev;
    stream = s->stream;
    return LUM_OK;
}

int scene_max_material_kind(const lum_scene* s) { return s ? s->max_mat_kind : 0; }

std::mutex& scene_mutex(lum_scene* s) { return s->mu; }

lum_status scene_view(lum_scene* s, const lum_render_params* params, SceneDev& dev, RenderDev& R, int& device) {
    if (!s) return fail(LUM_ERR_INVALID_ARGUMENT, "scene is null");
    lum_status st = check_params(params);
    if (st != LUM_OK) return st;
    if (sampled(*params))
        return fail(LUM_ERR_UNSUPPORTED, "adaptive sampling and the time limit are lum_render / lum_render_device "
                                         "/ lum_render_ldr features");
    st = make_render_dev(s, *params, R);
    if (st != LUM_OK) return st;
    dev = s->dev;
    device = s->device;
    return LUM_OK;
}

}  // namespace lum
