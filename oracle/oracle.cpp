// oracle.cpp -- TEST INFRASTRUCTURE, not part of the product.
//
// CPU f64 restatement of the Luminara path-tracing sample loop.  Only tests/,
// __graft_entry__.smoke() and bench.py's CPU-baseline leg load this library, and only as
// the checker.  Each function cites the Rust reference (src/<file>.rs:<lines>, paths
// relative to the Luminara project root) that it restates.
//
// Two RNG modes:
//   ORC_MODE_STREAM  the reference's own estimator: one SmallRng stream per image row seeded
//                    with row*seed (src/render.rs:1608), rejection samplers consuming a variable
//                    number of draws (src/vec3.rs:96-122).  SmallRng on 64-bit targets is
//                    xoshiro256++ seeded by SplitMix64 (rand 0.9.2; published algorithms of
//                    Blackman & Vigna), restated here.  No reference test pins its stream.
//   ORC_MODE_KEYED   the GPU estimator in f64: every draw comes from Philox4x32-10 keyed by
//                    (pixel, stratum, bounce, call) and the samplers are the direct (rejection
//                    free) mappings the CUDA kernels use.  Same distributions, different draw
//                    mapping; used for path-level comparisons with the device.
//
// Parity status: pinned against the reference's unit-test known answers only (the Rust
// reference cannot be built here); bitwise image parity with the reference is unpinned.

#include "oracle.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <limits>
#include <memory>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr double PI = 3.14159265358979323846;
constexpr double INF = std::numeric_limits<double>::infinity();

// ---------------------------------------------------------------------------------------
// Vec3 (src/vec3.rs:7-224)
// ---------------------------------------------------------------------------------------
struct V3 {
    double x, y, z;
};
inline V3 v3(double x, double y, double z) { return V3{x, y, z}; }
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
inline V3 operator*(V3 a, double t) { return {a.x * t, a.y * t, a.z * t}; }
inline V3 operator*(double t, V3 a) { return a * t; }
inline V3 operator/(V3 a, double t) { return {a.x / t, a.y / t, a.z / t}; }
inline V3& operator+=(V3& a, V3 b) { a = a + b; return a; }
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline double length_squared(V3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
inline double length(V3 a) { return std::sqrt(length_squared(a)); }
inline V3 cross(V3 a, V3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline V3 unit(V3 a) { return a / length(a); }                       // vec3.rs:53-57
inline bool near_zero(V3 a) {                                          // vec3.rs:59-62
    const double e = 1e-8;
    return std::fabs(a.x) < e && std::fabs(a.y) < e && std::fabs(a.z) < e;
}
inline V3 reflect(V3 v, V3 n) { return v - n * 2.0 * dot(v, n); }     // vec3.rs:64-66
inline V3 reflect_around(V3 v, V3 h) { return h * 2.0 * dot(v, h) - v; }  // vec3.rs:69-71
inline V3 refract(V3 v, V3 n, double eta) {                            // vec3.rs:73-78
    double cos_theta = std::fmin(dot(-v, n), 1.0);
    V3 r_perp = (v + n * cos_theta) * eta;
    V3 r_par = n * -std::sqrt(std::fabs(1.0 - length_squared(r_perp)));
    return r_perp + r_par;
}
inline V3 hadamard(V3 a, V3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
inline V3 vmin(V3 a, V3 b) { return {std::fmin(a.x, b.x), std::fmin(a.y, b.y), std::fmin(a.z, b.z)}; }
inline V3 vmax(V3 a, V3 b) { return {std::fmax(a.x, b.x), std::fmax(a.y, b.y), std::fmax(a.z, b.z)}; }
inline double axis(V3 v, int a) { return a == 0 ? v.x : (a == 1 ? v.y : v.z); }
inline V3 from(const double* p) { return {p[0], p[1], p[2]}; }
inline double to_radians(double d) { return d * (PI / 180.0); }       // Rust f64::to_radians
// Rust f64::clamp: NaN passes through.
inline double rclamp(double x, double lo, double hi) {
    if (x < lo) x = lo;
    if (x > hi) x = hi;
    return x;
}
// Rust `as usize` from f64: saturating, NaN -> 0.
inline uint64_t as_usize(double x) {
    if (!(x > 0.0)) return 0;
    if (x >= 18446744073709551615.0) return UINT64_MAX;
    return (uint64_t)x;
}
inline double fract(double x) { return x - std::trunc(x); }

// ---------------------------------------------------------------------------------------
// RNG
// ---------------------------------------------------------------------------------------
// SmallRng (rand 0.9.2, 64-bit): xoshiro256++ with SplitMix64 seed expansion; f64 draws are
// (next_u64 >> 11) * 2^-53.  Restated from the published algorithms.
struct Xoshiro {
    uint64_t s[4];
    static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    explicit Xoshiro(uint64_t state) {
        const uint64_t PHI = 0x9e3779b97f4a7c15ull;
        for (int i = 0; i < 4; ++i) {
            state += PHI;
            uint64_t z = state;
            z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
            z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
            s[i] = z ^ (z >> 31);
        }
    }
    Xoshiro(uint64_t a, uint64_t b, uint64_t c, uint64_t d) { s[0] = a; s[1] = b; s[2] = c; s[3] = d; }
    uint64_t next_u64() {
        uint64_t res = rotl(s[0] + s[3], 23) + s[0];
        uint64_t t = s[1] << 17;
        s[2] ^= s[0];
        s[3] ^= s[1];
        s[1] ^= s[2];
        s[0] ^= s[3];
        s[2] ^= t;
        s[3] = rotl(s[3], 45);
        return res;
    }
    double next_f64() { return (double)(next_u64() >> 11) * (1.0 / 9007199254740992.0); }
};

// Philox4x32-10 (Salmon et al., SC'11), the counter-based generator of the GPU path.
inline void philox4x32_10(const uint32_t in[4], const uint32_t key_in[2], uint32_t out[4]) {
    uint32_t c0 = in[0], c1 = in[1], c2 = in[2], c3 = in[3];
    uint32_t k0 = key_in[0], k1 = key_in[1];
    for (int r = 0; r < 10; ++r) {
        if (r > 0) {
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}
inline double u24(uint32_t x) { return (double)(x >> 8) * (1.0 / 16777216.0); }

// Draw source used by the integrator.  STREAM: every draw pulls the row stream in the
// reference's order.  KEYED: draws are addressed by (call, slot) inside the current bounce.
struct Sampler {
    int mode;
    Xoshiro* stream;
    uint32_t key[2];
    uint32_t pixel, stratum, bounce;
    double cache[6][4];
    bool have[6];
    void begin_bounce(uint32_t b) {
        bounce = b;
        for (int i = 0; i < 6; ++i) have[i] = false;
    }
    double keyed(int call, int slot) {
        if (!have[call]) {
            uint32_t ctr[4] = {pixel, stratum, bounce, (uint32_t)call};
            uint32_t o[4];
            philox4x32_10(ctr, key, o);
            for (int i = 0; i < 4; ++i) cache[call][i] = u24(o[i]);
            have[call] = true;
        }
        return cache[call][slot];
    }
    // A draw at (call, slot): the stream mode ignores the address.
    double draw(int call, int slot) { return mode == ORC_MODE_STREAM ? stream->next_f64() : keyed(call, slot); }
};
// Keyed call indices (must match the device mapping).
enum { CALL_CAMERA = 0, CALL_CAMERA2 = 1, CALL_SCATTER = 2, CALL_NEE = 3, CALL_EXTRA = 4, CALL_BLEND = 5 };

// Direct samplers of the keyed mode.
inline V3 keyed_unit_vector(double a, double b) {
    double z = 1.0 - 2.0 * a;
    double r = std::sqrt(std::fmax(0.0, 1.0 - z * z));
    double phi = 2.0 * PI * b;
    return {r * std::cos(phi), r * std::sin(phi), z};
}
inline V3 keyed_in_sphere(double a, double b, double c) { return keyed_unit_vector(a, b) * std::cbrt(c); }
inline V3 keyed_in_disk(double a, double b) {
    double r = std::sqrt(a), phi = 2.0 * PI * b;
    return {r * std::cos(phi), r * std::sin(phi), 0.0};
}

// Reference samplers (vec3.rs:96-122), stream mode.
inline V3 random_in_unit_sphere(Sampler& s, int call) {
    if (s.mode == ORC_MODE_KEYED)
        return keyed_in_sphere(s.draw(call, 0), s.draw(call, 1), s.draw(call, 2));
    for (;;) {
        double x = -1.0 + s.stream->next_f64() * 2.0;
        double y = -1.0 + s.stream->next_f64() * 2.0;
        double z = -1.0 + s.stream->next_f64() * 2.0;
        V3 v{x, y, z};
        if (length_squared(v) < 1.0) return v;
    }
}
inline V3 random_unit_vector(Sampler& s, int call, int slot0) {
    if (s.mode == ORC_MODE_KEYED) return keyed_unit_vector(s.draw(call, slot0), s.draw(call, slot0 + 1));
    return unit(random_in_unit_sphere(s, call));
}
// Metal/Isotropic/Dielectric-roughness in-sphere draws: keyed slots are given explicitly.
inline V3 random_in_unit_sphere_at(Sampler& s, int call, int slot0) {
    if (s.mode == ORC_MODE_KEYED)
        return keyed_in_sphere(s.draw(call, slot0), s.draw(call, slot0 + 1), s.draw(call, slot0 + 2));
    return random_in_unit_sphere(s, call);
}
inline V3 random_in_unit_disk(Sampler& s) {
    if (s.mode == ORC_MODE_KEYED) return keyed_in_disk(s.draw(CALL_CAMERA, 2), s.draw(CALL_CAMERA, 3));
    for (;;) {
        double x = s.stream->next_f64() * 2.0 - 1.0;
        double y = s.stream->next_f64() * 2.0 - 1.0;
        V3 v{x, y, 0.0};
        if (length_squared(v) < 1.0) return v;
    }
}

// ---------------------------------------------------------------------------------------
// Ray, AABB (src/ray.rs, src/aabb.rs:7-88)
// ---------------------------------------------------------------------------------------
struct Ray {
    V3 o, d;
    double time;
    V3 at(double t) const { return o + d * t; }
};

struct Aabb {
    V3 mn, mx;
    // aabb.rs:18-56; f64::max/min ignore NaN like fmax/fmin.
    bool hit(const Ray& r, double tmin, double tmax) const {
        for (int a = 0; a < 3; ++a) {
            double inv_d = 1.0 / axis(r.d, a);
            double t0 = (axis(mn, a) - axis(r.o, a)) * inv_d;
            double t1 = (axis(mx, a) - axis(r.o, a)) * inv_d;
            if (inv_d < 0.0) std::swap(t0, t1);
            tmin = std::fmax(t0, tmin);
            tmax = std::fmin(t1, tmax);
            if (a < 2 && tmax <= tmin) return false;
        }
        return tmax > tmin;
    }
    double surface_area() const {                                      // aabb.rs:59-62
        V3 d = mx - mn;
        return 2.0 * (d.x * d.y + d.y * d.z + d.z * d.x);
    }
};
inline Aabb surrounding(const Aabb& a, const Aabb& b) { return {vmin(a.mn, b.mn), vmax(a.mx, b.mx)}; }

// ---------------------------------------------------------------------------------------
// Textures and materials (src/texture.rs:9-50, src/material.rs:43-391, constant_medium.rs:77-89)
// ---------------------------------------------------------------------------------------
struct Material;
struct HitRecord {
    V3 p{0, 0, 0}, n{0, 0, 0};
    double t = 0, u = 0, v = 0;
    bool front_face = false;
    const Material* mat = nullptr;
    int32_t prim_id = -1;
    int32_t mat_index = -1;
    bool flat = false;   // planar primitive (used by the adjoint's hit-point derivative)
};
// hit.rs:19-43
inline void set_face(HitRecord& h, const Ray& r, V3 outward) {
    h.front_face = dot(r.d, outward) < 0.0;
    h.n = h.front_face ? outward : -outward;
}

struct Texture {
    int kind = LUM_TEX_SOLID;
    V3 even{0, 0, 0}, odd{0, 0, 0};
    double scale = 1.0;
    V3 value(double, double, V3 p) const {
        if (kind == LUM_TEX_SOLID) return even;                        // texture.rs:19-23
        double inv = 1.0 / scale;                                      // texture.rs:38-50
        int64_t x = (int64_t)std::floor(p.x * inv);
        int64_t y = (int64_t)std::floor(p.y * inv);
        int64_t z = (int64_t)std::floor(p.z * inv);
        return ((x + y + z) % 2 == 0) ? even : odd;
    }
};

struct Scatter {
    Ray ray;
    V3 att;
};

struct Material {
    int kind = LUM_MAT_LAMBERTIAN;
    Texture tex;
    V3 albedo{0, 0, 0};
    double fuzz = 0, ior = 1.5, roughness = 0, metallic = 0, intensity = 1, dispersion = 0;
    V3 tint{1, 1, 1};
    double extra[4] = {0, 0, 0, 0};   // the other materials' parameters (after their clamps)
    V3 color2{0, 0, 0};               // Subsurface scatter_color
    const Material* sub[2] = {nullptr, nullptr};   // Blend children

    bool is_specular() const {
        switch (kind) {
            case LUM_MAT_METAL: return true;                           // material.rs:90-92
            case LUM_MAT_DIELECTRIC: return true;                      // material.rs:145-147
            case LUM_MAT_MICROFACET: return metallic > 0.9 && roughness < 0.1;  // material.rs:323-326
            case LUM_MAT_TRANSPARENT: return true;                     // material.rs:437-439
            case LUM_MAT_IRIDESCENT: return true;                      // material.rs:495-497
            case LUM_MAT_ANISOTROPIC: return true;                     // material.rs:603-605
            default: return false;                                     // Blend: the trait default
        }
    }
    V3 emitted(double u, double v, V3 p) const {                       // material.rs:19-21, 241-243
        if (kind == LUM_MAT_EMISSIVE) return tex.value(u, v, p) * intensity;
        if (kind == LUM_MAT_BLEND)                                     // material.rs:417-420
            return sub[0]->emitted(u, v, p) * extra[0] + sub[1]->emitted(u, v, p) * (1.0 - extra[0]);
        return {0, 0, 0};
    }
    // Iridescent::thin_film_color (material.rs:469-491)
    static V3 thin_film(double cos_theta, double thickness, double film_ior) {
        double sin_theta = std::sqrt(1.0 - cos_theta * cos_theta);
        double sin_f = sin_theta / film_ior;
        double cos_f = std::sqrt(std::fmax(1.0 - sin_f * sin_f, 0.0));
        double opd = 2.0 * thickness * film_ior * cos_f;
        const double wl[3] = {650.0, 532.0, 450.0};
        double c[3];
        for (int i = 0; i < 3; ++i) {
            double ph = 2.0 * PI * opd / wl[i];
            double sn = std::sin(ph / 2.0);
            c[i] = sn * sn;
        }
        return {c[0], c[1], c[2]};
    }
    // The other materials' scatter (material.rs:408-865); keyed slots as on the device.
    bool scatter_other(const Ray& r, const HitRecord& h, Sampler& s, Scatter& out, int level) const {
        switch (kind) {
            case LUM_MAT_BLEND: {                                      // material.rs:408-415
                double x = s.draw(CALL_BLEND, level);
                return (x < extra[0] ? sub[0] : sub[1])->scatter(r, h, s, out, level + 1);
            }
            case LUM_MAT_TRANSPARENT:                                  // material.rs:429-435
                out.ray = {h.p, r.d, r.time};
                out.att = {1, 1, 1};
                return true;
            case LUM_MAT_IRIDESCENT: {                                 // material.rs:499-527
                V3 ud = unit(r.d);
                double ct = std::fmin(std::fabs(dot(-ud, h.n)), 1.0);
                out.att = hadamard(albedo, thin_film(ct, extra[0], ior));
                V3 dir = reflect(ud, h.n);
                if (roughness > 0.0) {
                    dir += random_in_unit_sphere_at(s, CALL_SCATTER, 0) * roughness;
                    if (dot(dir, h.n) <= 0.0) return false;
                }
                out.ray = {h.p, dir, r.time};
                return true;
            }
            case LUM_MAT_TOON: {                                       // material.rs:549-577
                V3 dir = h.n + random_unit_vector(s, CALL_SCATTER, 0);
                if (near_zero(dir)) dir = h.n;
                double ndl = std::fmax(dot(unit(dir), h.n), 0.0);
                double band = std::floor(ndl * extra[0]) / (extra[0] - 1.0);
                double q = rclamp(band, 0.0, 1.0);
                V3 view = unit(-r.d);
                V3 hv = unit(view + unit(dir));
                double spec = std::pow(std::fmax(dot(hv, h.n), 0.0), extra[1] * 100.0);
                out.ray = {h.p, dir, r.time};
                out.att = albedo * (q + (spec > 0.5 ? 0.3 : 0.0));
                return true;
            }
            case LUM_MAT_ANISOTROPIC: {                                // material.rs:607-641
                V3 refl = reflect(unit(r.d), h.n);
                int ax = (int)extra[2];
                V3 wt = ax == 0 ? v3(1, 0, 0) : (ax == 1 ? v3(0, 1, 0) : v3(0, 0, 1));
                V3 t = unit(wt - h.n * dot(wt, h.n));
                V3 b = cross(h.n, t);
                double r1 = s.draw(CALL_SCATTER, 0) * 2.0 * PI;
                double r2 = std::sqrt(s.draw(CALL_SCATTER, 1));
                V3 sc = unit(refl + t * (std::cos(r1) * r2 * extra[0]) + b * (std::sin(r1) * r2 * extra[1]));
                if (!(dot(sc, h.n) > 0.0)) return false;
                out.ray = {h.p, sc, r.time};
                out.att = albedo;
                return true;
            }
            case LUM_MAT_CLEARCOAT: {                                  // material.rs:664-707
                V3 ud = unit(r.d);
                double ct = std::fmin(std::fabs(dot(-ud, h.n)), 1.0);
                double r0 = (1.0 - ior) / (1.0 + ior);
                r0 = r0 * r0;
                double om = 1.0 - ct;
                double fr = r0 + (1.0 - r0) * (om * om * om * om * om);
                if (s.draw(CALL_SCATTER, 0) < fr * extra[0]) {
                    V3 refl = reflect(ud, h.n);
                    double rough = (1.0 - extra[0]) * 0.3;
                    V3 dir = refl;
                    if (rough > 0.001) {
                        V3 fz = refl + random_in_unit_sphere_at(s, CALL_SCATTER, 1) * rough;
                        if (dot(fz, h.n) > 0.0) dir = fz;
                    }
                    out.ray = {h.p, dir, r.time};
                    out.att = {1, 1, 1};
                    return true;
                }
                V3 dir = h.n + random_unit_vector(s, CALL_SCATTER, 1);
                if (near_zero(dir)) dir = h.n;
                out.ray = {h.p, dir, r.time};
                out.att = albedo;
                return true;
            }
            case LUM_MAT_VELVET: {                                     // material.rs:724-746
                V3 dir = h.n + random_unit_vector(s, CALL_SCATTER, 0);
                if (near_zero(dir)) dir = h.n;
                double ct = std::fabs(dot(-unit(r.d), h.n));
                double st = std::sqrt(std::fmax(1.0 - ct * ct, 0.0));
                out.ray = {h.p, dir, r.time};
                out.att = albedo * (1.0 + std::pow(st, 1.5) * extra[0]);
                return true;
            }
            case LUM_MAT_TRANSLUCENT: {                                // material.rs:769-797
                V3 dir;
                if (s.draw(CALL_SCATTER, 0) < extra[0]) {
                    V3 through = unit(r.d);
                    V3 below = -h.n + random_unit_vector(s, CALL_SCATTER, 1);
                    dir = through * (1.0 - extra[1]) + below * extra[1];
                    if (near_zero(dir)) dir = -h.n;
                } else {
                    dir = h.n + random_unit_vector(s, CALL_SCATTER, 1);
                    if (near_zero(dir)) dir = h.n;
                }
                out.ray = {h.p, dir, r.time};
                out.att = albedo;
                return true;
            }
            case LUM_MAT_SUBSURFACE: {                                 // material.rs:823-864
                double fr = reflectance(std::fabs(dot(unit(r.d), h.n)), 1.0 / 1.4);
                if (s.draw(CALL_SCATTER, 0) < fr) {
                    V3 dir = h.n + random_unit_vector(s, CALL_SCATTER, 1);
                    if (near_zero(dir)) dir = h.n;
                    out.ray = {h.p, dir, r.time};
                    out.att = albedo;
                    return true;
                }
                double mfp = extra[0];
                double step = -mfp * std::log(std::fmax(s.draw(CALL_SCATTER, 1), 1e-10));
                V3 exit = h.p + random_unit_vector(s, CALL_SCATTER, 2) * step;
                V3 ed = h.n + random_unit_vector(s, CALL_EXTRA, 0);
                ed = near_zero(ed) ? h.n : unit(ed);
                double k = -step / mfp;
                out.ray = {exit, ed, r.time};
                out.att = hadamard(albedo, v3(std::exp(k * (1.0 - color2.x)), std::exp(k * (1.0 - color2.y)),
                                              std::exp(k * (1.0 - color2.z))));
                return true;
            }
        }
        return false;
    }
    static double reflectance(double cosine, double ref_idx) {         // material.rs:138-141
        double r0 = (1.0 - ref_idx) / (1.0 + ref_idx);
        r0 = r0 * r0;
        double m = 1.0 - cosine;
        return r0 + (1.0 - r0) * (m * m * m * m * m);
    }
    static double schlick_g1(double n_dot_v, double k) { return n_dot_v / (n_dot_v * (1.0 - k) + k); }
    static double geometry(double ndv, double ndl, double rough) {     // material.rs:285-288
        double k = (rough + 1.0) * (rough + 1.0) / 8.0;
        return schlick_g1(ndv, k) * schlick_g1(ndl, k);
    }
    static V3 fresnel(double cos_theta, V3 f0) {                       // material.rs:291-294
        double m = std::fmax(1.0 - cos_theta, 0.0);
        double t = m * m * m * m * m;
        return f0 * (1.0 - t) + v3(1, 1, 1) * t;
    }
    // material.rs:297-319
    static V3 sample_ggx_normal(V3 n, double alpha, double r1, double r2) {
        double theta = std::atan(std::sqrt(alpha * alpha * r1 / (1.0 - r1 + 1e-10)));
        double phi = 2.0 * PI * r2;
        double st = std::sin(theta), ct = std::cos(theta);
        V3 h{st * std::cos(phi), st * std::sin(phi), ct};
        V3 up = std::fabs(n.y) < 0.999 ? v3(0, 1, 0) : v3(1, 0, 0);
        V3 tangent = unit(cross(up, n));
        V3 bitangent = cross(n, tangent);
        return unit(tangent * h.x + bitangent * h.y + n * h.z);
    }

    bool scatter(const Ray& r, const HitRecord& h, Sampler& s, Scatter& out, int level = 0) const {
        if (kind >= LUM_MAT_BLEND) return scatter_other(r, h, s, out, level);
        switch (kind) {
            case LUM_MAT_LAMBERTIAN: {                                 // material.rs:59-71
                V3 dir = h.n + random_unit_vector(s, CALL_SCATTER, 0);
                if (near_zero(dir)) dir = h.n;
                out.ray = {h.p, dir, r.time};
                out.att = tex.value(h.u, h.v, h.p);
                return true;
            }
            case LUM_MAT_METAL: {                                      // material.rs:94-106
                V3 refl = reflect(unit(r.d), h.n);
                V3 sc = refl + random_in_unit_sphere_at(s, CALL_SCATTER, 0) * fuzz;
                if (dot(sc, h.n) > 0.0) {
                    out.ray = {h.p, sc, r.time};
                    out.att = albedo;
                    return true;
                }
                return false;
            }
            case LUM_MAT_DIELECTRIC: {                                 // material.rs:149-213
                double ior_used = ior;
                V3 chan{1, 1, 1};
                if (dispersion > 0.0) {
                    uint32_t channel = (uint32_t)as_usize(s.draw(CALL_EXTRA, 0) * 3.0);
                    double off = channel == 0 ? -dispersion : (channel == 1 ? 0.0 : dispersion);
                    chan = channel == 0 ? v3(3, 0, 0) : (channel == 1 ? v3(0, 3, 0) : v3(0, 0, 3));
                    ior_used = ior + off;
                }
                double eta = h.front_face ? 1.0 / ior_used : ior_used;
                V3 ud = unit(r.d);
                double cos_t = std::fmin(dot(-ud, h.n), 1.0);
                double sin_t = std::sqrt(1.0 - cos_t * cos_t);
                bool cannot = eta * sin_t > 1.0;
                V3 dir;
                if (cannot) {
                    dir = reflect(ud, h.n);
                } else if (reflectance(cos_t, eta) > s.draw(CALL_SCATTER, 0)) {
                    dir = reflect(ud, h.n);
                } else {
                    dir = refract(ud, h.n, eta);
                }
                if (roughness > 0.0) dir += random_in_unit_sphere_at(s, CALL_SCATTER, 1) * roughness;
                V3 att;
                if (!h.front_face && !(tint.x == 1.0 && tint.y == 1.0 && tint.z == 1.0)) {
                    double dist = h.t;
                    att = {std::exp(-(1.0 - tint.x) * dist), std::exp(-(1.0 - tint.y) * dist),
                           std::exp(-(1.0 - tint.z) * dist)};
                } else {
                    att = tint;
                }
                if (dispersion > 0.0) att = hadamard(att, chan);
                out.ray = {h.p, dir, r.time};
                out.att = att;
                return true;
            }
            case LUM_MAT_EMISSIVE:                                     // material.rs:237-239
                return false;
            case LUM_MAT_MICROFACET: {                                 // material.rs:328-390
                double alpha = roughness * roughness;
                V3 v = unit(-r.d);
                V3 n = h.n;
                V3 alb = tex.value(h.u, h.v, h.p);
                double ndv = std::fmax(dot(n, v), 0.001);
                V3 f0 = v3(0.04, 0.04, 0.04) * (1.0 - metallic) + alb * metallic;
                V3 fw = fresnel(ndv, f0);
                double sp = rclamp((fw.x + fw.y + fw.z) / 3.0, 0.1, 0.9);
                if (s.draw(CALL_SCATTER, 0) < sp) {
                    double r1 = s.draw(CALL_SCATTER, 1);
                    double r2 = s.draw(CALL_SCATTER, 2);
                    V3 hh = sample_ggx_normal(n, alpha, r1, r2);
                    V3 l = reflect_around(v, hh);
                    double ndl = dot(n, l);
                    if (ndl <= 0.0) return false;
                    double ndh = std::fmax(dot(n, hh), 0.0);
                    double vdh = std::fmax(dot(v, hh), 0.0);
                    double g = geometry(ndv, ndl, roughness);
                    V3 f = fresnel(vdh, f0);
                    V3 w = ndh > 0.001 ? f * (g * vdh / (ndv * ndh)) : v3(0, 0, 0);
                    out.ray = {h.p, l, r.time};
                    out.att = w / sp;
                    return true;
                }
                V3 dir = n + random_unit_vector(s, CALL_SCATTER, 1);
                if (near_zero(dir)) dir = n;
                V3 kd = (v3(1, 1, 1) - fw) * (1.0 - metallic);
                out.ray = {h.p, dir, r.time};
                out.att = hadamard(kd, alb) / (1.0 - sp);
                return true;
            }
            case LUM_MAT_ISOTROPIC: {                                  // constant_medium.rs:81-89
                out.ray = {h.p, random_in_unit_sphere_at(s, CALL_SCATTER, 0), r.time};
                out.att = albedo;
                return true;
            }
        }
        return false;
    }
};

Material make_material(const lum_material& m) {
    Material out;
    out.kind = m.kind;
    out.tex.kind = m.texture;
    out.tex.even = from(m.color);
    out.tex.odd = from(m.color2);
    out.tex.scale = std::fabs(m.tex_scale) < 1e-10 ? 1.0 : m.tex_scale;  // texture.rs:32-35
    out.albedo = from(m.color);
    out.fuzz = std::fmin(m.fuzz, 1.0);                                  // material.rs:81-86
    out.ior = m.ior;
    out.roughness = m.roughness;
    out.metallic = m.metallic;
    if (m.kind == LUM_MAT_MICROFACET) {                                 // material.rs:255-261
        out.roughness = rclamp(m.roughness, 0.01, 1.0);
        out.metallic = rclamp(m.metallic, 0.0, 1.0);
    }
    out.intensity = m.intensity;
    out.dispersion = m.dispersion;
    out.tint = from(m.tint);
    out.color2 = from(m.color2);
    const double* e = m.extra;
    auto cl = [](double x, double lo, double hi) { return std::fmin(std::fmax(x, lo), hi); };
    switch (m.kind) {                                                   // the constructors' clamps
        case LUM_MAT_BLEND: out.extra[0] = cl(e[0], 0.0, 1.0); break;  // material.rs:402-406
        case LUM_MAT_IRIDESCENT:                                        // material.rs:459-466
            out.extra[0] = std::fmax(e[0], 100.0);
            out.ior = std::fmax(m.ior, 1.0);
            out.roughness = cl(m.roughness, 0.0, 1.0);
            break;
        case LUM_MAT_TOON:                                              // material.rs:538-545
            out.extra[0] = std::fmax(std::floor(cl(e[0], 0.0, 4294967295.0)), 2.0);
            out.extra[1] = std::fmax(e[1], 0.0);
            break;
        case LUM_MAT_ANISOTROPIC:                                       // material.rs:592-599
            out.extra[0] = cl(e[0], 0.001, 1.0);
            out.extra[1] = cl(e[1], 0.001, 1.0);
            out.extra[2] = std::fmin(std::floor(std::fmax(e[2], 0.0)), 2.0);
            break;
        case LUM_MAT_CLEARCOAT:                                         // material.rs:655-661
            out.extra[0] = cl(e[0], 0.0, 1.0);
            out.ior = std::fmax(m.ior, 1.0);
            break;
        case LUM_MAT_VELVET: out.extra[0] = cl(e[0], 0.0, 2.0); break;  // material.rs:718-720
        case LUM_MAT_TRANSLUCENT:                                       // material.rs:760-766
            out.extra[0] = cl(e[0], 0.0, 1.0);
            out.extra[1] = cl(e[1], 0.0, 1.0);
            break;
        case LUM_MAT_SUBSURFACE: out.extra[0] = std::fmax(e[0], 0.001); break;  // material.rs:812-818
        default: break;
    }
    return out;
}

// Links Blend children (indices into the same array); false when an index is out of range or
// Blends nest more than 4 deep (the device's limit).
bool link_blends(std::vector<Material>& ms, const lum_material* mats, uint32_t n) {
    for (uint32_t i = 0; i < n; ++i) {
        if (mats[i].kind != LUM_MAT_BLEND) continue;
        for (int k = 0; k < 2; ++k) {
            if (mats[i].sub[k] < 0 || (uint32_t)mats[i].sub[k] >= n) return false;
            ms[i].sub[k] = &ms[mats[i].sub[k]];
        }
    }
    std::function<bool(const Material*, int)> ok = [&](const Material* m, int lv) {
        if (m->kind != LUM_MAT_BLEND) return true;
        return lv < 4 && ok(m->sub[0], lv + 1) && ok(m->sub[1], lv + 1);
    };
    for (uint32_t i = 0; i < n; ++i)
        if (!ok(&ms[i], 0)) return false;
    return true;
}

// ---------------------------------------------------------------------------------------
// Hittables (src/hit.rs, sphere.rs, quad.rs, rect.rs, triangle.rs, obj.rs, disk.rs,
// plane.rs, transform.rs, constant_medium.rs, bvh.rs)
// ---------------------------------------------------------------------------------------
struct Hittable {
    virtual ~Hittable() = default;
    virtual bool hit(const Ray& r, double tmin, double tmax, HitRecord& rec) const = 0;
    virtual bool bbox(Aabb& out) const = 0;
};
using HPtr = std::unique_ptr<Hittable>;

struct Leaf : Hittable {
    const Material* mat = nullptr;
    int32_t prim_id = -1;
    int32_t mat_index = -1;
    bool flat = false;
    void tag(HitRecord& h) const {
        h.mat = mat;
        h.prim_id = prim_id;
        h.mat_index = mat_index;
        h.flat = flat;
    }
};

struct Sphere : Leaf {                                                  // sphere.rs:23-68
    V3 c;
    double r;
    bool hit(const Ray& ray, double tmin, double tmax, HitRecord& rec) const override {
        V3 oc = ray.o - c;
        double a = length_squared(ray.d);
        double half_b = dot(oc, ray.d);
        double cc = length_squared(oc) - r * r;
        double disc = half_b * half_b - a * cc;
        if (disc < 0.0) return false;
        double sq = std::sqrt(disc);
        double root = (-half_b - sq) / a;
        if (root < tmin || root > tmax) {
            root = (-half_b + sq) / a;
            if (root < tmin || root > tmax) return false;
        }
        rec.t = root;
        rec.p = ray.at(root);
        V3 on = (rec.p - c) / r;
        double theta = std::acos(-on.y);
        double phi = std::atan2(-on.z, on.x) + PI;
        rec.u = phi / (2.0 * PI);
        rec.v = theta / PI;
        set_face(rec, ray, on);
        tag(rec);
        return true;
    }
    bool bbox(Aabb& o) const override {
        V3 rr{r, r, r};
        o = {c - rr, c + rr};
        return true;
    }
};

struct MovingSphere : Leaf {                                            // sphere.rs:71-125
    V3 c0, c1;
    double r;
    bool hit(const Ray& ray, double tmin, double tmax, HitRecord& rec) const override {
        V3 c = c0 + (c1 - c0) * ray.time;
        V3 oc = ray.o - c;
        double a = length_squared(ray.d);
        double half_b = dot(oc, ray.d);
        double cc = length_squared(oc) - r * r;
        double disc = half_b * half_b - a * cc;
        if (disc < 0.0) return false;
        double sq = std::sqrt(disc);
        double root = (-half_b - sq) / a;
        if (root < tmin || root > tmax) {
            root = (-half_b + sq) / a;
            if (root < tmin || root > tmax) return false;
        }
        rec.t = root;
        rec.p = ray.at(root);
        V3 on = (rec.p - c) / r;
        double theta = std::acos(-on.y);
        double phi = std::atan2(-on.z, on.x) + PI;
        rec.u = phi / (2.0 * PI);
        rec.v = theta / PI;
        set_face(rec, ray, on);
        tag(rec);
        return true;
    }
    bool bbox(Aabb& o) const override {
        V3 rr{r, r, r};
        o = surrounding({c0 - rr, c0 + rr}, {c1 - rr, c1 + rr});
        return true;
    }
};

struct Quad : Leaf {                                                    // quad.rs:20-72
    Quad() { flat = true; }
    V3 q, u, v, n, w;
    double d;
    void init() {
        V3 nn = cross(u, v);
        n = unit(nn);
        d = dot(n, q);
        w = nn / dot(nn, nn);
    }
    bool hit(const Ray& ray, double tmin, double tmax, HitRecord& rec) const override {
        double denom = dot(n, ray.d);
        if (std::fabs(denom) < 1e-8) return false;
        double t = (d - dot(n, ray.o)) / denom;
        if (t < tmin || t > tmax) return false;
        V3 p = ray.at(t);
        V3 ph = p - q;
        double alpha = dot(w, cross(ph, v));
        double beta = dot(w, cross(u, ph));
        if (!(alpha >= 0.0 && alpha <= 1.0) || !(beta >= 0.0 && beta <= 1.0)) return false;
        rec.t = t;
        rec.p = p;
        rec.u = alpha;
        rec.v = beta;
        set_face(rec, ray, n);
        tag(rec);
        return true;
    }
    bool bbox(Aabb& o) const override {
        V3 p0 = q, p1 = q + u, p2 = q + v, p3 = q + u + v;
        V3 e{1e-4, 1e-4, 1e-4};
        o = {vmin(vmin(vmin(p0, p1), p2), p3) - e, vmax(vmax(vmax(p0, p1), p2), p3) + e};
        return true;
    }
};

// rect.rs:7-125: axis 0 = XY (z=k), 1 = XZ (y=k), 2 = YZ (x=k).
struct AxisRect : Leaf {
    AxisRect() { flat = true; }
    int plane;
    double a0, a1, b0, b1, k;
    bool hit(const Ray& ray, double tmin, double tmax, HitRecord& rec) const override {
        // (ka, kb, kk) = axes of the rect's first/second coordinate and its normal.
        int ka, kb, kk;
        V3 nrm;
        if (plane == 0) { ka = 0; kb = 1; kk = 2; nrm = {0, 0, 1}; }
        else if (plane == 1) { ka = 0; kb = 2; kk = 1; nrm = {0, 1, 0}; }
        else { ka = 1; kb = 2; kk = 0; nrm = {1, 0, 0}; }
        double t = (k - axis(ray.o, kk)) / axis(ray.d, kk);
        if (t < tmin || t > tmax) return false;
        double x = axis(ray.o, ka) + t * axis(ray.d, ka);
        double y = axis(ray.o, kb) + t * axis(ray.d, kb);
        if (x < a0 || x > a1 || y < b0 || y > b1) return false;
        rec.u = (x - a0) / (a1 - a0);
        rec.v = (y - b0) / (b1 - b0);
        rec.t = t;
        rec.p = ray.at(t);
        set_face(rec, ray, nrm);
        tag(rec);
        return true;
    }
    bool bbox(Aabb& o) const override {
        if (plane == 0) o = {{a0, b0, k - 0.0001}, {a1, b1, k + 0.0001}};
        else if (plane == 1) o = {{a0, k - 0.0001, b0}, {a1, k + 0.0001, b1}};
        else o = {{k - 0.0001, a0, b0}, {k + 0.0001, a1, b1}};
        return true;
    }
};

struct Triangle : Leaf {                       // triangle.rs:21-64, obj.rs:259-313
    Triangle() { flat = true; }
    V3 v0, v1, v2;
    bool has_normals = false;
    V3 n0, n1, n2;
    bool hit(const Ray& ray, double tmin, double tmax, HitRecord& rec) const override {
        V3 e1 = v1 - v0, e2 = v2 - v0;
        V3 h = cross(ray.d, e2);
        double a = dot(e1, h);
        if (std::fabs(a) < 1e-8) return false;
        double f = 1.0 / a;
        V3 s = ray.o - v0;
        double u = f * dot(s, h);
        if (!(u >= 0.0 && u <= 1.0)) return false;
        V3 q = cross(s, e1);
        double v = f * dot(ray.d, q);
        if (v < 0.0 || u + v > 1.0) return false;
        double t = f * dot(e2, q);
        if (t < tmin || t > tmax) return false;
        rec.t = t;
        rec.p = ray.at(t);
        V3 on = has_normals ? unit(n0 * (1.0 - u - v) + n1 * u + n2 * v) : unit(cross(e1, e2));
        rec.u = u;
        rec.v = v;
        set_face(rec, ray, on);
        tag(rec);
        return true;
    }
    bool bbox(Aabb& o) const override {
        V3 e{1e-4, 1e-4, 1e-4};
        o = {vmin(vmin(v0, v1), v2) - e, vmax(vmax(v0, v1), v2) + e};
        return true;
    }
};

struct Disk : Leaf {                                                    // disk.rs:16-65
    Disk() { flat = true; }
    V3 c, n;
    double r;
    bool hit(const Ray& ray, double tmin, double tmax, HitRecord& rec) const override {
        double denom = dot(n, ray.d);
        if (std::fabs(denom) < 1e-8) return false;
        double t = dot(c - ray.o, n) / denom;
        if (t < tmin || t > tmax) return false;
        V3 p = ray.at(t);
        V3 off = p - c;
        if (length_squared(off) > r * r) return false;
        double rr = length(off) / r;
        double theta = std::atan2(off.z, off.x);
        rec.u = theta / (2.0 * PI) + 0.5;
        rec.v = rr;
        rec.t = t;
        rec.p = p;
        set_face(rec, ray, n);
        tag(rec);
        return true;
    }
    bool bbox(Aabb& o) const override {
        V3 rr{r, r, r};
        o = {c - rr, c + rr};
        return true;
    }
};

struct Plane : Leaf {                                                   // plane.rs:18-74
    Plane() { flat = true; }
    V3 p0, n, ua, va;
    void init(V3 point, V3 normal) {
        p0 = point;
        n = near_zero(normal) ? v3(0, 1, 0) : unit(normal);
        V3 up = std::fabs(n.y) > 0.999 ? v3(1, 0, 0) : v3(0, 1, 0);
        ua = unit(cross(up, n));
        va = cross(n, ua);
    }
    bool hit(const Ray& ray, double tmin, double tmax, HitRecord& rec) const override {
        double denom = dot(n, ray.d);
        if (std::fabs(denom) < 1e-8) return false;
        double t = dot(p0 - ray.o, n) / denom;
        if (t < tmin || t > tmax) return false;
        V3 p = ray.at(t);
        V3 local = p - p0;
        rec.u = std::fabs(fract(dot(local, ua)));
        rec.v = std::fabs(fract(dot(local, va)));
        rec.t = t;
        rec.p = p;
        set_face(rec, ray, n);
        tag(rec);
        return true;
    }
    bool bbox(Aabb&) const override { return false; }
};

struct HittableList : Hittable {                                        // hit.rs:72-103
    std::vector<HPtr> objects;
    bool hit(const Ray& r, double tmin, double tmax, HitRecord& rec) const override {
        double closest = tmax;
        bool any = false;
        HitRecord tmp;
        for (auto& o : objects) {
            if (o->hit(r, tmin, closest, tmp)) {
                closest = tmp.t;
                rec = tmp;
                any = true;
            }
        }
        return any;
    }
    bool bbox(Aabb& out) const override {
        if (objects.empty()) return false;
        bool have = false;
        for (auto& o : objects) {
            Aabb b;
            if (o->bbox(b)) {
                out = have ? surrounding(out, b) : b;
                have = true;
            }
        }
        return have;
    }
};

struct Translate : Hittable {                                           // transform.rs:18-29
    HPtr inner;
    V3 off;
    bool hit(const Ray& r, double tmin, double tmax, HitRecord& rec) const override {
        Ray moved{r.o - off, r.d, 0.0};  // Ray::new drops the time
        if (!inner->hit(moved, tmin, tmax, rec)) return false;
        rec.p += off;
        return true;
    }
    bool bbox(Aabb& o) const override {
        Aabb b;
        if (!inner->bbox(b)) return false;
        o = {b.mn + off, b.mx + off};
        return true;
    }
};

// transform.rs:31-256: axis 0 = X, 1 = Y, 2 = Z.
struct Rotate : Hittable {
    HPtr inner;
    int ax;
    double s, c;
    bool has_box = false;
    Aabb box;
    // Forward rotation (object -> world) of a vector, per axis as in the reference.
    V3 fwd(V3 p) const {
        if (ax == 1) return {c * p.x + s * p.z, p.y, -s * p.x + c * p.z};
        if (ax == 0) return {p.x, c * p.y - s * p.z, s * p.y + c * p.z};
        return {c * p.x - s * p.y, s * p.x + c * p.y, p.z};
    }
    V3 inv(V3 p) const {
        if (ax == 1) return {c * p.x - s * p.z, p.y, s * p.x + c * p.z};
        if (ax == 0) return {p.x, c * p.y + s * p.z, -s * p.y + c * p.z};
        return {c * p.x + s * p.y, -s * p.x + c * p.y, p.z};
    }
    void init(double degrees) {
        double rad = to_radians(degrees);
        s = std::sin(rad);
        c = std::cos(rad);
        Aabb b;
        if (inner->bbox(b)) {
            V3 mn{INF, INF, INF}, mx{-INF, -INF, -INF};
            for (int i = 0; i < 2; ++i)
                for (int j = 0; j < 2; ++j)
                    for (int k = 0; k < 2; ++k) {
                        double x = i * b.mx.x + (1 - i) * b.mn.x;
                        double y = j * b.mx.y + (1 - j) * b.mn.y;
                        double z = k * b.mx.z + (1 - k) * b.mn.z;
                        V3 nv = fwd({x, y, z});
                        mn = vmin(mn, nv);
                        mx = vmax(mx, nv);
                    }
            box = {mn, mx};
            has_box = true;
        }
    }
    bool hit(const Ray& r, double tmin, double tmax, HitRecord& rec) const override {
        // RotateY builds its ray with Ray::new (time 0); RotateX/RotateZ keep the time.
        Ray rr{inv(r.o), inv(r.d), ax == 1 ? 0.0 : r.time};
        if (!inner->hit(rr, tmin, tmax, rec)) return false;
        rec.p = fwd(rec.p);
        rec.n = fwd(rec.n);
        return true;
    }
    bool bbox(Aabb& o) const override {
        if (!has_box) return false;
        o = box;
        return true;
    }
};

struct Scale : Hittable {                                               // transform.rs:258-284
    HPtr inner;
    double f, inv_f;
    bool hit(const Ray& r, double tmin, double tmax, HitRecord& rec) const override {
        Ray sr{r.o * inv_f, r.d * inv_f, 0.0};
        if (!inner->hit(sr, tmin, tmax, rec)) return false;
        rec.p = rec.p * f;
        rec.t *= f;
        return true;
    }
    bool bbox(Aabb& o) const override {
        Aabb b;
        if (!inner->bbox(b)) return false;
        o = {b.mn * f, b.mx * f};
        return true;
    }
};

struct ConstantMedium : Leaf {                                          // constant_medium.rs:25-74
    HPtr boundary;
    double neg_inv_density;
    bool hit(const Ray& ray, double tmin, double tmax, HitRecord& rec) const override {
        HitRecord h1, h2;
        if (!boundary->hit(ray, -INF, INF, h1)) return false;
        if (!boundary->hit(ray, h1.t + 0.0001, INF, h2)) return false;
        double t1 = std::fmax(h1.t, tmin);
        double t2 = std::fmin(h2.t, tmax);
        if (t1 >= t2) return false;
        if (t1 < 0.0) t1 = 0.0;
        double len = length(ray.d);
        double inside = (t2 - t1) * len;
        double hv = std::fabs(fract(ray.o.x * 73856093.0 + ray.o.y * 19349663.0 + ray.o.z * 83492791.0 +
                                    ray.d.x * 47392381.0));
        double hit_distance = neg_inv_density * std::log(std::fmax(1.0 - hv, 1e-10));
        if (hit_distance > inside) return false;
        double t = t1 + hit_distance / len;
        rec.t = t;
        rec.p = ray.at(t);
        rec.u = 0.0;
        rec.v = 0.0;
        set_face(rec, ray, v3(1, 0, 0));
        tag(rec);
        return true;
    }
    bool bbox(Aabb& o) const override { return boundary->bbox(o); }
};

struct BvhNode : Hittable {                                             // bvh.rs:6-68
    HPtr left, right;
    Aabb box;
    bool hit(const Ray& r, double tmin, double tmax, HitRecord& rec) const override {
        if (!box.hit(r, tmin, tmax)) return false;
        HitRecord lh;
        bool hl = left->hit(r, tmin, tmax, lh);
        double tr = hl ? lh.t : tmax;
        HitRecord rh;
        bool hr = right->hit(r, tmin, tr, rh);
        if (hr) { rec = rh; return true; }
        if (hl) { rec = lh; return true; }
        return false;
    }
    bool bbox(Aabb& o) const override { o = box; return true; }
};

inline double centroid_axis(const Aabb& b, int a) { return (axis(b.mn, a) + axis(b.mx, a)) * 0.5; }

// bvh.rs:71-163
std::pair<int, size_t> find_best_split(const std::vector<HPtr>& objs) {
    const size_t n = objs.size();
    const int B = 12;
    Aabb overall;
    objs[0]->bbox(overall);
    V3 cmin{INF, INF, INF}, cmax{-INF, -INF, -INF};
    for (auto& o : objs) {
        Aabb b;
        if (o->bbox(b)) {
            overall = surrounding(overall, b);
            V3 c = (b.mn + b.mx) * 0.5;
            cmin = vmin(cmin, c);
            cmax = vmax(cmax, c);
        }
    }
    double osa = overall.surface_area();
    if (osa < 1e-10) return {0, n / 2};
    int best_axis = 0;
    double best_cost = INF;
    size_t best_mid = n / 2;
    for (int a = 0; a < 3; ++a) {
        double extent = axis(cmax, a) - axis(cmin, a);
        if (extent < 1e-10) continue;
        size_t cnt[B] = {0};
        bool has[B] = {false};
        Aabb bb[B];
        for (auto& o : objs) {
            Aabb b;
            if (o->bbox(b)) {
                double c = (axis(b.mn, a) + axis(b.mx, a)) * 0.5;
                uint64_t k = as_usize((c - axis(cmin, a)) / extent * (double)B);
                if (k > B - 1) k = B - 1;
                cnt[k]++;
                bb[k] = has[k] ? surrounding(bb[k], b) : b;
                has[k] = true;
            }
        }
        for (int split = 1; split < B; ++split) {
            size_t lc = 0, rc = 0;
            bool lh = false, rh = false;
            Aabb lb, rb;
            for (int i = 0; i < split; ++i) {
                lc += cnt[i];
                if (has[i]) { lb = lh ? surrounding(lb, bb[i]) : bb[i]; lh = true; }
            }
            for (int i = split; i < B; ++i) {
                rc += cnt[i];
                if (has[i]) { rb = rh ? surrounding(rb, bb[i]) : bb[i]; rh = true; }
            }
            if (lc == 0 || rc == 0) continue;
            double lsa = lh ? lb.surface_area() : 0.0;
            double rsa = rh ? rb.surface_area() : 0.0;
            double cost = 1.0 + ((double)lc * lsa + (double)rc * rsa) / osa;
            if (cost < best_cost) {
                best_cost = cost;
                best_axis = a;
                best_mid = lc;
            }
        }
    }
    return {best_axis, best_mid};
}

// bvh.rs:16-58
HPtr build_bvh(std::vector<HPtr> objs) {
    const size_t n = objs.size();
    if (n == 1) return std::move(objs[0]);
    auto node = std::make_unique<BvhNode>();
    if (n == 2) {
        node->left = std::move(objs[0]);
        node->right = std::move(objs[1]);
    } else {
        auto [ax, mid] = find_best_split(objs);
        std::vector<double> keys(n);
        std::vector<size_t> order(n);
        for (size_t i = 0; i < n; ++i) {
            Aabb b;
            keys[i] = objs[i]->bbox(b) ? centroid_axis(b, ax) : 0.0;
            order[i] = i;
        }
        // sort_by is stable; partial_cmp falls back to Equal on NaN.
        std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return keys[a] < keys[b]; });
        std::vector<HPtr> sorted(n);
        for (size_t i = 0; i < n; ++i) sorted[i] = std::move(objs[order[i]]);
        size_t m = std::min(std::max(mid, (size_t)1), n - 1);
        std::vector<HPtr> l, r;
        for (size_t i = 0; i < m; ++i) l.push_back(std::move(sorted[i]));
        for (size_t i = m; i < n; ++i) r.push_back(std::move(sorted[i]));
        node->left = build_bvh(std::move(l));
        node->right = build_bvh(std::move(r));
    }
    Aabb lb, rb;
    node->left->bbox(lb);
    node->right->bbox(rb);
    node->box = surrounding(lb, rb);
    return node;
}

void bvh_stats(const Hittable* h, uint32_t depth, uint32_t& nodes, uint32_t& maxd) {
    auto* b = dynamic_cast<const BvhNode*>(h);
    if (!b) {
        maxd = std::max(maxd, depth);
        return;
    }
    nodes++;
    bvh_stats(b->left.get(), depth + 1, nodes, maxd);
    bvh_stats(b->right.get(), depth + 1, nodes, maxd);
}

// ---------------------------------------------------------------------------------------
// Lights, background, camera, filter
// ---------------------------------------------------------------------------------------
struct Light {
    int kind;
    V3 p0, u, v, n, e;
    double r;
};

// render.rs:1333-1343
inline void build_onb(V3 n, V3& a, V3& b) {
    if (n.z < -0.9999999) {
        a = {0, -1, 0};
        b = {-1, 0, 0};
        return;
    }
    double aa = 1.0 / (1.0 + n.z);
    double bb = -n.x * n.y * aa;
    a = {1.0 - n.x * n.x * aa, bb, -n.x};
    b = {bb, 1.0 - n.y * n.y * aa, -n.y};
}

struct Camera {                                                         // camera.rs:48-102
    V3 origin, llc, hor, ver, u, v, forward;
    double lens_radius;
    bool panorama = false;
    void init(const lum_camera& c) {
        double theta = to_radians(c.vfov_degrees);
        double h = std::tan(theta / 2.0);
        double vh = 2.0 * h;
        double vw = c.aspect_ratio * vh;
        V3 w = unit(from(c.look_from) - from(c.look_at));
        u = unit(cross(from(c.vup), w));
        v = cross(w, u);
        hor = u * vw * c.focus_dist;
        ver = v * vh * c.focus_dist;
        origin = from(c.look_from);
        llc = origin - hor / 2.0 - ver / 2.0 - w * c.focus_dist;
        lens_radius = c.aperture / 2.0;
        forward = w * -1.0;                                             // camera.rs:72-74
        panorama = c.panorama != 0;
    }
    Ray get_ray(double s, double t, Sampler& smp) const {
        if (panorama) {                                                 // camera.rs:83-90
            const double pi = 3.14159265358979323846;
            double theta = pi * (1.0 - t);
            double phi = 2.0 * pi * s - pi;
            V3 dir = forward * (std::sin(theta) * std::cos(phi)) + u * (std::sin(theta) * std::sin(phi)) +
                     v * std::cos(theta);
            double time = smp.draw(CALL_CAMERA2, 0);
            return {origin, unit(dir), time};
        }
        V3 rd = random_in_unit_disk(smp) * lens_radius;
        V3 off = u * rd.x + v * rd.y;
        double time = smp.draw(CALL_CAMERA2, 0);
        return {origin + off, llc + hor * s + ver * t - origin - off, time};
    }
};

double mitchell_1d(double x) {                                          // render.rs:220-237
    x = std::fabs(x);
    const double b = 1.0 / 3.0, c = 1.0 / 3.0;
    if (x < 1.0)
        return ((12.0 - 9.0 * b - 6.0 * c) * x * x * x + (-18.0 + 12.0 * b + 6.0 * c) * x * x + (6.0 - 2.0 * b)) / 6.0;
    if (x < 2.0)
        return ((-b - 6.0 * c) * x * x * x + (6.0 * b + 30.0 * c) * x * x + (-12.0 * b - 48.0 * c) * x +
                (8.0 * b + 24.0 * c)) / 6.0;
    return 0.0;
}
double filter_weight(int f, double dx, double dy) {                     // render.rs:201-216
    switch (f) {
        case LUM_FILTER_TRIANGLE:
            return std::fmax(1.0 - std::fabs(dx) * 2.0, 0.0) * std::fmax(1.0 - std::fabs(dy) * 2.0, 0.0);
        case LUM_FILTER_GAUSSIAN: {
            double sigma = 0.35;
            return std::exp(-(dx * dx + dy * dy) / (2.0 * sigma * sigma));
        }
        case LUM_FILTER_MITCHELL: return mitchell_1d(dx * 2.0) * mitchell_1d(dy * 2.0);
        default: return 1.0;
    }
}

// Equirectangular environment map (Background::EnvMap).
struct EnvMap {
    std::vector<float> px;
    uint32_t w = 0, h = 0;
};

V3 background(const lum_render_params& p, const Ray& r, const EnvMap* env) {   // render.rs:73-171
    switch (p.background) {
        case LUM_BG_STARFIELD: {                                        // render.rs:86-112
            V3 ud = unit(r.d);
            double t = 0.5 * (ud.y + 1.0);
            V3 space = v3(0.0, 0.0, 0.02) * (1.0 - t) + v3(0.02, 0.0, 0.05) * t;
            double scale = 500.0 * p.bg_star_density;
            int64_t ix = (int64_t)std::floor(ud.x * scale), iy = (int64_t)std::floor(ud.y * scale),
                    iz = (int64_t)std::floor(ud.z * scale);
            uint64_t hash = ((uint64_t)ix * 73856093ull) ^ ((uint64_t)iy * 19349663ull) ^ ((uint64_t)iz * 83492791ull);
            double star = (double)(hash % 10000) / 10000.0;
            if (!(star > 0.997)) return space;
            double rh = (double)((hash >> 8) % 100) / 100.0;
            V3 c = rh < 0.3 ? v3(1.0, 0.9, 0.8) : (rh < 0.6 ? v3(0.9, 0.9, 1.0) : v3(1, 1, 1));
            return space + c * (star * p.bg_star_brightness);
        }
        case LUM_BG_ENVMAP: {                                           // render.rs:113-151
            if (!env || env->w == 0) return {0, 0, 0};
            V3 ud = unit(r.d);
            double theta = std::acos(-ud.y);
            double phi = std::atan2(-ud.z, ud.x) + PI;
            double u = phi / (2.0 * PI), v = theta / PI;
            double fx = u * env->w - 0.5, fy = v * env->h - 0.5;
            int64_t w = env->w, h = env->h;
            int64_t x0 = (((int64_t)std::floor(fx)) % w + w) % w;
            int64_t y0 = (int64_t)rclamp(std::floor(fy), 0.0, (double)(h - 1));
            int64_t x1 = (x0 + 1) % w, y1 = std::min<int64_t>(y0 + 1, h - 1);
            double tx = fx - std::floor(fx), ty = fy - std::floor(fy);
            auto at = [&](int64_t x, int64_t y) {
                const float* q = &env->px[3 * (size_t)(y * w + x)];
                return v3(q[0], q[1], q[2]);
            };
            V3 c = at(x0, y0) * ((1.0 - tx) * (1.0 - ty)) + at(x1, y0) * (tx * (1.0 - ty)) +
                   at(x0, y1) * ((1.0 - tx) * ty) + at(x1, y1) * (tx * ty);
            return c * p.bg_intensity;
        }
        case LUM_BG_SOLID: return from(p.bg_color);
        case LUM_BG_GRADIENT: {
            V3 ud = unit(r.d);
            double t = 0.5 * (ud.y + 1.0);
            return from(p.bg_color) * (1.0 - t) + from(p.bg_color2) * t;
        }
        case LUM_BG_SUN: {
            V3 ud = unit(r.d);
            double t = 0.5 * (ud.y + 1.0);
            V3 sky = v3(1, 1, 1) * (1.0 - t) + from(p.bg_color2) * t;
            double sd = dot(ud, unit(from(p.bg_dir)));
            if (sd > 0.9995) return from(p.bg_color) * p.bg_intensity;
            if (sd > 0.995) {
                double glow = (sd - 0.995) / (0.9995 - 0.995);
                return sky + from(p.bg_color) * (p.bg_intensity * 0.3 * glow);
            }
            return sky;
        }
        default: {
            V3 ud = unit(r.d);
            double t = 0.5 * (ud.y + 1.0);
            return v3(1, 1, 1) * (1.0 - t) + v3(0.5, 0.7, 1.0) * t;
        }
    }
}

}  // namespace

// ---------------------------------------------------------------------------------------
// Scene: SceneWorld (src/scene.rs:774-839) built from the shared description
// ---------------------------------------------------------------------------------------
struct orc_scene {
    std::vector<Material> mats;
    EnvMap env;
    HPtr bvh;
    std::vector<HPtr> unbounded;
    std::vector<const Hittable*> top;   // every top-level object (tie queries)
    std::vector<Light> lights;
    std::vector<Aabb> object_boxes;
    std::vector<int> object_has_box;
    Camera cam;
    lum_camera cam_desc;

    bool hit(const Ray& r, double tmin, double tmax, HitRecord& rec) const {  // scene.rs:817-834
        double closest = tmax;
        bool any = false;
        HitRecord tmp;
        if (bvh && bvh->hit(r, tmin, closest, tmp)) {
            closest = tmp.t;
            rec = tmp;
            any = true;
        }
        for (auto& o : unbounded) {
            if (o->hit(r, tmin, closest, tmp)) {
                closest = tmp.t;
                rec = tmp;
                any = true;
            }
        }
        return any;
    }
};

namespace {

HPtr make_rect(int plane, double a0, double a1, double b0, double b1, double k, const Material* m, int mi, int32_t id) {
    auto r = std::make_unique<AxisRect>();
    r->plane = plane;
    r->a0 = a0; r->a1 = a1; r->b0 = b0; r->b1 = b1; r->k = k;
    r->mat = m; r->mat_index = mi; r->prim_id = id;
    return r;
}

// rect.rs:128-141: XY(zmax), XY(zmin), XZ(ymax), XZ(ymin), YZ(xmax), YZ(xmin)
void make_box(V3 mn, V3 mx, const Material* m, int mi, int32_t id0, std::vector<HPtr>& out) {
    out.push_back(make_rect(0, mn.x, mx.x, mn.y, mx.y, mx.z, m, mi, id0 + 0));
    out.push_back(make_rect(0, mn.x, mx.x, mn.y, mx.y, mn.z, m, mi, id0 + 1));
    out.push_back(make_rect(1, mn.x, mx.x, mn.z, mx.z, mx.y, m, mi, id0 + 2));
    out.push_back(make_rect(1, mn.x, mx.x, mn.z, mx.z, mn.y, m, mi, id0 + 3));
    out.push_back(make_rect(2, mn.y, mx.y, mn.z, mx.z, mx.x, m, mi, id0 + 4));
    out.push_back(make_rect(2, mn.y, mx.y, mn.z, mx.z, mn.x, m, mi, id0 + 5));
}

HPtr wrap_transform(HPtr obj, const lum_transform& xf) {
    for (int i = 0; i < xf.n_ops && i < LUM_MAX_XF_OPS; ++i) {
        const double* a = xf.arg[i];
        switch (xf.op[i]) {
            case LUM_XF_TRANSLATE: {
                auto t = std::make_unique<Translate>();
                t->inner = std::move(obj);
                t->off = from(a);
                obj = std::move(t);
                break;
            }
            case LUM_XF_ROTATE_X:
            case LUM_XF_ROTATE_Y:
            case LUM_XF_ROTATE_Z: {
                auto r = std::make_unique<Rotate>();
                r->inner = std::move(obj);
                r->ax = xf.op[i] == LUM_XF_ROTATE_X ? 0 : (xf.op[i] == LUM_XF_ROTATE_Y ? 1 : 2);
                r->init(a[0]);
                obj = std::move(r);
                break;
            }
            case LUM_XF_SCALE: {
                auto s = std::make_unique<Scale>();
                s->inner = std::move(obj);
                s->f = std::fabs(a[0]) < 1e-10 ? 1.0 : a[0];
                s->inv_f = 1.0 / s->f;
                obj = std::move(s);
                break;
            }
            default: break;
        }
    }
    return obj;
}

}  // namespace

extern "C" {

int orc_scene_create(const lum_scene_desc* d, orc_scene** out) {
    if (!d || !out) return 1;
    auto* s = new orc_scene();
    s->mats.reserve(d->n_materials);
    for (uint32_t i = 0; i < d->n_materials; ++i) s->mats.push_back(make_material(d->materials[i]));
    if (!link_blends(s->mats, d->materials, d->n_materials)) {
        delete s;
        return 3;
    }
    s->cam_desc = d->camera;
    s->cam.init(d->camera);
    std::vector<HPtr> world;
    int32_t id = 0;
    auto mat = [&](int mi) -> const Material* { return (mi >= 0 && (uint32_t)mi < s->mats.size()) ? &s->mats[mi] : nullptr; };
    for (uint32_t i = 0; i < d->n_objects; ++i) {
        const lum_object& o = d->objects[i];
        const Material* m = mat(o.material);
        HPtr obj;
        bool group_box = false;
        switch (o.kind) {
            case LUM_OBJ_SPHERE: {
                auto sp = std::make_unique<Sphere>();
                sp->c = from(o.p); sp->r = o.p[3];
                sp->mat = m; sp->mat_index = o.material; sp->prim_id = id++;
                obj = std::move(sp);
                break;
            }
            case LUM_OBJ_MOVING_SPHERE: {
                auto sp = std::make_unique<MovingSphere>();
                sp->c0 = from(o.p); sp->c1 = from(o.p + 3); sp->r = o.p[6];
                sp->mat = m; sp->mat_index = o.material; sp->prim_id = id++;
                obj = std::move(sp);
                break;
            }
            case LUM_OBJ_QUAD: {
                auto q = std::make_unique<Quad>();
                q->q = from(o.p); q->u = from(o.p + 3); q->v = from(o.p + 6);
                q->init();
                q->mat = m; q->mat_index = o.material; q->prim_id = id++;
                obj = std::move(q);
                break;
            }
            case LUM_OBJ_RECT_XY:
            case LUM_OBJ_RECT_XZ:
            case LUM_OBJ_RECT_YZ:
                obj = make_rect(o.kind - LUM_OBJ_RECT_XY, o.p[0], o.p[1], o.p[2], o.p[3], o.p[4], m, o.material, id++);
                break;
            case LUM_OBJ_TRIANGLE: {
                auto t = std::make_unique<Triangle>();
                t->v0 = from(o.p); t->v1 = from(o.p + 3); t->v2 = from(o.p + 6);
                t->mat = m; t->mat_index = o.material; t->prim_id = id++;
                obj = std::move(t);
                break;
            }
            case LUM_OBJ_DISK: {
                auto k = std::make_unique<Disk>();
                k->c = from(o.p);
                V3 nn = from(o.p + 3);
                k->n = near_zero(nn) ? v3(0, 1, 0) : unit(nn);
                k->r = o.p[6];
                k->mat = m; k->mat_index = o.material; k->prim_id = id++;
                obj = std::move(k);
                break;
            }
            case LUM_OBJ_PLANE: {
                auto pl = std::make_unique<Plane>();
                pl->init(from(o.p), from(o.p + 3));
                pl->mat = m; pl->mat_index = o.material; pl->prim_id = id++;
                obj = std::move(pl);
                break;
            }
            case LUM_OBJ_BOX: {
                std::vector<HPtr> sides;
                make_box(from(o.p), from(o.p + 3), m, o.material, id, sides);
                id += 6;
                if (o.transform >= 0) {
                    auto lst = std::make_unique<HittableList>();
                    lst->objects = std::move(sides);
                    obj = std::move(lst);
                    group_box = true;
                } else {
                    for (auto& sd : sides) world.push_back(std::move(sd));
                    continue;
                }
                break;
            }
            case LUM_OBJ_FOG_SPHERE:
            case LUM_OBJ_FOG_BOX: {
                auto cm = std::make_unique<ConstantMedium>();
                double density;
                if (o.kind == LUM_OBJ_FOG_SPHERE) {
                    auto sp = std::make_unique<Sphere>();
                    sp->c = from(o.p); sp->r = o.p[3];
                    cm->boundary = std::move(sp);
                    density = o.p[4];
                } else {
                    auto lst = std::make_unique<HittableList>();
                    make_box(from(o.p), from(o.p + 3), nullptr, -1, -1, lst->objects);
                    cm->boundary = std::move(lst);
                    density = o.p[6];
                }
                cm->neg_inv_density = -1.0 / density;
                cm->mat = m; cm->mat_index = o.material; cm->prim_id = id++;
                obj = std::move(cm);
                break;
            }
            default:
                delete s;
                return 2;
        }
        (void)group_box;
        if (o.transform >= 0) {
            if ((uint32_t)o.transform >= d->n_transforms) { delete s; return 1; }
            obj = wrap_transform(std::move(obj), d->transforms[o.transform]);
        }
        world.push_back(std::move(obj));
    }
    for (uint32_t mi = 0; mi < d->n_meshes; ++mi) {
        const lum_mesh& me = d->meshes[mi];
        for (uint32_t t = 0; t < me.n_triangles; ++t) {
            auto tr = std::make_unique<Triangle>();
            const uint32_t* ix = me.indices + 3 * (size_t)t;
            tr->v0 = from(me.positions + 3 * (size_t)ix[0]);
            tr->v1 = from(me.positions + 3 * (size_t)ix[1]);
            tr->v2 = from(me.positions + 3 * (size_t)ix[2]);
            if (me.normals) {
                tr->has_normals = true;
                tr->n0 = from(me.normals + 3 * (size_t)ix[0]);
                tr->n1 = from(me.normals + 3 * (size_t)ix[1]);
                tr->n2 = from(me.normals + 3 * (size_t)ix[2]);
            }
            int mat_i = me.tri_material ? me.tri_material[t] : me.material;
            tr->mat = mat(mat_i); tr->mat_index = mat_i; tr->prim_id = id++;
            world.push_back(std::move(tr));
        }
    }
    for (uint32_t i = 0; i < d->n_lights; ++i) {
        const lum_light& l = d->lights[i];
        s->lights.push_back({l.kind, from(l.p0), from(l.u), from(l.v), from(l.normal), from(l.emission), l.radius});
    }
    // SceneWorld::from_list: bounded objects into the BVH, unbounded into a list.
    std::vector<HPtr> bounded;
    for (auto& o : world) s->top.push_back(o.get());
    for (auto& o : world) {
        Aabb b;
        bool hb = o->bbox(b);
        s->object_boxes.push_back(b);
        s->object_has_box.push_back(hb ? 1 : 0);
        if (hb) bounded.push_back(std::move(o));
        else s->unbounded.push_back(std::move(o));
    }
    if (!bounded.empty()) s->bvh = build_bvh(std::move(bounded));
    *out = s;
    return 0;
}

void orc_scene_destroy(orc_scene* s) { delete s; }

int orc_scene_bbox(const orc_scene* s, int32_t i, double out[6]) {
    if (!s || i < 0 || (size_t)i >= s->object_boxes.size() || !s->object_has_box[i]) return 1;
    const Aabb& b = s->object_boxes[i];
    out[0] = b.mn.x; out[1] = b.mn.y; out[2] = b.mn.z;
    out[3] = b.mx.x; out[4] = b.mx.y; out[5] = b.mx.z;
    return 0;
}

int orc_bvh_stats(const orc_scene* s, uint32_t* n_nodes, uint32_t* depth) {
    uint32_t nn = 0, md = 0;
    if (s->bvh) bvh_stats(s->bvh.get(), 0, nn, md);
    *n_nodes = nn;
    *depth = md;
    return 0;
}

int orc_intersect(const orc_scene* s, const orc_ray* rays, uint32_t n, orc_hit* hits) {
    if (!s || (!rays && n) || (!hits && n)) return 1;
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        const orc_ray& r = rays[i];
        Ray ray{from(r.org), from(r.dir), r.time};
        HitRecord rec;
        orc_hit& h = hits[i];
        std::memset(&h, 0, sizeof(h));
        if (s->hit(ray, r.tmin, r.tmax, rec)) {
            h.t = rec.t; h.u = rec.u; h.v = rec.v;
            h.point[0] = rec.p.x; h.point[1] = rec.p.y; h.point[2] = rec.p.z;
            h.normal[0] = rec.n.x; h.normal[1] = rec.n.y; h.normal[2] = rec.n.z;
            h.prim_id = rec.prim_id;
            h.front_face = rec.front_face ? 1 : 0;
            h.material = rec.mat_index;
        } else {
            h.prim_id = -1;
            h.material = -1;
        }
    }
    return 0;
}

int orc_tie_count(const orc_scene* s, const orc_ray* rays, uint32_t n, double rel, double abs_eps, int32_t* counts) {
    if (!s || (!rays && n) || (!counts && n)) return 1;
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        const orc_ray& r = rays[i];
        Ray ray{from(r.org), from(r.dir), r.time};
        HitRecord rec;
        counts[i] = 0;
        if (!s->hit(ray, r.tmin, r.tmax, rec)) continue;
        double lo = std::fmax(r.tmin, rec.t - rel * rec.t - abs_eps), hi = rec.t + rel * rec.t + abs_eps;
        int c = 0;
        for (const Hittable* o : s->top) {
            HitRecord tmp;
            if (o->hit(ray, lo, hi, tmp)) ++c;
        }
        counts[i] = c;
    }
    return 0;
}

int orc_occluded(const orc_scene* s, const orc_ray* rays, uint32_t n, int32_t* occ) {
    if (!s || (!rays && n) || (!occ && n)) return 1;
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        const orc_ray& r = rays[i];
        Ray ray{from(r.org), from(r.dir), r.time};
        HitRecord rec;
        occ[i] = s->hit(ray, r.tmin, r.tmax, rec) ? 1 : 0;
    }
    return 0;
}

}  // extern "C"

namespace {

struct Counters {
    uint64_t segments = 0, shadow = 0;
};

// render.rs:1346-1466
V3 sample_direct_light(const orc_scene& sc, V3 hp, V3 normal, V3 albedo, Sampler& s, Counters& cnt) {
    const auto& lights = sc.lights;
    if (lights.empty()) return {0, 0, 0};
    uint64_t idx = as_usize(s.draw(CALL_NEE, 1) * (double)lights.size());
    idx = std::min<uint64_t>(idx, lights.size() - 1);
    const Light& L = lights[idx];
    V3 lp, ln, em;
    double area;
    if (L.kind == LUM_LIGHT_SPHERE) {
        V3 to_c = L.p0 - hp;
        double d2c = length_squared(to_c);
        if (d2c < L.r * L.r) return {0, 0, 0};
        double dc = std::sqrt(d2c);
        double stm = L.r / dc;
        double ctm = std::sqrt(std::fmax(1.0 - stm * stm, 0.0));
        double r1 = s.draw(CALL_NEE, 2), r2 = s.draw(CALL_NEE, 3);
        double ct = 1.0 - r1 * (1.0 - ctm);
        double st = std::sqrt(std::fmax(1.0 - ct * ct, 0.0));
        double phi = 2.0 * PI * r2;
        V3 w = to_c / dc;
        V3 a, b;
        build_onb(w, a, b);
        V3 dir = unit(a * (st * std::cos(phi)) + b * (st * std::sin(phi)) + w * ct);
        V3 oc = hp - L.p0;
        double bc = dot(oc, dir);
        double cc = length_squared(oc) - L.r * L.r;
        double disc = bc * bc - cc;
        double t;
        if (disc > 0.0) {
            double sq = std::sqrt(disc);
            double t1 = -bc - sq;
            t = t1 > 0.001 ? t1 : -bc + sq;
        } else {
            t = dc;
        }
        lp = hp + dir * t;
        ln = unit(lp - L.p0);
        double solid = 2.0 * PI * (1.0 - ctm);
        area = solid * t * t / std::fmax(std::fabs(dot(-dir, ln)), 0.001);
        em = L.e;
    } else if (L.kind == LUM_LIGHT_RECT) {
        double a = s.draw(CALL_NEE, 2), b = s.draw(CALL_NEE, 3);
        lp = L.p0 + L.u * a + L.v * b;
        area = length(cross(L.u, L.v));
        ln = L.n;
        em = L.e;
    } else {
        double r1 = s.draw(CALL_NEE, 2), r2 = s.draw(CALL_NEE, 3);
        double r = std::sqrt(r1) * L.r;
        double th = 2.0 * PI * r2;
        V3 w = L.n;
        V3 av = std::fabs(w.x) > 0.9 ? v3(0, 1, 0) : v3(1, 0, 0);
        V3 ut = unit(cross(w, av));
        V3 vt = cross(w, ut);
        lp = L.p0 + ut * (r * std::cos(th)) + vt * (r * std::sin(th));
        area = PI * L.r * L.r;
        ln = L.n;
        em = L.e;
    }
    V3 tl = lp - hp;
    double d2 = length_squared(tl);
    double dist = std::sqrt(d2);
    V3 dir = tl / dist;
    double ct = dot(normal, dir);
    if (ct <= 0.0) return {0, 0, 0};
    double ctl = std::fabs(dot(-dir, ln));
    if (ctl <= 0.001) return {0, 0, 0};
    Ray shadow{hp, dir, 0.0};
    HitRecord tmp;
    cnt.shadow++;
    if (sc.hit(shadow, 0.001, dist - 0.001, tmp)) return {0, 0, 0};
    return hadamard(em, albedo) * (ct * ctl * area * (double)lights.size() / (PI * d2));
}

// render.rs:1472-1537 (recursive form, stream mode)
V3 ray_color_stream(const orc_scene& sc, const lum_render_params& p, const Ray& r, Sampler& s, uint32_t depth,
                    bool skip_emission, Counters& cnt) {
    if (depth == 0) return {0, 0, 0};
    HitRecord h;
    cnt.segments++;
    if (sc.hit(r, 0.001, INF, h)) {
        V3 emitted = skip_emission || !h.mat ? v3(0, 0, 0) : h.mat->emitted(h.u, h.v, h.p);
        Scatter scat;
        if (h.mat && h.mat->scatter(r, h, s, scat)) {
            double mc = std::fmax(std::fmax(scat.att.x, scat.att.y), scat.att.z);
            double surv = rclamp(mc, 0.05, 1.0);
            if (depth < 47 && s.stream->next_f64() > surv) return emitted;
            double rrw = depth < 47 ? 1.0 / surv : 1.0;
            bool use_nee = !h.mat->is_specular() && !sc.lights.empty();
            V3 direct = use_nee ? sample_direct_light(sc, h.p, h.n, scat.att, s, cnt) : v3(0, 0, 0);
            V3 indirect = hadamard(scat.att, ray_color_stream(sc, p, scat.ray, s, depth - 1, use_nee, cnt)) * rrw;
            V3 res = emitted + direct + indirect;
            if (std::isnan(res.x) || std::isnan(res.y) || std::isnan(res.z)) return {0, 0, 0};
            return res;
        }
        return emitted;
    }
    return background(p, r, &sc.env);
}

// Keyed mode: the device estimator (iterative; draws addressed per bounce).  Same terms as
// the recursion above: L = sum_j B_j (e_j + d_j) with B_{j+1} = B_j * att_j * rrw_j; a NaN
// in level j drops that level and everything deeper (the recursion's guard).
V3 ray_color_keyed(const orc_scene& sc, const lum_render_params& p, Ray r, Sampler& s, uint32_t max_depth,
                   Counters& cnt) {
    V3 L{0, 0, 0}, B{1, 1, 1};
    bool skip = false;
    for (uint32_t b = 0; b < max_depth; ++b) {
        uint32_t depth = max_depth - b;
        s.begin_bounce(b);
        HitRecord h;
        cnt.segments++;
        if (!sc.hit(r, 0.001, INF, h)) {
            L += hadamard(B, background(p, r, &sc.env));
            break;
        }
        // Non-finite vertex: the recursion's NaN guard zeroes this level and deeper.
        if (!std::isfinite(h.p.x) || !std::isfinite(h.p.y) || !std::isfinite(h.p.z)) break;
        V3 e = skip || !h.mat ? v3(0, 0, 0) : h.mat->emitted(h.u, h.v, h.p);
        Scatter scat;
        if (!h.mat || !h.mat->scatter(r, h, s, scat)) {
            L += hadamard(B, e);
            break;
        }
        double dl2 = length_squared(scat.ray.d);
        if (!(dl2 > 0.0) || !std::isfinite(dl2)) {   // zero-radius in-sphere draw: next level is NaN
            L += hadamard(B, e);
            break;
        }
        double mc = std::fmax(std::fmax(scat.att.x, scat.att.y), scat.att.z);
        double surv = rclamp(mc, 0.05, 1.0);
        if (depth < 47 && s.draw(CALL_NEE, 0) > surv) {
            L += hadamard(B, e);
            break;
        }
        double rrw = depth < 47 ? 1.0 / surv : 1.0;
        bool use_nee = !h.mat->is_specular() && !sc.lights.empty();
        V3 dl = use_nee ? sample_direct_light(sc, h.p, h.n, scat.att, s, cnt) : v3(0, 0, 0);
        V3 term = e + dl;
        V3 nb = hadamard(B, scat.att) * rrw;
        if (std::isnan(term.x) || std::isnan(term.y) || std::isnan(term.z) || std::isnan(nb.x) ||
            std::isnan(nb.y) || std::isnan(nb.z))
            break;
        L += hadamard(B, term);
        B = nb;
        skip = use_nee;
        r = scat.ray;
    }
    return L;
}

struct Frame {
    size_t full_w, full_h, crop_x, crop_y, w, h;
    uint32_t sqrt_spp, s_begin, s_end;
};

Frame frame_of(const lum_render_params& p) {
    Frame f;
    f.full_w = std::max<uint32_t>(p.width, 1);
    f.full_h = std::max<uint32_t>(p.height, 1);
    if (p.has_crop) {                                                   // render.rs:1575-1583
        f.crop_x = std::min<size_t>(p.crop[0], f.full_w);
        f.crop_y = std::min<size_t>(p.crop[1], f.full_h);
        f.w = std::min<size_t>(p.crop[2], f.full_w);
        f.h = std::min<size_t>(p.crop[3], f.full_h);
    } else {
        f.crop_x = f.crop_y = 0;
        f.w = f.full_w;
        f.h = f.full_h;
    }
    f.sqrt_spp = (uint32_t)std::ceil(std::sqrt((double)p.samples_per_pixel));
    uint32_t total = f.sqrt_spp * f.sqrt_spp;
    f.s_begin = std::min(p.sample_begin, total);
    f.s_end = p.sample_count ? std::min(total, f.s_begin + p.sample_count) : total;
    return f;
}

V3 clamp_sample(V3 smp) {                                               // render.rs:1692-1697
    double lum = 0.2126 * smp.x + 0.7152 * smp.y + 0.0722 * smp.z;
    return lum > 100.0 ? smp * (100.0 / lum) : smp;
}

V3 trace_sample(const orc_scene& sc, const lum_render_params& p, const Ray& ray, Sampler& s, Counters& cnt) {
    return s.mode == ORC_MODE_STREAM ? ray_color_stream(sc, p, ray, s, p.max_depth, false, cnt)
                                     : ray_color_keyed(sc, p, ray, s, p.max_depth, cnt);
}

// One sample at the pixel centre after the time limit (render.rs:1612-1622): the lens and
// time draws as usual (stratum 0 in keyed mode), luminance-clamped, no filter.
V3 expired_sample(const orc_scene& sc, const lum_render_params& p, const Frame& f, Sampler& s, size_t gi, double y,
                  Counters& cnt) {
    s.stratum = 0;
    s.begin_bounce(0);
    double uc = ((double)gi + 0.5) / (double)(f.full_w - 1);
    double vc = (y + 0.5) / (double)(f.full_h - 1);
    Ray ray = sc.cam.get_ray(uc, vc, s);
    return clamp_sample(trace_sample(sc, p, ray, s, cnt));
}

// Adaptive sampling (render.rs:1624-1678): strata in order sy-major; Welford's running mean
// and squared deviations of the clamped luminance; stop once n >= min_samples, n > 1 and the
// standard error sqrt(var / n) is below the threshold.  The pixel is the running mean of the
// clamped samples (no pixel filter).
V3 adaptive_pixel(const orc_scene& sc, const lum_render_params& p, const Frame& f, Sampler& s, size_t gi, double y,
                  uint32_t min_samples, Counters& cnt, uint64_t& paths) {
    V3 mean{0, 0, 0};
    double m2_lum = 0.0, mean_lum = 0.0;
    uint32_t n = 0;
    const uint32_t total = f.sqrt_spp * f.sqrt_spp;
    for (uint32_t st = 0; st < total; ++st) {
        uint32_t sx = st % f.sqrt_spp, sy = st / f.sqrt_spp;
        s.stratum = st;
        s.begin_bounce(0);
        double uc = ((double)gi + ((double)sx + s.draw(CALL_CAMERA, 0)) / (double)f.sqrt_spp) / (double)(f.full_w - 1);
        double vc = (y + ((double)sy + s.draw(CALL_CAMERA, 1)) / (double)f.sqrt_spp) / (double)(f.full_h - 1);
        Ray ray = sc.cam.get_ray(uc, vc, s);
        V3 cl = clamp_sample(trace_sample(sc, p, ray, s, cnt));
        ++n;
        double lum = 0.2126 * cl.x + 0.7152 * cl.y + 0.0722 * cl.z;
        double d1 = lum - mean_lum;
        mean_lum += d1 / (double)n;
        double d2 = lum - mean_lum;
        m2_lum += d1 * d2;
        mean = mean + (cl - mean) / (double)n;
        if (n >= min_samples && n > 1) {
            double var = m2_lum / (double)(n - 1);
            if (std::sqrt(var / (double)n) < p.adaptive_threshold) break;
        }
    }
    paths += n;
    return mean;
}

}  // namespace

extern "C" {

}  // extern "C"

namespace {

// The sample loop of render.rs:1598-1706.  expire: 0 = the wall-clock time limit of the
// params (checked when a row starts, render.rs:1601-1605), 1 = every row starts after it.
// row_list (n_list entries, output row index = position in the list) renders an arbitrary set
// of rows in parallel instead of the range [row_begin, row_end).
// sums (4 doubles per pixel): the pixel's filter-weighted clamped radiance and filter-weight
// sums before the division of render.rs:1705 (plain sample loop only).
int render_rows(const orc_scene* sc, const lum_render_params* pp, int mode, int threads, uint32_t row_begin,
                uint32_t row_end, double* out, orc_stats* stats, int expire, const uint32_t* row_list = nullptr,
                uint32_t n_list = 0, double* sums = nullptr) {
    if (!sc || !pp || !out) return 1;
    const lum_render_params& p = *pp;
    Frame f = frame_of(p);
    const uint32_t actual_spp = f.sqrt_spp * f.sqrt_spp;
    if (mode == ORC_MODE_STREAM && (f.s_begin != 0 || f.s_end != actual_spp)) return 2;
    if (p.adaptive && (f.s_begin != 0 || f.s_end != actual_spp)) return 3;
    // render.rs:1592: minimum samples before the variance test
    const uint32_t min_samples = p.adaptive ? std::max<uint32_t>(actual_spp / 4, 16) : 0;
    std::atomic<bool> expired{expire != 0};
    row_end = std::min<uint32_t>(row_end, (uint32_t)f.h);
    if (row_list) {
        for (uint32_t k = 0; k < n_list; ++k)
            if (row_list[k] >= (uint32_t)f.h) return 4;
        row_begin = 0;
        row_end = n_list;
    }
    uint64_t segs = 0, shadows = 0, paths = 0;
    auto t0 = std::chrono::steady_clock::now();
#ifdef _OPENMP
    int nt = threads > 0 ? threads : omp_get_max_threads();
#else
    int nt = 1;
#endif
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt) reduction(+ : segs, shadows, paths)
    for (int64_t k = row_begin; k < (int64_t)row_end; ++k) {
        const int64_t j = k;                                            // output row
        size_t gj = (size_t)(row_list ? row_list[k] : k) + f.crop_y;
        Xoshiro rng((uint64_t)gj * p.seed);                             // render.rs:1608 (wrapping)
        Sampler s;
        s.mode = mode;
        s.stream = &rng;
        s.key[0] = (uint32_t)p.seed;
        s.key[1] = (uint32_t)(p.seed >> 32);
        double y = (double)(f.full_h - 1 - gj);
        Counters cnt;
        if (p.time_limit > 0.0 &&
            std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() > p.time_limit)
            expired.store(true, std::memory_order_relaxed);
        const bool row_expired = expired.load(std::memory_order_relaxed);
        for (size_t i = 0; i < f.w; ++i) {
            size_t gi = i + f.crop_x;
            V3 color{0, 0, 0};
            double tw = 0.0;
            s.pixel = (uint32_t)(gj * f.full_w + gi);
            double* o = out + ((size_t)j * f.w + i) * 3;
            if (row_expired || p.adaptive) {
                V3 px = row_expired ? expired_sample(*sc, p, f, s, gi, y, cnt)
                                    : adaptive_pixel(*sc, p, f, s, gi, y, min_samples, cnt, paths);
                paths += row_expired ? 1 : 0;
                o[0] = px.x * p.exposure;
                o[1] = px.y * p.exposure;
                o[2] = px.z * p.exposure;
                continue;
            }
            for (uint32_t st = f.s_begin; st < f.s_end; ++st) {
                uint32_t sx = st % f.sqrt_spp, sy = st / f.sqrt_spp;
                s.stratum = st;
                s.begin_bounce(0);
                double jx = ((double)sx + s.draw(CALL_CAMERA, 0)) / (double)f.sqrt_spp;  // render.rs:1685-1688
                double jy = ((double)sy + s.draw(CALL_CAMERA, 1)) / (double)f.sqrt_spp;
                double uc = ((double)gi + jx) / (double)(f.full_w - 1);
                double vc = (y + jy) / (double)(f.full_h - 1);
                Ray ray = sc->cam.get_ray(uc, vc, s);
                V3 smp = mode == ORC_MODE_STREAM ? ray_color_stream(*sc, p, ray, s, p.max_depth, false, cnt)
                                                 : ray_color_keyed(*sc, p, ray, s, p.max_depth, cnt);
                double lum = 0.2126 * smp.x + 0.7152 * smp.y + 0.0722 * smp.z;  // render.rs:1692-1697
                V3 cl = lum > 100.0 ? smp * (100.0 / lum) : smp;
                double w = filter_weight(p.pixel_filter, jx - 0.5, jy - 0.5);
                color += cl * w;
                tw += w;
            }
            paths += f.s_end - f.s_begin;
            if (sums) {
                double* q = sums + ((size_t)j * f.w + i) * 4;
                q[0] = color.x;
                q[1] = color.y;
                q[2] = color.z;
                q[3] = tw;
            }
            V3 px = tw > 0.0 ? color / tw : color;
            o[0] = px.x * p.exposure;
            o[1] = px.y * p.exposure;
            o[2] = px.z * p.exposure;
        }
        segs += cnt.segments;
        shadows += cnt.shadow;
    }
    auto t1 = std::chrono::steady_clock::now();
    if (stats) {
        stats->paths = paths;
        stats->segments = segs;
        stats->shadow_rays = shadows;
        stats->seconds = std::chrono::duration<double>(t1 - t0).count();
        stats->threads = nt;
    }
    return 0;
}

}  // namespace

extern "C" {

int orc_render_rows(const orc_scene* sc, const lum_render_params* pp, int mode, int threads, uint32_t row_begin,
                    uint32_t row_end, double* out, orc_stats* stats) {
    return render_rows(sc, pp, mode, threads, row_begin, row_end, out, stats, 0);
}

int orc_render_sums(const orc_scene* sc, const lum_render_params* p, int mode, int threads, double* sums,
                    orc_stats* st) {
    if (!sums || (p && (p->adaptive || p->time_limit > 0.0))) return 1;
    Frame f = frame_of(*p);
    std::vector<double> img((size_t)f.w * f.h * 3);
    return render_rows(sc, p, mode, threads, 0, (uint32_t)f.h, img.data(), st, 0, nullptr, 0, sums);
}

int orc_render_row_list(const orc_scene* sc, const lum_render_params* pp, int mode, int threads,
                        const uint32_t* rows, uint32_t n_rows, double* out, orc_stats* stats) {
    if (!rows && n_rows) return 1;
    return render_rows(sc, pp, mode, threads, 0, 0, out, stats, 0, rows, n_rows);
}

int orc_render(const orc_scene* sc, const lum_render_params* p, int mode, int threads, double* out, orc_stats* st) {
    Frame f = frame_of(*p);
    return render_rows(sc, p, mode, threads, 0, (uint32_t)f.h, out, st, 0);
}

int orc_render_expired(const orc_scene* sc, const lum_render_params* p, int mode, int threads, double* out,
                       orc_stats* st) {
    Frame f = frame_of(*p);
    return render_rows(sc, p, mode, threads, 0, (uint32_t)f.h, out, st, 1);
}

int orc_scene_set_envmap(orc_scene* sc, const float* rgb, uint32_t w, uint32_t h) {
    if (!sc) return 1;
    if (!rgb || !w || !h) {
        sc->env = EnvMap{};
        return 0;
    }
    sc->env.px.assign(rgb, rgb + 3 * (size_t)w * h);
    sc->env.w = w;
    sc->env.h = h;
    return 0;
}

// AOV passes (render.rs:3508-3568): one ray per pixel through the pixel centre.  Stream mode:
// the reference's per-pixel SmallRng seeded with (j * W + i) * seed (wrapping); keyed mode:
// the draws of (pixel, stratum 0, bounce 0) as on the device.
int orc_render_aov(const orc_scene* sc, const lum_render_params* pp, int mode, double* depth, uint8_t* normals,
                   uint8_t* albedo) {
    if (!sc || !pp) return 1;
    const lum_render_params& p = *pp;
    Frame f = frame_of(p);
    auto to_u8 = [](double x) -> uint8_t {            // Rust `as u8`: NaN -> 0, saturating
        if (!(x > 0.0)) return 0;
        if (x >= 255.0) return 255;
        return (uint8_t)x;
    };
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t j = 0; j < (int64_t)f.h; ++j) {
        size_t gj = (size_t)j + f.crop_y;
        double y = (double)(f.full_h - 1 - gj);
        for (size_t i = 0; i < f.w; ++i) {
            size_t gi = i + f.crop_x;
            size_t o = (size_t)j * f.w + i;
            Xoshiro rng(((uint64_t)gj * (uint64_t)f.full_w + (uint64_t)gi) * p.seed);
            Sampler s;
            s.mode = mode;
            s.stream = &rng;
            s.key[0] = (uint32_t)p.seed;
            s.key[1] = (uint32_t)(p.seed >> 32);
            s.pixel = (uint32_t)(gj * f.full_w + gi);
            s.stratum = 0;
            s.begin_bounce(0);
            double uc = ((double)gi + 0.5) / (double)(f.full_w - 1);
            double vc = (y + 0.5) / (double)(f.full_h - 1);
            Ray ray = sc->cam.get_ray(uc, vc, s);
            HitRecord h;
            double dv = 0.0;
            uint8_t nb[3] = {0, 0, 0}, ab[3] = {0, 0, 0};
            if (sc->hit(ray, 0.001, INF, h)) {
                dv = (double)(float)h.t;
                const double n[3] = {h.n.x, h.n.y, h.n.z};
                for (int c = 0; c < 3; ++c) nb[c] = to_u8(rclamp((n[c] * 0.5 + 0.5) * 255.0, 0.0, 255.0));
                Scatter sct;
                if (h.mat && h.mat->scatter(ray, h, s, sct)) {
                    const double a[3] = {sct.att.x, sct.att.y, sct.att.z};
                    for (int c = 0; c < 3; ++c) ab[c] = to_u8(rclamp(a[c], 0.0, 1.0) * 255.0);
                } else if (h.mat) {
                    V3 e = h.mat->emitted(h.u, h.v, h.p);
                    double me = std::fmax(std::fmax(e.x, std::fmax(e.y, e.z)), 1.0);
                    const double a[3] = {e.x, e.y, e.z};
                    for (int c = 0; c < 3; ++c) ab[c] = to_u8(rclamp(a[c] / me * 255.0, 0.0, 255.0));
                }
            }
            if (depth) depth[o] = dv;
            for (int c = 0; c < 3; ++c) {
                if (normals) normals[3 * o + c] = nb[c];
                if (albedo) albedo[3 * o + c] = ab[c];
            }
        }
    }
    return 0;
}

int orc_scatter_in(const lum_material* mats, uint32_t n_mats, uint32_t index, const double ray[7], const double hp[3],
                   const double on[3], double t, double u, double v, uint64_t seed, int n_iter, double* out) {
    if (!mats || index >= n_mats) return 1;
    std::vector<Material> ms;
    ms.reserve(n_mats);
    for (uint32_t i = 0; i < n_mats; ++i) ms.push_back(make_material(mats[i]));
    if (!link_blends(ms, mats, n_mats)) return 2;
    const Material& m = ms[index];
    Xoshiro rng(seed);
    Sampler s;
    s.mode = ORC_MODE_STREAM;
    s.stream = &rng;
    Ray r{from(ray), from(ray + 3), ray[6]};
    HitRecord h;
    h.p = from(hp);
    h.t = t;
    h.u = u;
    h.v = v;
    set_face(h, r, from(on));
    h.mat = &m;
    for (int i = 0; i < n_iter; ++i) {
        Scatter sc;
        bool ok = m.scatter(r, h, s, sc);
        double* o = out + (size_t)i * 11;
        o[0] = ok ? 1.0 : 0.0;
        o[1] = sc.ray.d.x; o[2] = sc.ray.d.y; o[3] = sc.ray.d.z;
        o[4] = sc.att.x; o[5] = sc.att.y; o[6] = sc.att.z;
        o[7] = h.front_face ? 1.0 : 0.0;
        o[8] = sc.ray.o.x; o[9] = sc.ray.o.y; o[10] = sc.ray.o.z;
        if (!ok) o[1] = o[2] = o[3] = o[4] = o[5] = o[6] = o[8] = o[9] = o[10] = 0.0;
    }
    return 0;
}

int orc_scatter(const lum_material* lm, const double ray[7], const double hp[3], const double on[3], double t,
                double u, double v, uint64_t seed, int n_iter, double* out) {
    std::vector<double> full((size_t)std::max(n_iter, 0) * 11);
    int rc = orc_scatter_in(lm, 1, 0, ray, hp, on, t, u, v, seed, n_iter, full.data());
    if (rc) return rc;
    for (int i = 0; i < n_iter; ++i)
        for (int k = 0; k < 8; ++k) out[(size_t)i * 8 + k] = full[(size_t)i * 11 + k];
    return 0;
}

double orc_emitted(const lum_material* mats, uint32_t n_mats, uint32_t index, double u, double v,
                   const double p[3]) {
    std::vector<Material> ms;
    for (uint32_t i = 0; i < n_mats; ++i) ms.push_back(make_material(mats[i]));
    if (index >= n_mats || !link_blends(ms, mats, n_mats)) return NAN;
    V3 e = ms[index].emitted(u, v, from(p));
    return e.x + e.y + e.z;
}

int orc_is_specular(const lum_material* m) { return make_material(*m).is_specular() ? 1 : 0; }

double orc_thin_film(double cos_theta, double thickness, double film_ior, int channel) {
    V3 c = Material::thin_film(cos_theta, thickness, film_ior);
    return channel == 0 ? c.x : (channel == 1 ? c.y : c.z);
}

double orc_schlick(double c, double r) { return Material::reflectance(c, r); }

double orc_ggx_d(double ndh, double alpha) {                            // material.rs:273-277
    double a2 = alpha * alpha;
    double den = ndh * ndh * (a2 - 1.0) + 1.0;
    return a2 / (PI * den * den);
}

int orc_camera_ray(const lum_camera* c, double s, double t, uint64_t seed, double out[7]) {
    Camera cam;
    cam.init(*c);
    Xoshiro rng(seed);
    Sampler smp;
    smp.mode = ORC_MODE_STREAM;
    smp.stream = &rng;
    Ray r = cam.get_ray(s, t, smp);
    out[0] = r.o.x; out[1] = r.o.y; out[2] = r.o.z;
    out[3] = r.d.x; out[4] = r.d.y; out[5] = r.d.z;
    out[6] = r.time;
    return 0;
}

double orc_filter_weight(int f, double dx, double dy) { return filter_weight(f, dx, dy); }

int orc_sample_direct_light(const orc_scene* sc, const double p[3], const double n[3], const double alb[3],
                            uint64_t seed, int n_iter, double* out) {
    Xoshiro rng(seed);
    Sampler s;
    s.mode = ORC_MODE_STREAM;
    s.stream = &rng;
    Counters cnt;
    for (int i = 0; i < n_iter; ++i) {
        V3 r = sample_direct_light(*sc, from(p), from(n), from(alb), s, cnt);
        out[3 * i] = r.x; out[3 * i + 1] = r.y; out[3 * i + 2] = r.z;
    }
    return 0;
}

int orc_aabb_hit(const double mn[3], const double mx[3], const double ray[7], double tmin, double tmax) {
    Aabb b{from(mn), from(mx)};
    Ray r{from(ray), from(ray + 3), ray[6]};
    return b.hit(r, tmin, tmax) ? 1 : 0;
}

void orc_refract(const double v[3], const double n[3], double eta, double out[3]) {
    V3 r = refract(from(v), from(n), eta);
    out[0] = r.x; out[1] = r.y; out[2] = r.z;
}
void orc_reflect(const double v[3], const double n[3], double out[3]) {
    V3 r = reflect(from(v), from(n));
    out[0] = r.x; out[1] = r.y; out[2] = r.z;
}

void orc_stream_u64(uint64_t seed, uint32_t n, uint64_t* out) {
    Xoshiro r(seed);
    for (uint32_t i = 0; i < n; ++i) out[i] = r.next_u64();
}
void orc_stream_f64(uint64_t seed, uint32_t n, double* out) {
    Xoshiro r(seed);
    for (uint32_t i = 0; i < n; ++i) out[i] = r.next_f64();
}
void orc_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) { philox4x32_10(ctr, key, out); }
void orc_xoshiro_from_state(const uint64_t state[4], uint32_t n, uint64_t* out) {
    Xoshiro r(state[0], state[1], state[2], state[3]);
    for (uint32_t i = 0; i < n; ++i) out[i] = r.next_u64();
}
void orc_seed_state(uint64_t seed, uint64_t out[4]) {
    Xoshiro r(seed);
    for (int i = 0; i < 4; ++i) out[i] = r.s[i];
}

}  // extern "C"

// =======================================================================================
// f64 adjoint of the keyed estimator (the checker for the device's lum_backward).
//
// Forward-mode dual numbers over groups of 16 material parameters at a time.  Each
// path is re-traced in f64 and the primal values take every branch (Russian roulette, the
// microfacet lobe, the primitive hit, shadow visibility), so the result is the derivative of
// the estimator with those decisions held.  With detach = 1 the Russian-roulette survival and
// the microfacet lobe probability are constants (the device adjoint's estimator: the terms
// their derivatives add have zero mean); detach = 0 keeps them, which is the plain derivative
// of the per-sample image and is what a tiny-step finite difference of orc_render measures.
// The hit point moves on the tangent plane of a flat primitive and is held on curved ones;
// shading normals are constant.  Parameters: albedo of Lambertian / Metal / Microfacet (the
// texel used), Microfacet roughness, and emission (colour * intensity) of Emissive materials
// and of the NEE lights that carry them (light_material).  Metal, Dielectric and Isotropic
// scatter directions, and sphere-light NEE terms as functions of the shading point, are held.
// =======================================================================================
namespace {

constexpr int ND = 16;
struct Dd {
    double v = 0.0;
    double d[ND] = {};
};
inline Dd dcst(double x) {
    Dd r;
    r.v = x;
    return r;
}
inline Dd operator+(const Dd& a, const Dd& b) {
    Dd r;
    r.v = a.v + b.v;
    for (int k = 0; k < ND; ++k) r.d[k] = a.d[k] + b.d[k];
    return r;
}
inline Dd operator-(const Dd& a, const Dd& b) {
    Dd r;
    r.v = a.v - b.v;
    for (int k = 0; k < ND; ++k) r.d[k] = a.d[k] - b.d[k];
    return r;
}
inline Dd operator-(const Dd& a) {
    Dd r;
    r.v = -a.v;
    for (int k = 0; k < ND; ++k) r.d[k] = -a.d[k];
    return r;
}
inline Dd operator*(const Dd& a, const Dd& b) {
    Dd r;
    r.v = a.v * b.v;
    for (int k = 0; k < ND; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
    return r;
}
inline Dd operator*(const Dd& a, double s) {
    Dd r;
    r.v = a.v * s;
    for (int k = 0; k < ND; ++k) r.d[k] = a.d[k] * s;
    return r;
}
inline Dd operator*(double s, const Dd& a) { return a * s; }
inline Dd operator+(const Dd& a, double s) {
    Dd r = a;
    r.v += s;
    return r;
}
inline Dd operator+(double s, const Dd& a) { return a + s; }
inline Dd operator-(const Dd& a, double s) { return a + (-s); }
inline Dd operator-(double s, const Dd& a) { return (-a) + s; }
inline Dd operator/(const Dd& a, const Dd& b) {
    Dd r;
    r.v = a.v / b.v;
    for (int k = 0; k < ND; ++k) r.d[k] = (a.d[k] - r.v * b.d[k]) / b.v;
    return r;
}
inline Dd operator/(const Dd& a, double s) { return a * (1.0 / s); }
inline Dd operator/(double s, const Dd& b) { return dcst(s) / b; }
inline Dd dsqrt(const Dd& a) {
    Dd r;
    r.v = std::sqrt(a.v);
    double h = r.v > 0.0 ? 0.5 / r.v : 0.0;
    for (int k = 0; k < ND; ++k) r.d[k] = a.d[k] * h;
    return r;
}
inline Dd dmax(const Dd& a, double lo) { return a.v >= lo ? a : dcst(lo); }
inline Dd dclamp(const Dd& a, double lo, double hi) { return a.v < lo ? dcst(lo) : (a.v > hi ? dcst(hi) : a); }
inline Dd dabs(const Dd& a) { return a.v >= 0.0 ? a : -a; }
inline Dd dmax3(const Dd& a, const Dd& b, const Dd& c) {
    const Dd& m = a.v >= b.v ? a : b;
    return m.v >= c.v ? m : c;
}

struct DV {
    Dd x, y, z;
};
inline DV dv(V3 a) { return {dcst(a.x), dcst(a.y), dcst(a.z)}; }
inline V3 val(const DV& a) { return {a.x.v, a.y.v, a.z.v}; }
inline DV operator+(const DV& a, const DV& b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline DV operator-(const DV& a, const DV& b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline DV operator-(const DV& a) { return {-a.x, -a.y, -a.z}; }
inline DV operator*(const DV& a, const Dd& s) { return {a.x * s, a.y * s, a.z * s}; }
inline DV operator*(const DV& a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline DV operator*(V3 a, const Dd& s) { return {s * a.x, s * a.y, s * a.z}; }
inline DV had(const DV& a, const DV& b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
inline Dd ddot(const DV& a, const DV& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline Dd ddot(V3 a, const DV& b) { return b.x * a.x + b.y * a.y + b.z * a.z; }
inline DV dunit(const DV& a) { return a * (1.0 / dsqrt(ddot(a, a))); }
inline bool dnan(const DV& a) { return std::isnan(a.x.v) || std::isnan(a.y.v) || std::isnan(a.z.v); }

// Parameter layout: albedo 3*m+c, roughness 3*n+m, emission 4*n+3*m+c (n materials).
struct AdjCtx {
    const orc_scene* sc;
    const lum_render_params* p;
    const int32_t* light_mat;
    int n_mat;
    int begin;
    bool detach;
    bool score;                // with detach: add the NEE survival score term
    const double* direction;   // non-null: one slot, seeded with this direction over all parameters
    Dd param(double v, int idx) const {
        Dd r = dcst(v);
        if (direction) {
            r.d[0] = direction[idx];
            return r;
        }
        int k = idx - begin;
        if (k >= 0 && k < ND) r.d[k] = 1.0;
        return r;
    }
    DV albedo(int m, V3 a) const { return {param(a.x, 3 * m), param(a.y, 3 * m + 1), param(a.z, 3 * m + 2)}; }
    Dd rough(int m, double r) const { return param(r, 3 * n_mat + m); }
    DV emission(int m, V3 e) const {
        if (m < 0) return dv(e);
        return {param(e.x, 4 * n_mat + 3 * m), param(e.y, 4 * n_mat + 3 * m + 1), param(e.z, 4 * n_mat + 3 * m + 2)};
    }
};

inline DV dfresnel(const Dd& cos_theta, const DV& f0) {                // material.rs:291-294
    Dd m = dmax(1.0 - cos_theta, 0.0);
    Dd t = m * m * m * m * m;
    return {f0.x * (1.0 - t) + t, f0.y * (1.0 - t) + t, f0.z * (1.0 - t) + t};
}

// Attenuation and outgoing direction of a scatter whose primal outcome is `sc` (material.rs).
// att uses the lobe probability as the context says (held or not); att_full never holds it.
void scatter_dual(const AdjCtx& C, const Material& m, int mi, const HitRecord& h, const DV& d_in, Sampler& s,
                  const Scatter& sc, DV& att, DV& att_full, DV& dir) {
    dir = dv(sc.ray.d);
    switch (m.kind) {
        case LUM_MAT_LAMBERTIAN:
            att = C.albedo(mi, m.tex.value(h.u, h.v, h.p));
            att_full = att;
            return;
        case LUM_MAT_METAL:
            att = C.albedo(mi, m.albedo);
            att_full = att;
            return;
        case LUM_MAT_MICROFACET: {                                     // material.rs:328-390
            V3 n = h.n;
            DV alb = C.albedo(mi, m.tex.value(h.u, h.v, h.p));
            Dd rr = C.rough(mi, m.roughness);
            DV v = dunit(-d_in);
            Dd ndv = dmax(ddot(n, v), 0.001);
            DV f0 = DV{dcst(0.04 * (1.0 - m.metallic)), dcst(0.04 * (1.0 - m.metallic)), dcst(0.04 * (1.0 - m.metallic))} +
                    alb * m.metallic;
            DV fw = dfresnel(ndv, f0);
            Dd sp_full = dclamp((fw.x + fw.y + fw.z) / 3.0, 0.1, 0.9);
            Dd sp = C.detach ? dcst(sp_full.v) : sp_full;
            if (s.draw(CALL_SCATTER, 0) < sp.v) {
                double r1 = s.draw(CALL_SCATTER, 1), r2 = s.draw(CALL_SCATTER, 2);
                Dd alpha = rr * rr;
                Dd tan2 = alpha * alpha * (r1 / (1.0 - r1 + 1e-10));     // tan^2 of atan(...) (material.rs:297-319)
                Dd ct = 1.0 / dsqrt(1.0 + tan2);
                Dd st = dsqrt(tan2) * ct;
                double phi = 2.0 * PI * r2;
                V3 up = std::fabs(n.y) < 0.999 ? v3(0, 1, 0) : v3(1, 0, 0);
                V3 tg = unit(cross(up, n));
                V3 bt = cross(n, tg);
                DV hh = dunit(tg * (st * std::cos(phi)) + bt * (st * std::sin(phi)) + n * ct);
                Dd vh = ddot(v, hh);
                dir = hh * (vh * 2.0) - v;
                Dd ndl = ddot(n, dir);
                Dd ndh = dmax(ddot(n, hh), 0.0);
                Dd vdh = dmax(vh, 0.0);
                Dd k = (rr + 1.0) * (rr + 1.0) / 8.0;                    // material.rs:280-288
                Dd g = (ndv / (ndv * (1.0 - k) + k)) * (ndl / (ndl * (1.0 - k) + k));
                DV f = dfresnel(vdh, f0);
                if (ndh.v > 0.001) {
                    Dd c = g * vdh / (ndv * ndh);
                    att = f * (c / sp);
                    att_full = f * (c / sp_full);
                } else {
                    att = att_full = dv(v3(0, 0, 0));
                }
                return;
            }
            DV kd = DV{1.0 - fw.x, 1.0 - fw.y, 1.0 - fw.z} * (1.0 - m.metallic);
            att = had(kd, alb) * (1.0 / (1.0 - sp));
            att_full = had(kd, alb) * (1.0 / (1.0 - sp_full));
            return;
        }
        default:
            att = att_full = dv(sc.att);
            return;
    }
}

// render.rs:1346-1466 with the shading point as a dual; the light point, visibility and the
// early-outs come from the primal.
DV nee_dual(const AdjCtx& C, const DV& hp, V3 normal, const DV& att, Sampler& s, Counters& cnt) {
    const orc_scene& sc = *C.sc;
    const auto& lights = sc.lights;
    V3 hv = val(hp);
    V3 prim = sample_direct_light(sc, hv, normal, val(att), s, cnt);
    if (prim.x == 0.0 && prim.y == 0.0 && prim.z == 0.0) return dv(v3(0, 0, 0));
    uint64_t idx = as_usize(s.draw(CALL_NEE, 1) * (double)lights.size());
    idx = std::min<uint64_t>(idx, lights.size() - 1);
    const Light& L = lights[idx];
    DV em = C.emission(C.light_mat ? C.light_mat[idx] : -1, L.e);
    if (L.kind == LUM_LIGHT_SPHERE) {
        // held constant in the shading point: the primal factor prim / (em * att)
        V3 a = val(att);
        double gx = em.x.v * a.x != 0.0 ? prim.x / (em.x.v * a.x) : 0.0;
        double gy = em.y.v * a.y != 0.0 ? prim.y / (em.y.v * a.y) : 0.0;
        double gz = em.z.v * a.z != 0.0 ? prim.z / (em.z.v * a.z) : 0.0;
        DV ea = had(em, att);
        return {ea.x * gx, ea.y * gy, ea.z * gz};
    }
    V3 lp;
    double area;
    if (L.kind == LUM_LIGHT_RECT) {
        double a = s.draw(CALL_NEE, 2), b = s.draw(CALL_NEE, 3);
        lp = L.p0 + L.u * a + L.v * b;
        area = length(cross(L.u, L.v));
    } else {
        double r1 = s.draw(CALL_NEE, 2), r2 = s.draw(CALL_NEE, 3);
        double r = std::sqrt(r1) * L.r;
        double th = 2.0 * PI * r2;
        V3 w = L.n;
        V3 av = std::fabs(w.x) > 0.9 ? v3(0, 1, 0) : v3(1, 0, 0);
        V3 ut = unit(cross(w, av));
        V3 vt = cross(w, ut);
        lp = L.p0 + ut * (r * std::cos(th)) + vt * (r * std::sin(th));
        area = PI * L.r * L.r;
    }
    DV tl = dv(lp) - hp;
    Dd d2 = ddot(tl, tl);
    Dd dist = dsqrt(d2);
    DV dir = tl * (1.0 / dist);
    Dd ct = ddot(normal, dir);
    Dd ctl = dabs(ddot(-L.n, dir));
    Dd gterm = ct * ctl * (area * (double)lights.size() / PI) / d2;
    return had(em, att) * gterm;
}

// One keyed path (ray_color_keyed above) with dual radiance.
DV path_dual(const AdjCtx& C, Ray r, Sampler& s, uint32_t max_depth, Counters& cnt) {
    const orc_scene& sc = *C.sc;
    DV L = dv(v3(0, 0, 0)), B = dv(v3(1, 1, 1));
    DV o = dv(r.o), d = dv(r.d);
    bool skip = false;
    for (uint32_t b = 0; b < max_depth; ++b) {
        uint32_t depth = max_depth - b;
        s.begin_bounce(b);
        HitRecord h;
        cnt.segments++;
        if (!sc.hit(r, 0.001, INF, h)) {
            L = L + had(B, dv(background(*C.p, r, &C.sc->env)));
            break;
        }
        if (!std::isfinite(h.p.x) || !std::isfinite(h.p.y) || !std::isfinite(h.p.z)) break;
        DV P = dv(h.p);
        if (h.flat) {                     // intersection with the hit primitive's plane
            Dd nd = ddot(h.n, d);
            if (std::fabs(nd.v) > 1e-12) {
                Dd t = ddot(h.n, dv(h.p) - o) / nd;
                P = o + d * t;
                P.x.v = h.p.x;
                P.y.v = h.p.y;
                P.z.v = h.p.z;
            }
        }
        DV e = dv(v3(0, 0, 0));
        if (!skip && h.mat && h.mat->kind == LUM_MAT_EMISSIVE) e = C.emission(h.mat_index, h.mat->emitted(h.u, h.v, h.p));
        Scatter scat;
        if (!h.mat || !h.mat->scatter(r, h, s, scat)) {
            L = L + had(B, e);
            break;
        }
        double dl2 = length_squared(scat.ray.d);
        if (!(dl2 > 0.0) || !std::isfinite(dl2)) {
            L = L + had(B, e);
            break;
        }
        DV att, att_full, dir;
        scatter_dual(C, *h.mat, h.mat_index, h, d, s, scat, att, att_full, dir);
        double mc = std::fmax(std::fmax(scat.att.x, scat.att.y), scat.att.z);
        double surv = rclamp(mc, 0.05, 1.0);
        if (depth < 47 && s.draw(CALL_NEE, 0) > surv) {
            L = L + had(B, e);
            break;
        }
        Dd rrw = dcst(1.0);
        if (depth < 47) rrw = C.detach ? dcst(1.0 / surv) : 1.0 / dclamp(dmax3(att.x, att.y, att.z), 0.05, 1.0);
        bool use_nee = !h.mat->is_specular() && !sc.lights.empty();
        DV dl = use_nee ? nee_dual(C, P, h.n, att, s, cnt) : dv(v3(0, 0, 0));
        // The NEE term is evaluated only on paths that survive Russian roulette and is not
        // divided by the survival probability (render.rs:1497-1524), so its expectation carries
        // a factor surv(theta).  With probabilities held, the unbiased derivative adds the
        // score term (surv'/surv) * term, surv' taken in full (lobe probability included).
        if (C.detach && C.score && use_nee && depth < 47) {
            Dd sf = dclamp(dmax3(att_full.x, att_full.y, att_full.z), 0.05, 1.0);
            Dd ratio = sf / sf.v;
            dl = {dl.x * ratio, dl.y * ratio, dl.z * ratio};
        }
        DV term = e + dl;
        DV nb = had(B, att) * rrw;
        if (dnan(term) || dnan(nb)) break;
        L = L + had(B, term);
        B = nb;
        skip = use_nee;
        r = scat.ray;
        o = P;
        d = dir;
    }
    return L;
}

}  // namespace

extern "C" {

static int adjoint_impl(const orc_scene* sc, const lum_render_params* pp, const double* dl_dimage,
                        const int32_t* light_material, int mode, int threads, const double* direction,
                        double* d_albedo, double* d_roughness, double* d_emission, double* out_rgb);

int orc_adjoint(const orc_scene* sc, const lum_render_params* pp, const double* dl_dimage, const int32_t* light_material,
                int detach, int threads, double* d_albedo, double* d_roughness, double* d_emission, double* out_rgb) {
    if (!sc || !pp || !dl_dimage || !d_albedo || !d_roughness || !d_emission) return 1;
    return adjoint_impl(sc, pp, dl_dimage, light_material, detach, threads, nullptr, d_albedo, d_roughness, d_emission,
                        out_rgb);
}

int orc_adjoint_dir(const orc_scene* sc, const lum_render_params* pp, const double* dl_dimage,
                    const int32_t* light_material, int detach, int threads, const double* direction, double* out) {
    if (!sc || !pp || !dl_dimage || !direction || !out) return 1;
    const size_t n = sc->mats.size();
    std::vector<double> da(3 * n + 1), dr(n + 1), de(3 * n + 1);
    int rc = adjoint_impl(sc, pp, dl_dimage, light_material, detach, threads, direction, da.data(), dr.data(), de.data(),
                          nullptr);
    *out = da[0];
    return rc;
}

// mode: 0 plain, 1 probabilities held with the survival score term, 2 held without it.
static int adjoint_impl(const orc_scene* sc, const lum_render_params* pp, const double* dl_dimage,
                        const int32_t* light_material, int mode, int threads, const double* direction,
                        double* d_albedo, double* d_roughness, double* d_emission, double* out_rgb) {
    const lum_render_params& p = *pp;
    Frame f = frame_of(p);
    const int n_mat = (int)sc->mats.size();
    const int n_par = 7 * n_mat;
    std::vector<double> grad((size_t)n_par, 0.0);
#ifdef _OPENMP
    int nt = threads > 0 ? threads : omp_get_max_threads();
#else
    int nt = 1;
    (void)threads;
#endif
    const int n_pass = direction ? 1 : std::max(n_par, 1);
    for (int begin = 0; begin < n_pass; begin += ND) {
        AdjCtx C{sc, pp, light_material, n_mat, begin, mode != 0, mode == 1, direction};
        const bool write_img = out_rgb && begin == 0;
#pragma omp parallel num_threads(nt)
        {
            double gl[ND] = {};
#pragma omp for schedule(dynamic, 1)
            for (int64_t j = 0; j < (int64_t)f.h; ++j) {
                size_t gj = (size_t)j + f.crop_y;
                Sampler s;
                s.mode = ORC_MODE_KEYED;
                s.stream = nullptr;
                s.key[0] = (uint32_t)p.seed;
                s.key[1] = (uint32_t)(p.seed >> 32);
                double y = (double)(f.full_h - 1 - gj);
                Counters cnt;
                for (size_t i = 0; i < f.w; ++i) {
                    size_t gi = i + f.crop_x;
                    DV color = dv(v3(0, 0, 0));
                    double tw = 0.0;
                    s.pixel = (uint32_t)(gj * f.full_w + gi);
                    for (uint32_t st = f.s_begin; st < f.s_end; ++st) {
                        uint32_t sx = st % f.sqrt_spp, sy = st / f.sqrt_spp;
                        s.stratum = st;
                        s.begin_bounce(0);
                        double jx = ((double)sx + s.draw(CALL_CAMERA, 0)) / (double)f.sqrt_spp;
                        double jy = ((double)sy + s.draw(CALL_CAMERA, 1)) / (double)f.sqrt_spp;
                        double uc = ((double)gi + jx) / (double)(f.full_w - 1);
                        double vc = (y + jy) / (double)(f.full_h - 1);
                        Ray ray = sc->cam.get_ray(uc, vc, s);
                        DV smp = path_dual(C, ray, s, p.max_depth, cnt);
                        Dd lum = 0.2126 * smp.x + 0.7152 * smp.y + 0.0722 * smp.z;   // render.rs:1692-1697
                        DV cl = lum.v > 100.0 ? smp * (100.0 / lum) : smp;
                        double w = filter_weight(p.pixel_filter, jx - 0.5, jy - 0.5);
                        color = color + cl * w;
                        tw += w;
                    }
                    DV px = tw > 0.0 ? color * (1.0 / tw) : color;
                    const double* g = dl_dimage + ((size_t)j * f.w + i) * 3;
                    for (int k = 0; k < ND; ++k)
                        gl[k] += p.exposure * (g[0] * px.x.d[k] + g[1] * px.y.d[k] + g[2] * px.z.d[k]);
                    if (write_img) {
                        double* o = out_rgb + ((size_t)j * f.w + i) * 3;
                        o[0] = px.x.v * p.exposure;
                        o[1] = px.y.v * p.exposure;
                        o[2] = px.z.v * p.exposure;
                    }
                }
            }
#pragma omp critical
            if (direction) grad[0] += gl[0];
            else
                for (int k = 0; k < ND && begin + k < n_par; ++k) grad[(size_t)begin + k] += gl[k];
        }
    }
    if (direction) {
        d_albedo[0] = n_par > 0 ? grad[0] : 0.0;
        return 0;
    }
    for (int m = 0; m < n_mat; ++m) {
        for (int c = 0; c < 3; ++c) {
            d_albedo[3 * m + c] = grad[(size_t)3 * m + c];
            d_emission[3 * m + c] = grad[(size_t)4 * n_mat + 3 * m + c];
        }
        d_roughness[m] = grad[(size_t)3 * n_mat + m];
    }
    return 0;
}

}  // extern "C"
