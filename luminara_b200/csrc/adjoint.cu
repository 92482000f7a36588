// adjoint.cu -- path-replay adjoint of the renderer: d(loss)/d(per-material albedo,
// roughness, emission) given dL/d(image).
//
// Forward estimator (the megakernel's, src/render.rs:1472-1537 in iterative form): per path
// L = sum_j B_j (e_j + n_j) with B_{j+1} = B_j att_j rrw_j, n_j the NEE term
// E_L att_j G_j vis_j; the pixel is the mean of the luminance-clamped L over its strata.
//
// The backward kernel replays each path from its RNG key with the forward's own functions
// (start_path, trace, shade), records the vertices, then sweeps them backwards:
//   w_j = a (.) B_j                          a = J_clamp^T dLoss/dI / N
//   grad(e_j)  += w_j                        emission of the hit material when counted
//   grad(E_L)  += w_j (.) att_j G_j vis_j     emission of the light's material
//   abar_j      = w_j (.) (rrw_j S_{j+1} + E_L G_j vis_j)      S_{j+1}: the suffix sum
//   grad(albedo, roughness) += abar_j . d att_j / d(albedo, roughness)
// Russian-roulette survival and the microfacet lobe probability are treated as constants:
// the expectation of the estimator does not depend on them, so these per-path derivatives are
// unbiased.  Roughness also moves the GGX-sampled direction; that dependence is carried to
// later vertices by reverse-mode adjoints of the vertex position and direction:
//   - att_j and the specular direction l_j as functions of (incoming direction, roughness),
//     differentiated with 4-wide forward-mode duals,
//   - the NEE geometry term G_j as a function of the vertex position (rect and disk lights),
//   - the ray/surface intersection p_j = p_{j-1} + t d_j with Jacobian M = I - d n^T/(n.d).
// Visibility changes (edges, occlusion) are not differentiated; shading normals of curved
// surfaces are taken as constant along the path; Metal/Dielectric/Isotropic directions stop
// the direction adjoint.  Gradients accumulate in shared memory per block, then globally.
#include <cuda_runtime.h>

#include <chrono>
#include <cstdio>
#include <cstring>
#include <vector>

#include "kernels.h"
#include "scene_access.h"
#include "tracer.cuh"

namespace lum {
namespace adj {

constexpr int kMaxVerts = 16;   // recorded vertices per path; lum_backward rejects deeper paths
constexpr unsigned kFullMask = 0xffffffffu;

// ---------------------------------------------------------------- 4-wide forward duals
struct D4 {
    float v, d[4];
};
__device__ __forceinline__ D4 cst(float x) { return {x, {0.f, 0.f, 0.f, 0.f}}; }
__device__ __forceinline__ D4 seed(float x, int k) {
    D4 r = cst(x);
    r.d[k] = 1.0f;
    return r;
}
__device__ __forceinline__ D4 operator+(D4 a, D4 b) {
    D4 r{a.v + b.v, {}};
    for (int k = 0; k < 4; ++k) r.d[k] = a.d[k] + b.d[k];
    return r;
}
__device__ __forceinline__ D4 operator-(D4 a, D4 b) {
    D4 r{a.v - b.v, {}};
    for (int k = 0; k < 4; ++k) r.d[k] = a.d[k] - b.d[k];
    return r;
}
__device__ __forceinline__ D4 operator-(D4 a) {
    D4 r{-a.v, {}};
    for (int k = 0; k < 4; ++k) r.d[k] = -a.d[k];
    return r;
}
__device__ __forceinline__ D4 operator*(D4 a, D4 b) {
    D4 r{a.v * b.v, {}};
    for (int k = 0; k < 4; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
    return r;
}
__device__ __forceinline__ D4 operator*(D4 a, float s) {
    D4 r{a.v * s, {}};
    for (int k = 0; k < 4; ++k) r.d[k] = a.d[k] * s;
    return r;
}
__device__ __forceinline__ D4 operator*(float s, D4 a) { return a * s; }
__device__ __forceinline__ D4 operator+(D4 a, float s) {
    a.v += s;
    return a;
}
__device__ __forceinline__ D4 operator+(float s, D4 a) { return a + s; }
__device__ __forceinline__ D4 operator-(float s, D4 a) { return (-a) + s; }
__device__ __forceinline__ D4 operator/(D4 a, D4 b) {
    float inv = 1.0f / b.v;
    D4 r{a.v * inv, {}};
    for (int k = 0; k < 4; ++k) r.d[k] = (a.d[k] - r.v * b.d[k]) * inv;
    return r;
}
__device__ __forceinline__ D4 operator/(float s, D4 b) { return cst(s) / b; }
__device__ __forceinline__ D4 operator/(D4 a, float s) { return a * (1.0f / s); }
__device__ __forceinline__ D4 dsqrt(D4 a) {
    float s = sqrtf(a.v);
    D4 r{s, {}};
    float h = s > 0.0f ? 0.5f / s : 0.0f;
    for (int k = 0; k < 4; ++k) r.d[k] = a.d[k] * h;
    return r;
}
__device__ __forceinline__ D4 dmax(D4 a, float lo) { return a.v >= lo ? a : cst(lo); }
__device__ __forceinline__ D4 dabs(D4 a) { return a.v >= 0.0f ? a : -a; }

struct VD {
    D4 x, y, z;
};
__device__ __forceinline__ VD vd(V a) { return {cst(a.x), cst(a.y), cst(a.z)}; }
__device__ __forceinline__ VD operator+(VD a, VD b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ VD operator-(VD a, VD b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ VD operator*(VD a, D4 s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ VD operator*(V a, D4 s) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ D4 ddot(VD a, VD b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ D4 ddot(V a, VD b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ VD dunit(VD a) {
    D4 inv = 1.0f / dsqrt(ddot(a, a));
    return a * inv;
}

// Microfacet att (material.rs:328-390) and, for the specular lobe, the sampled direction l,
// as functions of the incoming ray direction d (dual slots 0..2) and roughness r (slot 3).
// The lobe probability sp is a constant here.  drho = d att / d albedo (diagonal, values).
__device__ void microfacet_dual(V n, V d, float r, V rho, float m, float u1, float u2, bool spec, float sp, VD& att,
                                VD& l, V& drho) {
    VD dd{seed(d.x, 0), seed(d.y, 1), seed(d.z, 2)};
    D4 rr = seed(r, 3);
    VD v = dunit(VD{-dd.x, -dd.y, -dd.z});
    D4 ndv = dmax(ddot(n, v), 0.001f);
    float f0[3] = {0.04f * (1.0f - m) + rho.x * m, 0.04f * (1.0f - m) + rho.y * m, 0.04f * (1.0f - m) + rho.z * m};
    if (spec) {
        D4 alpha = rr * rr;
        D4 tan2 = alpha * alpha * (u1 / (1.0f - u1 + 1e-10f));
        D4 ct = 1.0f / dsqrt(1.0f + tan2);
        D4 st = dsqrt(tan2) * ct;
        float sp_, cp_;
        sincospif(2.0f * u2, &sp_, &cp_);
        V up = fabsf(n.y) < 0.999f ? mk(0.f, 1.f, 0.f) : mk(1.f, 0.f, 0.f);
        V tg = unit(cross(up, n));
        V bt = cross(n, tg);
        VD h = dunit(tg * (st * cp_) + bt * (st * sp_) + n * ct);
        D4 vh = ddot(v, h);
        l = h * (vh * 2.0f) - v;
        D4 ndl = ddot(n, l);
        D4 ndh = dmax(ddot(n, h), 0.0f);
        D4 vdh = dmax(vh, 0.0f);
        D4 k = (rr + 1.0f) * (rr + 1.0f) * 0.125f;
        D4 g = (ndv / (ndv * (1.0f - k) + k)) * (ndl / (ndl * (1.0f - k) + k));
        D4 om = dmax(1.0f - vdh, 0.0f);
        D4 om2 = om * om;
        D4 t = om2 * om2 * om;
        D4 common = ndh.v > 0.001f ? g * vdh / (ndv * ndh) * (1.0f / sp) : cst(0.0f);
        att.x = (f0[0] * (1.0f - t) + t) * common;
        att.y = (f0[1] * (1.0f - t) + t) * common;
        att.z = (f0[2] * (1.0f - t) + t) * common;
        float dr = m * (1.0f - t.v) * common.v;
        drho = mk(dr, dr, dr);
    } else {
        D4 om = dmax(1.0f - ndv, 0.0f);
        D4 om2 = om * om;
        D4 t = om2 * om2 * om;
        float s = (1.0f - m) / (1.0f - sp);
        D4 F0 = f0[0] * (1.0f - t) + t, F1 = f0[1] * (1.0f - t) + t, F2 = f0[2] * (1.0f - t) + t;
        att.x = (1.0f - F0) * (s * rho.x);
        att.y = (1.0f - F1) * (s * rho.y);
        att.z = (1.0f - F2) * (s * rho.z);
        drho = mk(s * ((1.0f - F0.v) - rho.x * m * (1.0f - t.v)), s * ((1.0f - F1.v) - rho.y * m * (1.0f - t.v)),
                  s * ((1.0f - F2.v) - rho.z * m * (1.0f - t.v)));
        l = VD{cst(0.f), cst(0.f), cst(0.f)};
    }
}

// NEE geometry term G(p) = cos * cos_l * A * N / (pi d^2) for a fixed light point y, with
// its gradient with respect to the shading point p (render.rs:1439-1465).
__device__ float nee_geometry(V p, V n, V y, V nl, float area_n, V& grad) {
    VD pd{seed(p.x, 0), seed(p.y, 1), seed(p.z, 2)};
    VD tl = vd(y) - pd;
    D4 d2 = ddot(tl, tl);
    D4 dist = dsqrt(d2);
    VD dir = tl * (1.0f / dist);
    D4 ct = ddot(n, dir);
    D4 ctl = dabs(ddot(-nl, dir) * 1.0f);
    D4 G = ct * ctl * (area_n / CUDART_PI_F) / d2;
    grad = mk(G.d[0], G.d[1], G.d[2]);
    return G.v;
}

struct Vert {
    V p, n, d_in, B;   // hit point, facing normal, incoming direction, throughput to this vertex
    float t;           // p = previous origin + t * d_in
    int mat;
    uint32_t flags;    // bit0 continued (att applies), bit1 emission counted, bit2 NEE valid,
                       // bit3 NEE visible, bit4 specular lobe, bit5 flat surface
};
enum : uint32_t { VF_CONT = 1, VF_EMIT = 2, VF_NEE = 4, VF_VIS = 8, VF_SPEC = 16, VF_FLAT = 32 };

struct Grads {
    float* albedo;     // 3 per material
    float* rough;      // 1 per material
    float* emission;   // 3 per material
};

__device__ __forceinline__ void add_grad(float* smem, int n_mat, const Grads& g, int mat, int field, float v) {
    if (v == 0.0f || mat < 0) return;
    if (smem) atomicAdd(smem + field * n_mat + mat, v);
    else if (field < 3) atomicAdd(g.albedo + 3 * mat + field, v);
    else if (field == 3) atomicAdd(g.rough + mat, v);
    else atomicAdd(g.emission + 3 * mat + (field - 4), v);
}

__device__ __forceinline__ int prim_type(const SceneDev& S, int prim) {
    return prim <= -2 ? 100 : (__ldg(S.meta + prim) & 15);
}

// One path: forward replay with the forward's functions, then the backward sweep.
__device__ void path_adjoint(const SceneDev& S, const RenderDev& R, uint32_t gi, uint32_t gj, uint32_t pixel,
                             uint32_t st, V gpix, float inv_wsum, const int* light_mat, int* stack, uint32_t& err,
                             float* smem, int n_mat, const Grads& G, Vert* verts) {
    Path P;
    start_path(S, R, gi, gj, pixel, st, P);
    int K = 0;
    V bg = mk(0.f, 0.f, 0.f);
    bool bg_hit = false;
    const uint32_t maxd = min(R.max_depth, (uint32_t)kMaxVerts);
    while (P.bounce < maxd) {
        Hit h;
        h.t = CUDART_INF_F;
        h.prim = -1;
        h.b1 = h.b2 = 0.0f;
        const Ray in = P.ray;
        const V B = P.beta;
        const bool skip = P.skip_emission;
        const bool found = trace(S, in, 0.001f, false, h, stack, err);
        if (!found) {
            bg = background(R, in);
            bg_hit = true;
            break;
        }
        Vert& vx = verts[K];
        Surface sf = surface_of(S, in, h);
        vx.p = sf.p;
        vx.n = sf.n;
        vx.d_in = in.d;
        vx.B = B;
        vx.t = h.t;
        vx.mat = sf.mat;
        int pt = prim_type(S, h.prim);
        vx.flags = (pt == PT_QUAD || pt == PT_TRIANGLE || pt == PT_DISK || pt == 100) ? VF_FLAT : 0u;
        if (!skip && S.mats[sf.mat].kind == 4) vx.flags |= VF_EMIT;
        ++K;
        Pending pend;
        const uint32_t b0 = P.bounce;
        const int stt = shade(S, R, pixel, P, true, h, pend);
        if (P.bounce > b0) vx.flags |= VF_CONT;                         // scatter survived RR
        if (S.mats[sf.mat].kind == 5 && (vx.flags & VF_CONT)) {
            // lobe of the microfacet sample: draw 0 of CALL_SCATTER against sp (material.rs:345)
            float4 su = draw4(R.key0, R.key1, pixel, st, b0, CALL_SCATTER);
            const MatDev& m = S.mats[sf.mat];
            V alb = tex_value(m, sf.p);
            V v = unit(-in.d);
            float ndv = fmaxf(dot(sf.n, v), 0.001f);
            V f0 = mk(0.04f, 0.04f, 0.04f) * (1.0f - m.metallic) + alb * m.metallic;
            V fw = fresnel(ndv, f0);
            float sp = fminf(fmaxf((fw.x + fw.y + fw.z) * (1.0f / 3.0f), 0.1f), 0.9f);
            if (su.x < sp) vx.flags |= VF_SPEC;
        }
        if (stt == ST_SHADOW) {
            vx.flags |= VF_NEE;
            Ray sr{P.ray.o, pend.dir, 0.0f};
            Hit sh;
            sh.t = pend.tmax;
            sh.prim = -1;
            if (!trace(S, sr, 0.001f, true, sh, stack, err)) {
                vx.flags |= VF_VIS;
                P.L = P.L + pend.contrib;
            }
        }
        if (!(vx.flags & VF_CONT)) break;
        if (stt == ST_DONE) break;
    }
    // adjoint of L through the luminance clamp (render.rs:1692-1697), mean over strata
    const V Lw = mk(0.2126f, 0.7152f, 0.0722f);
    float lum = dot(Lw, P.L);
    V a = gpix * inv_wsum;
    if (lum > 100.0f) {                          // f(L) = 100 L / lum(L)
        float s = 100.0f / lum;
        float la = dot(a, P.L);
        a = (a - Lw * (la / lum)) * s;
    }
    float wf = filter_weight(R.pixel_filter, P.jx - 0.5f, P.jy - 0.5f);
    a = a * wf;
    // backward sweep
    V S_next = bg_hit ? bg : mk(0.f, 0.f, 0.f);
    V Dbar = mk(0.f, 0.f, 0.f);   // adjoint of the outgoing direction of the current vertex
    V Pbar = mk(0.f, 0.f, 0.f);   // adjoint of the position of the next vertex, pulled back below
    for (int j = K - 1; j >= 0; --j) {
        const Vert& vx = verts[j];
        const MatDev& m = S.mats[vx.mat];
        const V w = mul(a, vx.B);
        V c = mk(0.f, 0.f, 0.f);
        V e = emitted(m, vx.p);
        if (vx.flags & VF_EMIT) {
            c = c + e;
            add_grad(smem, n_mat, G, vx.mat, 4, w.x);
            add_grad(smem, n_mat, G, vx.mat, 5, w.y);
            add_grad(smem, n_mat, G, vx.mat, 6, w.z);
        }
        V PbarJ = mk(0.f, 0.f, 0.f);   // adjoint of this vertex's position
        V DbarIn = mk(0.f, 0.f, 0.f);  // adjoint of this vertex's incoming direction
        if (vx.flags & VF_CONT) {
            const uint32_t bounce = (uint32_t)j;
            const uint32_t depth = R.max_depth - bounce;
            float4 su = draw4(R.key0, R.key1, pixel, st, bounce, CALL_SCATTER);
            float4 nu = draw4(R.key0, R.key1, pixel, st, bounce, CALL_NEE);
            VD att;
            VD l;
            V drho = mk(0.f, 0.f, 0.f);
            bool dual = false;
            V att_v;
            if (m.kind == 5) {
                V alb = tex_value(m, vx.p);
                V v = unit(-vx.d_in);
                float ndv = fmaxf(dot(vx.n, v), 0.001f);
                V f0 = mk(0.04f, 0.04f, 0.04f) * (1.0f - m.metallic) + alb * m.metallic;
                V fw = fresnel(ndv, f0);
                float sp = fminf(fmaxf((fw.x + fw.y + fw.z) * (1.0f / 3.0f), 0.1f), 0.9f);
                microfacet_dual(vx.n, vx.d_in, m.roughness, alb, m.metallic, su.y, su.z, (vx.flags & VF_SPEC) != 0, sp,
                                att, l, drho);
                att_v = mk(att.x.v, att.y.v, att.z.v);
                dual = true;
            } else if (m.kind == 1 || m.kind == 2) {
                att_v = m.kind == 1 ? tex_value(m, vx.p) : mk(m.color);
                drho = mk(1.f, 1.f, 1.f);
            } else if (m.kind == 3) {                 // dielectric: attenuation without parameters here
                att_v = mk(m.tint);
            } else {                                  // isotropic
                att_v = mk(m.color);
            }
            float surv = fminf(fmaxf(fmaxf(fmaxf(att_v.x, att_v.y), att_v.z), 0.05f), 1.0f);
            float rrw = depth < 47 ? 1.0f / surv : 1.0f;
            V abar = mul(w, S_next * rrw);
            V nee = mk(0.f, 0.f, 0.f);
            if ((vx.flags & VF_NEE) && (vx.flags & VF_VIS)) {
                // recompute the NEE sample (render.rs:1358-1437) for the light emission and G
                int nl = S.n_lights;
                int li = min((int)(nu.y * (float)nl), nl - 1);
                const LightDev& Lt = S.lights[li];
                Ray srr;
                float tmax;
                V contrib;
                if (sample_light(S, vx.p, vx.n, att_v, nu, srr, tmax, contrib)) {
                    V EL = mk(Lt.e);
                    // contrib = EL * att * Gval ; recover Gval from one channel-free form
                    V y;
                    bool has_geo = false;
                    if (Lt.kind == 2) {
                        y = mk(Lt.p0) + mk(Lt.u) * nu.z + mk(Lt.v) * nu.w;
                        has_geo = true;
                    } else if (Lt.kind == 3) {
                        float r = sqrtf(nu.z) * Lt.radius, sp2, cp2;
                        sincospif(2.0f * nu.w, &sp2, &cp2);
                        V wl = mk(Lt.n);
                        V av = fabsf(wl.x) > 0.9f ? mk(0.f, 1.f, 0.f) : mk(1.f, 0.f, 0.f);
                        V ut = unit(cross(wl, av));
                        V vt = cross(wl, ut);
                        y = mk(Lt.p0) + ut * (r * cp2) + vt * (r * sp2);
                        has_geo = true;
                    }
                    float Gv;
                    V gradG = mk(0.f, 0.f, 0.f);
                    if (has_geo) {
                        Gv = nee_geometry(vx.p, vx.n, y, mk(Lt.n), Lt.area * (float)nl, gradG);
                    } else {
                        float ea = EL.x * att_v.x;
                        Gv = ea != 0.0f ? contrib.x / ea : 0.0f;
                    }
                    nee = mul(EL, att_v) * Gv;
                    abar = abar + mul(w, EL) * Gv;
                    int lm = light_mat ? light_mat[li] : -1;
                    V gE = mul(w, att_v) * Gv;
                    add_grad(smem, n_mat, G, lm, 4, gE.x);
                    add_grad(smem, n_mat, G, lm, 5, gE.y);
                    add_grad(smem, n_mat, G, lm, 6, gE.z);
                    float s = dot(mul(w, EL), att_v);
                    PbarJ = PbarJ + gradG * s;
                }
            }
            c = c + nee;
            // albedo / roughness through att
            add_grad(smem, n_mat, G, vx.mat, 0, abar.x * drho.x);
            add_grad(smem, n_mat, G, vx.mat, 1, abar.y * drho.y);
            add_grad(smem, n_mat, G, vx.mat, 2, abar.z * drho.z);
            if (dual) {
                float gr = abar.x * att.x.d[3] + abar.y * att.y.d[3] + abar.z * att.z.d[3];
                DbarIn = DbarIn + mk(abar.x * att.x.d[0] + abar.y * att.y.d[0] + abar.z * att.z.d[0],
                                     abar.x * att.x.d[1] + abar.y * att.y.d[1] + abar.z * att.z.d[1],
                                     abar.x * att.x.d[2] + abar.y * att.y.d[2] + abar.z * att.z.d[2]);
                if (vx.flags & VF_SPEC) {                 // outgoing direction l(d_in, r)
                    gr += Dbar.x * l.x.d[3] + Dbar.y * l.y.d[3] + Dbar.z * l.z.d[3];
                    for (int k = 0; k < 3; ++k) {
                        float dk = Dbar.x * l.x.d[k] + Dbar.y * l.y.d[k] + Dbar.z * l.z.d[k];
                        if (k == 0) DbarIn.x += dk;
                        else if (k == 1) DbarIn.y += dk;
                        else DbarIn.z += dk;
                    }
                }
                add_grad(smem, n_mat, G, vx.mat, 3, gr);
            }
            S_next = c + mul(att_v, S_next) * rrw;
        } else {
            S_next = c;
        }
        // position adjoint of this vertex, then through p_j = p_{j-1} + t d_j
        PbarJ = PbarJ + Pbar;
        if (vx.flags & VF_FLAT) {
            float nd = dot(vx.n, vx.d_in);
            if (fabsf(nd) > 1e-12f) {
                V MtP = PbarJ - vx.n * (dot(vx.d_in, PbarJ) / nd);
                Pbar = MtP;                      // adjoint of the previous vertex's position
                DbarIn = DbarIn + MtP * vx.t;
            } else {
                Pbar = mk(0.f, 0.f, 0.f);
            }
        } else {
            Pbar = mk(0.f, 0.f, 0.f);
        }
        // the incoming direction of vertex j is the outgoing direction of vertex j-1; only a
        // microfacet vertex's direction depends on parameters (handled at j-1 via Dbar)
        Dbar = DbarIn;
    }
}

__global__ void __launch_bounds__(128) k_backward(SceneDev S, RenderDev R, const float* __restrict__ dldi,
                                                  const int* __restrict__ light_mat, Grads G, int n_mat,
                                                  int use_smem, WorkCounters* wc) {
    extern __shared__ int smem_raw[];
    int* stack = smem_raw + threadIdx.x;
    float* gsm = use_smem ? reinterpret_cast<float*>(smem_raw + kStackDepth * blockDim.x) : nullptr;
    if (gsm)
        for (int k = threadIdx.x; k < 7 * n_mat; k += blockDim.x) gsm[k] = 0.0f;
    __syncthreads();
    Vert verts[kMaxVerts];
    const int lane = threadIdx.x & 31;
    uint32_t err = 0;
    for (;;) {
        uint32_t task = 0;
        if (lane == 0) task = atomicAdd(&wc->next_task, 1u);
        task = __shfl_sync(kFullMask, task, 0);
        if (task >= R.n_tasks) break;
        const uint32_t i = (task % R.tiles_x) * 8 + (lane & 7);
        const uint32_t j = (task / R.tiles_x) * 4 + (lane >> 3);
        if (i < R.w && j < R.h) {
            const uint32_t gi = i + R.crop_x, gj = j + R.crop_y;
            const uint32_t pixel = gj * R.full_w + gi;
            const float* g = dldi + 3 * ((size_t)j * R.w + i);
            V gpix = mk(g[0], g[1], g[2]) * R.exposure;
            // pixel = sum_s f(L_s) w_s / sum_s w_s (render.rs:1699-1705)
            float wsum = 0.0f;
            for (uint32_t st = R.s_begin; st < R.s_end; ++st) {
                float4 c = draw4(R.key0, R.key1, pixel, st, 0, CALL_CAMERA);
                uint32_t sx = st % R.sqrt_spp, sy = st / R.sqrt_spp;
                float inv_n = 1.0f / (float)R.sqrt_spp;
                wsum += filter_weight(R.pixel_filter, ((float)sx + c.x) * inv_n - 0.5f, ((float)sy + c.y) * inv_n - 0.5f);
            }
            float inv_wsum = wsum > 0.0f ? 1.0f / wsum : 1.0f;
            if (gpix.x != 0.0f || gpix.y != 0.0f || gpix.z != 0.0f)
                for (uint32_t st = R.s_begin; st < R.s_end; ++st)
                    path_adjoint(S, R, gi, gj, pixel, st, gpix, inv_wsum, light_mat, stack, err, gsm, n_mat, G, verts);
        }
    }
    __syncthreads();
    if (gsm) {
        for (int k = threadIdx.x; k < 7 * n_mat; k += blockDim.x) {
            float v = gsm[k];
            if (v == 0.0f) continue;
            int field = k / n_mat, mat = k % n_mat;
            if (field < 3) atomicAdd(G.albedo + 3 * mat + field, v);
            else if (field == 3) atomicAdd(G.rough + mat, v);
            else atomicAdd(G.emission + 3 * mat + (field - 4), v);
        }
    }
    if (err) atomicOr(&wc->error_flags, err);
}

}  // namespace adj
}  // namespace lum

namespace {

lum_status adj_cuda(cudaError_t e, const char* what) {
    char msg[256];
    snprintf(msg, sizeof msg, "%s: %s", what, cudaGetErrorString(e));
    cudaGetLastError();
    return lum::set_error(e == cudaErrorMemoryAllocation ? LUM_ERR_OUT_OF_MEMORY : LUM_ERR_CUDA, msg);
}

}  // namespace

extern "C" {

lum_status lum_forward(lum_scene* scene, const lum_render_params* params, float* out_rgb, lum_stats* stats) {
    return lum_render(scene, params, out_rgb, stats);
}

lum_status lum_backward(lum_scene* scene, const lum_render_params* params, const float* dL_dimage,
                        const int32_t* light_material, float* d_albedo, float* d_roughness, float* d_emission,
                        lum_stats* stats) {
    using namespace lum;
    auto t0 = std::chrono::steady_clock::now();
    if (!scene || !params || !dL_dimage || !d_albedo || !d_roughness || !d_emission)
        return set_error(LUM_ERR_INVALID_ARGUMENT, "null argument");
    SceneDev dev;
    RenderDev R;
    cudaStream_t stream;
    lum_status st = prepare_render(scene, params, dev, R, stream);
    if (st != LUM_OK) return st;
    if (R.max_depth > (uint32_t)adj::kMaxVerts)
        return set_error(LUM_ERR_UNSUPPORTED, "lum_backward supports max_depth <= 16");
    const int n_mat = dev.n_mats;
    if (light_material)
        for (int k = 0; k < dev.n_lights; ++k)
            if (light_material[k] < -1 || light_material[k] >= n_mat)
                return set_error(LUM_ERR_INVALID_ARGUMENT, "light_material names no material");
    const size_t px = (size_t)R.w * R.h;
    std::memset(d_albedo, 0, sizeof(float) * 3 * n_mat);
    std::memset(d_roughness, 0, sizeof(float) * n_mat);
    std::memset(d_emission, 0, sizeof(float) * 3 * n_mat);
    if (px == 0 || R.s_end <= R.s_begin || n_mat == 0) return LUM_OK;
    size_t bytes_img = sizeof(float) * 3 * px, bytes_g = sizeof(float) * 7 * n_mat, bytes_lm = sizeof(int) * (dev.n_lights + 1);
    char* buf = nullptr;
    cudaError_t e = cudaMalloc(&buf, bytes_img + bytes_g + bytes_lm + sizeof(WorkCounters) + 1024);
    if (e != cudaSuccess) return adj_cuda(e, "cudaMalloc");
    float* d_img = (float*)buf;
    float* d_g = (float*)(buf + bytes_img);
    int* d_lm = (int*)(buf + bytes_img + bytes_g);
    WorkCounters* wc = (WorkCounters*)(((size_t)(buf + bytes_img + bytes_g + bytes_lm) + 255) & ~(size_t)255);
    std::vector<int> lm(dev.n_lights + 1, -1);
    if (light_material)
        for (int k = 0; k < dev.n_lights; ++k) lm[k] = light_material[k];
    adj::Grads G{d_g, d_g + 3 * n_mat, d_g + 4 * n_mat};
    cudaEvent_t ev0, ev1;
    cudaEventCreate(&ev0);
    cudaEventCreate(&ev1);
    bool ok = (e = cudaMemcpyAsync(d_img, dL_dimage, bytes_img, cudaMemcpyHostToDevice, stream)) == cudaSuccess &&
              (e = cudaMemcpyAsync(d_lm, lm.data(), bytes_lm, cudaMemcpyHostToDevice, stream)) == cudaSuccess &&
              (e = cudaMemsetAsync(d_g, 0, bytes_g, stream)) == cudaSuccess &&
              (e = cudaMemsetAsync(wc, 0, sizeof(WorkCounters), stream)) == cudaSuccess;
    float ms = 0.0f;
    WorkCounters counters{};
    if (ok) {
        const size_t stack = (size_t)kStackDepth * 128 * sizeof(int);
        int use_smem = (stack + bytes_g) <= 160 * 1024 ? 1 : 0;
        size_t smem = stack + (use_smem ? bytes_g : 0);
        cudaFuncSetAttribute(adj::k_backward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        int occ = 0, nsm = 0, devi = 0;
        cudaGetDevice(&devi);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, devi);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, adj::k_backward, 128, smem);
        int grid = nsm * (occ > 0 ? occ : 1);
        int need = (int)((R.n_tasks + 3) / 4);
        if (grid > need) grid = need > 0 ? need : 1;
        cudaEventRecord(ev0, stream);
        adj::k_backward<<<grid, 128, smem, stream>>>(dev, R, d_img, d_lm, G, n_mat, use_smem, wc);
        e = cudaGetLastError();
        ok = e == cudaSuccess;
        cudaEventRecord(ev1, stream);
    }
    std::vector<float> hg(7 * (size_t)n_mat);
    if (ok)
        ok = (e = cudaMemcpyAsync(hg.data(), d_g, bytes_g, cudaMemcpyDeviceToHost, stream)) == cudaSuccess &&
             (e = cudaMemcpyAsync(&counters, wc, sizeof counters, cudaMemcpyDeviceToHost, stream)) == cudaSuccess &&
             (e = cudaStreamSynchronize(stream)) == cudaSuccess;
    if (ok) cudaEventElapsedTime(&ms, ev0, ev1);
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
    cudaFree(buf);
    if (!ok) return adj_cuda(e, "lum_backward");
    std::memcpy(d_albedo, hg.data(), sizeof(float) * 3 * n_mat);
    std::memcpy(d_roughness, hg.data() + 3 * n_mat, sizeof(float) * n_mat);
    std::memcpy(d_emission, hg.data() + 4 * n_mat, sizeof(float) * 3 * n_mat);
    if (stats) {
        std::memset(stats, 0, sizeof *stats);
        stats->paths = px * (R.s_end - R.s_begin);
        stats->kernel_ms = ms;
        stats->total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        stats->error_flags = counters.error_flags;
    }
    if (counters.error_flags) return set_error(LUM_ERR_KERNEL, "backward kernel reported error flags");
    return LUM_OK;
}

}  // extern "C"
