// adjoint.cu -- path-replay adjoint of the renderer: d(loss)/d(per-material albedo,
// roughness, emission) given dL/d(image).
//
// Forward estimator (the megakernel's, src/render.rs:1472-1537 in iterative form): per path
// L = sum_j B_j (e_j + n_j) with B_{j+1} = B_j att_j rrw_j, n_j the NEE term
// E_L att_j G_j vis_j; the pixel is the mean of the luminance-clamped L over its strata.
//
// The backward pass replays each path from its RNG key with the forward's own functions
// (start_path, trace, shade) in a replay kernel that records the path's vertices into a
// staging buffer (one chunk of tiles at a time), then a sweep kernel walks each path's
// vertices backwards (one thread per path, no traversal):
//   w_j = a (.) B_j                          a = J_clamp^T dLoss/dI / N
//   grad(e_j)  += w_j                        emission of the hit material when counted
//   grad(E_L)  += w_j (.) att_j G_j vis_j     emission of the light's material
//   abar_j      = w_j (.) (rrw_j S_{j+1} + E_L G_j vis_j)      S_{j+1}: the suffix sum
//   grad(albedo, roughness) += abar_j . d att_j / d(albedo, roughness)
// Russian-roulette survival and the microfacet lobe probability are held constant in the
// weights they divide (those weights make the expectation independent of them).  The one
// exception is the NEE term, which the reference adds only on paths that survive Russian
// roulette without dividing by the survival probability, so its expectation is surv * term;
// its derivative gets the score term (surv'/surv) * term with surv' in full.  The result is an
// unbiased estimate of the derivative of the expected image.  Roughness also moves the GGX-sampled direction; that dependence is carried to
// later vertices by reverse-mode adjoints of the vertex position and direction:
//   - att_j and the specular direction l_j as functions of (incoming direction, roughness),
//     differentiated with 4-wide forward-mode duals,
//   - the NEE geometry term G_j as a function of the vertex position (rect and disk lights),
//   - the ray/surface intersection p_j = p_{j-1} + t d_j with Jacobian M = I - d n^T/(n.d).
// Visibility changes (edges, occlusion) are not differentiated; shading normals of curved
// surfaces are taken as constant along the path; Metal/Dielectric/Isotropic directions stop
// the direction adjoint.  Gradients accumulate in shared memory per block, then globally.
// Splitting replay and sweep keeps each kernel's instruction footprint small (the fused form
// stalled on instruction fetch) and lets the sweep run one path per thread at full width.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "kernels.h"
#include "scene_access.h"
#include "tracer.cuh"

namespace lum {
namespace adj {

constexpr int kMaxVerts = 16;   // recorded vertices per path; lum_backward rejects deeper paths
constexpr unsigned kFullMask = 0xffffffffu;

// ---------------------------------------------------------------- N-wide forward duals
template <int N>
struct Dn {
    float v, d[N];
};
template <int N>
__device__ __forceinline__ Dn<N> cst(float x) {
    Dn<N> r;
    r.v = x;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = 0.0f;
    return r;
}
template <int N>
__device__ __forceinline__ Dn<N> seed(float x, int k) {
    Dn<N> r = cst<N>(x);
    r.d[k] = 1.0f;
    return r;
}
template <int N>
__device__ __forceinline__ Dn<N> operator+(Dn<N> a, Dn<N> b) {
    Dn<N> r;
    r.v = a.v + b.v;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = a.d[k] + b.d[k];
    return r;
}
template <int N>
__device__ __forceinline__ Dn<N> operator-(Dn<N> a, Dn<N> b) {
    Dn<N> r;
    r.v = a.v - b.v;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = a.d[k] - b.d[k];
    return r;
}
template <int N>
__device__ __forceinline__ Dn<N> operator-(Dn<N> a) {
    Dn<N> r;
    r.v = -a.v;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = -a.d[k];
    return r;
}
template <int N>
__device__ __forceinline__ Dn<N> operator*(Dn<N> a, Dn<N> b) {
    Dn<N> r;
    r.v = a.v * b.v;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
    return r;
}
template <int N>
__device__ __forceinline__ Dn<N> operator*(Dn<N> a, float s) {
    Dn<N> r;
    r.v = a.v * s;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = a.d[k] * s;
    return r;
}
template <int N>
__device__ __forceinline__ Dn<N> operator*(float s, Dn<N> a) { return a * s; }
template <int N>
__device__ __forceinline__ Dn<N> operator+(Dn<N> a, float s) {
    a.v += s;
    return a;
}
template <int N>
__device__ __forceinline__ Dn<N> operator+(float s, Dn<N> a) { return a + s; }
template <int N>
__device__ __forceinline__ Dn<N> operator-(float s, Dn<N> a) { return (-a) + s; }
template <int N>
__device__ __forceinline__ Dn<N> operator/(Dn<N> a, Dn<N> b) {
    float inv = 1.0f / b.v;
    Dn<N> r;
    r.v = a.v * inv;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = (a.d[k] - r.v * b.d[k]) * inv;
    return r;
}
template <int N>
__device__ __forceinline__ Dn<N> operator/(float s, Dn<N> b) { return cst<N>(s) / b; }
template <int N>
__device__ __forceinline__ Dn<N> operator/(Dn<N> a, float s) { return a * (1.0f / s); }
template <int N>
__device__ __forceinline__ Dn<N> dsqrt(Dn<N> a) {
    float s = sqrtf(a.v);
    Dn<N> r;
    r.v = s;
    float h = s > 0.0f ? 0.5f / s : 0.0f;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = a.d[k] * h;
    return r;
}
template <int N>
__device__ __forceinline__ Dn<N> dmax(Dn<N> a, float lo) { return a.v >= lo ? a : cst<N>(lo); }
template <int N>
__device__ __forceinline__ Dn<N> dabs(Dn<N> a) { return a.v >= 0.0f ? a : -a; }

template <int N>
struct VDn {
    Dn<N> x, y, z;
};
template <int N>
__device__ __forceinline__ VDn<N> vd(V a) { return {cst<N>(a.x), cst<N>(a.y), cst<N>(a.z)}; }
template <int N>
__device__ __forceinline__ VDn<N> operator+(VDn<N> a, VDn<N> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <int N>
__device__ __forceinline__ VDn<N> operator-(VDn<N> a, VDn<N> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <int N>
__device__ __forceinline__ VDn<N> operator*(VDn<N> a, Dn<N> s) { return {a.x * s, a.y * s, a.z * s}; }
template <int N>
__device__ __forceinline__ VDn<N> operator*(V a, Dn<N> s) { return {s * a.x, s * a.y, s * a.z}; }
template <int N>
__device__ __forceinline__ Dn<N> ddot(VDn<N> a, VDn<N> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <int N>
__device__ __forceinline__ Dn<N> ddot(V a, VDn<N> b) { return b.x * a.x + b.y * a.y + b.z * a.z; }
template <int N>
__device__ __forceinline__ VDn<N> dunit(VDn<N> a) {
    Dn<N> inv = 1.0f / dsqrt(ddot(a, a));
    return a * inv;
}

// Microfacet att (material.rs:328-390) and, for the specular lobe, the sampled direction l.
// N = 4: functions of the incoming direction d (dual slots 0..2) and roughness r (slot 3);
// N = 1: of roughness only (slot 0).  The lobe probability sp is a constant here.  drho =
// d att / d albedo (diagonal, values).
template <int N>
__device__ void microfacet_dual(V n, V d, float r, V rho, float m, float u1, float u2, bool spec, float sp, VDn<N>& att,
                                VDn<N>& l, V& drho, float& dsp_dalb, V& dsp_dd) {
    VDn<N> dd = vd<N>(d);
    if constexpr (N == 4) {
        dd.x.d[0] = 1.0f;
        dd.y.d[1] = 1.0f;
        dd.z.d[2] = 1.0f;
    }
    Dn<N> rr = seed<N>(r, N - 1);
    VDn<N> v = dunit(VDn<N>{-dd.x, -dd.y, -dd.z});
    Dn<N> ndv = dmax(ddot(n, v), 0.001f);
    float f0[3] = {0.04f * (1.0f - m) + rho.x * m, 0.04f * (1.0f - m) + rho.y * m, 0.04f * (1.0f - m) + rho.z * m};
    {   // the lobe probability sp = clamp(mean Fresnel(ndv, f0), 0.1, 0.9) and its derivatives
        Dn<N> omn = dmax(1.0f - ndv, 0.0f);
        Dn<N> omn2 = omn * omn;
        Dn<N> tn = omn2 * omn2 * omn;
        Dn<N> spr = (tn * (3.0f - f0[0] - f0[1] - f0[2]) + (f0[0] + f0[1] + f0[2])) * (1.0f / 3.0f);
        const bool active = spr.v > 0.1f && spr.v < 0.9f;
        dsp_dalb = active ? m * (1.0f - tn.v) * (1.0f / 3.0f) : 0.0f;
        dsp_dd = mk(0.f, 0.f, 0.f);
        if constexpr (N == 4)
            if (active) dsp_dd = mk(spr.d[0], spr.d[1], spr.d[2]);
    }
    if (spec) {
        Dn<N> alpha = rr * rr;
        Dn<N> tan2 = alpha * alpha * (u1 / (1.0f - u1 + 1e-10f));
        Dn<N> ct = 1.0f / dsqrt(1.0f + tan2);
        Dn<N> st = dsqrt(tan2) * ct;
        float sp_, cp_;
        sincospif(2.0f * u2, &sp_, &cp_);
        V up = fabsf(n.y) < 0.999f ? mk(0.f, 1.f, 0.f) : mk(1.f, 0.f, 0.f);
        V tg = unit(cross(up, n));
        V bt = cross(n, tg);
        VDn<N> h = dunit(tg * (st * cp_) + bt * (st * sp_) + n * ct);
        Dn<N> vh = ddot(v, h);
        l = h * (vh * 2.0f) - v;
        Dn<N> ndl = ddot(n, l);
        Dn<N> ndh = dmax(ddot(n, h), 0.0f);
        Dn<N> vdh = dmax(vh, 0.0f);
        Dn<N> k = (rr + 1.0f) * (rr + 1.0f) * 0.125f;
        Dn<N> g = (ndv / (ndv * (1.0f - k) + k)) * (ndl / (ndl * (1.0f - k) + k));
        Dn<N> om = dmax(1.0f - vdh, 0.0f);
        Dn<N> om2 = om * om;
        Dn<N> t = om2 * om2 * om;
        Dn<N> common = ndh.v > 0.001f ? g * vdh / (ndv * ndh) * (1.0f / sp) : cst<N>(0.0f);
        att.x = (f0[0] * (1.0f - t) + t) * common;
        att.y = (f0[1] * (1.0f - t) + t) * common;
        att.z = (f0[2] * (1.0f - t) + t) * common;
        float dr = m * (1.0f - t.v) * common.v;
        drho = mk(dr, dr, dr);
    } else {
        Dn<N> om = dmax(1.0f - ndv, 0.0f);
        Dn<N> om2 = om * om;
        Dn<N> t = om2 * om2 * om;
        float s = (1.0f - m) / (1.0f - sp);
        Dn<N> F0 = f0[0] * (1.0f - t) + t, F1 = f0[1] * (1.0f - t) + t, F2 = f0[2] * (1.0f - t) + t;
        att.x = (1.0f - F0) * (s * rho.x);
        att.y = (1.0f - F1) * (s * rho.y);
        att.z = (1.0f - F2) * (s * rho.z);
        drho = mk(s * ((1.0f - F0.v) - rho.x * m * (1.0f - t.v)), s * ((1.0f - F1.v) - rho.y * m * (1.0f - t.v)),
                  s * ((1.0f - F2.v) - rho.z * m * (1.0f - t.v)));
        l = vd<N>(mk(0.f, 0.f, 0.f));
    }
}

// Diffuse-lobe microfacet att and d att / d albedo as plain values (no direction adjoint).
__device__ __forceinline__ V microfacet_diffuse(V n, V d, V rho, float m, float sp, V& drho, float& dsp_dalb) {
    float ndv = fmaxf(dot(n, unit(-d)), 0.001f);
    float om = fmaxf(1.0f - ndv, 0.0f);
    float om2 = om * om;
    float t = om2 * om2 * om;
    float s = (1.0f - m) / (1.0f - sp);
    V f0 = mk(0.04f, 0.04f, 0.04f) * (1.0f - m) + rho * m;
    const float spr = (t * (3.0f - f0.x - f0.y - f0.z) + (f0.x + f0.y + f0.z)) * (1.0f / 3.0f);
    dsp_dalb = spr > 0.1f && spr < 0.9f ? m * (1.0f - t) * (1.0f / 3.0f) : 0.0f;
    V F = f0 * (1.0f - t) + mk(t, t, t);
    drho = mk(s * ((1.0f - F.x) - rho.x * m * (1.0f - t)), s * ((1.0f - F.y) - rho.y * m * (1.0f - t)),
              s * ((1.0f - F.z) - rho.z * m * (1.0f - t)));
    return mk((1.0f - F.x) * s * rho.x, (1.0f - F.y) * s * rho.y, (1.0f - F.z) * s * rho.z);
}

// NEE geometry term G(p) = cos * cos_l * A * N / (pi d^2) for a fixed light point y
// (render.rs:1439-1465); with GRAD, also its gradient with respect to the shading point p.
template <bool GRAD>
__device__ float nee_geometry(V p, V n, V y, V nl, float area_n, V& grad) {
    if constexpr (GRAD) {
        VDn<3> pd = vd<3>(p);
        pd.x.d[0] = 1.0f;
        pd.y.d[1] = 1.0f;
        pd.z.d[2] = 1.0f;
        VDn<3> tl = vd<3>(y) - pd;
        Dn<3> d2 = ddot(tl, tl);
        Dn<3> dist = dsqrt(d2);
        VDn<3> dir = tl * (1.0f / dist);
        Dn<3> ct = ddot(n, dir);
        Dn<3> ctl = dabs(ddot(-nl, dir));
        Dn<3> G = ct * ctl * (area_n / CUDART_PI_F) / d2;
        grad = mk(G.d[0], G.d[1], G.d[2]);
        return G.v;
    } else {
        V tl = y - p;
        float d2 = len2(tl);
        V dir = tl * rsqrtf(d2);
        return dot(n, dir) * fabsf(dot(-nl, dir)) * (area_n / CUDART_PI_F) / d2;
    }
}

struct alignas(16) Vert {
    V p, n, d_in, B;   // hit point, facing normal, incoming direction, throughput to this vertex
    float t;           // p = previous origin + t * d_in
    float sp;          // microfacet lobe probability (when the material is Microfacet)
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

// Flags of a replayed vertex after its shading step at bounce b0 (now at bounce b1), and the
// microfacet lobe probability sp (material.rs:340-345).
__device__ __forceinline__ uint32_t vertex_flags(const SceneDev& S, const RenderDev& R, uint32_t pixel, uint32_t st,
                                                 uint32_t b0, uint32_t b1, int prim, const Surface& sf, V d_in,
                                                 bool skip, float& sp) {
    const int pt = prim_type(S, prim);
    uint32_t f = (pt == PT_QUAD || pt == PT_TRIANGLE || pt == PT_DISK || pt == 100) ? VF_FLAT : 0u;
    const MatDev& m = S.mats[sf.mat];
    if (!skip && m.kind == 4) f |= VF_EMIT;
    sp = 0.0f;
    if (b1 > b0) f |= VF_CONT;                                         // scatter survived RR
    if (m.kind == 5 && (f & VF_CONT)) {
        float4 su = draw4(R.key0, R.key1, pixel, st, b0, CALL_SCATTER);
        V alb = tex_value(m, sf.p);
        V v = unit(-d_in);
        float ndv = fmaxf(dot(sf.n, v), 0.001f);
        V f0 = mk(0.04f, 0.04f, 0.04f) * (1.0f - m.metallic) + alb * m.metallic;
        V fw = fresnel(ndv, f0);
        sp = fminf(fmaxf((fw.x + fw.y + fw.z) * (1.0f / 3.0f), 0.1f), 0.9f);
        if (su.x < sp) f |= VF_SPEC;
    }
    return f;
}

// The NEE term of vertex vx (light emission EL, attenuation att, geometry G) and, with GEO,
// dG/dp.  Returns false when the sample is void.
template <bool GEO>
__device__ __forceinline__ bool nee_term(const SceneDev& S, const Vert& vx, V att, float4 nu, int& li, V& EL, float& Gv,
                                         V& gradG) {
    const int nl = S.n_lights;
    li = min((int)(nu.y * (float)nl), nl - 1);
    const LightDev& Lt = S.lights[li];
    Ray srr;
    float tmax;
    V contrib;
    if (!sample_light(S, vx.p, vx.n, att, nu, srr, tmax, contrib)) return false;
    EL = mk(Lt.e);
    gradG = mk(0.f, 0.f, 0.f);
    if (Lt.kind == 2 || Lt.kind == 3) {
        V y;
        if (Lt.kind == 2) {
            y = mk(Lt.p0) + mk(Lt.u) * nu.z + mk(Lt.v) * nu.w;
        } else {
            float r = sqrtf(nu.z) * Lt.radius, sp2, cp2;
            sincospif(2.0f * nu.w, &sp2, &cp2);
            V wl = mk(Lt.n);
            V av = fabsf(wl.x) > 0.9f ? mk(0.f, 1.f, 0.f) : mk(1.f, 0.f, 0.f);
            V ut = unit(cross(wl, av));
            V vt = cross(wl, ut);
            y = mk(Lt.p0) + ut * (r * cp2) + vt * (r * sp2);
        }
        Gv = nee_geometry<GEO>(vx.p, vx.n, y, mk(Lt.n), Lt.area * (float)nl, gradG);
    } else {                                   // sphere light: G held constant in p
        float ea = EL.x * att.x;
        Gv = ea != 0.0f ? contrib.x / ea : 0.0f;
    }
    return true;
}

// Per-path record of the replay (one slot per path of the chunk).
struct alignas(16) PathHead {
    V L;            // radiance of the path (input of the luminance clamp)
    float jx;
    V bg;           // background radiance after the last vertex (0 if the path ended on a surface)
    float jy;
    int K;          // recorded vertices; -1 = no path in this slot
    uint32_t pixel; // global pixel id (RNG key)
    uint32_t local; // j * w + i within the output
    uint32_t st;    // stratum
};

// The backward sweep of one replayed path: K vertices at vb[k * stride].
//   w_j = a (.) B_j ; grad(e_j) += w_j ; grad(E_L) += w_j (.) att_j G_j ;
//   abar_j = w_j (.) (rrw_j S_{j+1} + E_L G_j) ; grad(albedo, roughness) += abar_j . d att_j
// Position and direction adjoints are needed only behind the first specular-lobe microfacet
// vertex (the only parameter-dependent direction), so vertices up to it take the cheap form.
__device__ void sweep_path(const SceneDev& S, const RenderDev& R, const PathHead& ph, V gpix, float inv_wsum,
                           const int* light_mat, float* smem, int n_mat, const Grads& G, const Vert* vb, size_t stride) {
    const uint32_t pixel = ph.pixel, st = ph.st;
    const int K = ph.K;
    // adjoint of L through the luminance clamp (render.rs:1692-1697), mean over strata
    const V Lw = mk(0.2126f, 0.7152f, 0.0722f);
    float lum = dot(Lw, ph.L);
    V a = gpix * inv_wsum;
    if (lum > 100.0f) {                          // f(L) = 100 L / lum(L)
        float s = 100.0f / lum;
        float la = dot(a, ph.L);
        a = (a - Lw * (la / lum)) * s;
    }
    float wf = filter_weight(R.pixel_filter, ph.jx - 0.5f, ph.jy - 0.5f);
    a = a * wf;
    int first_spec = K;
    for (int q = 0; q < K; ++q)
        if (vb[(size_t)q * stride].flags & VF_SPEC) {
            first_spec = q;
            break;
        }
    V S_next = ph.bg;
    V Dbar = mk(0.f, 0.f, 0.f);   // adjoint of the outgoing direction of the current vertex
    V Pbar = mk(0.f, 0.f, 0.f);   // adjoint of the position of the next vertex, pulled back below
    for (int j = K - 1; j >= 0; --j) {
        const Vert vx = vb[(size_t)j * stride];
        const MatDev& m = S.mats[vx.mat];
        const bool geo = j > first_spec;   // this vertex's position/direction depend on parameters
        const V w = mul(a, vx.B);
        V c = mk(0.f, 0.f, 0.f);
        if (vx.flags & VF_EMIT) {
            c = emitted(m, vx.p);
            add_grad(smem, n_mat, G, vx.mat, 4, w.x);
            add_grad(smem, n_mat, G, vx.mat, 5, w.y);
            add_grad(smem, n_mat, G, vx.mat, 6, w.z);
        }
        V PbarJ = mk(0.f, 0.f, 0.f);   // adjoint of this vertex's position
        V DbarIn = mk(0.f, 0.f, 0.f);  // adjoint of this vertex's incoming direction
        if (vx.flags & VF_CONT) {
            const uint32_t depth = R.max_depth - (uint32_t)j;
            const float4 su = draw4(R.key0, R.key1, pixel, st, (uint32_t)j, CALL_SCATTER);
            const bool spec = (vx.flags & VF_SPEC) != 0;
            V att_v, drho = mk(0.f, 0.f, 0.f);
            V datt[4] = {};               // d att / d (d_in.x, d_in.y, d_in.z, roughness), sp held
            V dl[4] = {};                 // d l / d (same), specular lobe
            float dsp_dalb = 0.0f;        // d sp / d albedo (each channel), microfacet
            V dsp_dd = mk(0.f, 0.f, 0.f); // d sp / d d_in
            if (m.kind == 5) {
                V alb = tex_value(m, vx.p);
                if (geo) {
                    VDn<4> att, l;
                    microfacet_dual<4>(vx.n, vx.d_in, m.roughness, alb, m.metallic, su.y, su.z, spec, vx.sp, att, l,
                                       drho, dsp_dalb, dsp_dd);
                    att_v = mk(att.x.v, att.y.v, att.z.v);
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        datt[k] = mk(att.x.d[k], att.y.d[k], att.z.d[k]);
                        dl[k] = mk(l.x.d[k], l.y.d[k], l.z.d[k]);
                    }
                } else if (spec) {
                    VDn<1> att, l;
                    V unused;
                    microfacet_dual<1>(vx.n, vx.d_in, m.roughness, alb, m.metallic, su.y, su.z, true, vx.sp, att, l,
                                       drho, dsp_dalb, unused);
                    att_v = mk(att.x.v, att.y.v, att.z.v);
                    datt[3] = mk(att.x.d[0], att.y.d[0], att.z.d[0]);
                    dl[3] = mk(l.x.d[0], l.y.d[0], l.z.d[0]);
                } else {
                    att_v = microfacet_diffuse(vx.n, vx.d_in, alb, m.metallic, vx.sp, drho, dsp_dalb);
                }
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
                const float4 nu = draw4(R.key0, R.key1, pixel, st, (uint32_t)j, CALL_NEE);
                int li;
                V EL, gradG;
                float Gv;
                bool ok = geo ? nee_term<true>(S, vx, att_v, nu, li, EL, Gv, gradG)
                              : nee_term<false>(S, vx, att_v, nu, li, EL, Gv, gradG);
                if (ok) {
                    nee = mul(EL, att_v) * Gv;
                    c = c + nee;
                    abar = abar + mul(w, EL) * Gv;
                    int lm = light_mat ? light_mat[li] : -1;
                    V gE = mul(w, att_v) * Gv;
                    add_grad(smem, n_mat, G, lm, 4, gE.x);
                    add_grad(smem, n_mat, G, lm, 5, gE.y);
                    add_grad(smem, n_mat, G, lm, 6, gE.z);
                    if (geo) PbarJ = PbarJ + gradG * dot(mul(w, EL), att_v);
                }
            }
            // The NEE term is added only on paths that survive Russian roulette and is not divided
            // by the survival probability (render.rs:1497-1524): its expectation carries surv(att),
            // so the unbiased derivative adds (surv'/surv) * (NEE contribution), surv' taken with
            // the lobe probability's own dependence on albedo and direction.
            V ga = mul(abar, drho);                          // albedo gradient of this vertex
            float gr_score = 0.0f;
            V dscore = mk(0.f, 0.f, 0.f);                    // its incoming-direction part
            const float mx = fmaxf(fmaxf(att_v.x, att_v.y), att_v.z);
            if (depth < 47 && mx > 0.05f && mx < 1.0f && (nee.x != 0.0f || nee.y != 0.0f || nee.z != 0.0f)) {
                const int cs = att_v.x == mx ? 0 : (att_v.y == mx ? 1 : 2);
                const float coef = dot(w, nee) / mx;
                if (m.kind == 1 || m.kind == 2) {
                    ga = ga + mk(cs == 0 ? coef : 0.f, cs == 1 ? coef : 0.f, cs == 2 ? coef : 0.f);
                } else if (m.kind == 5) {
                    // d att_c / d albedo_k = drho_c [c == k] + att_c * (-1/sp | 1/(1-sp)) * dsp/dalbedo_k
                    const float sl = (spec ? -1.0f / vx.sp : 1.0f / (1.0f - vx.sp)) * mx;
                    const float dc = cs == 0 ? drho.x : (cs == 1 ? drho.y : drho.z);
                    const float common = coef * sl * dsp_dalb;
                    ga = ga + mk(common + (cs == 0 ? coef * dc : 0.f), common + (cs == 1 ? coef * dc : 0.f),
                                 common + (cs == 2 ? coef * dc : 0.f));
                    auto comp = [cs](V v) { return cs == 0 ? v.x : (cs == 1 ? v.y : v.z); };
                    gr_score = coef * comp(datt[3]);
                    if (geo) dscore = (mk(comp(datt[0]), comp(datt[1]), comp(datt[2])) + dsp_dd * sl) * coef;
                }
            }
            // albedo / roughness through att
            add_grad(smem, n_mat, G, vx.mat, 0, ga.x);
            add_grad(smem, n_mat, G, vx.mat, 1, ga.y);
            add_grad(smem, n_mat, G, vx.mat, 2, ga.z);
            if (m.kind == 5) {
                float gr = dot(abar, datt[3]) + gr_score;
                if (spec) gr += dot(Dbar, dl[3]);            // outgoing direction l(d_in, r)
                add_grad(smem, n_mat, G, vx.mat, 3, gr);
                if (geo) {
                    DbarIn = mk(dot(abar, datt[0]), dot(abar, datt[1]), dot(abar, datt[2])) + dscore;
                    if (spec) DbarIn = DbarIn + mk(dot(Dbar, dl[0]), dot(Dbar, dl[1]), dot(Dbar, dl[2]));
                }
            }
            S_next = c + mul(att_v, S_next) * rrw;
        } else {
            S_next = c;
        }
        if (!geo) {
            Dbar = mk(0.f, 0.f, 0.f);
            Pbar = mk(0.f, 0.f, 0.f);
            continue;
        }
        // position adjoint of this vertex, then through p_j = p_{j-1} + t d_j
        PbarJ = PbarJ + Pbar;
        Pbar = mk(0.f, 0.f, 0.f);
        if (vx.flags & VF_FLAT) {
            float nd = dot(vx.n, vx.d_in);
            if (fabsf(nd) > 1e-12f) {
                V MtP = PbarJ - vx.n * (dot(vx.d_in, PbarJ) / nd);
                Pbar = MtP;                      // adjoint of the previous vertex's position
                DbarIn = DbarIn + MtP * vx.t;
            }
        }
        // the incoming direction of vertex j is the outgoing direction of vertex j-1; only a
        // microfacet vertex's direction depends on parameters (used at j-1 via Dbar)
        Dbar = DbarIn;
    }
}

#ifndef LUM_ADJ_MIN_BLOCKS
#define LUM_ADJ_MIN_BLOCKS 5
#endif

constexpr uint32_t kReplayStrata = 8;   // strata per replay task (tile x stratum group)

// Replay kernel: the forward megakernel's state machine (same functions, same RNG keys, one
// traversal per loop iteration for every tracing lane) over the tiles [t0, t1), a task being
// one 8x4 tile and a group of kReplayStrata strata.  Each path's vertices and head go to the
// chunk's slots: slot = ((tile - t0) * n_strata + s) * 32 + lane, vertex k of a slot at
// verts[k * n_slots + slot].
// CLS: the scene class (tracer.cuh), as for the megakernel's class builds.
template <int CLS>
__global__ void __launch_bounds__(128, LUM_ADJ_MIN_BLOCKS) k_replay(SceneDev S, RenderDev R, const float* __restrict__ dldi,
                                                                  uint32_t t0, uint32_t t1, PathHead* __restrict__ heads,
                                                                  Vert* __restrict__ verts, size_t n_slots,
                                                                  float* __restrict__ inv_wsum_px, WorkCounters* wc) {
    extern __shared__ int smem_raw[];
    int* stack = smem_raw + threadIdx.x;
    const int lane = threadIdx.x & 31;
    uint32_t err = 0;
    const uint32_t n_st = R.s_end - R.s_begin;
    const uint32_t n_groups = (n_st + kReplayStrata - 1) / kReplayStrata;
    const uint32_t n_tasks = (t1 - t0) * n_groups;
    enum : int { A_IDLE = 0, A_CLOSEST = 1, A_SHADOW = 2, A_DONE = 3 };
    for (;;) {
        uint32_t task = 0;
        if (lane == 0) task = atomicAdd(&wc->next_task, 1u);
        task = __shfl_sync(kFullMask, task, 0);
        if (task >= n_tasks) break;
        const uint32_t tile = t0 + task / n_groups, group = task % n_groups;
        const uint32_t s_lo = R.s_begin + group * kReplayStrata, s_hi = min(R.s_end, s_lo + kReplayStrata);
        const uint32_t i = (tile % R.tiles_x) * 8 + (lane & 7);
        const uint32_t j = (tile / R.tiles_x) * 4 + (lane >> 3);
        const bool valid = i < R.w && j < R.h;
        const uint32_t gi = i + R.crop_x, gj = j + R.crop_y;
        const uint32_t pixel = gj * R.full_w + gi;
        const size_t slot_base = (size_t)(tile - t0) * n_st * 32 + lane;
        uint32_t st = s_hi;
        if (valid) {
            const float* g = dldi + 3 * ((size_t)j * R.w + i);
            if (g[0] != 0.0f || g[1] != 0.0f || g[2] != 0.0f) st = s_lo;
        }
        if (valid && group == 0) {
            // pixel = sum_s f(L_s) w_s / sum_s w_s (render.rs:1699-1705)
            float wsum = 0.0f;
            if (R.pixel_filter == LUM_FILTER_BOX) {
                wsum = (float)n_st;
            } else {
                for (uint32_t s2 = R.s_begin; s2 < R.s_end; ++s2) {
                    float4 c = draw4(R.key0, R.key1, pixel, s2, 0, CALL_CAMERA);
                    uint32_t sx = s2 % R.sqrt_spp, sy = s2 / R.sqrt_spp;
                    float inv_n = 1.0f / (float)R.sqrt_spp;
                    wsum += filter_weight(R.pixel_filter, ((float)sx + c.x) * inv_n - 0.5f,
                                          ((float)sy + c.y) * inv_n - 0.5f);
                }
            }
            inv_wsum_px[(size_t)j * R.w + i] = wsum > 0.0f ? 1.0f / wsum : 1.0f;
        }
        if (st == s_hi)                                 // nothing to replay for this lane
            for (uint32_t s2 = s_lo; s2 < s_hi; ++s2) heads[slot_base + (size_t)(s2 - R.s_begin) * 32].K = -1;
        int state = A_IDLE;
        uint32_t cur = 0;
        int K = 0;
        uint32_t vflags = 0;
        float vsp = 0.0f;
        V bg = mk(0.f, 0.f, 0.f);
        Path P;
        Pending pend;
        Hit h;                  // closest hit so far of the lane's walk
        Trav tv;                // place of a suspended walk
        bool found = false, walking = false;
        for (;;) {
            if (state == A_IDLE && st < s_hi) {
                start_path<philox_unroll<CLS>()>(S, R, gi, gj, pixel, st, P);
                cur = st++;
                K = 0;
                bg = mk(0.f, 0.f, 0.f);
                state = R.max_depth > 0 ? A_CLOSEST : A_DONE;
            }
            if (!__any_sync(kFullMask, state != A_IDLE)) break;
            const size_t slot = slot_base + (size_t)(cur - R.s_begin) * 32;
            if (state == A_CLOSEST || state == A_SHADOW) {
                const bool shadow = state == A_SHADOW;
                Ray r;
                r.o = P.ray.o;
                r.d = shadow ? pend.dir : P.ray.d;
                r.time = shadow ? 0.0f : P.ray.time;
                if (!walking) {
                    h.t = shadow ? pend.tmax : CUDART_INF_F;
                    h.prim = -1;
                    h.b1 = h.b2 = 0.0f;
                    tv.node = S.n_nodes > 0 ? 0 : kSentinel;
                    tv.sp = 0;
                    found = false;
                }
                walking = !trace_resume<false, false, LUM_SUSPEND_LANES, CLS>(S, r, 0.001f, shadow, h, found, tv, stack,
                                                                             err);
                if (walking) {
                    // suspended: resumes in a later iteration
                } else if (shadow) {
                    if (!found) {
                        P.L = P.L + pend.contrib;
                        vflags |= VF_VIS;
                    }
                    verts[(size_t)(K - 1) * n_slots + slot].flags = vflags;
                    state = P.bounce >= R.max_depth ? A_DONE : A_CLOSEST;
                } else if (!found) {
                    bg = background(S, R, P.ray);                     // render.rs:1535
                    P.L = P.L + mul(P.beta, bg);
                    state = A_DONE;
                } else {
                    const Ray in = P.ray;
                    const V B = P.beta;
                    const bool skip = P.skip_emission;
                    Surface sf = surface_of<false, CLS>(S, in, h);
                    const bool finite = isfinite(sf.p.x) && isfinite(sf.p.y) && isfinite(sf.p.z);
                    const uint32_t b0 = P.bounce;
                    // the adjoint rejects the other materials: the base-material shading
                    const int stt = shade<-1, false, true, false, CLS>(S, R, pixel, P, true, h, pend);
                    if (finite) {
                        Vert& vx = verts[(size_t)K * n_slots + slot];
                        vx.p = sf.p;
                        vx.n = sf.n;
                        vx.d_in = in.d;
                        vx.B = B;
                        vx.t = h.t;
                        vx.mat = sf.mat;
                        vflags = vertex_flags(S, R, pixel, cur, b0, P.bounce, h.prim, sf, in.d, skip, vsp);
                        if (stt == ST_SHADOW) vflags |= VF_NEE;
                        vx.sp = vsp;
                        vx.flags = vflags;
                        ++K;
                    }
                    state = stt == ST_SHADOW ? A_SHADOW : (stt == ST_CLOSEST ? A_CLOSEST : A_DONE);
                }
            }
            if (state == A_DONE) {
                PathHead ph;
                ph.L = P.L;
                ph.jx = P.jx;
                ph.bg = bg;
                ph.jy = P.jy;
                ph.K = K;
                ph.pixel = pixel;
                ph.local = j * R.w + i;
                ph.st = cur;
                heads[slot] = ph;
                state = A_IDLE;
            }
        }
    }
    if (err) atomicOr(&wc->error_flags, err);
}

// Sweep kernel: one path slot per thread (grid-stride over n_slots; vertex k of a slot at
// verts[k * stride + slot]), gradients accumulated per block in shared memory when use_smem,
// else with global atomics.
__global__ void __launch_bounds__(128) k_sweep(SceneDev S, RenderDev R, const float* __restrict__ dldi,
                                               const int* __restrict__ light_mat, const PathHead* __restrict__ heads,
                                               const Vert* __restrict__ verts, size_t n_slots, size_t stride,
                                               const float* __restrict__ inv_wsum_px, Grads G, int n_mat, int use_smem) {
    extern __shared__ float gsm_raw[];
    float* gsm = use_smem ? gsm_raw : nullptr;
    if (gsm)
        for (int k = threadIdx.x; k < 7 * n_mat; k += blockDim.x) gsm[k] = 0.0f;
    __syncthreads();
    for (size_t slot = (size_t)blockIdx.x * blockDim.x + threadIdx.x; slot < n_slots;
         slot += (size_t)gridDim.x * blockDim.x) {
        const PathHead ph = heads[slot];
        if (ph.K <= 0) continue;
        const float* g = dldi + 3 * (size_t)ph.local;
        const V gpix = mk(g[0], g[1], g[2]) * R.exposure;
        sweep_path(S, R, ph, gpix, inv_wsum_px[ph.local], light_mat, gsm, n_mat, G, verts + slot, stride);
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
    if (params && (params->adaptive || params->time_limit > 0.0))
        return lum::set_error(LUM_ERR_UNSUPPORTED, "the differentiable render has no adaptive sampling or time limit");
    return lum_render(scene, params, out_rgb, stats);
}

lum_status lum_backward(lum_scene* scene, const lum_render_params* params, const float* dL_dimage,
                        const int32_t* light_material, float* d_albedo, float* d_roughness, float* d_emission,
                        lum_stats* stats) {
    using namespace lum;
    auto t0 = std::chrono::steady_clock::now();
    if (!scene || !params || !dL_dimage || !d_albedo || !d_roughness || !d_emission)
        return set_error(LUM_ERR_INVALID_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> lk(scene_mutex(scene));
    SceneDev dev;
    RenderDev R;
    cudaStream_t stream;
    lum_status st = prepare_render(scene, params, dev, R, stream);
    if (st != LUM_OK) return st;
    if (R.max_depth > (uint32_t)adj::kMaxVerts)
        return set_error(LUM_ERR_UNSUPPORTED, "lum_backward supports max_depth <= 16");
    if (scene_max_material_kind(scene) > LUM_MAT_ISOTROPIC)
        return set_error(LUM_ERR_UNSUPPORTED, "lum_backward differentiates Lambertian, Metal, Dielectric, Emissive, "
                                              "Microfacet and Isotropic materials only");
    const int n_mat = dev.n_mats;
    if (light_material)
        for (int k = 0; k < dev.n_lights; ++k)
            if (light_material[k] < -1 || light_material[k] >= n_mat)
                return set_error(LUM_ERR_INVALID_ARGUMENT, "light_material names no material");
    const size_t px = (size_t)R.w * R.h;
    std::memset(d_albedo, 0, sizeof(float) * 3 * n_mat);
    std::memset(d_roughness, 0, sizeof(float) * n_mat);
    std::memset(d_emission, 0, sizeof(float) * 3 * n_mat);
    if (px == 0 || R.s_end <= R.s_begin || n_mat == 0 || R.max_depth == 0) return LUM_OK;
    // Paths are replayed a chunk of tiles at a time into a staging buffer of vertex records
    // (bounded, at most 8 GiB or a quarter of free device memory), then swept.
    const uint32_t n_st = R.s_end - R.s_begin;
    const size_t per_tile = (size_t)32 * n_st * (sizeof(adj::PathHead) + (size_t)R.max_depth * sizeof(adj::Vert));
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    const size_t budget = std::max<size_t>(per_tile, std::min<size_t>((size_t)8 << 30, free_b / 4));
    const uint32_t chunk_tiles = (uint32_t)std::min<size_t>(R.n_tasks, budget / per_tile);
    const size_t n_slots = (size_t)chunk_tiles * 32 * n_st;
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    const size_t bytes_img = sizeof(float) * 3 * px, bytes_g = sizeof(float) * 7 * n_mat,
                 bytes_lm = sizeof(int) * (dev.n_lights + 1), bytes_ws = sizeof(float) * px,
                 bytes_heads = sizeof(adj::PathHead) * n_slots,
                 bytes_verts = sizeof(adj::Vert) * n_slots * R.max_depth;
    const size_t o_g = al(bytes_img), o_lm = o_g + al(bytes_g), o_ws = o_lm + al(bytes_lm), o_wc = o_ws + al(bytes_ws),
                 o_heads = o_wc + al(sizeof(WorkCounters)), o_verts = o_heads + al(bytes_heads),
                 total = o_verts + al(bytes_verts);
    char* buf = nullptr;
    cudaError_t e = cudaMalloc(&buf, total);
    if (e != cudaSuccess) return adj_cuda(e, "cudaMalloc");
    float* d_img = (float*)buf;
    float* d_g = (float*)(buf + o_g);
    int* d_lm = (int*)(buf + o_lm);
    float* d_ws = (float*)(buf + o_ws);
    WorkCounters* wc = (WorkCounters*)(buf + o_wc);
    adj::PathHead* d_heads = (adj::PathHead*)(buf + o_heads);
    adj::Vert* d_verts = (adj::Vert*)(buf + o_verts);
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
        int nsm = 0, devi = 0;
        cudaGetDevice(&devi);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, devi);
        const size_t stack = (size_t)kStackDepth * 128 * sizeof(int);
        auto replay = dev.cls == CLS_QUAD ? adj::k_replay<CLS_QUAD>
                    : dev.cls == CLS_MESH ? adj::k_replay<CLS_MESH> : adj::k_replay<CLS_ALL>;
        int occ_r = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_r, replay, 128, stack);
        // Gradients accumulate per block in shared memory when the material table fits
        // (LUM_ADJ_GRADS=smem|global overrides), else with global atomics.
        int use_smem = bytes_g <= 64 * 1024 ? 1 : 0;
        if (const char* env = std::getenv("LUM_ADJ_GRADS")) {
            if (!std::strcmp(env, "smem") && bytes_g <= 200 * 1024) use_smem = 1;
            if (!std::strcmp(env, "global")) use_smem = 0;
        }
        const size_t smem_s = use_smem ? bytes_g : 0;
        if (smem_s > 48 * 1024) cudaFuncSetAttribute(adj::k_sweep, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_s);
        int occ_s = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_s, adj::k_sweep, 128, smem_s);
        const uint32_t n_groups = (n_st + adj::kReplayStrata - 1) / adj::kReplayStrata;
        const int grid_r = (int)std::min<size_t>((size_t)nsm * std::max(occ_r, 1), ((size_t)chunk_tiles * n_groups + 3) / 4);
        const int grid_s = (int)std::min<size_t>((size_t)nsm * std::max(occ_s, 1), (n_slots + 127) / 128);
        cudaEventRecord(ev0, stream);
        for (uint32_t c0 = 0; ok && c0 < R.n_tasks; c0 += chunk_tiles) {
            const uint32_t c1 = std::min<uint32_t>(R.n_tasks, c0 + chunk_tiles);
            const size_t slots = (size_t)(c1 - c0) * 32 * n_st;
            e = cudaMemsetAsync(&wc->next_task, 0, sizeof(uint32_t), stream);
            if (e == cudaSuccess) {
                replay<<<grid_r, 128, stack, stream>>>(dev, R, d_img, c0, c1, d_heads, d_verts, n_slots, d_ws, wc);
                e = cudaGetLastError();
            }
            if (e == cudaSuccess) {
                const int gs = (int)std::min<size_t>((size_t)grid_s, (slots + 127) / 128);
                adj::k_sweep<<<gs, 128, smem_s, stream>>>(dev, R, d_img, d_lm, d_heads, d_verts, slots, n_slots, d_ws, G,
                                                           n_mat, use_smem);
                e = cudaGetLastError();
            }
            ok = e == cudaSuccess;
        }
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
