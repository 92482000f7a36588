// tonemap.cu -- linear HDR image -> RGBA8 on the GPU: exposure (optionally automatic), the
// reference's per-pixel colour chain, tone curve and sRGB quantisation.
//
// The chain restates render::render's per-pixel loop (src/render.rs:3100-3260) for its
// colour steps, with the tone curves and gamma_correct of src/render.rs:3608-3658 and the
// auto-exposure key value of src/render.rs:2594-2606 (log-average luminance,
// src/render.rs:525-540).  The colour steps run in f64 like the reference's; the tone curve and
// sRGB power run in f32 with an f64 re-evaluation near byte boundaries (tone_gamma), so the
// bytes agree with an f64 restatement except where a last-bit difference meets a boundary.
//
// Kernels (HBM-bound: 12 bytes in, 4 bytes out per pixel):
//   k_loglum   fixed grid of 256 x 256 threads, each summing ln(1e-4 + max(lum, 0)) (f32 log,
//              f64 sum) over a grid stride, a shared-memory tree per block -> 256 partials.  The
//              grid does not depend on the device, so the sum is reproducible.
//   k_tonemap  4 pixels per thread: three 16-byte loads of 12 floats, one 16-byte store of
//              4 RGBA pixels (a scalar tail with byte stores for pixel counts not divisible
//              by 4, or for buffers that are not 16-byte aligned).  With auto-exposure each block first
//              sums the 256 partials in the same fixed order.  The common chain (no optional
//              step) reads each channel's byte from a table of the chain's 255 byte thresholds
//              (one entry lookup per channel, see ByteTable); chains with optional steps, and
//              tone curves whose table does not fit, take the f32 path with its f64 fallback.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <type_traits>
#include <vector>

#include "../../include/luminara_gpu.h"
#include "kernels.h"
#include "scene_access.h"

namespace lum {
namespace tone {

constexpr int kLogBlocks = 256;
constexpr int kLogThreads = 256;
constexpr int kThreads = 256;
static_assert(kLogBlocks * sizeof(double) <= LUM_TONEMAP_SCRATCH_BYTES, "scratch too small");

struct Chain {
    lum_tonemap_params p;
    double cos_h, sin_h;          // hue rotation
    int16_t bright_off;           // (brightness * 255) as i16
    bool wb, hue, sat, grade, bright, contrast, sepia, tint, balance;
    bool extra;                   // any step beyond exposure, tone curve and gamma
    float inv_gamma;              // 1/gamma, or 0 for the sRGB transfer function
};

// Rust's `as u8` from f64: truncation, saturating, NaN -> 0.
__host__ __device__ __forceinline__ uint32_t sat_u8(double x) {
    if (!(x > 0.0)) return 0u;
    if (x >= 255.0) return 255u;
    return (uint32_t)x;
}

__host__ __device__ __forceinline__ double clamp01(double x) { return fmin(fmax(x, 0.0), 1.0); }

// Tone curves (src/render.rs:3608-3641).
__host__ __device__ __forceinline__ double tone_curve(int kind, double x) {
    x = fmax(x, 0.0);   // f64::max ignores NaN
    switch (kind) {
        case LUM_TONEMAP_REINHARD:
            return x / (1.0 + x);
        case LUM_TONEMAP_FILMIC: {
            auto uc2 = [](double v) {
                const double a = 0.15, b = 0.50, c = 0.10, d = 0.20, e = 0.02, f = 0.30;
                return ((v * (a * v + c * b) + d * e) / (v * (a * v + b) + d * f)) - e / f;
            };
            return clamp01(uc2(x) / uc2(11.2));
        }
        case LUM_TONEMAP_NONE:
            return clamp01(x);
        default: {
            const double a = 2.51, b = 0.03, c = 2.43, d = 0.59, e = 0.14;
            return clamp01((x * (a * x + b)) / (x * (c * x + d) + e));
        }
    }
}

// Tone curve in f32 (the fast path of tone_gamma below).
__device__ __forceinline__ float tone_curve_f(int kind, float x) {
    x = fmaxf(x, 0.0f);
    switch (kind) {
        case LUM_TONEMAP_REINHARD:
            return x / (1.0f + x);
        case LUM_TONEMAP_FILMIC: {
            auto uc2 = [](float v) {
                const float a = 0.15f, b = 0.50f, c = 0.10f, d = 0.20f, e = 0.02f, f = 0.30f;
                return ((v * (a * v + c * b) + d * e) / (v * (a * v + b) + d * f)) - e / f;
            };
            return fminf(fmaxf(uc2(x) / uc2(11.2f), 0.0f), 1.0f);
        }
        case LUM_TONEMAP_NONE:
            return fminf(fmaxf(x, 0.0f), 1.0f);
        default: {
            const float a = 2.51f, b = 0.03f, c = 2.43f, d = 0.59f, e = 0.14f;
            return fminf(fmaxf((x * (a * x + b)) / (x * (c * x + d) + e), 0.0f), 1.0f);
        }
    }
}

// gamma_correct (src/render.rs:3648-3658): sRGB transfer function (gamma <= 0) or 1/gamma
// power, plus the dither offset, quantised as (s + dither).clamp(0, 0.999) * 256.
__host__ __device__ __forceinline__ double quantised(double s, double dither) {
    double q = s + dither;
    if (q != q) return -1.0;
    return fmin(fmax(q, 0.0), 0.999) * 256.0;
}

__host__ __device__ __forceinline__ double srgb64(double x, double gamma) {
    if (gamma > 0.0) return pow(x, 1.0 / gamma);
    return x <= 0.0031308 ? 12.92 * x : 1.055 * pow(x, 1.0 / 2.4) - 0.055;
}

// Tone curve + gamma_correct of one channel.  The tone curve and the power run in f32: from an
// exact f64 input their result moves the scaled value q by less than 1e-4 of a byte step.  Only
// when q lies within 1e-3 of an integer, where truncation could then differ from the f64
// result, is the channel evaluated again in f64; so the bytes are those of the f64 formulas at
// a fraction of their cost.
__device__ __noinline__ double tone_gamma64(int kind, double x, double gamma, double dither) {
    return quantised(srgb64(clamp01(tone_curve(kind, x)), gamma), dither);
}

__device__ __forceinline__ uint32_t tone_gamma(int kind, double x, double gamma, double dither) {
    if (x != x) return 0u;
    const float t = tone_curve_f(kind, (float)x);
    float sf;
    if (gamma > 0.0) sf = powf(t, (float)(1.0 / gamma));
    else sf = t <= 0.0031308f ? 12.92f * t : 1.055f * powf(t, 1.0f / 2.4f) - 0.055f;
    double q = quantised((double)sf, dither);
    const double fr = q - floor(q);
    if (fr < 2e-3 || fr > 1.0 - 2e-3) q = tone_gamma64(kind, x, gamma, dither);
    return q < 0.0 ? 0u : sat_u8(q);
}

// One pixel of the full chain (src/render.rs:3100-3260); pixel p = j * w + i of the output.
__device__ __noinline__ uint32_t pixel_full(const Chain& C, double r, double g, double b, uint32_t p, uint32_t w,
                                            uint32_t h, double exposure) {
    const lum_tonemap_params& P = C.p;
    uint32_t i = 0, j = 0;
    if (P.vignette > 0.0 || P.dither) {
        j = p / w;
        i = p - j * w;
    }
    double vf = 1.0;
    if (P.vignette > 0.0) {
        const double cx = ((double)i + 0.5) / (double)w - 0.5, cy = ((double)j + 0.5) / (double)h - 0.5;
        vf = fmax(1.0 - (cx * cx + cy * cy) * P.vignette * 4.0, 0.0);
    }
    double cr = r * exposure * vf, cg = g * exposure * vf, cb = b * exposure * vf;
    if (C.wb) {
        cr *= 1.0 + P.white_balance * 0.1;
        cb *= 1.0 - P.white_balance * 0.1;
        cg *= 1.0 + P.white_balance * 0.02;
    }
    if (C.hue) {   // rotation about the grey axis (Rodrigues)
        const double k = 1.0 / 3.0, s3 = 1.0 / sqrt(3.0), ca = C.cos_h, sa = C.sin_h;
        const double d = ca + k * (1.0 - ca), m = k * (1.0 - ca) - s3 * sa, p = k * (1.0 - ca) + s3 * sa;
        const double nr = cr * d + cg * m + cb * p;
        const double ng = cr * p + cg * d + cb * m;
        const double nb = cr * m + cg * p + cb * d;
        cr = fmax(nr, 0.0);
        cg = fmax(ng, 0.0);
        cb = fmax(nb, 0.0);
    }
    if (C.sat) {
        const double lum = 0.2126 * cr + 0.7152 * cg + 0.0722 * cb;
        cr = lum + (cr - lum) * P.saturation;
        cg = lum + (cg - lum) * P.saturation;
        cb = lum + (cb - lum) * P.saturation;
    }
    if (C.grade) {
        const double lum = fmax(0.2126 * cr + 0.7152 * cg + 0.0722 * cb, 0.0);
        const double t = clamp01(lum / (lum + 1.0));
        cr *= P.grade_shadows[0] * (1.0 - t) + P.grade_highlights[0] * t;
        cg *= P.grade_shadows[1] * (1.0 - t) + P.grade_highlights[1] * t;
        cb *= P.grade_shadows[2] * (1.0 - t) + P.grade_highlights[2] * t;
    }
    double dither = 0.0;
    if (P.dither) {   // 4x4 Bayer matrix (src/render.rs:3187-3195), (value - 0.5) / 255
        const uint64_t bayer = 0x5D7F91B36E4CA280ull;   // rows {0,8,2,10} {12,4,14,6} {3,11,1,9} {15,7,13,5}
        const uint32_t v = (uint32_t)(bayer >> (4 * ((j & 3) * 4 + (i & 3)))) & 15u;
        dither = ((double)v / 16.0 - 0.5) / 255.0;
    }
    uint32_t R = tone_gamma(P.tone_map, cr, P.gamma, dither), G = tone_gamma(P.tone_map, cg, P.gamma, dither),
             B = tone_gamma(P.tone_map, cb, P.gamma, dither);
    if (C.bright) {
        R = (uint32_t)min(max((int)R + (int)C.bright_off, 0), 255);
        G = (uint32_t)min(max((int)G + (int)C.bright_off, 0), 255);
        B = (uint32_t)min(max((int)B + (int)C.bright_off, 0), 255);
    }
    if (C.contrast) {
        auto con = [&](uint32_t v) { return sat_u8(fmin(fmax((((double)v / 255.0 - 0.5) * P.contrast + 0.5) * 255.0, 0.0), 255.0)); };
        R = con(R);
        G = con(G);
        B = con(B);
    }
    if (C.sepia) {
        const double fr = R / 255.0, fg = G / 255.0, fb = B / 255.0, s = P.sepia;
        const double sr = fmin(fr * 0.393 + fg * 0.769 + fb * 0.189, 1.0);
        const double sg = fmin(fr * 0.349 + fg * 0.686 + fb * 0.168, 1.0);
        const double sb = fmin(fr * 0.272 + fg * 0.534 + fb * 0.131, 1.0);
        R = sat_u8((fr * (1.0 - s) + sr * s) * 255.0);
        G = sat_u8((fg * (1.0 - s) + sg * s) * 255.0);
        B = sat_u8((fb * (1.0 - s) + sb * s) * 255.0);
    }
    if (C.tint) {
        R = sat_u8(fmin(fmax((R / 255.0 * P.tint[0]) * 255.0, 0.0), 255.0));
        G = sat_u8(fmin(fmax((G / 255.0 * P.tint[1]) * 255.0, 0.0), 255.0));
        B = sat_u8(fmin(fmax((B / 255.0 * P.tint[2]) * 255.0, 0.0), 255.0));
    }
    if (C.balance) {
        R = sat_u8(fmin(fmax(R * P.color_balance[0], 0.0), 255.0));
        G = sat_u8(fmin(fmax(G * P.color_balance[1], 0.0), 255.0));
        B = sat_u8(fmin(fmax(B * P.color_balance[2], 0.0), 255.0));
    }
    if (P.posterize >= 2) {
        const double L = (double)P.posterize;
        auto post = [&](uint32_t v) { return sat_u8(fmin(fmax(round((v / 255.0) * (L - 1.0)) / (L - 1.0) * 255.0, 0.0), 255.0)); };
        R = post(R);
        G = post(G);
        B = post(B);
    }
    return R | (G << 8) | (B << 16) | (255u << 24);
}

// Fast channel path: tone curve KIND and the sRGB / 1/gamma power in f32 with the hardware
// reciprocal and __powf (exp2 of log2), then the exact f64 evaluation (tone_gamma64) only when
// the scaled value lies within kGuard of a byte boundary.  Values below one step are byte 0
// either way.
template <int KIND>
__device__ __forceinline__ float tone_fast(float x) {
    x = fmaxf(x, 0.0f);
    if constexpr (KIND == LUM_TONEMAP_REINHARD) {
        return __fdividef(x, 1.0f + x);
    } else if constexpr (KIND == LUM_TONEMAP_FILMIC) {
        auto uc2 = [](float v) {
            const float a = 0.15f, b = 0.50f, c = 0.10f, d = 0.20f, e = 0.02f, f = 0.30f;
            return __fdividef(fmaf(v, fmaf(a, v, c * b), d * e), fmaf(v, fmaf(a, v, b), d * f)) - e / f;
        };
        const float white = 1.0f / uc2(11.2f);
        return fminf(fmaxf(uc2(x) * white, 0.0f), 1.0f);
    } else if constexpr (KIND == LUM_TONEMAP_NONE) {
        return fminf(x, 1.0f);
    } else {
        const float a = 2.51f, b = 0.03f, c = 2.43f, d = 0.59f, e = 0.14f;
        return fminf(fmaxf(__fdividef(x * fmaf(a, x, b), fmaf(x, fmaf(c, x, d), e)), 0.0f), 1.0f);
    }
}

// Guard window, in byte steps, around each quantisation boundary.  Worst case of the f32 path:
// 1 ulp for the exposure product, 2 ulp __fdividef, 6 ulp __powf (2 + floor(1.173 |y log2 t|)
// with y = 1/2.4 and t >= 0.0031308), a few ulp of fmaf/scaling: < 1.1e-6 relative, i.e. at most
// 2.7e-4 of a step at the top of the range.  The window keeps a 2x margin over that.
constexpr float kGuard = 6e-4f;

// v: the channel before exposure; the exact f64 input of the fallback is (double)v * exposure.
template <int KIND>
__device__ __forceinline__ uint32_t tone_gamma_fast(float v, float exposure32, double exposure, float inv_gamma) {
    const float x = v * exposure32;
    if (x != x) return 0u;
    const float t = tone_fast<KIND>(x);
    float sv;
    if (inv_gamma > 0.0f) sv = __powf(t, inv_gamma);
    else sv = t <= 0.0031308f ? 12.92f * t : fmaf(1.055f, __powf(t, 1.0f / 2.4f), -0.055f);
    const float q = fminf(fmaxf(sv, 0.0f), 0.999f) * 256.0f;
    const float fr = q - floorf(q);
    if (fr > 1.0f - kGuard || (fr < kGuard && q >= 1.0f)) {
        const double q64 = tone_gamma64(KIND, (double)v * exposure, inv_gamma > 0.0f ? 1.0 / (double)inv_gamma : 0.0,
                                        0.0);
        return q64 < 0.0 ? 0u : sat_u8(q64);
    }
    return (uint32_t)q;
}

// Byte tables of the common chain.  Without dither, vignette or the other optional steps, a
// channel's byte is a non-decreasing step function of x = (double)v * exposure: the tone curve,
// the sRGB or 1/gamma power and the quantisation are all monotone.  So it is fixed by the 255
// thresholds T_k = min{x : byte(x) >= k}, found once per (tone curve, gamma) on the host by
// bisection over the f64 bit patterns with the reference's own f64 formulas (the host's libm
// pow, as the f64 restatement uses) -- exact, not a fit.  The kernel finds x's byte from one
// table entry: positive doubles order like their bit patterns, and the bucket of x is its top
// 19 bits (sign, exponent, 7 mantissa bits), chosen so that no bucket holds two thresholds.
// Entry i (a u64): byte at the bucket's lower end in bits 56-63, the low 45 bits of the bucket's
// threshold (or 2^45: none) in bits 0-45; x's byte is that base, plus one if x's low 45 bits reach
// the threshold's.  Entry 0 stands for every bucket below the first, entry nb + 1 for every
// bucket above the last.  Non-finite, huge or non-positive x take the f64 path as before.
constexpr int kTabShift = 45;                                  // 52 - 7 mantissa bits
constexpr unsigned long long kTabLowMask = (1ull << kTabShift) - 1ull;
constexpr int kTabMaxEntries = 4096;                           // nb + 2 per table
constexpr int kTabSlots = 16;                                  // (tone curve, gamma) pairs per device

struct ByteTable {
    const unsigned long long* tab;   // device address of the slot, or null: no table
    long long k0;                    // bucket key of entry 1
    int nb;                          // buckets with an entry of their own
};

static __device__ __align__(256) unsigned long long g_byte_tables[kTabSlots][kTabMaxEntries];

template <int KIND>
__device__ __forceinline__ uint32_t tone_table(float v, double exposure, const ByteTable& T, float inv_gamma) {
    const double x = (double)v * exposure;
    if (!(x > 0.0)) return 0u;                                 // NaN, zero and negatives: byte 0
    if (!(x < 1e30)) {
        const double q64 = tone_gamma64(KIND, x, inv_gamma > 0.0f ? 1.0 / (double)inv_gamma : 0.0, 0.0);
        return q64 < 0.0 ? 0u : sat_u8(q64);
    }
    const long long b = __double_as_longlong(x);
    const long long i = min(max((b >> kTabShift) - T.k0 + 1, 0ll), (long long)T.nb + 1);
    const unsigned long long e = __ldg(T.tab + i);
    return (uint32_t)(e >> 56) + (((unsigned long long)b & kTabLowMask) >= (e & (2ull * kTabLowMask + 1ull)) ? 1u : 0u);
}

// tone_table for an exposure 2^k (k2 = k): x = (double)v * 2^k is exact, so x's bits follow from v's
// and the bucket key and the compare against the entry's threshold bits are done in 32-bit
// integer arithmetic, with no f64 conversion or multiply.  For v normal and positive, x's
// exponent field is v's + k + 896 and its mantissa v's shifted left 29 bits: key = x_bits >> 45 =
// (v_bits >> 16) + ((k + 896) << 7), and x's bits below the key are (v_bits & 0xFFFF) << 29.
// Zero, negative, non-finite, denormal and very large v (x at or above 2^99: the f64 formulas
// take x >= 1e30) go through tone_table itself, so the bytes are tone_table's in every case.
template <int KIND>
__device__ __forceinline__ uint32_t tone_table_pow2(float v, int k2, double exposure, const ByteTable& T,
                                                    float inv_gamma) {
    const uint32_t u = __float_as_uint(v);
    const int ef = (int)(u >> 23) + k2 + 896;                  // x's biased f64 exponent (v > 0)
    if (u - 0x00800000u >= 0x7F000000u || ef < 1 || ef >= 1023 + 99)
        return tone_table<KIND>(v, exposure, T, inv_gamma);    // v <= 0, denormal, inf/NaN; x tiny or huge
    const int key = (int)(u >> 16) + ((k2 + 896) << 7);
    const int i = min(max(key - (int)T.k0 + 1, 0), T.nb + 1);
    const unsigned long long e = __ldg(T.tab + i);
    const uint32_t th = (uint32_t)(e >> 32) & 0x3FFFu, tl = (uint32_t)e;   // threshold bits 0-45
    const uint32_t m = u & 0xFFFFu, mh = m >> 3, ml = m << 29;              // x's bits 0-44
    return (uint32_t)(e >> 56) + ((mh > th || (mh == th && ml >= tl)) ? 1u : 0u);
}

template <int KIND>
__device__ __forceinline__ uint32_t pixel_table_pow2(float r, float g, float b, int k2, double exposure,
                                                     const ByteTable& T, float inv_gamma) {
    const uint32_t R = tone_table_pow2<KIND>(r, k2, exposure, T, inv_gamma);
    const uint32_t G = tone_table_pow2<KIND>(g, k2, exposure, T, inv_gamma);
    const uint32_t B = tone_table_pow2<KIND>(b, k2, exposure, T, inv_gamma);
    return R | (G << 8) | (B << 16) | (255u << 24);
}

template <int KIND>
__device__ __forceinline__ uint32_t pixel_table(float r, float g, float b, double exposure, const ByteTable& T,
                                                float inv_gamma) {
    const uint32_t R = tone_table<KIND>(r, exposure, T, inv_gamma);
    const uint32_t G = tone_table<KIND>(g, exposure, T, inv_gamma);
    const uint32_t B = tone_table<KIND>(b, exposure, T, inv_gamma);
    return R | (G << 8) | (B << 16) | (255u << 24);
}

// The common chain -- exposure, tone curve KIND, sRGB or gamma -- inline, in f32 with the exact
// f64 fallback near byte boundaries (the channel values stay f32 until the fallback needs them);
// used when no byte table is available.
template <int KIND>
__device__ __forceinline__ uint32_t pixel_fast(float r, float g, float b, float e32, double exposure, float inv_gamma) {
    const uint32_t R = tone_gamma_fast<KIND>(r, e32, exposure, inv_gamma);
    const uint32_t G = tone_gamma_fast<KIND>(g, e32, exposure, inv_gamma);
    const uint32_t B = tone_gamma_fast<KIND>(b, e32, exposure, inv_gamma);
    return R | (G << 8) | (B << 16) | (255u << 24);
}

// Any chain: the fast path, or pixel_full (kept out of line so the hot loop stays small in the
// instruction cache) when an optional step is on.
template <int KIND>
__device__ __forceinline__ uint32_t pixel_rgba(const Chain& C, float r, float g, float b, uint32_t p, uint32_t w,
                                               uint32_t h, float e32, double exposure) {
    if (C.extra) return pixel_full(C, r, g, b, p, w, h, exposure);
    return pixel_fast<KIND>(r, g, b, e32, exposure, C.inv_gamma);
}

__device__ __forceinline__ double log_lum(float r, float g, float b) {
    const double lum = 0.2126 * (double)r + 0.7152 * (double)g + 0.0722 * (double)b;
    return (double)logf((float)(1e-4 + fmax(lum, 0.0)));   // f32 log, f64 sum
}

// VEC: 4 pixels per step from three 16-byte loads (hdr 16-byte aligned).
template <bool VEC>
__global__ void __launch_bounds__(kLogThreads) k_loglum(const float* __restrict__ hdr, uint32_t n, double* __restrict__ partials) {
    __shared__ double sh[kLogThreads];
    double acc = 0.0;
    const uint32_t t0 = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
    uint32_t from = 0;
    if constexpr (VEC) {
        const float4* in = reinterpret_cast<const float4*>(hdr);
        const uint32_t n4 = n / 4;
        for (uint32_t q = t0; q < n4; q += stride) {
            const float4 a = in[3 * q], b = in[3 * q + 1], c = in[3 * q + 2];
            acc += (log_lum(a.x, a.y, a.z) + log_lum(a.w, b.x, b.y)) + (log_lum(b.z, b.w, c.x) + log_lum(c.y, c.z, c.w));
        }
        from = 4 * n4;
    }
    for (uint32_t p = from + t0; p < n; p += stride)
        acc += log_lum(hdr[3 * (size_t)p], hdr[3 * (size_t)p + 1], hdr[3 * (size_t)p + 2]);
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int s = kLogThreads / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) partials[blockIdx.x] = sh[0];
}

template <bool VEC, int KIND>
__global__ void __launch_bounds__(kThreads, 6) k_tonemap(const float* __restrict__ hdr, uint32_t w, uint32_t h, const __grid_constant__ Chain C,
                                                      double exposure, const double* __restrict__ partials,
                                                      uint8_t* __restrict__ rgba, const ByteTable T) {
    __shared__ double s_exposure;
    if (partials) {   // auto-exposure: key value 0.18 over the log-average luminance
        if (threadIdx.x == 0) {
            double sum = 0.0;
            for (int k = 0; k < kLogBlocks; ++k) sum += partials[k];
            const size_t n = (size_t)w * h;
            const double log_avg = n ? exp(sum / (double)n) : 0.0;
            s_exposure = (log_avg > 1e-6 ? 0.18 / log_avg : 1.0) * exposure;
        }
        __syncthreads();
        exposure = s_exposure;
    }
    const uint32_t n = w * h;
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t t0 = blockIdx.x * blockDim.x + threadIdx.x;
    const float e32 = (float)exposure;
    uint32_t scalar_from = 0;
    if constexpr (VEC) {
        const uint32_t n4 = n / 4;
        const float4* in = reinterpret_cast<const float4*>(hdr);
        uint4* out = reinterpret_cast<uint4*>(rgba);
        const long long eb = __double_as_longlong(exposure);
        const int k2 = (int)((eb >> 52) & 0x7FF) - 1023;
        const bool pow2 = exposure > 0.0 && (eb & 0xFFFFFFFFFFFFFll) == 0 && k2 > -1000 && k2 < 1000;
        if (!C.extra && T.tab && pow2) {   // byte table, exposure 2^k2: integer keys (uniform branch)
            const float ig = C.inv_gamma;
            for (uint32_t q = t0; q < n4; q += stride) {
                const float4 a = __ldcs(in + 3 * q), b = __ldcs(in + 3 * q + 1), c = __ldcs(in + 3 * q + 2);
                __stcs(out + q, make_uint4(pixel_table_pow2<KIND>(a.x, a.y, a.z, k2, exposure, T, ig),
                                           pixel_table_pow2<KIND>(a.w, b.x, b.y, k2, exposure, T, ig),
                                           pixel_table_pow2<KIND>(b.z, b.w, c.x, k2, exposure, T, ig),
                                           pixel_table_pow2<KIND>(c.y, c.z, c.w, k2, exposure, T, ig)));
            }
        } else if (!C.extra && T.tab) {   // the common chain from its byte table (uniform branch, hoisted)
            const float ig = C.inv_gamma;
            for (uint32_t q = t0; q < n4; q += stride) {
                const float4 a = __ldcs(in + 3 * q), b = __ldcs(in + 3 * q + 1), c = __ldcs(in + 3 * q + 2);
                __stcs(out + q, make_uint4(pixel_table<KIND>(a.x, a.y, a.z, exposure, T, ig),
                                           pixel_table<KIND>(a.w, b.x, b.y, exposure, T, ig),
                                           pixel_table<KIND>(b.z, b.w, c.x, exposure, T, ig),
                                           pixel_table<KIND>(c.y, c.z, c.w, exposure, T, ig)));
            }
        } else if (!C.extra) {     // the common chain in f32 with the exact fallback
            const float ig = C.inv_gamma;
            for (uint32_t q = t0; q < n4; q += stride) {
                const float4 a = __ldcs(in + 3 * q), b = __ldcs(in + 3 * q + 1), c = __ldcs(in + 3 * q + 2);
                __stcs(out + q, make_uint4(pixel_fast<KIND>(a.x, a.y, a.z, e32, exposure, ig),
                                           pixel_fast<KIND>(a.w, b.x, b.y, e32, exposure, ig),
                                           pixel_fast<KIND>(b.z, b.w, c.x, e32, exposure, ig),
                                           pixel_fast<KIND>(c.y, c.z, c.w, e32, exposure, ig)));
            }
        } else {
            for (uint32_t q = t0; q < n4; q += stride) {
                const float4 a = in[3 * q], b = in[3 * q + 1], c = in[3 * q + 2];
                const uint32_t p = 4 * q;
                out[q] = make_uint4(pixel_rgba<KIND>(C, a.x, a.y, a.z, p, w, h, e32, exposure),
                                    pixel_rgba<KIND>(C, a.w, b.x, b.y, p + 1, w, h, e32, exposure),
                                    pixel_rgba<KIND>(C, b.z, b.w, c.x, p + 2, w, h, e32, exposure),
                                    pixel_rgba<KIND>(C, c.y, c.z, c.w, p + 3, w, h, e32, exposure));
            }
        }
        scalar_from = 4 * n4;
    }
    for (uint32_t p = scalar_from + t0; p < n; p += stride) {   // any output alignment: byte stores
        const uint32_t v = pixel_rgba<KIND>(C, hdr[3 * (size_t)p], hdr[3 * (size_t)p + 1], hdr[3 * (size_t)p + 2], p,
                                            w, h, e32, exposure);
        rgba[4 * (size_t)p] = (uint8_t)v;
        rgba[4 * (size_t)p + 1] = (uint8_t)(v >> 8);
        rgba[4 * (size_t)p + 2] = (uint8_t)(v >> 16);
        rgba[4 * (size_t)p + 3] = (uint8_t)(v >> 24);
    }
}

Chain make_chain(const lum_tonemap_params& p) {
    Chain C;
    C.p = p;
    const double ang = p.hue_shift * (3.14159265358979323846 / 180.0);
    C.cos_h = std::cos(ang);
    C.sin_h = std::sin(ang);
    double bo = p.brightness * 255.0;
    bo = bo != bo ? 0.0 : (bo > 32767.0 ? 32767.0 : (bo < -32768.0 ? -32768.0 : bo));
    C.bright_off = (int16_t)bo;
    auto ne1 = [](const double* v) { return v[0] != 1.0 || v[1] != 1.0 || v[2] != 1.0; };
    C.wb = std::fabs(p.white_balance) > 1e-6;
    C.hue = std::fabs(p.hue_shift) > 1e-6;
    C.sat = std::fabs(p.saturation - 1.0) > 1e-6;
    C.grade = ne1(p.grade_shadows) || ne1(p.grade_highlights);
    C.bright = std::fabs(p.brightness) > 1e-6;
    C.contrast = std::fabs(p.contrast - 1.0) > 1e-6;
    C.sepia = p.sepia > 0.0;
    C.tint = p.tint[0] < 1.0 || p.tint[1] < 1.0 || p.tint[2] < 1.0;
    C.balance = std::fabs(p.color_balance[0] - 1.0) > 1e-6 || std::fabs(p.color_balance[1] - 1.0) > 1e-6 ||
                std::fabs(p.color_balance[2] - 1.0) > 1e-6;
    C.inv_gamma = p.gamma > 0.0 ? (float)(1.0 / p.gamma) : 0.0f;
    C.extra = p.vignette > 0.0 || p.dither || p.posterize >= 2 || C.wb || C.hue || C.sat || C.grade || C.bright ||
              C.contrast || C.sepia || C.tint || C.balance;
    return C;
}

// Host side of the byte tables: the chain's byte for an exact f64 x (gamma <= 0: sRGB).
static uint32_t host_byte(int kind, double x, double gamma) {
    return sat_u8(quantised(srgb64(clamp01(tone_curve(kind, x)), gamma), 0.0));
}

static long long dbits(double x) {
    long long b;
    std::memcpy(&b, &x, sizeof b);
    return b;
}
static double bdouble(long long b) {
    double x;
    std::memcpy(&x, &b, sizeof x);
    return x;
}

// Builds the entries of one table; false when the chain is not the step function the table
// encodes (a bucket with two thresholds, too many buckets, or a byte that does not match).
static bool build_byte_table(int kind, double gamma, std::vector<unsigned long long>& ent, long long& k0, int& nb) {
    const long long top = dbits(1e30);
    std::vector<long long> th;                                  // bit patterns of T_1 .. T_bmax
    const uint32_t bmax = host_byte(kind, 1e30, gamma);
    if (host_byte(kind, bdouble(1), gamma) != 0u) return false;  // smallest positive x must be byte 0
    for (uint32_t k = 1; k <= bmax; ++k) {
        long long lo = th.empty() ? 0 : th.back() - 1, hi = top;   // byte(lo) < k <= byte(hi)
        if (lo < 0) lo = 0;
        while (hi - lo > 1) {
            const long long m = lo + (hi - lo) / 2;
            if (host_byte(kind, bdouble(m), gamma) >= k) hi = m;
            else lo = m;
        }
        th.push_back(hi);
    }
    if (th.empty()) return false;
    k0 = th.front() >> kTabShift;
    const long long k1 = th.back() >> kTabShift;
    nb = (int)(k1 - k0 + 1);
    if (nb + 2 > kTabMaxEntries) return false;
    ent.assign(nb + 2, 0ull);
    ent[0] = 2ull * kTabLowMask + 1ull;                          // below: byte 0, no threshold
    ent[nb + 1] = ((unsigned long long)bmax << 56) | (2ull * kTabLowMask + 1ull);
    size_t t = 0;                                               // thresholds at or below the bucket start
    for (int i = 0; i < nb; ++i) {
        const long long key = k0 + i, lo = key << kTabShift, hi = (key + 1) << kTabShift;
        while (t < th.size() && th[t] <= lo) ++t;
        const uint32_t base = (uint32_t)t;
        if (host_byte(kind, bdouble(lo), gamma) != base) return false;        // not monotone here
        unsigned long long thr = 2ull * kTabLowMask + 1ull;     // none
        if (t < th.size() && th[t] < hi) {
            if (t + 1 < th.size() && th[t + 1] < hi) return false;            // two in one bucket
            thr = (unsigned long long)th[t] & kTabLowMask;
        }
        ent[i + 1] = ((unsigned long long)base << 56) | thr;
    }
    return true;
}

// One table per (device, tone curve, gamma), uploaded once into a slot of g_byte_tables.
struct TableSlot {
    int device, kind;
    long long gamma_bits;
    ByteTable T;
};

static ByteTable byte_table(int kind, double gamma) {
    static std::mutex mu;
    static std::vector<TableSlot> slots;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return ByteTable{nullptr, 0, 0};
    if (!(gamma > 0.0)) gamma = 0.0;
    const long long gb = dbits(gamma);
    std::lock_guard<std::mutex> lk(mu);
    int used = 0;
    for (const TableSlot& sl : slots) {
        if (sl.device != dev) continue;
        if (sl.kind == kind && sl.gamma_bits == gb) return sl.T;
        ++used;
    }
    TableSlot sl{dev, kind, gb, ByteTable{nullptr, 0, 0}};
    std::vector<unsigned long long> ent;
    void* base = nullptr;
    if (used < kTabSlots && build_byte_table(kind, gamma, ent, sl.T.k0, sl.T.nb) &&
        cudaGetSymbolAddress(&base, g_byte_tables) == cudaSuccess &&
        cudaMemcpyToSymbol(g_byte_tables, ent.data(), ent.size() * sizeof(unsigned long long),
                           (size_t)used * kTabMaxEntries * sizeof(unsigned long long)) == cudaSuccess)
        sl.T.tab = static_cast<const unsigned long long*>(base) + (size_t)used * kTabMaxEntries;
    cudaGetLastError();
    if (!sl.T.tab) sl.kind = -1 - kind;                         // remembered as "no table"
    slots.push_back(sl);
    return sl.T;
}

}  // namespace tone

cudaError_t launch_tonemap(const float* hdr, uint32_t w, uint32_t h, const lum_tonemap_params& tm, double exposure,
                           double* scratch, uint8_t* rgba, cudaStream_t stream) {
    const size_t n = (size_t)w * h;
    if (n == 0) return cudaSuccess;
    if (n >= ((size_t)1 << 32)) return cudaErrorInvalidValue;   // 32-bit pixel indices
    const double* partials = nullptr;
    const bool vec = (((uintptr_t)hdr | (uintptr_t)rgba) & 15) == 0;
    if (tm.auto_exposure) {
        if (((uintptr_t)hdr & 15) == 0)
            tone::k_loglum<true><<<tone::kLogBlocks, tone::kLogThreads, 0, stream>>>(hdr, (uint32_t)n, scratch);
        else
            tone::k_loglum<false><<<tone::kLogBlocks, tone::kLogThreads, 0, stream>>>(hdr, (uint32_t)n, scratch);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        partials = scratch;
    }
    const tone::Chain C = tone::make_chain(tm);
    const tone::ByteTable T = C.extra ? tone::ByteTable{nullptr, 0, 0} : tone::byte_table(tm.tone_map, tm.gamma);
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const size_t work = vec ? (n + 3) / 4 : n;
    // at most two resident waves (6 blocks/SM), threads looping over the rest: on B200 the 1080p
    // frame 20.5 -> 18.4 us against one block per 256 quads (2.3 waves), the 8K frame unchanged
    const int grid = (int)std::min<size_t>((work + tone::kThreads - 1) / tone::kThreads, (size_t)nsm * 12);
    auto go = [&](auto kind) {
        constexpr int K = decltype(kind)::value;
        if (vec)
            tone::k_tonemap<true, K><<<grid, tone::kThreads, 0, stream>>>(hdr, (uint32_t)w, (uint32_t)h, C, exposure,
                                                                          partials, rgba, T);
        else
            tone::k_tonemap<false, K><<<grid, tone::kThreads, 0, stream>>>(hdr, (uint32_t)w, (uint32_t)h, C, exposure,
                                                                           partials, rgba, T);
    };
    switch (tm.tone_map) {
        case LUM_TONEMAP_REINHARD: go(std::integral_constant<int, LUM_TONEMAP_REINHARD>()); break;
        case LUM_TONEMAP_FILMIC: go(std::integral_constant<int, LUM_TONEMAP_FILMIC>()); break;
        case LUM_TONEMAP_NONE: go(std::integral_constant<int, LUM_TONEMAP_NONE>()); break;
        default: go(std::integral_constant<int, LUM_TONEMAP_ACES>()); break;
    }
    return cudaGetLastError();
}

}  // namespace lum

extern "C" {

void lum_tonemap_default(lum_tonemap_params* out) {
    if (!out) return;
    std::memset(out, 0, sizeof *out);
    out->tone_map = LUM_TONEMAP_ACES;                                   // src/render.rs:176-182
    out->exposure = 1.0;
    out->gamma = 0.0;
    out->saturation = 1.0;
    out->contrast = 1.0;
    for (int c = 0; c < 3; ++c) {
        out->grade_shadows[c] = out->grade_highlights[c] = 1.0;
        out->tint[c] = out->color_balance[c] = 1.0;
    }
}

lum_status lum_tonemap_device(const float* d_hdr_rgb, uint32_t width, uint32_t height, const lum_tonemap_params* tm,
                              void* d_scratch, uint8_t* d_rgba, void* stream) {
    if (!tm) return lum::set_error(LUM_ERR_INVALID_ARGUMENT, "null tone-map parameters");
    if ((size_t)width * height == 0) return LUM_OK;
    if ((size_t)width * height >= ((size_t)1 << 32))
        return lum::set_error(LUM_ERR_TOO_LARGE, "tone map supports fewer than 2^32 pixels");
    if (!d_hdr_rgb || !d_rgba) return lum::set_error(LUM_ERR_INVALID_ARGUMENT, "null image buffer");
    if ((uintptr_t)d_hdr_rgb & 3u) return lum::set_error(LUM_ERR_INVALID_ARGUMENT, "d_hdr_rgb is not 4-byte aligned");
    if (d_scratch && ((uintptr_t)d_scratch & 7u))
        return lum::set_error(LUM_ERR_INVALID_ARGUMENT, "d_scratch is not 8-byte aligned");
    if (tm->auto_exposure && !d_scratch)
        return lum::set_error(LUM_ERR_INVALID_ARGUMENT, "auto_exposure needs LUM_TONEMAP_SCRATCH_BYTES of device scratch");
    if (tm->tone_map < LUM_TONEMAP_ACES || tm->tone_map > LUM_TONEMAP_NONE)
        return lum::set_error(LUM_ERR_INVALID_ARGUMENT, "unknown tone_map");
    cudaError_t e = lum::launch_tonemap(d_hdr_rgb, width, height, *tm, tm->exposure, (double*)d_scratch, d_rgba,
                                        (cudaStream_t)stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return lum::set_error(LUM_ERR_CUDA, cudaGetErrorString(e));
    }
    return LUM_OK;
}

}  // extern "C"
