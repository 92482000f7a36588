// render_task.cuh -- one warp's render task: an 8x4 tile of one frame and a range of its strata.
//
// The task's (pixel, stratum) pairs form one pool that the warp's lanes draw from through a
// shared-memory counter: a lane whose path ends takes the next pair, so no lane idles while the
// task has paths left (a lane that owned one pixel would wait, at the end of every task, for the
// lane with the longest paths).  Pairs are numbered stratum-major, so the warp starts on one
// stratum of every pixel of the tile, as coherent as one path per pixel.  Every loop iteration
// runs exactly one traversal per active lane -- the closest hit of a path segment or the any hit
// of an NEE shadow ray, through the same code -- then that lane's shading step, so traversal
// stays convergent across lanes at different bounces.
//
// Each finished path adds its clamped, filter-weighted radiance and its filter weight to the
// tile's per-pixel sums in 64-bit fixed point (2^-32 units, shared-memory atomics): integer sums
// do not depend on the order in which paths finish, so the image is deterministic and equal
// whichever kernel (megakernel, batched megakernel, wavefront) traced the paths.
#pragma once

#include "tracer.cuh"

namespace lum {

constexpr double kFixScale = 4294967296.0;   // 2^32

// v * 2^32 is exact in f32 (a power-of-two scale; the clamped samples are far below overflow),
// so rounding it to an integer in f32 gives the same value as llrint((double)v * 2^32), without
// the f64 conversions.
__device__ __forceinline__ unsigned long long to_fixed(float v) {
    return (unsigned long long)__float2ll_rn(v * 4294967296.0f);
}

// *p += to_fixed(x) on a shared-memory sum as two 32-bit atomic adds: the low word's add returns
// its old value, a wrap of the low word carries one into the high word.  Each wrap is counted
// exactly once, so the 64-bit sum is exact (mod 2^64) and independent of the order of the adds.
// On B200 this measured 2% faster on the sphere-field frame than one 64-bit shared atomic add.
__device__ __forceinline__ void add_fixed(unsigned long long* p, float x) {
    const unsigned long long v = to_fixed(x);
    uint32_t* w = reinterpret_cast<uint32_t*>(p);
    const uint32_t lo = (uint32_t)v, hi = (uint32_t)(v >> 32);
    const uint32_t old = atomicAdd(w, lo);
    const uint32_t h = hi + ((uint32_t)(old + lo) < old ? 1u : 0u);
    if (h) atomicAdd(w + 1, h);
}

// Pixel value from its fixed-point sums (render.rs:1705 and the exposure of 2610-2624).
__device__ __forceinline__ void fixed_pixel(const unsigned long long* a, float exposure, float* o) {
    const double w = (double)(long long)a[3] / kFixScale;
    const double inv = w > 0.0 ? 1.0 / w : 1.0;
    for (int c = 0; c < 3; ++c) o[c] = (float)((double)(long long)a[c] / kFixScale * inv) * exposure;
}

// One lane's traversal and shading step (state ST_CLOSEST or ST_SHADOW): the closest hit of its
// path segment or the any hit of its NEE shadow ray, walked (or resumed) through the same code,
// then the shading step once the walk is complete.  A walk suspended by trace_resume leaves the
// state unchanged and resumes in a later iteration.
template <bool COUNT, bool EXT, bool NEE, bool SPH, int SUSPEND, int CLS>
__device__ __forceinline__ void path_step(const SceneDev& S, const RenderDev& R, uint32_t pixel, int& state, Path& P,
                                          Pending& pend, Hit& h, Trav& tv, bool& found, bool& walking, V* stash,
                                          int* stack, uint32_t& err, uint32_t& nseg, uint32_t& nsh,
                                          TestTally* tally) {
    const bool shadow = state == ST_SHADOW;
    Ray r;
    r.o = P.ray.o;
    r.d = shadow ? pend.dir : P.ray.d;
    r.time = shadow ? 0.0f : P.ray.time;                      // Ray::new (render.rs:1457)
    if (!walking) {
        h.t = shadow ? (EXT ? fabsf(pend.tmax) : pend.tmax) : CUDART_INF_F;
        h.prim = -1;
        h.b1 = h.b2 = 0.0f;
        tv.node = S.n_nodes > 0 ? 0 : kSentinel;
        tv.sp = 0;
        found = false;
    }
    walking = !trace_resume<COUNT, SPH, SUSPEND, CLS>(S, r, 0.001f, shadow, h, found, tv, stack, err, tally);
    if (walking) return;
    if (shadow) {
        ++nsh;
        if (!found) P.L = P.L + pend.contrib;
        shadow_done<EXT>(P, pend, stash);
        state = P.bounce >= R.max_depth ? ST_DONE : ST_CLOSEST;
    } else {
        ++nseg;
        state = shade<-1, EXT, NEE, SPH, CLS>(S, R, pixel, P, found, h, pend, stash);
    }
}

// Runs the task; on return acc[k][0..3] (k < tw * th, pixel (k % tw, k / tw) of the tile) hold
// the sums.  acc (32 x 4) and *next are the warp's shared memory; the call zeroes them.
// EXT: the scene may use the other materials or backgrounds; NEE: it has lights; SPH: its
// primitives are spheres and its materials the basic four (shade's and trace's template flags).
template <bool COUNT, bool EXT = true, bool NEE = true, bool SPH = false, int SUSPEND = LUM_SUSPEND_LANES,
          int CLS = CLS_ALL>
__device__ __forceinline__ void tile_task(const SceneDev& S, const RenderDev& R, uint32_t x0, uint32_t y0,
                                          uint32_t tw, uint32_t th, uint32_t s_lo, uint32_t s_hi,
                                          unsigned long long (*acc)[4], uint32_t* next, V* exit_stash, int* stack,
                                          uint32_t& err, uint32_t& nseg, uint32_t& nsh, TestTally* tally) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    acc[lane][0] = acc[lane][1] = acc[lane][2] = acc[lane][3] = 0ull;
    if (lane == 0) *next = 0u;
    __syncwarp(full);
    const uint32_t nv = tw * th;
    const uint32_t n_items = s_hi > s_lo ? nv * (s_hi - s_lo) : 0u;
    int state = ST_IDLE;
    uint32_t cur = 0, pixel = 0;
    Path P;
    Pending pend;
    Hit h;                    // closest hit so far of the lane's walk
    Trav tv;                  // place of a suspended walk
    bool found = false, walking = false;
    for (;;) {
        if (state == ST_IDLE) {
            const uint32_t idx = atomicAdd(next, 1u);
            if (idx < n_items) {
                cur = idx % nv;
                const uint32_t st = s_lo + idx / nv;
                const uint32_t gi = x0 + cur % tw + R.crop_x, gj = y0 + cur / tw + R.crop_y;
                pixel = gj * R.full_w + gi;
                start_path<philox_unroll<CLS>()>(S, R, gi, gj, pixel, st, P);
                state = R.max_depth > 0 ? ST_CLOSEST : ST_DONE;
            }
        }
        if (!__any_sync(full, state != ST_IDLE)) break;
        if (state == ST_CLOSEST || state == ST_SHADOW)
            path_step<COUNT, EXT, NEE, SPH, SUSPEND, CLS>(S, R, pixel, state, P, pend, h, tv, found, walking,
                                                          exit_stash + lane, stack, err, nseg, nsh, tally);
        if (state == ST_DONE) {
            const float4 v = path_sample(R, P.L, P.jx, P.jy);
            add_fixed(&acc[cur][0], v.x);
            add_fixed(&acc[cur][1], v.y);
            add_fixed(&acc[cur][2], v.z);
            add_fixed(&acc[cur][3], v.w);
            state = ST_IDLE;
        }
    }
    __syncwarp(full);
}

}  // namespace lum
