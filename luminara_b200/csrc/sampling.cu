// sampling.cu -- the in-loop branches of the sample loop: adaptive sampling and the time limit
// (render.rs:1592-1678), as one persistent kernel over 8x4 tiles.
//
// Time limit: a tile whose task starts after the limit renders one sample per pixel at the
// pixel centre, luminance-clamped, unfiltered (the reference decides per row when the row
// starts, render.rs:1601-1623; here per tile when its task starts).  The clock starts at a
// %globaltimer stamp taken on the stream just before the render kernel.
//
// Without adaptive sampling, a tile that starts in time traces all its (pixel, stratum) pairs
// into tile_task's fixed-point sums, so it equals lum_render's tile bit for bit.
//
// Adaptive sampling runs a tile in rounds of kRoundStrata strata over its still-active pixels.
// In a round the warp's lanes draw (pixel, stratum) pairs from one pool, as tile_task does,
// and store each clamped sample in shared memory; then lane p walks its pixel's samples in
// stratum order through Welford's update and the stopping test -- the reference's sequential
// loop, so a pixel stops at the same sample count as there, given the same sample values.
// Samples traced past a pixel's stopping point in its last round are dropped (fewer than
// kRoundStrata per pixel).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <mutex>
#include <utility>
#include <vector>

#include "kernels.h"
#include "render_task.cuh"
#include "tracer.cuh"

namespace lum {
namespace {

constexpr int kSampThreads = 128;
constexpr int kSampWarps = kSampThreads / 32;
constexpr uint32_t kRoundStrata = 16;
constexpr unsigned kAll = 0xffffffffu;

// Luminance clamp of one sample (render.rs:1692-1697), rounded like path_sample.
__device__ __forceinline__ V clamp_sample(V L) {
    const float lum = __fadd_rn(__fadd_rn(__fmul_rn(0.2126f, L.x), __fmul_rn(0.7152f, L.y)), __fmul_rn(0.0722f, L.z));
    if (!(lum > 100.0f)) return L;
    const float k = __fdiv_rn(100.0f, lum);
    return V{__fmul_rn(L.x, k), __fmul_rn(L.y, k), __fmul_rn(L.z, k)};
}

// One warp's pool of paths: item idx < n_slots * n_st is slot idx % n_slots, stratum
// st_lo + idx / n_slots; slot s is the tile pixel slot_px[s].  centre: the time limit's one
// centre sample (n_st = 1, stratum 0).  With acc, each finished path adds its clamped,
// filter-weighted value to acc[tile pixel] in fixed point (tile_task's sums; the call zeroes
// acc); without, its clamped sample goes to smp[stratum - st_lo][tile pixel].  One copy of
// the traversal and shading code serves every kind of tile.
template <bool EXT, bool NEE, bool SPH>
__device__ __forceinline__ void sample_pool(const SceneDev& S, const RenderDev& R, uint32_t x0, uint32_t y0, uint32_t tw,
                            const uint32_t* slot_px, uint32_t n_slots, uint32_t st_lo, uint32_t n_st, bool centre,
                            unsigned long long (*acc)[4], float (*smp)[32][3], uint32_t* next, V* exit_stash,
                            int* stack, uint32_t& err, uint32_t& nseg, uint32_t& nsh) {
    const int lane = threadIdx.x & 31;
    if (acc) acc[lane][0] = acc[lane][1] = acc[lane][2] = acc[lane][3] = 0ull;
    if (lane == 0) *next = 0u;
    __syncwarp(kAll);
    const uint32_t n_items = n_slots * n_st;
    int state = ST_IDLE;
    uint32_t px = 0, k = 0, pixel = 0;
    Path P;
    Pending pend;
    Hit h;                    // closest hit so far of the lane's walk
    Trav tv;                  // place of a suspended walk
    bool found = false, walking = false;
    for (;;) {
        if (state == ST_IDLE) {
            const uint32_t idx = atomicAdd(next, 1u);
            if (idx < n_items) {
                px = slot_px[idx % n_slots];
                k = idx / n_slots;
                const uint32_t gi = x0 + px % tw + R.crop_x, gj = y0 + px / tw + R.crop_y;
                pixel = gj * R.full_w + gi;
                if (centre)
                    start_path_centre(S, R, gi, gj, pixel, P);
                else
                    start_path(S, R, gi, gj, pixel, st_lo + k, P);
                state = R.max_depth > 0 ? ST_CLOSEST : ST_DONE;
            }
        }
        if (!__any_sync(kAll, state != ST_IDLE)) break;
        if (state == ST_CLOSEST || state == ST_SHADOW) {
            const bool shadow = state == ST_SHADOW;
            Ray r;
            r.o = P.ray.o;
            r.d = shadow ? pend.dir : P.ray.d;
            r.time = shadow ? 0.0f : P.ray.time;                  // Ray::new (render.rs:1457)
            if (!walking) {
                h.t = shadow ? (EXT ? fabsf(pend.tmax) : pend.tmax) : CUDART_INF_F;
                h.prim = -1;
                h.b1 = h.b2 = 0.0f;
                tv.node = S.n_nodes > 0 ? 0 : kSentinel;
                tv.sp = 0;
                found = false;
            }
            walking = !trace_resume<false, SPH, LUM_SUSPEND_LANES>(S, r, 0.001f, shadow, h, found, tv, stack, err);
            if (walking) {
                // suspended: resumes in a later iteration
            } else if (shadow) {
                ++nsh;
                if (!found) P.L = P.L + pend.contrib;
                shadow_done<EXT>(P, pend, exit_stash + lane);
                state = P.bounce >= R.max_depth ? ST_DONE : ST_CLOSEST;
            } else {
                ++nseg;
                state = shade<-1, EXT, NEE, SPH>(S, R, pixel, P, found, h, pend, exit_stash + lane);
            }
        }
        if (state == ST_DONE) {
            if (acc) {
                const float4 v = path_sample(R, P.L, P.jx, P.jy);
                add_fixed(&acc[px][0], v.x);
                add_fixed(&acc[px][1], v.y);
                add_fixed(&acc[px][2], v.z);
                add_fixed(&acc[px][3], v.w);
            } else {
                const V c = clamp_sample(P.L);
                smp[k][px][0] = c.x;
                smp[k][px][1] = c.y;
                smp[k][px][2] = c.z;
            }
            state = ST_IDLE;
        }
    }
    __syncwarp(kAll);
}

__global__ void k_stamp(WorkCounters* wc) { wc->t0_ns = globaltimer(); }

template <bool ADAPTIVE, bool EXT, bool NEE, bool SPH>
__global__ void __launch_bounds__(kSampThreads, ADAPTIVE ? 4 : 5) k_render_sampled(SceneDev S, RenderDev R, SamplingDev A,
                                                                    float* __restrict__ out, WorkCounters* wc) {
    extern __shared__ int s_stack[];
    __shared__ unsigned long long s_acc[kSampWarps][32][4];
    __shared__ float s_smp[kSampWarps][ADAPTIVE ? kRoundStrata : 1][32][3];
    __shared__ uint32_t s_slot[kSampWarps][32];
    __shared__ uint32_t s_next[kSampWarps];
    __shared__ V s_exit[kSampWarps][32];            // deferred Subsurface origins
    int* stack = s_stack + threadIdx.x;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t err = 0, nseg = 0, nsh = 0;
    unsigned long long kept = 0;
    const uint32_t total = R.sqrt_spp * R.sqrt_spp;
    for (;;) {
        uint32_t task = 0, expired = 0;
        if (lane == 0) {
            task = atomicAdd(&wc->next_task, 1u);
            if (A.limit_ns) expired = globaltimer() - wc->t0_ns > A.limit_ns ? 1u : 0u;
        }
        task = __shfl_sync(kAll, task, 0);
        expired = __shfl_sync(kAll, expired, 0);
        if (task >= R.n_tasks) break;
        const uint32_t x0 = (task % R.tiles_x) * 8, y0 = (task / R.tiles_x) * 4;
        const uint32_t tw = min(8u, R.w - x0), th = min(4u, R.h - y0), nv = tw * th;
        float* o = lane < (int)nv ? out + 3 * ((size_t)(y0 + lane / tw) * R.w + x0 + lane % tw) : nullptr;
        // One pool call site per kernel (a single inlined copy of traversal and shading): an
        // expired tile is one round of centre samples, a tile without adaptive sampling one
        // round of all its strata into the fixed-point sums, an adaptive tile rounds of
        // kRoundStrata strata over its active pixels.
        double mean_lum = 0.0, m2_lum = 0.0, mean[3] = {0.0, 0.0, 0.0};   // Welford (render.rs:1628-1667)
        uint32_t n = 0;
        bool active = o != nullptr;
        const bool fixed_sums = !ADAPTIVE && !expired;
        for (uint32_t lo = 0;; lo += kRoundStrata) {
            const unsigned act = __ballot_sync(kAll, active);
            if (!act) break;
            if (active) s_slot[wid][__popc(act & ((1u << lane) - 1u))] = lane;
            const uint32_t st_lo = expired ? 0u : ADAPTIVE ? lo : R.s_begin;
            const uint32_t n_st = expired ? 1u : ADAPTIVE ? min(kRoundStrata, total - lo) : R.s_end - R.s_begin;
            sample_pool<EXT, NEE, SPH>(S, R, x0, y0, tw, s_slot[wid], __popc(act), st_lo, n_st, expired != 0,
                        fixed_sums ? s_acc[wid] : nullptr, s_smp[wid], &s_next[wid], s_exit[wid], stack, err, nseg,
                        nsh);
            if (active) {
                if (expired) {
                    for (int c = 0; c < 3; ++c) o[c] = s_smp[wid][0][lane][c] * R.exposure;
                    kept += 1;
                    active = false;
                } else if (!ADAPTIVE) {
                    fixed_pixel(s_acc[wid][lane], R.exposure, o);
                    kept += n_st;
                    active = false;
                } else {
                    for (uint32_t k = 0; k < n_st; ++k) {
                        const float* c = s_smp[wid][k][lane];
                        ++n;
                        const double lum = 0.2126 * (double)c[0] + 0.7152 * (double)c[1] + 0.0722 * (double)c[2];
                        const double d1 = lum - mean_lum;
                        mean_lum += d1 / (double)n;
                        m2_lum += d1 * (lum - mean_lum);
                        for (int q = 0; q < 3; ++q) mean[q] += ((double)c[q] - mean[q]) / (double)n;
                        if (n >= A.min_samples && n > 1 && sqrt(m2_lum / (double)(n - 1) / (double)n) < A.threshold) {
                            active = false;
                            break;
                        }
                    }
                    if (n >= total) active = false;
                    if (!active) {
                        for (int q = 0; q < 3; ++q) o[q] = (float)mean[q] * R.exposure;
                        kept += n;
                    }
                }
            }
            __syncwarp(kAll);   // the round's results are read before the next round writes
        }
        __syncwarp(kAll);
    }
    unsigned long long s = nseg, h = nsh;
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
        s += __shfl_xor_sync(kAll, s, d);
        h += __shfl_xor_sync(kAll, h, d);
        kept += __shfl_xor_sync(kAll, kept, d);
        err |= __shfl_xor_sync(kAll, err, d);
    }
    if (lane == 0) {
        atomicAdd(&wc->segments, s);
        atomicAdd(&wc->shadow_rays, h);
        atomicAdd(&wc->samples, kept);
        if (err) atomicOr(&wc->error_flags, err);
    }
}

int num_sms() {
    static const int n = [] {   // initialised once, thread-safe
        int dev = 0, sms = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        return sms > 0 ? sms : 148;
    }();
    return n;
}

template <bool ADAPTIVE, bool EXT, bool NEE, bool SPH>
cudaError_t launch_t(const SceneDev& S, const RenderDev& R, const SamplingDev& A, float* out, WorkCounters* wc,
                     cudaStream_t stream) {
    // the traversal stack sized to the scene's BVH; resident blocks per stack size (cached)
    const size_t stack = (size_t)S.stack_depth * kSampThreads * sizeof(int);
    static std::mutex mu;
    static bool attr = false;
    static std::vector<std::pair<size_t, int>> occ_of;
    int occ = 0;
    {
        std::lock_guard<std::mutex> lk(mu);
        if (!attr) {
            cudaFuncSetAttribute(k_render_sampled<ADAPTIVE, EXT, NEE, SPH>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)((size_t)kStackDepth * kSampThreads * sizeof(int)));
            attr = true;
        }
        for (const auto& e : occ_of)
            if (e.first == stack) occ = e.second;
        if (occ <= 0) {
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_render_sampled<ADAPTIVE, EXT, NEE, SPH>, kSampThreads,
                                                          stack);
            if (occ <= 0) occ = 1;
            occ_of.push_back({stack, occ});
        }
    }
    k_stamp<<<1, 1, 0, stream>>>(wc);
    int grid = num_sms() * occ;
    const int needed = (int)std::min<uint64_t>(((uint64_t)R.n_tasks + kSampWarps - 1) / kSampWarps, 1u << 30);
    grid = std::max(1, std::min(grid, needed));
    k_render_sampled<ADAPTIVE, EXT, NEE, SPH><<<grid, kSampThreads, stack, stream>>>(S, R, A, out, wc);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_render_sampled(const SceneDev& S, const RenderDev& R, const SamplingDev& A, float* out,
                                  WorkCounters* wc, cudaStream_t stream) {
    // scenes without the other materials and backgrounds, without lights, or made of spheres
    // with the basic materials run kernels built without the code they cannot reach
    const bool nee = S.n_lights > 0;
    if (R.ext) {
        if (nee)
            return A.adaptive ? launch_t<true, true, true, false>(S, R, A, out, wc, stream)
                              : launch_t<false, true, true, false>(S, R, A, out, wc, stream);
        return A.adaptive ? launch_t<true, true, false, false>(S, R, A, out, wc, stream)
                          : launch_t<false, true, false, false>(S, R, A, out, wc, stream);
    }
    if (S.spheres_basic) {
        if (nee)
            return A.adaptive ? launch_t<true, false, true, true>(S, R, A, out, wc, stream)
                              : launch_t<false, false, true, true>(S, R, A, out, wc, stream);
        return A.adaptive ? launch_t<true, false, false, true>(S, R, A, out, wc, stream)
                          : launch_t<false, false, false, true>(S, R, A, out, wc, stream);
    }
    if (nee)
        return A.adaptive ? launch_t<true, false, true, false>(S, R, A, out, wc, stream)
                          : launch_t<false, false, true, false>(S, R, A, out, wc, stream);
    return A.adaptive ? launch_t<true, false, false, false>(S, R, A, out, wc, stream)
                      : launch_t<false, false, false, false>(S, R, A, out, wc, stream);
}

}  // namespace lum
