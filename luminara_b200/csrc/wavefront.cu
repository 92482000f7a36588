// wavefront.cu -- batched persistent wavefront tracer (many scenes per launch sequence).
//
// The same estimator as the megakernel (tracer.cuh: start_path, trace, shade), organised as
// a wavefront over a pool of Q path slots in HBM (structure of arrays), for batches of many
// scenes of uneven size, resolution and spp.  One iteration:
//   generate   pop free slots, start camera paths for the next work items (work item =
//              (scene, stratum, pixel) in scene order; keyed RNG, so every path is the one the
//              megakernel traces for the same key)
//   extend     closest hit of every active path; classify the hit into a material queue
//   shade<k>   one kernel per material kind (Lambertian, Metal, Dielectric, Emissive,
//              Microfacet, Isotropic) plus a generic kernel for misses and for batches whose
//              queue is below the sort threshold; emits next rays and NEE shadow rays
//   shadow     any-hit of the shadow rays; adds unoccluded contributions
//   bookkeep   one thread swaps the double-buffered queues and flags completion
// Queue sizes live in device memory, so every iteration is the same kernel sequence: G
// iterations are captured once into a CUDA graph and relaunched until the batch is done.
// Finished paths add their clamped, filter-weighted radiance to per-pixel 64-bit fixed-point
// accumulators (2^-32 units) with integer atomics, which makes the image independent of the
// order in which paths finish.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include <sys/stat.h>

#include "kernels.h"
#include "scene_access.h"
#include "render_task.cuh"
#include "tracer.cuh"

namespace lum {
namespace wf {

constexpr int kQueues = 7;                     // 0 generic; 1..6 = material kinds
constexpr double kFix = 4294967296.0;          // fixed-point scale of the accumulators
constexpr unsigned kFullMask = 0xffffffffu;

struct Ctl {
    unsigned long long work_next, work_total;
    unsigned long long segments, shadow_rays;
    unsigned long long t0_ns;
    uint32_t cur;
    uint32_t ext_n[2];
    uint32_t free_n;
    uint32_t shadow_n;
    uint32_t mat_n[kQueues];
    uint32_t iteration;
    uint32_t error_flags;
    uint32_t done;
};

struct Pool {
    float4* o_t;      // origin, time
    float4* d_jx;     // direction, jitter x
    float4* beta_jy;  // throughput, jitter y
    float4* L;        // radiance
    uint4* ids;       // scene, RNG pixel key, output pixel, stratum | bounce << 24 | skip << 31
    float4* hit;      // t, prim (bits), b1, b2
    float4* sdir;     // shadow direction, t max
    float4* scon;     // shadow contribution, flags (1: finish after the shadow, 2: origin in sorg)
    float4* sorg;     // shadow origin when it is not the path's origin (Subsurface exit points)
    uint32_t* ext[2];
    uint32_t* freeq;
    uint32_t* shadowq;
    uint32_t* matq[kQueues];
    uint32_t Q;
};

struct Tables {
    const SceneDev* scenes;
    const RenderDev* renders;
    const unsigned long long* prefix;      // n + 1 work prefix sums
    const unsigned long long* acc_off;     // per-scene first pixel in acc
    unsigned long long* acc;               // 4 per pixel: r, g, b, weight
    unsigned long long* done_count;
    const unsigned long long* scene_total;
    unsigned long long* finish_ns;
    uint32_t* finish_iter;
    uint32_t n;
    uint32_t sort_threshold;
};

// Appends `value` to queue q; lanes of the warp with the same queue share one atomic.
__device__ __forceinline__ void append(uint32_t* q, uint32_t* counter, uint32_t value, unsigned group) {
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(group) - 1;
    const unsigned below = group & ((1u << lane) - 1u);
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(counter, (uint32_t)__popc(group));
    base = __shfl_sync(group, base, leader);
    q[base + __popc(below)] = value;
}

__device__ __forceinline__ void load_path(const Pool& pl, uint32_t s, Path& P, uint4& id) {
    float4 a = pl.o_t[s], b = pl.d_jx[s], c = pl.beta_jy[s], l = pl.L[s];
    id = pl.ids[s];
    P.ray.o = xyz(a);
    P.ray.time = a.w;
    P.ray.d = xyz(b);
    P.jx = b.w;
    P.beta = xyz(c);
    P.jy = c.w;
    P.L = xyz(l);
    P.stratum = id.w & 0xFFFFFFu;
    P.bounce = (id.w >> 24) & 0x7Fu;
    P.skip_emission = (id.w >> 31) != 0;
}

__device__ __forceinline__ void store_path(const Pool& pl, uint32_t s, const Path& P, uint32_t scene, uint32_t key,
                                           uint32_t out_idx) {
    pl.o_t[s] = make_float4(P.ray.o.x, P.ray.o.y, P.ray.o.z, P.ray.time);
    pl.d_jx[s] = make_float4(P.ray.d.x, P.ray.d.y, P.ray.d.z, P.jx);
    pl.beta_jy[s] = make_float4(P.beta.x, P.beta.y, P.beta.z, P.jy);
    pl.L[s] = make_float4(P.L.x, P.L.y, P.L.z, 0.0f);
    pl.ids[s] = make_uint4(scene, key, out_idx,
                           (P.stratum & 0xFFFFFFu) | ((P.bounce & 0x7Fu) << 24) | (P.skip_emission ? 0x80000000u : 0u));
}

__device__ __forceinline__ long long fix(float v) { return (long long)to_fixed(v); }

// A finished path: luminance clamp and filter weight (render.rs:1692-1701) into the
// fixed-point accumulators of its pixel; per-scene completion bookkeeping.
__device__ __forceinline__ void finish(const Tables& T, const Ctl* ctl, const RenderDev& R, uint32_t scene,
                                       uint32_t out_idx, const Path& P) {
    const float4 v = path_sample(R, P.L, P.jx, P.jy);
    unsigned long long* a = T.acc + 4 * (T.acc_off[scene] + out_idx);
    atomicAdd(a + 0, (unsigned long long)fix(v.x));
    atomicAdd(a + 1, (unsigned long long)fix(v.y));
    atomicAdd(a + 2, (unsigned long long)fix(v.z));
    atomicAdd(a + 3, (unsigned long long)fix(v.w));
    // per-scene completion count: one atomic per scene among the warp's finishing lanes (every
    // finishing path adding 1 to one of a few counters serialised on them)
    const unsigned grp = __match_any_sync(__activemask(), scene);
    const int lane = threadIdx.x & 31, leader = __ffs(grp) - 1;
    unsigned long long base = 0;
    if (lane == leader) base = atomicAdd(T.done_count + scene, (unsigned long long)__popc(grp));
    base = __shfl_sync(grp, base, leader);
    const unsigned long long k = base + (unsigned long long)__popc(grp & ((1u << lane) - 1u)) + 1ull;
    if (k == T.scene_total[scene]) {
        T.finish_ns[scene] = globaltimer();
        T.finish_iter[scene] = ctl->iteration;
    }
}

__global__ void k_init(Pool pl, Ctl* ctl) {
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < pl.Q; i += stride) pl.freeq[i] = pl.Q - 1u - i;
    if (blockIdx.x == 0 && threadIdx.x == 0) ctl->t0_ns = globaltimer();
}

__global__ void k_generate(Pool pl, Tables T, Ctl* ctl) {
    const uint32_t cur = ctl->cur;
    const unsigned long long next = ctl->work_next, total = ctl->work_total;
    const uint32_t free_n = ctl->free_n;
    const uint32_t n_gen = (uint32_t)min((unsigned long long)free_n, total - next);
    const uint32_t base = ctl->ext_n[cur];
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_gen; i += stride) {
        const uint32_t slot = pl.freeq[free_n - 1u - i];
        const unsigned long long w = next + i;
        uint32_t lo = 0, hi = T.n;                                  // scene: prefix[s] <= w < prefix[s+1]
        while (hi - lo > 1) {
            uint32_t mid = (lo + hi) >> 1;
            if (T.prefix[mid] <= w) lo = mid; else hi = mid;
        }
        const uint32_t s = lo;
        const RenderDev R = T.renders[s];
        const unsigned long long local = w - T.prefix[s];
        const uint32_t npix = R.w * R.h;
        const uint32_t stratum = R.s_begin + (uint32_t)(local / npix);
        const uint32_t p = (uint32_t)(local % npix);
        const uint32_t gi = p % R.w + R.crop_x, gj = p / R.w + R.crop_y;
        const uint32_t key = gj * R.full_w + gi;
        Path P;
        const SceneDev S = T.scenes[s];
        start_path(S, R, gi, gj, key, stratum, P);
        store_path(pl, slot, P, s, key, p);
        pl.ext[cur][base + i] = slot;
    }
}

__global__ void k_post_generate(Ctl* ctl) {
    const uint32_t cur = ctl->cur;
    const uint32_t n_gen = (uint32_t)min((unsigned long long)ctl->free_n, ctl->work_total - ctl->work_next);
    ctl->ext_n[cur] += n_gen;
    ctl->free_n -= n_gen;
    ctl->work_next += n_gen;
}

__global__ void k_extend(Pool pl, Tables T, Ctl* ctl) {
    extern __shared__ int s_stack[];
    int* stack = s_stack + threadIdx.x;
    const uint32_t cur = ctl->cur;
    const uint32_t n = ctl->ext_n[cur];
    const bool sorted = n >= T.sort_threshold;
    const uint32_t stride = gridDim.x * blockDim.x;
    uint32_t err = 0, segs = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint32_t slot = pl.ext[cur][i];
        const float4 a = pl.o_t[slot], b = pl.d_jx[slot];
        const uint4 id = pl.ids[slot];
        const SceneDev S = T.scenes[id.x];
        const uint32_t bounce = (id.w >> 24) & 0x7Fu;
        Hit h;
        h.t = CUDART_INF_F;
        h.prim = -1;
        h.b1 = h.b2 = 0.0f;
        bool found = false;
        if (bounce < T.renders[id.x].max_depth) {
            Ray r{xyz(a), xyz(b), a.w};
            found = trace(S, r, 0.001f, false, h, stack, err);
            ++segs;
        }
        pl.hit[slot] = make_float4(h.t, __int_as_float(found ? h.prim : -1), h.b1, h.b2);
        int q = 0;
        if (found && sorted) {
            int mat = h.prim <= -2 ? S.planes[-2 - h.prim].material : (__ldg(S.meta + h.prim) >> 4);
            q = S.mats[mat].kind;
            if (q < 1 || q >= kQueues) q = 0;
        }
        const unsigned group = __match_any_sync(__activemask(), q);
        append(pl.matq[q], &ctl->mat_n[q], slot, group);
    }
    unsigned long long s = segs;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(kFullMask, s, o);
    if ((threadIdx.x & 31) == 0 && s) atomicAdd(&ctl->segments, s);
    if (err) atomicOr(&ctl->error_flags, err);
}

template <int Q>
__global__ void k_shade(Pool pl, Tables T, Ctl* ctl) {
    const uint32_t n = ctl->mat_n[Q];
    const uint32_t nxt = ctl->cur ^ 1u;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint32_t slot = pl.matq[Q][i];
        Path P;
        uint4 id;
        load_path(pl, slot, P, id);
        const float4 hv = pl.hit[slot];
        Hit h;
        h.t = hv.x;
        h.prim = __float_as_int(hv.y);
        h.b1 = hv.z;
        h.b2 = hv.w;
        const RenderDev R = T.renders[id.x];
        int st;
        Pending pend;
        V exit;                                                        // deferred Subsurface origin
        if (P.bounce >= R.max_depth) {
            st = ST_DONE;                                              // depth == 0 -> black
        } else {
            const SceneDev S = T.scenes[id.x];
            st = shade<Q == 0 ? -1 : Q>(S, R, id.y, P, h.prim != -1, h, pend, &exit);
        }
        // a deferred Subsurface origin: the pool keeps the next segment's origin, the shadow
        // query its own (sorg)
        const bool moved = st == ST_SHADOW && pend.tmax < 0.0f;
        const V shadow_org = P.ray.o;
        if (moved) P.ray.o = exit;
        store_path(pl, slot, P, id.x, id.y, id.z);
        if (st == ST_DONE) {
            finish(T, ctl, R, id.x, id.z, P);
            append(pl.freeq, &ctl->free_n, slot, __activemask());
        } else {
            bool cont = st == ST_CLOSEST || P.bounce < R.max_depth;
            if (st == ST_SHADOW) {
                if (moved) pl.sorg[slot] = make_float4(shadow_org.x, shadow_org.y, shadow_org.z, 0.0f);
                pl.sdir[slot] = make_float4(pend.dir.x, pend.dir.y, pend.dir.z, fabsf(pend.tmax));
                pl.scon[slot] = make_float4(pend.contrib.x, pend.contrib.y, pend.contrib.z,
                                            (cont ? 0.0f : 1.0f) + (moved ? 2.0f : 0.0f));
                append(pl.shadowq, &ctl->shadow_n, slot, __activemask());
            }
            if (cont) append(pl.ext[nxt], &ctl->ext_n[nxt], slot, __activemask());
        }
    }
}

__global__ void k_shadow(Pool pl, Tables T, Ctl* ctl) {
    extern __shared__ int s_stack[];
    int* stack = s_stack + threadIdx.x;
    const uint32_t n = ctl->shadow_n;
    const uint32_t stride = gridDim.x * blockDim.x;
    uint32_t err = 0, cnt = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint32_t slot = pl.shadowq[i];
        const uint4 id = pl.ids[slot];
        const float4 sd = pl.sdir[slot], sc = pl.scon[slot];
        const int flags = (int)sc.w;
        const float4 o = (flags & 2) ? pl.sorg[slot] : pl.o_t[slot];
        Ray r{xyz(o), xyz(sd), 0.0f};                                 // Ray::new (render.rs:1457)
        Hit h;
        h.t = sd.w;
        h.prim = -1;
        ++cnt;
        const SceneDev S = T.scenes[id.x];
        const bool occluded = trace(S, r, 0.001f, true, h, stack, err);
        if (!occluded) {
            float4 l = pl.L[slot];
            l.x += sc.x;
            l.y += sc.y;
            l.z += sc.z;
            pl.L[slot] = l;
        }
        if (flags & 1) {
            Path P;
            uint4 id2;
            load_path(pl, slot, P, id2);
            finish(T, ctl, T.renders[id.x], id.x, id.z, P);
            append(pl.freeq, &ctl->free_n, slot, __activemask());
        }
    }
    unsigned long long s = cnt;
    for (int o2 = 16; o2 > 0; o2 >>= 1) s += __shfl_xor_sync(kFullMask, s, o2);
    if ((threadIdx.x & 31) == 0 && s) atomicAdd(&ctl->shadow_rays, s);
    if (err) atomicOr(&ctl->error_flags, err);
}

__global__ void k_post_iteration(Ctl* ctl, uint32_t Q) {
    const uint32_t cur = ctl->cur;
    ctl->ext_n[cur] = 0;
    ctl->cur = cur ^ 1u;
    for (int k = 0; k < kQueues; ++k) ctl->mat_n[k] = 0;
    ctl->shadow_n = 0;
    ctl->iteration += 1;
    if (ctl->ext_n[cur ^ 1u] > Q || ctl->free_n > Q) ctl->error_flags |= LUM_KERR_QUEUE_OVERFLOW;
    ctl->done = (ctl->work_next >= ctl->work_total && ctl->ext_n[cur ^ 1u] == 0) ? 1u : 0u;
}

// Fixed-point sums -> f32 RGB (render.rs:1705 and :2616-2618).
__global__ void k_finalize(Tables T, float* const* outs) {
    const uint32_t s = blockIdx.y;
    const RenderDev& R = T.renders[s];
    const uint32_t npix = R.w * R.h;
    float* out = outs[s];
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < npix; p += gridDim.x * blockDim.x) {
        const unsigned long long* a = T.acc + 4 * (T.acc_off[s] + p);
        double w = (double)(long long)a[3] / kFix;
        double inv = w > 0.0 ? 1.0 / w : 1.0;
        for (int c = 0; c < 3; ++c) out[3 * (size_t)p + c] = (float)((double)(long long)a[c] / kFix * inv) * R.exposure;
    }
}

// Batched megakernel: the megakernel's per-pixel path-regeneration loop (k_render) over one
// warp-task queue that spans every scene, one persistent launch for the batch.  A task is one
// 8x4 tile of one scene and one group of at most kGroupStrata of its strata; scenes are queued
// heaviest task first (order[]).
// Each task runs as the plain megakernel's (tile_task: the warp's lanes share the task's
// (pixel, stratum) pairs) and adds its fixed-point pixel sums to the scene's accumulators;
// k_finalize writes the images, equal bit for bit to lum_render's.  Scene descriptors are
// read in place (constant or global memory) rather than copied per task.
constexpr uint32_t kLanes = 4;           // streams of the streams mode
constexpr uint32_t kGroupStrata = 256;   // whole tiles up to 256 spp: the batch's queue is long anyway

// Scene and render descriptors of batches of up to kConstScenes scenes live in constant memory,
// indexed by a warp-uniform scene index: read through the constant cache like the plain
// megakernel's kernel parameters.  Larger batches read them from global memory.
constexpr uint32_t kConstScenes = 128;
__constant__ SceneDev c_scenes[kConstScenes];
__constant__ RenderDev c_renders[kConstScenes];

template <bool CONST_TABLES>
__global__ void __launch_bounds__(128, 5) k_render_multi(Tables T, const unsigned long long* task_prefix,
                                                         const uint32_t* order, const uint2* groups, Ctl* ctl,
                                                         uint32_t* next_task) {
    extern __shared__ int s_stack[];
    __shared__ unsigned long long s_acc[4][32][4];
    __shared__ uint32_t s_next[4];
    __shared__ V s_exit[4][32];                  // deferred Subsurface origins
    int* stack = s_stack + threadIdx.x;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const unsigned long long total = task_prefix[T.n];
    uint32_t err = 0, nseg = 0, nsh = 0;
    for (;;) {
        uint32_t task = 0;
        if (lane == 0) task = atomicAdd(next_task, 1u);
        task = __shfl_sync(kFullMask, task, 0);
        if (task >= total) break;
        uint32_t lo = 0, hi = T.n;
        while (hi - lo > 1) {
            uint32_t mid = (lo + hi) >> 1;
            if (task_prefix[mid] <= task) lo = mid; else hi = mid;
        }
        const uint32_t s = order[lo];
        const SceneDev& S = CONST_TABLES ? c_scenes[s] : T.scenes[s];
        const RenderDev& R = CONST_TABLES ? c_renders[s] : T.renders[s];
        const uint2 grp = groups[s];                       // (n_groups, strata per group)
        const uint32_t t = task - (uint32_t)task_prefix[lo];
        const uint32_t tile = t / grp.x, group = t - tile * grp.x;
        const uint32_t x0 = (tile % R.tiles_x) * 8, y0 = (tile / R.tiles_x) * 4;
        const uint32_t tw = min(8u, R.w - x0), th = min(4u, R.h - y0);
        const uint32_t s_lo = R.s_begin + group * grp.y;
        const uint32_t s_hi = min(R.s_end, s_lo + grp.y);
        tile_task<false>(S, R, x0, y0, tw, th, s_lo, s_hi, s_acc[wid], &s_next[wid], s_exit[wid], stack, err, nseg,
                         nsh, nullptr);
        if (lane < (int)(tw * th)) {
            const uint32_t i = x0 + lane % tw, j = y0 + lane / tw;
            unsigned long long* a = T.acc + 4 * (T.acc_off[s] + (size_t)j * R.w + i);
            for (int c = 0; c < 4; ++c) atomicAdd(a + c, s_acc[wid][lane][c]);
        }
        __syncwarp(kFullMask);
        if (lane == 0) {
            unsigned long long k = atomicAdd(T.done_count + s, 1ull) + 1ull;
            if (k == task_prefix[lo + 1] - task_prefix[lo]) T.finish_ns[s] = globaltimer();
        }
    }
    unsigned long long a = nseg, b = nsh;
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(kFullMask, a, o);
        b += __shfl_xor_sync(kFullMask, b, o);
        err |= __shfl_xor_sync(kFullMask, err, o);
    }
    if (lane == 0) {
        atomicAdd(&ctl->segments, a);
        atomicAdd(&ctl->shadow_rays, b);
        if (err) atomicOr(&ctl->error_flags, err);
    }
}

}  // namespace wf
}  // namespace lum

// ----------------------------------------------------------------------------- host side
namespace {

using lum::wf::Ctl;
using lum::wf::kQueues;

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

lum_status wf_cuda(cudaError_t e, const char* what) {
    char msg[256];
    snprintf(msg, sizeof msg, "%s: %s", what, cudaGetErrorString(e));
    cudaGetLastError();
    return lum::set_error(e == cudaErrorMemoryAllocation ? LUM_ERR_OUT_OF_MEMORY : LUM_ERR_CUDA, msg);
}

#define WF(call, what)                                \
    do {                                              \
        cudaError_t e_ = (call);                      \
        if (e_ != cudaSuccess) return wf_cuda(e_, what); \
    } while (0)

int sm_count(int device) {
    int n = 0;
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, device);
    return n > 0 ? n : 148;
}

}  // namespace

struct lum_batch {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    uint32_t n = 0;
    lum_batch_config cfg{};
    std::vector<lum::RenderDev> R;
    std::vector<lum::SceneDev> S;                  // host copies (constant tables of megakernel mode)
    std::vector<unsigned long long> scene_total;
    unsigned long long total_work = 0;
    size_t total_pixels = 0;
    std::vector<unsigned long long> acc_off;
    void* d_mem = nullptr;
    lum::wf::Pool pool{};
    lum::wf::Tables T{};
    Ctl* ctl = nullptr;
    float** d_out_table = nullptr;
    float* d_staging = nullptr;                 // per-scene device images for host outputs
    uint32_t* h_done = nullptr;                 // pinned
    int grid_queue = 0, grid_trace = 0, block = 128;
    size_t stack_bytes = 0;
    unsigned long long* d_tile_prefix = nullptr;   // megakernel mode: task prefix in queue order
    uint32_t* d_next_task = nullptr;
    uint32_t* d_order = nullptr;                   // queue position -> scene
    uint2* d_groups = nullptr;                     // per scene: (stratum groups, strata per group)
    int grid_mega = 0;
    // streams mode
    std::vector<cudaStream_t> lanes;
    std::vector<cudaEvent_t> scene_ev;            // per scene: its last kernel done
    std::vector<uint32_t> lane_order;             // launch order (heaviest first)
    lum::WorkCounters* d_wc = nullptr;            // per scene
};

namespace {

lum_status enqueue_iteration(lum_batch* b) {
    using namespace lum::wf;
    const int blk = b->block;
    k_generate<<<b->grid_queue, blk, 0, b->stream>>>(b->pool, b->T, b->ctl);
    k_post_generate<<<1, 1, 0, b->stream>>>(b->ctl);
    k_extend<<<b->grid_trace, blk, b->stack_bytes, b->stream>>>(b->pool, b->T, b->ctl);
    k_shade<0><<<b->grid_queue, blk, 0, b->stream>>>(b->pool, b->T, b->ctl);
    k_shade<1><<<b->grid_queue, blk, 0, b->stream>>>(b->pool, b->T, b->ctl);
    k_shade<2><<<b->grid_queue, blk, 0, b->stream>>>(b->pool, b->T, b->ctl);
    k_shade<3><<<b->grid_queue, blk, 0, b->stream>>>(b->pool, b->T, b->ctl);
    k_shade<4><<<b->grid_queue, blk, 0, b->stream>>>(b->pool, b->T, b->ctl);
    k_shade<5><<<b->grid_queue, blk, 0, b->stream>>>(b->pool, b->T, b->ctl);
    k_shade<6><<<b->grid_queue, blk, 0, b->stream>>>(b->pool, b->T, b->ctl);
    k_shadow<<<b->grid_trace, blk, b->stack_bytes, b->stream>>>(b->pool, b->T, b->ctl);
    k_post_iteration<<<1, 1, 0, b->stream>>>(b->ctl, b->pool.Q);
    return LUM_OK;
}

std::mutex g_const_mu;   // guards the constant scene tables of megakernel-mode renders

// Streams mode: each scene is lum_render's launch (the megakernel, the task plan lum_render
// chooses, the scene's slice of the batch accumulators as the split tiles' fixed-point sums),
// issued heaviest first round robin over the lanes with no host synchronisation in
// between, so the hardware starts a scene's CTAs as the previous scenes' CTAs retire.
lum_status run_lanes(lum_batch* b, float* const* d_outs, double* scene_done_ms, lum_batch_stats* stats,
                     std::chrono::steady_clock::time_point t0) {
    using namespace lum::wf;
    WF(cudaMemsetAsync(b->d_wc, 0, sizeof(lum::WorkCounters) * b->n, b->stream), "memset counters");
    WF(cudaEventRecord(b->ev0, b->stream), "event");
    for (cudaStream_t l : b->lanes) WF(cudaStreamWaitEvent(l, b->ev0, 0), "fork");
    for (uint32_t q = 0; q < b->n; ++q) {
        const uint32_t s = b->lane_order[q];
        cudaStream_t l = b->lanes[q % b->lanes.size()];
        const lum::RenderDev& R = b->R[s];
        if (R.n_tasks > 0 && R.s_end > R.s_begin) {
            // the scene's slice of the batch accumulators (32 bytes per pixel) as the split tiles'
            // scratch: as many tiles are split as it holds
            const lum::RenderGroups grp = lum::render_groups(R);
            WF(lum::launch_render_grouped(b->S[s], R, d_outs[s], b->d_wc + s, l, b->T.acc + 4 * b->acc_off[s],
                                          32 * (size_t)R.w * R.h, grp), "render launch");
        } else if (R.w > 0 && R.h > 0) {
            WF(cudaMemsetAsync(d_outs[s], 0, sizeof(float) * 3 * (size_t)R.w * R.h, l), "memset image");
        }
        WF(cudaEventRecord(b->scene_ev[s], l), "event");
    }
    for (uint32_t s = 0; s < b->n; ++s) WF(cudaStreamWaitEvent(b->stream, b->scene_ev[s], 0), "join");
    WF(cudaEventRecord(b->ev1, b->stream), "event");
    std::vector<lum::WorkCounters> wc(b->n);
    WF(cudaMemcpyAsync(wc.data(), b->d_wc, sizeof(lum::WorkCounters) * b->n, cudaMemcpyDeviceToHost, b->stream),
       "counters");
    WF(cudaStreamSynchronize(b->stream), "batch");
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, b->ev0, b->ev1);
    unsigned long long segs = 0, shadows = 0;
    uint32_t flags = 0;
    for (uint32_t s = 0; s < b->n; ++s) {
        segs += wc[s].segments;
        shadows += wc[s].shadow_rays;
        flags |= wc[s].error_flags;
        if (scene_done_ms) {
            float d = 0.0f;
            cudaEventElapsedTime(&d, b->ev0, b->scene_ev[s]);
            scene_done_ms[s] = d;
        }
    }
    if (stats) {
        stats->paths = b->total_work;
        stats->segments = segs;
        stats->shadow_rays = shadows;
        stats->device_ms = ms;
        stats->total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        stats->graph_launches = 0;
        stats->iterations = 1;
        stats->error_flags = flags;
    }
    if (flags) return lum::set_error(LUM_ERR_KERNEL, "streams-mode batch reported error flags");
    return LUM_OK;
}

lum_status run_batch(lum_batch* b, float* const* d_outs, double* scene_done_ms, lum_batch_stats* stats) {
    using namespace lum::wf;
    auto t0 = std::chrono::steady_clock::now();
    WF(cudaSetDevice(b->device), "cudaSetDevice");
    if (b->cfg.mode == LUM_BATCH_STREAMS) return run_lanes(b, d_outs, scene_done_ms, stats, t0);
    WF(cudaMemcpyAsync(b->d_out_table, d_outs, sizeof(float*) * b->n, cudaMemcpyHostToDevice, b->stream), "outs");
    WF(cudaMemsetAsync(b->T.acc, 0, sizeof(unsigned long long) * 4 * b->total_pixels, b->stream), "memset acc");
    WF(cudaMemsetAsync(b->T.done_count, 0, sizeof(unsigned long long) * b->n, b->stream), "memset done");
    WF(cudaMemsetAsync(b->T.finish_ns, 0, sizeof(unsigned long long) * b->n, b->stream), "memset finish");
    Ctl c{};
    c.work_total = b->total_work;
    c.free_n = b->pool.Q;
    WF(cudaMemcpyAsync(b->ctl, &c, sizeof c, cudaMemcpyHostToDevice, b->stream), "ctl");
    WF(cudaEventRecord(b->ev0, b->stream), "event");
    if (b->cfg.mode == LUM_BATCH_MEGAKERNEL) {
        // the constant tables are per device: one megakernel-mode render at a time uploads and
        // uses them (this call synchronises its stream before returning)
        std::unique_lock<std::mutex> lk(g_const_mu, std::defer_lock);
        if (b->n <= kConstScenes) {
            lk.lock();
            WF(cudaMemcpyToSymbolAsync(c_scenes, b->S.data(), sizeof(lum::SceneDev) * b->n, 0, cudaMemcpyHostToDevice,
                                       b->stream), "scene table");
            WF(cudaMemcpyToSymbolAsync(c_renders, b->R.data(), sizeof(lum::RenderDev) * b->n, 0,
                                       cudaMemcpyHostToDevice, b->stream), "render table");
        }
        WF(cudaMemsetAsync(b->d_next_task, 0, sizeof(uint32_t), b->stream), "memset");
        k_init<<<1, 32, 0, b->stream>>>(b->pool, b->ctl);             // t0 only (pool is empty)
        WF(cudaGraphLaunch(b->exec, b->stream), "cudaGraphLaunch");
        k_finalize<<<dim3(64, b->n), 256, 0, b->stream>>>(b->T, b->d_out_table);
        WF(cudaGetLastError(), "finalize launch");
        WF(cudaEventRecord(b->ev1, b->stream), "event");
        Ctl out{};
        std::vector<unsigned long long> fin(b->n);
        WF(cudaMemcpyAsync(&out, b->ctl, sizeof out, cudaMemcpyDeviceToHost, b->stream), "ctl");
        WF(cudaMemcpyAsync(fin.data(), b->T.finish_ns, sizeof(unsigned long long) * b->n, cudaMemcpyDeviceToHost,
                           b->stream), "finish");
        WF(cudaStreamSynchronize(b->stream), "batch");
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, b->ev0, b->ev1);
        if (scene_done_ms)
            for (uint32_t s = 0; s < b->n; ++s)
                scene_done_ms[s] = fin[s] ? (double)(fin[s] - out.t0_ns) * 1e-6 : -1.0;
        if (stats) {
            stats->paths = b->total_work;
            stats->segments = out.segments;
            stats->shadow_rays = out.shadow_rays;
            stats->device_ms = ms;
            stats->total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
            stats->graph_launches = 1;
            stats->iterations = 1;
            stats->error_flags = out.error_flags;
        }
        if (out.error_flags) return lum::set_error(LUM_ERR_KERNEL, "batched megakernel reported error flags");
        return LUM_OK;
    }
    k_init<<<b->grid_queue, b->block, 0, b->stream>>>(b->pool, b->ctl);
    WF(cudaGetLastError(), "init launch");
    // Every graph launch runs iters_per_graph iterations; each pass retires at least one
    // bounce of every active path, so max_depth + 2 passes per pool refill bound the total.
    uint32_t max_depth = 0;
    for (const auto& r : b->R) max_depth = std::max(max_depth, r.max_depth);
    const unsigned long long refills = (b->total_work + b->pool.Q - 1) / b->pool.Q;
    const unsigned long long cap_iters = (refills + 2) * (2ull * max_depth + 4) + 64;
    unsigned long long cap_launches = cap_iters / b->cfg.iters_per_graph + 2;
    // Diagnostic: LUM_BATCH_MAX_LAUNCHES=n lowers the cap, so the cap's error path
    // (LUM_KERR_ITERATION_CAP) can be exercised without a runaway loop.
    if (const char* ml = std::getenv("LUM_BATCH_MAX_LAUNCHES")) {
        const long long m = std::strtoll(ml, nullptr, 10);
        if (m >= 1 && (unsigned long long)m < cap_launches) cap_launches = (unsigned long long)m;
    }
    uint32_t launches = 0;
    bool done = false;
    while (!done) {
        if (launches >= cap_launches) break;
        WF(cudaGraphLaunch(b->exec, b->stream), "cudaGraphLaunch");
        ++launches;
        WF(cudaMemcpyAsync(b->h_done, &b->ctl->done, sizeof(uint32_t), cudaMemcpyDeviceToHost, b->stream), "done");
        WF(cudaStreamSynchronize(b->stream), "batch");
        done = *b->h_done != 0;
    }
    dim3 fgrid(64, b->n);
    k_finalize<<<fgrid, 256, 0, b->stream>>>(b->T, b->d_out_table);
    WF(cudaGetLastError(), "finalize launch");
    WF(cudaEventRecord(b->ev1, b->stream), "event");
    Ctl out{};
    WF(cudaMemcpyAsync(&out, b->ctl, sizeof out, cudaMemcpyDeviceToHost, b->stream), "ctl");
    std::vector<unsigned long long> fin(b->n);
    WF(cudaMemcpyAsync(fin.data(), b->T.finish_ns, sizeof(unsigned long long) * b->n, cudaMemcpyDeviceToHost,
                       b->stream), "finish");
    WF(cudaStreamSynchronize(b->stream), "batch");
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, b->ev0, b->ev1);
    if (scene_done_ms)
        for (uint32_t s = 0; s < b->n; ++s)
            scene_done_ms[s] = fin[s] ? (double)(fin[s] - out.t0_ns) * 1e-6 : -1.0;
    uint32_t flags = out.error_flags | (done ? 0u : (uint32_t)LUM_KERR_ITERATION_CAP);
    if (stats) {
        stats->paths = b->total_work;
        stats->segments = out.segments;
        stats->shadow_rays = out.shadow_rays;
        stats->device_ms = ms;
        stats->total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        stats->graph_launches = launches;
        stats->iterations = out.iteration;
        stats->error_flags = flags;
    }
    if (flags) {
        char msg[128];
        snprintf(msg, sizeof msg, "wavefront batch reported error flags 0x%x", flags);
        return lum::set_error(LUM_ERR_KERNEL, msg);
    }
    return LUM_OK;
}

lum_status create_batch(lum_scene* const* scenes, const lum_render_params* params, uint32_t n,
                        const lum_batch_config& cfg, lum_batch** out) {
    using namespace lum::wf;
    auto* b = new lum_batch();
    auto fail_out = [&](lum_status st) {
        lum_batch_destroy(b);
        return st;
    };
    b->n = n;
    b->cfg = cfg;
    b->R.resize(n);
    std::vector<lum::SceneDev> S(n);
    for (uint32_t s = 0; s < n; ++s) {
        int dev = 0;
        lum_status st = lum::scene_view(scenes[s], &params[s], S[s], b->R[s], dev);
        if (st != LUM_OK) return fail_out(st);
        if (s == 0) b->device = dev;
        if (dev != b->device) return fail_out(lum::set_error(LUM_ERR_INVALID_ARGUMENT, "batch scenes on different devices"));
        if (b->R[s].max_depth > 127) return fail_out(lum::set_error(LUM_ERR_UNSUPPORTED, "batched max_depth above 127"));
        if (b->R[s].sqrt_spp * b->R[s].sqrt_spp > (1u << 24))
            return fail_out(lum::set_error(LUM_ERR_UNSUPPORTED, "batched strata above 2^24"));
    }
    std::vector<unsigned long long> prefix(n + 1, 0);
    b->acc_off.resize(n);
    b->scene_total.resize(n);
    for (uint32_t s = 0; s < n; ++s) {
        const auto& r = b->R[s];
        unsigned long long px = (unsigned long long)r.w * r.h;
        b->scene_total[s] = px * (r.s_end - r.s_begin);
        prefix[s + 1] = prefix[s] + b->scene_total[s];
        b->acc_off[s] = b->total_pixels;
        b->total_pixels += px;
    }
    b->total_work = prefix[n];
    b->S = S;
    const bool mega = cfg.mode == LUM_BATCH_MEGAKERNEL, lanes = cfg.mode == LUM_BATCH_STREAMS;
    if (cfg.mode != LUM_BATCH_WAVEFRONT && !mega && !lanes)
        return fail_out(lum::set_error(LUM_ERR_INVALID_ARGUMENT, "unknown batch mode"));
    // megakernel mode: tasks of one tile x one group of <= kGroupStrata strata, scenes queued
    // by decreasing task cost (strata per task x log2 of the primitive count), so the longest
    // tasks start first and the batch ends on short ones
    std::vector<uint2> groups(n);
    std::vector<uint32_t> order(n);
    std::vector<double> task_cost(n);
    for (uint32_t s = 0; s < n; ++s) {
        const uint32_t n_st = b->R[s].s_end > b->R[s].s_begin ? b->R[s].s_end - b->R[s].s_begin : 0;
        const uint32_t gs = std::max(1u, std::min(n_st, kGroupStrata));
        groups[s] = make_uint2(n_st ? (n_st + gs - 1) / gs : 0, gs);
        task_cost[s] = (double)gs * (2.0 + std::log2(1.0 + (double)S[s].n_prims)) * std::max(1u, b->R[s].max_depth);
        order[s] = s;
    }
    std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) { return task_cost[x] > task_cost[y]; });
    std::vector<unsigned long long> tile_prefix(n + 1, 0);
    for (uint32_t k = 0; k < n; ++k) {
        const uint32_t s = order[k];
        tile_prefix[k + 1] = tile_prefix[k] + (unsigned long long)b->R[s].n_tasks * groups[s].x;
    }
    if (tile_prefix[n] > 0xFFFFFFFFull) return fail_out(lum::set_error(LUM_ERR_TOO_LARGE, "too many tiles in batch"));
    const uint32_t Q = mega || lanes ? 1024u : cfg.pool_paths;
    if (Q < 1024 || Q > (1u << 24)) return fail_out(lum::set_error(LUM_ERR_INVALID_ARGUMENT, "pool_paths out of range"));
    if (!mega && cfg.block_threads != 128 && cfg.block_threads != 256)
        return fail_out(lum::set_error(LUM_ERR_INVALID_ARGUMENT, "block_threads must be 128 or 256"));
    if (!mega && (cfg.iters_per_graph < 1 || cfg.iters_per_graph > 64))
        return fail_out(lum::set_error(LUM_ERR_INVALID_ARGUMENT, "iters_per_graph out of range"));
    b->block = mega || lanes ? 128 : (int)cfg.block_threads;
    b->stack_bytes = (size_t)lum::kStackDepth * b->block * sizeof(int);

    // one allocation: pool SoA, queues, tables, accumulators, staging images
    size_t off = 0;
    auto take = [&](size_t bytes) {
        size_t o = off;
        off = align256(off + bytes);
        return o;
    };
    size_t o_ot = take(16ull * Q), o_dj = take(16ull * Q), o_bj = take(16ull * Q), o_L = take(16ull * Q);
    size_t o_ids = take(16ull * Q), o_hit = take(16ull * Q), o_sd = take(16ull * Q), o_sc = take(16ull * Q);
    size_t o_so = take(16ull * Q);
    size_t o_ext0 = take(4ull * Q), o_ext1 = take(4ull * Q), o_free = take(4ull * Q), o_shq = take(4ull * Q);
    size_t o_mq[kQueues];
    for (int k = 0; k < kQueues; ++k) o_mq[k] = take(4ull * Q);
    size_t o_scenes = take(sizeof(lum::SceneDev) * n), o_renders = take(sizeof(lum::RenderDev) * n);
    size_t o_prefix = take(8ull * (n + 1)), o_accoff = take(8ull * n), o_acc = take(32ull * b->total_pixels);
    size_t o_done = take(8ull * n), o_total = take(8ull * n), o_fin = take(8ull * n), o_finit = take(4ull * n);
    size_t o_ctl = take(sizeof(Ctl)), o_outs = take(sizeof(float*) * n);
    size_t o_stage = take(12ull * b->total_pixels);
    size_t o_tpre = take(8ull * (n + 1)), o_next = take(4), o_order = take(4ull * n), o_groups = take(8ull * n);
    size_t o_wc = take(sizeof(lum::WorkCounters) * n);
    cudaError_t e = cudaSetDevice(b->device);
    if (e != cudaSuccess) return fail_out(wf_cuda(e, "cudaSetDevice"));
    if ((e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaEventCreate(&b->ev0)) != cudaSuccess || (e = cudaEventCreate(&b->ev1)) != cudaSuccess ||
        (e = cudaMalloc(&b->d_mem, off)) != cudaSuccess ||
        (e = cudaHostAlloc((void**)&b->h_done, sizeof(uint32_t), cudaHostAllocDefault)) != cudaSuccess)
        return fail_out(wf_cuda(e, "batch allocation"));
    char* m = (char*)b->d_mem;
    Pool& pl = b->pool;
    pl.o_t = (float4*)(m + o_ot); pl.d_jx = (float4*)(m + o_dj); pl.beta_jy = (float4*)(m + o_bj);
    pl.L = (float4*)(m + o_L); pl.ids = (uint4*)(m + o_ids); pl.hit = (float4*)(m + o_hit);
    pl.sdir = (float4*)(m + o_sd); pl.scon = (float4*)(m + o_sc); pl.sorg = (float4*)(m + o_so);
    pl.ext[0] = (uint32_t*)(m + o_ext0); pl.ext[1] = (uint32_t*)(m + o_ext1);
    pl.freeq = (uint32_t*)(m + o_free); pl.shadowq = (uint32_t*)(m + o_shq);
    for (int k = 0; k < kQueues; ++k) pl.matq[k] = (uint32_t*)(m + o_mq[k]);
    pl.Q = Q;
    Tables& T = b->T;
    T.scenes = (const lum::SceneDev*)(m + o_scenes);
    T.renders = (const lum::RenderDev*)(m + o_renders);
    T.prefix = (const unsigned long long*)(m + o_prefix);
    T.acc_off = (const unsigned long long*)(m + o_accoff);
    T.acc = (unsigned long long*)(m + o_acc);
    T.done_count = (unsigned long long*)(m + o_done);
    T.scene_total = (const unsigned long long*)(m + o_total);
    T.finish_ns = (unsigned long long*)(m + o_fin);
    T.finish_iter = (uint32_t*)(m + o_finit);
    T.n = n;
    T.sort_threshold = cfg.sort_threshold;
    b->ctl = (Ctl*)(m + o_ctl);
    b->d_out_table = (float**)(m + o_outs);
    b->d_staging = (float*)(m + o_stage);
    b->d_tile_prefix = (unsigned long long*)(m + o_tpre);
    b->d_next_task = (uint32_t*)(m + o_next);
    b->d_order = (uint32_t*)(m + o_order);
    b->d_groups = (uint2*)(m + o_groups);
    b->d_wc = (lum::WorkCounters*)(m + o_wc);
    if ((e = cudaMemcpy(m + o_scenes, S.data(), sizeof(lum::SceneDev) * n, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(m + o_renders, b->R.data(), sizeof(lum::RenderDev) * n, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(m + o_prefix, prefix.data(), 8ull * (n + 1), cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(m + o_accoff, b->acc_off.data(), 8ull * n, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(m + o_total, b->scene_total.data(), 8ull * n, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(m + o_tpre, tile_prefix.data(), 8ull * (n + 1), cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(m + o_order, order.data(), 4ull * n, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(m + o_groups, groups.data(), 8ull * n, cudaMemcpyHostToDevice)) != cudaSuccess)
        return fail_out(wf_cuda(e, "batch upload"));

    // grids: persistent-style, sized to the SM count and the kernels' occupancy
    const int sms = sm_count(b->device);
    int occ_q = 0, occ_t = 0;
    cudaFuncSetAttribute(k_extend, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b->stack_bytes);
    cudaFuncSetAttribute(k_shadow, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b->stack_bytes);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_q, k_shade<5>, b->block, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_t, k_extend, b->block, b->stack_bytes);
    b->grid_queue = sms * std::max(occ_q, 1);
    b->grid_trace = sms * std::max(occ_t, 1);

    int occ_m = 0;
    for (auto fn : {k_render_multi<true>, k_render_multi<false>})
        cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)((size_t)lum::kStackDepth * 128 * sizeof(int)));
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_m, k_render_multi<true>, 128,
                                                  (size_t)lum::kStackDepth * 128 * sizeof(int));
    b->grid_mega = sms * std::max(occ_m, 1);

    if (lanes) {
        // streams mode: scenes launched by decreasing estimated time (paths x task cost per
        // stratum), round robin over kLanes streams
        b->lanes.assign(kLanes, nullptr);
        for (auto& l : b->lanes)
            if ((e = cudaStreamCreateWithFlags(&l, cudaStreamNonBlocking)) != cudaSuccess)
                return fail_out(wf_cuda(e, "cudaStreamCreate"));
        b->scene_ev.assign(n, nullptr);
        for (auto& ev : b->scene_ev)
            if ((e = cudaEventCreate(&ev)) != cudaSuccess) return fail_out(wf_cuda(e, "cudaEventCreate"));
        std::vector<double> est(n);
        for (uint32_t s = 0; s < n; ++s)
            est[s] = (double)b->scene_total[s] * task_cost[s] / std::max(1u, groups[s].y);
        b->lane_order.resize(n);
        for (uint32_t s = 0; s < n; ++s) b->lane_order[s] = s;
        std::stable_sort(b->lane_order.begin(), b->lane_order.end(),
                         [&](uint32_t x, uint32_t y) { return est[x] > est[y]; });
        *out = b;
        return LUM_OK;
    }

    // capture the batch's kernels into one graph: iters_per_graph wavefront iterations, or
    // the single persistent megakernel launch
    if ((e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
        return fail_out(wf_cuda(e, "cudaStreamBeginCapture"));
    if (mega) {
        if (n <= kConstScenes)
            k_render_multi<true><<<b->grid_mega, 128, (size_t)lum::kStackDepth * 128 * sizeof(int), b->stream>>>(
                b->T, b->d_tile_prefix, b->d_order, b->d_groups, b->ctl, b->d_next_task);
        else
            k_render_multi<false><<<b->grid_mega, 128, (size_t)lum::kStackDepth * 128 * sizeof(int), b->stream>>>(
                b->T, b->d_tile_prefix, b->d_order, b->d_groups, b->ctl, b->d_next_task);
    } else {
        for (uint32_t g = 0; g < cfg.iters_per_graph; ++g) enqueue_iteration(b);
    }
    e = cudaStreamEndCapture(b->stream, &b->graph);
    if (e != cudaSuccess) return fail_out(wf_cuda(e, "cudaStreamEndCapture"));
    if ((e = cudaGraphInstantiate(&b->exec, b->graph, 0)) != cudaSuccess)
        return fail_out(wf_cuda(e, "cudaGraphInstantiate"));
    *out = b;
    return LUM_OK;
}

// ---------------------------------------------------------------- autotuner
std::mutex g_tune_mu;

std::string tune_cache_path() {
    const char* p = std::getenv("LUM_AUTOTUNE_CACHE");
    if (p && *p) return p;
    const char* home = std::getenv("HOME");
    return std::string(home ? home : "/tmp") + "/.cache/luminara_b200_autotune.txt";
}

std::string batch_key(lum_scene* const* scenes, const lum_render_params* params, uint32_t n, int device) {
    cudaDeviceProp prop{};
    cudaGetDeviceProperties(&prop, device);
    unsigned long long paths = 0, pixels = 0, prims = 0, depth = 0;
    for (uint32_t s = 0; s < n; ++s) {
        uint32_t np = 0;
        lum_scene_info(scenes[s], &np, nullptr, nullptr, nullptr);
        prims += np;
        unsigned long long w = std::max(params[s].width, 1u), h = std::max(params[s].height, 1u);
        unsigned long long st = (unsigned long long)std::ceil(std::sqrt((double)params[s].samples_per_pixel));
        pixels += w * h;
        paths += w * h * st * st;
        depth += params[s].max_depth;
    }
    char buf[512];
    snprintf(buf, sizeof buf, "%s|n=%u|paths=%llu|pixels=%llu|prims=%llu|depth=%llu", prop.name, n, paths, pixels,
             prims, depth);
    for (char* c = buf; *c; ++c)
        if (*c == ' ') *c = '_';
    return buf;
}

bool tune_lookup(const std::string& key, lum_batch_config& cfg) {
    FILE* f = fopen(tune_cache_path().c_str(), "r");
    if (!f) return false;
    char line[512];
    bool found = false;
    while (fgets(line, sizeof line, f)) {
        char k[384];
        unsigned q, blk, thr, it, mode;
        if (sscanf(line, "%383s %u %u %u %u %u", k, &q, &blk, &thr, &it, &mode) == 6 && key == k) {
            std::memset(&cfg, 0, sizeof cfg);
            cfg.pool_paths = q;
            cfg.block_threads = blk;
            cfg.sort_threshold = thr;
            cfg.iters_per_graph = it;
            cfg.mode = mode;
            found = true;
        }
    }
    fclose(f);
    return found;
}

void tune_store(const std::string& key, const lum_batch_config& cfg, double ms) {
    std::string path = tune_cache_path();
    size_t slash = path.find_last_of('/');
    if (slash != std::string::npos && slash > 0) mkdir(path.substr(0, slash).c_str(), 0755);   // may exist
    FILE* f = fopen(path.c_str(), "a");
    if (!f) return;
    fprintf(f, "%s %u %u %u %u %u %.3f\n", key.c_str(), cfg.pool_paths, cfg.block_threads, cfg.sort_threshold,
            cfg.iters_per_graph, cfg.mode, ms);
    fclose(f);
}

}  // namespace

extern "C" {

lum_status lum_batch_default_config(lum_batch_config* cfg) {
    if (!cfg) return lum::set_error(LUM_ERR_INVALID_ARGUMENT, "null argument");
    std::memset(cfg, 0, sizeof *cfg);
    cfg->pool_paths = 1u << 20;
    cfg->block_threads = 128;
    cfg->sort_threshold = 1u << 16;
    cfg->iters_per_graph = 8;
    cfg->mode = LUM_BATCH_WAVEFRONT;
    return LUM_OK;
}

lum_status lum_batch_autotune(lum_scene* const* scenes, const lum_render_params* params, uint32_t n,
                              lum_batch_config* out, double* best_ms) {
    if (!scenes || !params || !out || n == 0) return lum::set_error(LUM_ERR_INVALID_ARGUMENT, "null argument");
    int device = 0;
    {
        lum::SceneDev d;
        lum::RenderDev r;
        lum_status st = lum::scene_view(scenes[0], &params[0], d, r, device);
        if (st != LUM_OK) return st;
    }
    std::lock_guard<std::mutex> lk(g_tune_mu);
    std::string key = batch_key(scenes, params, n, device);
    if (tune_lookup(key, *out)) {
        if (best_ms) *best_ms = -1.0;
        return LUM_OK;
    }
    // Two rounds of successive halving: every candidate on a calibration batch of the same
    // scenes with an eighth of each scene's strata, then the three fastest on a quarter of the
    // strata (the short first round favours configurations that hide per-scene tails, which
    // matter less at full size).
    auto calibration = [&](uint32_t div) {
        std::vector<lum_render_params> cal(params, params + n);
        for (auto& p : cal) {
            uint32_t sq = (uint32_t)std::ceil(std::sqrt((double)p.samples_per_pixel));
            uint32_t total = sq * sq;
            uint32_t cnt = p.sample_count ? p.sample_count : total;
            p.sample_count = std::max(1u, cnt / div);
        }
        return cal;
    };
    const uint32_t pools[] = {1u << 19, 1u << 20, 1u << 21};
    const uint32_t blocks[] = {128, 256};
    const uint32_t thresholds[] = {0u, 1u << 16, 0xFFFFFFFFu};
    std::vector<lum_batch_config> cands;
    {
        lum_batch_config c{};
        lum_batch_default_config(&c);
        c.mode = LUM_BATCH_MEGAKERNEL;
        cands.push_back(c);
        c.mode = LUM_BATCH_STREAMS;
        cands.push_back(c);
    }
    for (uint32_t q : pools)
        for (uint32_t blk : blocks)
            for (uint32_t thr : thresholds) {
                lum_batch_config c{};
                c.pool_paths = q;
                c.block_threads = blk;
                c.sort_threshold = thr;
                c.iters_per_graph = 8;
                c.mode = LUM_BATCH_WAVEFRONT;
                cands.push_back(c);
            }
    // device ms of one render (after a warm-up render), or a negative value when it failed
    auto time_cand = [&](const std::vector<lum_render_params>& cal, const lum_batch_config& c) {
        lum_batch* b = nullptr;
        if (create_batch(scenes, cal.data(), n, c, &b) != LUM_OK) return -1.0;
        lum_batch_stats st{};
        std::vector<float*> outs(n);
        size_t off = 0;
        for (uint32_t s = 0; s < n; ++s) {
            outs[s] = b->d_staging + 3 * off;
            off += (size_t)b->R[s].w * b->R[s].h;
        }
        lum_status rs = run_batch(b, outs.data(), nullptr, &st);   // warm-up
        if (rs == LUM_OK) rs = run_batch(b, outs.data(), nullptr, &st);
        lum_batch_destroy(b);
        return rs == LUM_OK ? st.device_ms : -1.0;
    };
    std::vector<std::pair<double, size_t>> round1;
    {
        const auto cal = calibration(8);
        for (size_t i = 0; i < cands.size(); ++i) {
            const double t = time_cand(cal, cands[i]);
            if (t >= 0.0) round1.push_back({t, i});
        }
    }
    std::sort(round1.begin(), round1.end());
    lum_batch_config best{};
    double best_t = 1e30;
    {
        const auto cal = calibration(4);
        for (size_t k = 0; k < round1.size() && k < 3; ++k) {
            const double t = time_cand(cal, cands[round1[k].second]);
            if (t >= 0.0 && t < best_t) {
                best_t = t;
                best = cands[round1[k].second];
            }
        }
    }
    if (best_t >= 1e30) return lum::set_error(LUM_ERR_CUDA, "autotune: no configuration ran");
    *out = best;
    if (best_ms) *best_ms = best_t;
    tune_store(key, best, best_t);
    return LUM_OK;
}

lum_status lum_batch_create(lum_scene* const* scenes, const lum_render_params* params, uint32_t n,
                            const lum_batch_config* cfg, lum_batch** out) {
    if (!scenes || !params || !out || n == 0) return lum::set_error(LUM_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    lum_batch_config c{};
    if (cfg) {
        c = *cfg;
    } else {
        lum_status st = lum_batch_autotune(scenes, params, n, &c, nullptr);
        if (st != LUM_OK) return st;
    }
    return create_batch(scenes, params, n, c, out);
}

lum_status lum_batch_config_of(const lum_batch* b, lum_batch_config* cfg) {
    if (!b || !cfg) return lum::set_error(LUM_ERR_INVALID_ARGUMENT, "null argument");
    *cfg = b->cfg;
    return LUM_OK;
}

lum_status lum_batch_render_device(lum_batch* b, float* const* d_outs, double* scene_done_ms,
                                   lum_batch_stats* stats) {
    if (!b || !d_outs) return lum::set_error(LUM_ERR_INVALID_ARGUMENT, "null argument");
    return run_batch(b, d_outs, scene_done_ms, stats);
}

lum_status lum_batch_render(lum_batch* b, float* const* outs, double* scene_done_ms, lum_batch_stats* stats) {
    if (!b || !outs) return lum::set_error(LUM_ERR_INVALID_ARGUMENT, "null argument");
    std::vector<float*> dev(b->n);
    size_t off = 0;
    for (uint32_t s = 0; s < b->n; ++s) {
        dev[s] = b->d_staging + 3 * off;
        off += (size_t)b->R[s].w * b->R[s].h;
    }
    auto t0 = std::chrono::steady_clock::now();
    lum_status st = run_batch(b, dev.data(), scene_done_ms, stats);
    if (st != LUM_OK && st != LUM_ERR_KERNEL) return st;
    for (uint32_t s = 0; s < b->n; ++s) {
        size_t bytes = 12ull * b->R[s].w * b->R[s].h;
        if (bytes && outs[s]) WF(cudaMemcpyAsync(outs[s], dev[s], bytes, cudaMemcpyDeviceToHost, b->stream), "D2H");
    }
    WF(cudaStreamSynchronize(b->stream), "D2H");
    if (stats) stats->total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return st;
}

lum_status lum_batch_destroy(lum_batch* b) {
    if (!b) return LUM_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    for (cudaStream_t l : b->lanes) {
        cudaStreamSynchronize(l);
        cudaStreamDestroy(l);
    }
    for (cudaEvent_t e : b->scene_ev) cudaEventDestroy(e);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    if (b->d_mem) cudaFree(b->d_mem);
    if (b->h_done) cudaFreeHost(b->h_done);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return LUM_OK;
}

}  // extern "C"
