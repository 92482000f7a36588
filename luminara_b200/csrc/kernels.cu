// kernels.cu -- CUDA kernels of the path-tracing core and their launchers (sm_100a).
//
//   k_render      the single-scene megakernel (camera -> closest hit -> scatter/NEE/RR ->
//                 per-pixel accumulation), replacing render.rs:1598-1706 + ray_color.
//   k_intersect   closest hit of a ray set (SceneWorld::hit, scene.rs:816-834).
//   k_occluded    any hit of a ray set (the NEE shadow query, render.rs:1457-1460).
#include <cuda_runtime.h>

#include <algorithm>

#include <chrono>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <utility>
#include <vector>

#include "kernels.h"
#include "scene_access.h"
#include "render_task.cuh"
#include "tracer.cuh"

namespace lum {

constexpr int kRenderThreads = 128;
// Minimum resident blocks per SM requested from the register allocator for the general
// megakernel builds (6 -> 80 registers, 24-58 bytes of spills; on B200 3-6% faster than 5 blocks
// at 93 registers without spills on the box-room, diff-quads and dense-mesh frames).  The
// scene-class builds (LUM_RENDER_CLASS_BLOCKS) run 7 blocks at 72 registers: more warps to hide
// the node and triangle fetch latency outweigh their larger spills (40-124 bytes) -- on B200 the
// dense mesh 194.2 -> 185.4 ms, the 512x512 quad frame 9.66 -> 9.33 ms, the box room unchanged
// (8 blocks: box room 3% slower).  The sphere builds use 7 blocks without lights (72 registers,
// no spills; 8 blocks at 64 registers gained nothing) and 6 with them.
#ifndef LUM_RENDER_MIN_BLOCKS
#define LUM_RENDER_MIN_BLOCKS 6
#endif
#ifndef LUM_RENDER_CLASS_BLOCKS
#define LUM_RENDER_CLASS_BLOCKS 7
#endif
constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ void flush_counters(WorkCounters* wc, uint32_t err, uint32_t nseg, uint32_t nsh) {
    unsigned long long s = nseg, h = nsh;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_xor_sync(kFull, s, o);
        h += __shfl_xor_sync(kFull, h, o);
        err |= __shfl_xor_sync(kFull, err, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&wc->segments, s);
        atomicAdd(&wc->shadow_rays, h);
        if (err) atomicOr(&wc->error_flags, err);
    }
}

// Persistent megakernel.  Each warp takes tasks of the launch's TaskPlan from a global counter:
// an 8x4 pixel tile and all of its strata, or, for the split tiles at the end of the list, a
// group of them.  tile_task (render_task.cuh) runs the task with the warp's lanes drawing
// (pixel, stratum) pairs from one pool and adding each finished path to the tile's fixed-point
// pixel sums.  A whole tile's task then writes its pixels; a split tile's tasks add their sums
// to the tile's sums in global memory, which k_split_finalize turns into pixels (raw-sum
// renders add every task's sums to the per-pixel sums instead).  Integer sums make the image
// deterministic and the same however the frame was split.
// The SPH builds are small enough for more blocks per SM without spills (72 registers without
// NEE, 80 with); their shared memory then fits when the traversal stack is sized to the scene's
// BVH (SceneDev::stack_depth).
// CLS (CLS_QUAD, CLS_MESH): general builds carrying only the primitive tests and light samplers
// of one scene class (SceneDev::cls).
template <bool COUNT, bool EXT, bool NEE, bool SPH, int CLS = CLS_ALL>
__global__ void __launch_bounds__(kRenderThreads, SPH ? (NEE ? 6 : 7) : CLS != CLS_ALL ? LUM_RENDER_CLASS_BLOCKS
                                                                               : LUM_RENDER_MIN_BLOCKS)
    k_render(SceneDev S, RenderDev R, float* __restrict__ out, WorkCounters* wc, TaskPlan TP) {
    extern __shared__ int s_stack[];
    __shared__ unsigned long long s_acc[kRenderThreads / 32][32][4];
    __shared__ uint32_t s_next[kRenderThreads / 32];
    __shared__ V s_exit[kRenderThreads / 32][32];      // deferred Subsurface origins (EXT only)
    int* stack = s_stack + threadIdx.x;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t err = 0, nseg = 0, nsh = 0;
    TestTally tally{};
    for (;;) {
        uint32_t task = 0;
        if (lane == 0) task = atomicAdd(&wc->next_task, 1u);
        task = __shfl_sync(kFull, task, 0);
        if (task >= TP.n_total) break;
        uint32_t tile, s_lo = R.s_begin, s_hi = R.s_end;
        if (task < TP.n_whole) {
            tile = task;
        } else {
            const uint32_t t2 = task - TP.n_whole;
            const uint32_t k = t2 / TP.n_groups, g = t2 - k * TP.n_groups;
            tile = TP.n_whole + k;
            s_lo = R.s_begin + g * TP.group_strata;
            s_hi = min(R.s_end, s_lo + TP.group_strata);
        }
        const uint32_t x0 = (tile % R.tiles_x) * 8, y0 = (tile / R.tiles_x) * 4;
        const uint32_t tw = min(8u, R.w - x0), th = min(4u, R.h - y0);
        tile_task<COUNT, EXT, NEE, SPH, LUM_SUSPEND_LANES, CLS>(S, R, x0, y0, tw, th, s_lo, s_hi, s_acc[wid],
                                                                &s_next[wid], s_exit[wid], stack, err, nseg, nsh,
                                                                &tally);
        if (lane < (int)(tw * th)) {
            const uint32_t i = x0 + lane % tw, j = y0 + lane / tw;
            const unsigned long long* a = s_acc[wid][lane];
            if (TP.pix_sums || task >= TP.n_whole) {   // raw-sum renders; split tiles
                unsigned long long* g = TP.pix_sums ? TP.pix_sums + 4 * ((size_t)j * R.w + i)
                                                    : TP.tile_sums + 128 * (size_t)(tile - TP.n_whole) + 4 * lane;
                for (int c = 0; c < 4; ++c) atomicAdd(g + c, a[c]);
            } else {
                fixed_pixel(a, R.exposure, out + 3 * ((size_t)j * R.w + i));
            }
        }
        __syncwarp(kFull);   // the sums are read before the next task clears them
    }
    flush_counters(wc, err, nseg, nsh);
    if constexpr (COUNT) {
        atomicAdd(&wc->tally.node, tally.node);
        for (int k = 0; k < 6; ++k) atomicAdd(&wc->tally.prim[k], tally.prim[k]);
        atomicAdd(&wc->tally.plane, tally.plane);
    }
}

// Pixels of the split tiles (TaskPlan::tile_sums): one thread per pixel slot of a split tile.
__global__ void k_split_finalize(RenderDev R, TaskPlan TP, uint32_t n_split, float* __restrict__ out) {
    const uint32_t n_tiles = TP.n_whole + n_split;
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < 32u * n_split; q += gridDim.x * blockDim.x) {
        const uint32_t k = q >> 5, p = q & 31u, tile = TP.n_whole + k;
        if (tile >= n_tiles) break;
        const uint32_t x0 = (tile % R.tiles_x) * 8, y0 = (tile / R.tiles_x) * 4;
        const uint32_t tw = min(8u, R.w - x0), th = min(4u, R.h - y0);
        if (p >= tw * th) continue;
        const uint32_t i = x0 + p % tw, j = y0 + p / tw;
        fixed_pixel(TP.tile_sums + 128 * (size_t)k + 4 * p, R.exposure, out + 3 * ((size_t)j * R.w + i));
    }
}

// Pixels from per-pixel fixed-point sums (the raw-sum renders' finalize).
__global__ void k_fixed_finalize(const unsigned long long* __restrict__ gacc, size_t n_px, float exposure,
                                 float* __restrict__ out) {
    for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < n_px; p += (size_t)gridDim.x * blockDim.x)
        fixed_pixel(gacc + 4 * p, exposure, out + 3 * p);
}

// u, v of a hit as the reference's HitRecord carries them (uv per primitive type).
__device__ void hit_uv(const SceneDev& S, const Ray& ray, const Hit& h, const Surface& sf, float& u, float& v) {
    u = v = 0.0f;
    if (h.prim <= -2) {                                                // plane.rs:60-62
        const PlaneDev& P = S.planes[-2 - h.prim];
        V local = sf.p - mk(P.p);
        float a = dot(local, mk(P.ua)), b = dot(local, mk(P.va));
        u = fabsf(a - truncf(a));
        v = fabsf(b - truncf(b));
        return;
    }
    int type = __ldg(S.meta + h.prim) & 15;
    float4 a = ldp(S, h.prim, 0);
    if (type == PT_SPHERE) {                                           // sphere.rs:48-52
        float4 b = ldp(S, h.prim, 1);
        V c = xyz(a);
        if (b.w != 0.0f) c = fma3(xyz(b) - c, ray.time, c);
        V on = (sf.p - c) * (1.0f / a.w);
        float theta = acosf(fminf(fmaxf(-on.y, -1.0f), 1.0f));
        float phi = atan2f(-on.z, on.x) + CUDART_PI_F;
        u = phi / (2.0f * CUDART_PI_F);
        v = theta / CUDART_PI_F;
    } else if (type == PT_QUAD) {
        float t, uv[2];
        if (hit_quad(a, ldp(S, h.prim, 1), ldp(S, h.prim, 2), ldp(S, h.prim, 3), ray, -CUDART_INF_F, CUDART_INF_F, t, uv)) {
            u = uv[0];
            v = uv[1];
        }
    } else if (type == PT_TRIANGLE) {
        u = h.b1;
        v = h.b2;
    } else if (type == PT_DISK) {                                      // disk.rs:38-41
        V off = sf.p - xyz(a);
        u = atan2f(off.z, off.x) / (2.0f * CUDART_PI_F) + 0.5f;
        v = sqrtf(len2(off)) / a.w;
    }
}

__global__ void __launch_bounds__(kRenderThreads) k_intersect(SceneDev S, const lum_ray* __restrict__ rays, uint32_t n,
                                                              lum_hit* __restrict__ hits, WorkCounters* wc) {
    extern __shared__ int s_stack[];
    int* stack = s_stack + threadIdx.x;
    uint32_t err = 0;
    for (uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += gridDim.x * blockDim.x) {
        lum_ray r = rays[idx];
        Ray ray{mk(r.org), mk(r.dir), r.time};
        Hit h;
        h.t = r.tmax;
        h.prim = -1;
        h.b1 = h.b2 = 0.0f;
        lum_hit out;
        out.reserved = 0;
        if (trace(S, ray, r.tmin, false, h, stack, err)) {
            Surface sf = surface_of(S, ray, h);
            out.t = h.t;
            hit_uv(S, ray, h, sf, out.u, out.v);
            out.normal[0] = sf.n.x;
            out.normal[1] = sf.n.y;
            out.normal[2] = sf.n.z;
            out.prim_id = h.prim <= -2 ? S.planes[-2 - h.prim].orig_id : __ldg(S.orig + h.prim);
            out.front_face = sf.front ? 1 : 0;
            out.material = sf.mat;
        } else {
            out.t = r.tmax;
            out.u = out.v = 0.0f;
            out.normal[0] = out.normal[1] = out.normal[2] = 0.0f;
            out.prim_id = -1;
            out.front_face = 0;
            out.material = -1;
        }
        hits[idx] = out;
    }
    if (err) atomicOr(&wc->error_flags, err);
}

__global__ void __launch_bounds__(kRenderThreads) k_occluded(SceneDev S, const lum_ray* __restrict__ rays, uint32_t n,
                                                             int32_t* __restrict__ occ, WorkCounters* wc) {
    extern __shared__ int s_stack[];
    int* stack = s_stack + threadIdx.x;
    uint32_t err = 0;
    for (uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += gridDim.x * blockDim.x) {
        lum_ray r = rays[idx];
        Ray ray{mk(r.org), mk(r.dir), r.time};
        Hit h;
        h.t = r.tmax;
        h.prim = -1;
        occ[idx] = trace(S, ray, r.tmin, true, h, stack, err) ? 1 : 0;
    }
    if (err) atomicOr(&wc->error_flags, err);
}

// ------------------------------------------------------------------------------ launchers
static int num_sms() {
    static const int n = [] {   // initialised once, thread-safe
        int dev = 0, sms = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        return sms > 0 ? sms : 148;
    }();
    return n;
}

static size_t stack_bytes(int threads) { return (size_t)kStackDepth * threads * sizeof(int); }

static int render_occupancy() {
    static const int occ = [] {   // initialised once, thread-safe
        for (auto fn : {k_render<false, false, false, false>, k_render<false, false, true, false>,
                        k_render<false, true, false, false>, k_render<false, true, true, false>,
                        k_render<false, false, false, true>, k_render<false, false, true, true>,
                        k_render<true, false, true, false>, k_render<true, true, true, false>,
                        k_render<false, false, false, false, CLS_QUAD>, k_render<false, false, true, false, CLS_QUAD>,
                        k_render<false, false, false, false, CLS_MESH>, k_render<false, false, true, false, CLS_MESH>})
            cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)stack_bytes(kRenderThreads));
        int o = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, k_render<false, false, true, false>, kRenderThreads,
                                                      stack_bytes(kRenderThreads));
        return o > 0 ? o : 4;
    }();
    return occ;
}

// Resident blocks per SM of a megakernel build with `smem` bytes of stack (cached).
static int kernel_occupancy(const void* fn, size_t smem) {
    static std::mutex mu;
    static std::vector<std::pair<std::pair<const void*, size_t>, int>> cache;
    std::lock_guard<std::mutex> lk(mu);
    for (const auto& e : cache)
        if (e.first.first == fn && e.first.second == smem) return e.second;
    int occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, kRenderThreads, smem);
    if (occ <= 0) occ = render_occupancy();
    cache.push_back({{fn, smem}, occ});
    return occ;
}

// Task plans.  A frame with fewer 8x4 tiles than LUM_SMALL_FRAME_TILES per resident warp splits
// every tile into stratum groups until the launch has about LUM_SMALL_FRAME_TASKS tasks per
// warp (groups of at least LUM_MIN_GROUP_STRATA strata), and widens the groups to
// LUM_PREF_GROUP_STRATA strata where the launch keeps LUM_SMALL_FRAME_TILES tasks per warp: a
// task ends when its warp's slowest lane does, so very short tasks pay that wait too often, but
// a launch with fewer tasks than warps leaves SMs idle.  Measured on B200 (kernel time):
//   512x512 x 64 spp quads (8192 tiles)     2 groups of 32 strata 10.26 ms, 4 of 16  9.66 ms
//   256x256 x 64 spp box room (2048 tiles)  7 groups of 10        1.99 ms, 14 of 5   2.02 ms,
//                                           8 of 8                 1.94 ms
//   128x128 x 16 spp box room (512 tiles)   4 groups of 4          0.29 ms, 2 of 8    0.43 ms
// A larger frame can also split its last LUM_TAIL_TILES_PER_WARP x (resident warps) tiles into
// LUM_TAIL_GROUPS groups, so that the launch ends on short tasks; on the 1080p frames (spheres
// 256 spp, dense mesh 144 spp) that gained nothing -- the warps still running at the end of a
// launch issue faster as the others exit -- so it is off (0).
#ifndef LUM_SMALL_FRAME_TILES
#define LUM_SMALL_FRAME_TILES 4
#endif
#ifndef LUM_SMALL_FRAME_TASKS
#define LUM_SMALL_FRAME_TASKS 8
#endif
#ifndef LUM_MIN_GROUP_STRATA
#define LUM_MIN_GROUP_STRATA 4
#endif
#ifndef LUM_PREF_GROUP_STRATA
#define LUM_PREF_GROUP_STRATA 8
#endif
#ifndef LUM_TAIL_TILES_PER_WARP
#define LUM_TAIL_TILES_PER_WARP 0
#endif
#ifndef LUM_TAIL_GROUPS
#define LUM_TAIL_GROUPS 8
#endif

// Scratch bytes of one split tile: 32 pixels x 4 fixed-point sums.
constexpr size_t kSplitTileBytes = 32 * 4 * sizeof(unsigned long long);

RenderGroups render_groups(const RenderDev& R) {
    const uint32_t n_st = R.s_end > R.s_begin ? R.s_end - R.s_begin : 0;
    RenderGroups g{1, n_st, R.n_tasks};
    if (R.n_tasks == 0 || n_st < 2) return g;
    const uint64_t warps = (uint64_t)num_sms() * render_occupancy() * (kRenderThreads / 32);
    uint64_t groups, split;
    if ((uint64_t)R.n_tasks < (uint64_t)LUM_SMALL_FRAME_TILES * warps) {
        groups = ((uint64_t)LUM_SMALL_FRAME_TASKS * warps + R.n_tasks - 1) / R.n_tasks;
        groups = std::min<uint64_t>(groups, n_st / LUM_MIN_GROUP_STRATA);
        const uint64_t wide = n_st / LUM_PREF_GROUP_STRATA;   // groups of the preferred size
        if (groups > wide && wide * R.n_tasks >= (uint64_t)LUM_SMALL_FRAME_TILES * warps) groups = wide;
        split = R.n_tasks;
    } else {
        groups = std::min<uint64_t>(LUM_TAIL_GROUPS, n_st / LUM_MIN_GROUP_STRATA);
        split = std::min<uint64_t>(R.n_tasks, (uint64_t)LUM_TAIL_TILES_PER_WARP * warps);
    }
    if (groups <= 1 || split == 0) return g;
    g.group_strata = (uint32_t)((n_st + groups - 1) / groups);
    g.n_groups = (n_st + g.group_strata - 1) / g.group_strata;   // no empty group
    g.n_whole = R.n_tasks - (uint32_t)split;
    return g;
}

size_t render_scratch_bytes(const RenderDev& R, const RenderGroups& g) {
    if (g.n_groups <= 1 || g.n_whole >= R.n_tasks) return 0;
    return (size_t)(R.n_tasks - g.n_whole) * kSplitTileBytes;
}

// The megakernel launch of plan `grp`.  pix_sums non-null: the launch leaves the frame's
// fixed-point sums there (zeroed first) and writes no pixels.  Otherwise split tiles need
// `scratch` (render_scratch_bytes); only as many tiles are split as its `scratch_bytes` hold,
// the others are rendered whole.
template <bool COUNT>
static cudaError_t launch_render_t(const SceneDev& S, const RenderDev& R, float* out, WorkCounters* wc,
                                   cudaStream_t stream, int blocks_per_sm, RenderGroups grp, void* scratch,
                                   size_t scratch_bytes, unsigned long long* pix_sums) {
    const int occ = render_occupancy();
    if (blocks_per_sm <= 0) blocks_per_sm = occ;
    const uint32_t n_tiles = R.n_tasks;
    const uint32_t n_st = R.s_end > R.s_begin ? R.s_end - R.s_begin : 0;
    TaskPlan TP{};
    TP.n_whole = n_tiles;
    TP.n_groups = 1;
    TP.group_strata = n_st;
    if (grp.n_groups > 1 && grp.n_whole < n_tiles) {
        uint64_t k = n_tiles - grp.n_whole;
        if (!pix_sums) k = std::min<uint64_t>(k, scratch ? scratch_bytes / kSplitTileBytes : 0);
        if (k > 0) {
            TP.n_whole = n_tiles - (uint32_t)k;
            TP.n_groups = grp.n_groups;
            TP.group_strata = grp.group_strata;
            if (!pix_sums) {
                TP.tile_sums = static_cast<unsigned long long*>(scratch);
                cudaError_t e = cudaMemsetAsync(scratch, 0, (size_t)k * kSplitTileBytes, stream);
                if (e != cudaSuccess) return e;
            }
        }
    }
    const uint64_t n_total = (uint64_t)TP.n_whole + (uint64_t)(n_tiles - TP.n_whole) * TP.n_groups;
    if (n_total > 0xFFFFFFF0ull) return cudaErrorInvalidValue;
    TP.n_total = (uint32_t)n_total;
    TP.pix_sums = pix_sums;
    if (pix_sums) {
        cudaError_t e = cudaMemsetAsync(pix_sums, 0, 32 * (size_t)R.w * R.h, stream);
        if (e != cudaSuccess) return e;
    }
    const bool nee = COUNT || S.n_lights > 0;
    const bool sph = !COUNT && !R.ext && S.spheres_basic;
    const int cls = (COUNT || R.ext || sph) ? (int)CLS_ALL : S.cls;
    auto kernel = R.ext ? (nee ? k_render<COUNT, true, true, false> : k_render<COUNT, true, COUNT, false>)
                : sph   ? (nee ? k_render<COUNT, false, true, !COUNT> : k_render<COUNT, false, COUNT, !COUNT>)
                : cls == CLS_QUAD ? (nee ? k_render<COUNT, false, true, false, CLS_QUAD>
                                         : k_render<COUNT, false, COUNT, false, CLS_QUAD>)
                : cls == CLS_MESH ? (nee ? k_render<COUNT, false, true, false, CLS_MESH>
                                         : k_render<COUNT, false, COUNT, false, CLS_MESH>)
                        : (nee ? k_render<COUNT, false, true, false> : k_render<COUNT, false, COUNT, false>);
    // the traversal stack sized to the scene's BVH; resident blocks for that size
    const size_t smem = (size_t)S.stack_depth * kRenderThreads * sizeof(int);
    if (blocks_per_sm == occ) blocks_per_sm = kernel_occupancy((const void*)kernel, smem);
    int grid = num_sms() * blocks_per_sm;
    int blocks_needed = (int)((n_total + 3) / 4);   // 4 warps per block, one task per warp at least
    if (grid > blocks_needed) grid = blocks_needed > 0 ? blocks_needed : 1;
    // (kernel above: scenes without the other materials and backgrounds, without lights, or
    // made of spheres with the basic materials run builds without the code they cannot reach;
    // the counter build is the general one: the same paths either way)
    kernel<<<grid, kRenderThreads, smem, stream>>>(S, R, out, wc, TP);
    cudaError_t e = cudaGetLastError();
    const uint32_t n_split = n_tiles - TP.n_whole;
    if (e != cudaSuccess || pix_sums || n_split == 0) return e;
    const int fgrid = (int)std::min<size_t>((32 * (size_t)n_split + 255) / 256, (size_t)num_sms() * 8);
    k_split_finalize<<<fgrid, 256, 0, stream>>>(R, TP, n_split, out);
    return cudaGetLastError();
}

cudaError_t launch_render_sums(const SceneDev& S, const RenderDev& R, unsigned long long* sums, WorkCounters* wc,
                               cudaStream_t stream) {
    return launch_render_t<false>(S, R, nullptr, wc, stream, 0, render_groups(R), nullptr, 0, sums);
}

cudaError_t launch_fixed_finalize(const unsigned long long* sums, size_t n_px, float exposure, float* out,
                                  cudaStream_t stream) {
    if (n_px == 0) return cudaSuccess;
    const int cgrid = (int)std::min<size_t>((n_px + 255) / 256, (size_t)num_sms() * 8);
    k_fixed_finalize<<<cgrid, 256, 0, stream>>>(sums, n_px, exposure, out);
    return cudaGetLastError();
}

cudaError_t launch_render(const SceneDev& S, const RenderDev& R, float* out, WorkCounters* wc, cudaStream_t stream,
                          int blocks_per_sm) {
    return launch_render_t<false>(S, R, out, wc, stream, blocks_per_sm, RenderGroups{1, 0, R.n_tasks}, nullptr, 0,
                                  nullptr);
}

cudaError_t launch_render_grouped(const SceneDev& S, const RenderDev& R, float* out, WorkCounters* wc,
                                  cudaStream_t stream, void* scratch, size_t scratch_bytes, RenderGroups groups) {
    return launch_render_t<false>(S, R, out, wc, stream, 0, groups, scratch, scratch_bytes, nullptr);
}

cudaError_t launch_render_counted(const SceneDev& S, const RenderDev& R, float* out, WorkCounters* wc,
                                  cudaStream_t stream) {
    return launch_render_t<true>(S, R, out, wc, stream, 0, RenderGroups{1, 0, R.n_tasks}, nullptr, 0, nullptr);
}

cudaError_t launch_intersect(const SceneDev& S, const lum_ray* rays, uint32_t n, lum_hit* hits, WorkCounters* wc,
                             cudaStream_t stream) {
    int grid = (int)((n + kRenderThreads - 1) / kRenderThreads);
    int cap = num_sms() * 16;
    if (grid > cap) grid = cap;
    if (grid < 1) grid = 1;
    k_intersect<<<grid, kRenderThreads, stack_bytes(kRenderThreads), stream>>>(S, rays, n, hits, wc);
    return cudaGetLastError();
}

cudaError_t launch_occluded(const SceneDev& S, const lum_ray* rays, uint32_t n, int32_t* occ, WorkCounters* wc,
                            cudaStream_t stream) {
    int grid = (int)((n + kRenderThreads - 1) / kRenderThreads);
    int cap = num_sms() * 16;
    if (grid > cap) grid = cap;
    if (grid < 1) grid = 1;
    k_occluded<<<grid, kRenderThreads, stack_bytes(kRenderThreads), stream>>>(S, rays, n, occ, wc);
    return cudaGetLastError();
}

}  // namespace lum

// ------------------------------------------------------------------ allocation-free render
// lum_render_noalloc (include/luminara_gpu.h): the megakernel writes into a fixed device
// array instead of device memory obtained from cudaMalloc.  Layout: WorkCounters in the
// first 256 bytes, then up to LUM_NOALLOC_MAX_PIXELS RGB float pixels.  In host code
// g_noalloc_scratch names a host-side stand-in, not the device array, so its device address
// is looked up per device with cudaGetSymbolAddress and passed to the kernel.
namespace {

constexpr size_t kNoAllocCounterBytes = 256;
constexpr size_t kNoAllocBytes = kNoAllocCounterBytes + (size_t)LUM_NOALLOC_MAX_PIXELS * 3 * sizeof(float);
static_assert(sizeof(lum::WorkCounters) <= kNoAllocCounterBytes, "counters must fit the header slot");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
void* g_noalloc_addr[kMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device (looked up once per device).
lum_status noalloc_scratch(void** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return lum::set_error(LUM_ERR_CUDA, cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return lum::set_error(LUM_ERR_TOO_LARGE, "device ordinal above 63");
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
        void* ptr = nullptr;
        e = cudaGetSymbolAddress((void**)&ptr, g_noalloc_scratch);
        if (e != cudaSuccess || !ptr) {
            char msg[256];
            snprintf(msg, sizeof msg, "cudaGetSymbolAddress of the no-alloc scratch failed: %s", cudaGetErrorString(e));
            return lum::set_error(LUM_ERR_CUDA, msg);
        }
        g_noalloc_addr[dev] = ptr;
    }
    *out = g_noalloc_addr[dev];
    return LUM_OK;
}

}  // namespace

// Called by lum_scene_create with the scene's device current.
void lum::noalloc_preload() {
    void* unused = nullptr;
    if (noalloc_scratch(&unused) != LUM_OK) lum::set_error(LUM_OK, "");   // reported again by the render
}

namespace {

lum_status noalloc_cuda(cudaError_t e, const char* what) {
    char msg[256];
    snprintf(msg, sizeof msg, "%s: %s", what, cudaGetErrorString(e));
    return lum::set_error(LUM_ERR_CUDA, msg);
}

}  // namespace

extern "C" lum_status lum_render_noalloc(lum_scene* scene, const lum_render_params* params, float* out_rgb,
                                         lum_stats* stats) {
    auto t0 = std::chrono::steady_clock::now();
    if (!scene || !params || !out_rgb) return lum::set_error(LUM_ERR_INVALID_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> lk(lum::scene_mutex(scene));
    lum::SceneDev dev;
    lum::RenderDev R;
    cudaStream_t stream;
    lum_status st = lum::prepare_render(scene, params, dev, R, stream);
    if (st != LUM_OK) return st;
    const size_t pixels = (size_t)R.w * R.h;
    if (pixels > LUM_NOALLOC_MAX_PIXELS) {
        char msg[256];
        snprintf(msg, sizeof msg, "lum_render_noalloc: a %u x %u image needs %zu pixels of scratch; the maximum is %u",
                 R.w, R.h, pixels, (unsigned)LUM_NOALLOC_MAX_PIXELS);
        return lum::set_error(LUM_ERR_TOO_LARGE, msg);
    }
    if (stats) std::memset(stats, 0, sizeof *stats);
    if (pixels == 0) return LUM_OK;
    void* base = nullptr;
    st = noalloc_scratch(&base);
    if (st != LUM_OK) return st;
    auto* wc = reinterpret_cast<lum::WorkCounters*>(base);
    float* image = reinterpret_cast<float*>(static_cast<unsigned char*>(base) + kNoAllocCounterBytes);
    const size_t bytes = pixels * 3 * sizeof(float);
    cudaError_t e = cudaMemsetAsync(wc, 0, sizeof(lum::WorkCounters), stream);   // counters start at zero
    if (e != cudaSuccess) return noalloc_cuda(e, "cudaMemsetAsync");
    if (R.n_tasks > 0 && R.s_end > R.s_begin) {
        e = lum::launch_render(dev, R, image, wc, stream, 0);
        if (e != cudaSuccess) return noalloc_cuda(e, "render launch");
    } else {
        e = cudaMemsetAsync(image, 0, bytes, stream);
        if (e != cudaSuccess) return noalloc_cuda(e, "cudaMemsetAsync");
    }
    lum::WorkCounters counters{};
    if ((e = cudaMemcpyAsync(out_rgb, image, bytes, cudaMemcpyDeviceToHost, stream)) != cudaSuccess ||
        (e = cudaMemcpyAsync(&counters, wc, sizeof counters, cudaMemcpyDeviceToHost, stream)) != cudaSuccess ||
        (e = cudaStreamSynchronize(stream)) != cudaSuccess)
        return noalloc_cuda(e, "lum_render_noalloc");
    if (stats) {
        stats->paths = (uint64_t)pixels * (R.s_end - R.s_begin);
        stats->segments = counters.segments;
        stats->shadow_rays = counters.shadow_rays;
        stats->total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        stats->error_flags = counters.error_flags;
    }
    if (counters.error_flags) return lum::set_error(LUM_ERR_KERNEL, "render kernel reported error flags");
    return LUM_OK;
}

