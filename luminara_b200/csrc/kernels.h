// kernels.h -- host-side declarations of the kernel launchers (internal to the library).
#pragma once

#include <cuda_runtime.h>

#include "../../include/luminara_gpu.h"
#include "device_scene.h"

namespace lum {

// Launches the megakernel on `stream`, whole tiles only (no scratch).  `wc` must be zeroed
// beforehand.  blocks_per_sm <= 0 picks the occupancy limit.
cudaError_t launch_render(const SceneDev& S, const RenderDev& R, float* out, WorkCounters* wc, cudaStream_t stream,
                          int blocks_per_sm);
// Task plan of a megakernel launch (TaskPlan, device_scene.h): tiles [0, n_whole) whole, the
// rest split into n_groups stratum groups.  Small frames split every tile; larger frames render
// whole tiles (splitting their last tiles is available, LUM_TAIL_TILES_PER_WARP, and off).
struct RenderGroups {
    uint32_t n_groups;      // groups per split tile (1 = no split)
    uint32_t group_strata;  // strata per group
    uint32_t n_whole;       // tiles rendered whole
};
RenderGroups render_groups(const RenderDev& R);
// Device scratch the split tiles of plan `g` need (0 without split tiles).
size_t render_scratch_bytes(const RenderDev& R, const RenderGroups& g);
// The megakernel with plan `groups`; `scratch` (render_scratch_bytes) holds the split tiles'
// sums and is cleared by the launch.  With less scratch fewer tiles are split.
cudaError_t launch_render_grouped(const SceneDev& S, const RenderDev& R, float* out, WorkCounters* wc,
                                  cudaStream_t stream, void* scratch, size_t scratch_bytes, RenderGroups groups);
// The megakernel leaving the frame's raw per-pixel sums (4 u64 fixed-point values per pixel:
// filter-weighted R, G, B and the filter weight, 2^-32 units) in `sums`, zeroed by the launch;
// no pixels are written.  Sums of disjoint stratum ranges add.
cudaError_t launch_render_sums(const SceneDev& S, const RenderDev& R, unsigned long long* sums, WorkCounters* wc,
                               cudaStream_t stream);
// Pixels (exposure applied) of n_px fixed-point sums.
cudaError_t launch_fixed_finalize(const unsigned long long* sums, size_t n_px, float exposure, float* out,
                                  cudaStream_t stream);
// Counter build of the megakernel: same image, plus node/primitive test tallies in wc->tally.
cudaError_t launch_render_counted(const SceneDev& S, const RenderDev& R, float* out, WorkCounters* wc,
                                  cudaStream_t stream);
// The in-loop branches of the sample loop (render.rs:1601-1678): adaptive sampling and the
// time limit.
struct SamplingDev {
    uint32_t adaptive;        // 1 = adaptive sampling
    uint32_t min_samples;     // max(spp / 4, 16)
    double threshold;         // standard-error threshold
    unsigned long long limit_ns;   // 0 = no time limit
};
// Renders a frame with adaptive sampling and/or a time limit (one task per 8x4 tile, all
// strata).  wc must be zeroed; wc->samples receives the samples kept.
cudaError_t launch_render_sampled(const SceneDev& S, const RenderDev& R, const SamplingDev& A, float* out,
                                  WorkCounters* wc, cudaStream_t stream);
// AOV passes into device buffers (any may be null): depth W*H floats, normals and albedo
// W*H*3 bytes.
cudaError_t launch_aov(const SceneDev& S, const RenderDev& R, float* depth, uint8_t* normals, uint8_t* albedo,
                       WorkCounters* wc, cudaStream_t stream);
cudaError_t launch_intersect(const SceneDev& S, const lum_ray* rays, uint32_t n, lum_hit* hits, WorkCounters* wc,
                             cudaStream_t stream);
cudaError_t launch_occluded(const SceneDev& S, const lum_ray* rays, uint32_t n, int32_t* occ, WorkCounters* wc,
                            cudaStream_t stream);

// Linear HDR (3 floats per pixel) -> RGBA8 through the colour chain of lum_tonemap_params at
// `exposure`; `scratch` (LUM_TONEMAP_SCRATCH_BYTES) is used with auto-exposure.
cudaError_t launch_tonemap(const float* hdr, uint32_t w, uint32_t h, const lum_tonemap_params& tm, double exposure,
                           double* scratch, uint8_t* rgba, cudaStream_t stream);

}  // namespace lum
