// device_scene.h -- layouts shared by the host builder and the CUDA kernels.
//
// Everything the kernels read is flattened into structure-of-arrays buffers in HBM:
//   nodes   BVH2 nodes, 64 B each (both child boxes inline, so one node fetch tests two boxes)
//   prims   world-space primitive records 0-2, 48 B per primitive (transforms already applied):
//           what the sphere, triangle, disk and fog tests read
//   prims3  record 3, 16 B per primitive: the quad test's plane and a triangle's shading normal
//   meta    per-primitive (material << 4 | type)
//   orig    per-primitive id in description order (for hit records)
//   planes  unbounded planes, tested linearly after the BVH (src/scene.rs:826-831)
//   mats    materials, lights: small tables read through the read-only path
#pragma once

#include <stdint.h>

#include "../../include/luminara_gpu.h"

namespace lum {

// Primitive types (low 4 bits of meta)
enum PrimType : int32_t {
    PT_SPHERE = 0,    // a=(c, r)        b=(c1, moving?1:0)
    PT_QUAD = 1,      // a=(Q, w.Q)      b=(u, |u x v|)    c=(v, 0)  d=(w, outward sign); w = (u x v)/|u x v|^2
    PT_TRIANGLE = 2,  // a=(v0, 0)       b=(e1, 0)         c=(e2, 0) d=(n_geom, smooth-normal index or -1)
    PT_DISK = 3,      // a=(c, r)        b=(n, 0)
    PT_FOG_SPHERE = 4,// a=(c, r)        c=(neg_inv_density, 0, 0, 0)
    PT_FOG_BOX = 5    // a=(min, 0)      b=(max, 0)        c=(neg_inv_density, 0, 0, 0)
};

constexpr int kStackDepth = 64;     // traversal stack entries per thread
constexpr int kMaxBlendDepth = 4;   // nesting levels of Blend materials (checked by lum_scene_create)
constexpr int kMaxBvhDepth = 62;    // the builder keeps every leaf at most this deep
constexpr int kMedianDepth = 40;    // below this depth the builder splits at the object median

struct alignas(16) MatDev {
    float color[3];
    int32_t kind;
    float color2[3];
    int32_t tex;
    float tint[3];
    float tex_scale;
    float fuzz;
    float ior;
    float roughness;
    float metallic;
    float intensity;
    float dispersion;
    int32_t tint_white;
    int32_t specular;
    float extra[4];      // per-kind parameters of the other materials (lum_material.extra)
    int32_t sub[2];      // Blend: the blended materials
    int32_t n_emit;      // Blend: emissive leaves below it (entries of SceneDev::blend_emit)
    int32_t emit_first;  // Blend: its first entry in SceneDev::blend_emit
};

// A Blend's emission flattened: sum over its emissive leaves of weight * emitted(leaf), the
// weight being the product of the ratios (or 1 - ratio) on the way down.
struct BlendEmit {
    int32_t leaf;
    float weight;
};

struct alignas(16) LightDev {
    float p0[3];
    int32_t kind;
    float u[3];
    float radius;
    float v[3];
    float area;
    float n[3];
    float pad0;
    float e[3];
    float pad1;
};

struct alignas(16) PlaneDev {
    float p[3];
    int32_t material;
    float n[3];
    int32_t orig_id;
    float ua[3];
    float pad0;
    float va[3];
    float pad1;
};

struct CameraDev {
    float origin[3];
    float llc[3];
    float hor[3];
    float ver[3];
    float u[3];          // right (panorama basis)
    float v[3];          // up (panorama basis)
    float lens_radius;
    float fwd[3];        // -w: the panorama's forward axis
    int32_t panorama;    // 1: equirectangular camera (camera.rs:83-90)
};

// Device scene: raw pointers into the scene's device allocation.
struct SceneDev {
    const void* nodes;       // float4[4 * n_nodes]
    const void* prims;       // float4[3 * n_prims]: records 0-2
    const void* prims3;      // float4[n_prims]: record 3
    const int32_t* meta;     // n_prims
    const int32_t* orig;     // n_prims
    const float* smooth_n;   // 9 floats per smooth triangle (n0, n1, n2)
    const MatDev* mats;
    const LightDev* lights;
    const PlaneDev* planes;
    int32_t n_nodes;
    int32_t n_prims;
    int32_t n_lights;
    int32_t n_planes;
    int32_t n_mats;
    int32_t spheres_basic;   // every primitive is a static sphere and every material Lambertian /
                             // Metal / Dielectric / Emissive (planes allowed): the SPH kernels apply
    int32_t stack_depth;     // traversal stack entries this BVH can need (<= kStackDepth)
    int32_t moving;          // some sphere moves: camera rays draw their time
    int32_t cls;             // scene class of the general megakernel build (CLS_*, tracer.cuh)
    int32_t pad_cls;
    const BlendEmit* blend_emit;   // emissive leaves of Blend materials
    const float* env;        // environment map, env_w * env_h RGB floats (or null)
    uint32_t env_w, env_h;
    CameraDev cam;
};

// Task list of one megakernel launch.  The frame's 8x4 tiles are numbered row-major; tiles
// [0, n_whole) are one task each (every stratum), tiles [n_whole, n_tiles) are split into
// n_groups tasks of group_strata consecutive strata (the last group may be shorter).  Whole
// tiles come first, so the launch ends on short tasks.
//   pix_sums   non-null: every task adds its sums to these per-pixel fixed-point sums (4 u64 per
//              pixel) and no pixels are written (raw-sum renders);
//   tile_sums  otherwise the split tiles' tasks add their sums here (128 u64 per split tile: 32
//              pixels x 4; zeroed before the launch), and k_split_finalize writes their pixels.
struct TaskPlan {
    uint32_t n_whole;
    uint32_t n_groups;
    uint32_t group_strata;
    uint32_t n_total;          // tasks: n_whole + (n_tiles - n_whole) * n_groups
    unsigned long long* pix_sums;
    unsigned long long* tile_sums;
};

// Test counts of the counter build (node visits test two child boxes each).
struct alignas(16) TestTally {
    unsigned long long node;
    unsigned long long prim[6];   // by PrimType
    unsigned long long plane;
};

// Work/scratch block of one render launch (global memory, zeroed before each launch).
struct alignas(16) WorkCounters {
    uint32_t next_task;
    uint32_t error_flags;
    uint32_t pad0, pad1;
    unsigned long long segments;
    unsigned long long shadow_rays;
    TestTally tally;
    unsigned long long samples;   // camera samples kept (adaptive / time-limited renders)
    unsigned long long t0_ns;     // start of a time-limited render (%globaltimer)
};

struct RenderDev {
    uint32_t full_w, full_h;
    uint32_t crop_x, crop_y, w, h;
    uint32_t sqrt_spp, s_begin, s_end;
    uint32_t max_depth;
    uint32_t key0, key1;
    int32_t background, pixel_filter;
    float bg_color[3], bg_color2[3], bg_dir[3];
    float bg_intensity;
    float exposure;
    uint32_t tiles_x, n_tasks;
    float star_density, star_brightness;   // STARFIELD background
    uint32_t ext;            // the scene or background uses the other materials / backgrounds
    uint32_t pad_ext;
};

}  // namespace lum
