/*
 * oracle.h -- TEST INFRASTRUCTURE, not part of the product.
 *
 * CPU f64 restatement of the Luminara per-pixel sample loop, used only by tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg as the checker.  Nothing in
 * luminara_b200/ links or calls it.
 *
 * Parity status: the Rust reference cannot be built on this machine (no cargo/rustc, no
 * vendored crates), so this restatement is pinned against the reference's own unit-test
 * known answers (restated in tests/test_oracle_kat.py), not against reference output.
 * Bitwise image parity with the reference is unpinned: its RNG (rand 0.9.2 SmallRng) is
 * restated from the published xoshiro256++/SplitMix64 definitions, but no reference test
 * pins RNG-stream values.
 */
#ifndef LUMINARA_ORACLE_H
#define LUMINARA_ORACLE_H

#include "../include/luminara_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_scene orc_scene;

enum { ORC_MODE_STREAM = 0, ORC_MODE_KEYED = 1 };

typedef struct orc_stats {
    uint64_t paths;
    uint64_t segments;
    uint64_t shadow_rays;
    double seconds;
    int32_t threads;
    int32_t reserved;
} orc_stats;

/* A ray in double precision: org[3], tmin, dir[3], tmax, time, pad. */
typedef struct orc_ray {
    double org[3];
    double tmin;
    double dir[3];
    double tmax;
    double time;
    double pad;
} orc_ray;

typedef struct orc_hit {
    double t, u, v;
    double point[3];
    double normal[3];
    int32_t prim_id;
    int32_t front_face;
    int32_t material;
    int32_t reserved;
} orc_hit;

int orc_scene_create(const lum_scene_desc* desc, orc_scene** out);
void orc_scene_destroy(orc_scene* s);
/* Closest hit of each ray (SceneWorld::hit).  hits[i].prim_id < 0 on a miss. */
int orc_intersect(const orc_scene* s, const orc_ray* rays, uint32_t n, orc_hit* hits);
/* Number of top-level objects hit within [t(1-rel)-abs_eps, t(1+rel)+abs_eps] around each
 * ray's closest hit t (0 on a miss); > 1 marks a tie such as coplanar coincident faces. */
int orc_tie_count(const orc_scene* s, const orc_ray* rays, uint32_t n, double rel, double abs_eps, int32_t* counts);
/* Shadow query: occluded[i] = world.hit(ray).is_some(). */
int orc_occluded(const orc_scene* s, const orc_ray* rays, uint32_t n, int32_t* occluded);
/* render(): the stratified loop, or the adaptive loop when p->adaptive, and the time limit
 * (p->time_limit, wall clock, checked when a row starts); out_rgb = W*H*3 doubles (exposure
 * applied, not cast to f32); stats->paths counts the samples traced (the reference's rays). */
int orc_render(const orc_scene* s, const lum_render_params* p, int mode, int threads,
               double* out_rgb, orc_stats* stats);
/* As orc_render with every row starting after the time limit: one sample per pixel at the
 * pixel centre (render.rs:1612-1622). */
int orc_render_expired(const orc_scene* s, const lum_render_params* p, int mode, int threads,
                       double* out_rgb, orc_stats* stats);
/* Renders only rows [row_begin, row_end) of the (cropped) image into out_rgb rows of the
 * same index; used for bounded CPU-baseline samples. */
int orc_render_rows(const orc_scene* s, const lum_render_params* p, int mode, int threads,
                    uint32_t row_begin, uint32_t row_end, double* out_rgb, orc_stats* stats);
/* The sample loop's per-pixel sums before the division of render.rs:1705: W*H*4 doubles
 * (filter-weighted clamped R, G, B and the filter weight).  Sums of disjoint stratum ranges add
 * (keyed mode; stream mode needs all strata). */
int orc_render_sums(const orc_scene* s, const lum_render_params* p, int mode, int threads, double* sums,
                    orc_stats* stats);
/* Renders the image rows rows[0..n_rows) (any order, OpenMP over the list) into out_rgb, row k of
 * the output holding image row rows[k]: a bounded sample of a frame spread over its height that
 * still keeps every host thread busy. */
int orc_render_row_list(const orc_scene* s, const lum_render_params* p, int mode, int threads,
                        const uint32_t* rows, uint32_t n_rows, double* out_rgb, orc_stats* stats);

/* Environment map of LUM_BG_ENVMAP: width*height*3 floats, top row first (NULL removes it). */
int orc_scene_set_envmap(orc_scene* s, const float* rgb, uint32_t width, uint32_t height);
/* AOV passes (render.rs:3508-3568): depth (W*H doubles, the f32 value of t), normals and
 * albedo (W*H*3 bytes); any may be NULL. */
int orc_render_aov(const orc_scene* s, const lum_render_params* p, int mode, double* depth, uint8_t* normals,
                   uint8_t* albedo);

/* Known-answer helpers mirroring the reference's unit tests. */
/* Material::scatter of mats[index] (Blend children index the same array); n_iter rows of 11:
 * ok, dir[3], att[3], front_face, origin[3]. */
int orc_scatter_in(const lum_material* mats, uint32_t n_mats, uint32_t index, const double ray[7],
                   const double hit_point[3], const double outward_normal[3], double t, double u, double v,
                   uint64_t seed, int n_iter, double* out);
/* Sum of the three channels of mats[index].emitted(u, v, p). */
double orc_emitted(const lum_material* mats, uint32_t n_mats, uint32_t index, double u, double v, const double p[3]);
int orc_is_specular(const lum_material* m);
/* Iridescent::thin_film_color channel (0 r, 1 g, 2 b). */
double orc_thin_film(double cos_theta, double thickness, double film_ior, int channel);
int orc_scatter(const lum_material* m, const double ray[7], const double hit_point[3],
                const double outward_normal[3], double t, double u, double v, uint64_t seed,
                int n_iter, double* out /* n_iter * 8: ok, dir[3], att[3], front */);
double orc_schlick(double cosine, double ref_idx);
double orc_ggx_d(double n_dot_h, double alpha);
int orc_camera_ray(const lum_camera* c, double s, double t, uint64_t seed, double out[7]);
double orc_filter_weight(int filter, double dx, double dy);
int orc_sample_direct_light(const orc_scene* s, const double p[3], const double n[3],
                            const double albedo[3], uint64_t seed, int n_iter, double* out);
int orc_aabb_hit(const double mn[3], const double mx[3], const double ray[7], double tmin,
                 double tmax);
int orc_scene_bbox(const orc_scene* s, int32_t object_index, double out[6]);
int orc_bvh_stats(const orc_scene* s, uint32_t* n_nodes, uint32_t* depth);
/* Vector helpers (vec3.rs): refract, reflect. */
void orc_refract(const double v[3], const double n[3], double eta, double out[3]);
void orc_reflect(const double v[3], const double n[3], double out[3]);
/* RNG pins: SmallRng stream outputs and Philox4x32-10 blocks. */
void orc_stream_u64(uint64_t seed, uint32_t n, uint64_t* out);
void orc_stream_f64(uint64_t seed, uint32_t n, double* out);
/* f64 adjoint of the keyed estimator for a given dL/d(image) (W*H*3 doubles): gradients with
 * respect to per-material albedo (3/material), roughness (1/material) and emission
 * (3/material).  detach = 1: Russian-roulette survival and microfacet lobe probabilities held
 * constant (the device adjoint's estimator); 0: the plain per-sample derivative.  out_rgb (may
 * be NULL) receives the primal image. */
int orc_adjoint(const orc_scene* s, const lum_render_params* p, const double* dl_dimage,
                const int32_t* light_material, int detach, int threads, double* d_albedo,
                double* d_roughness, double* d_emission, double* out_rgb);
/* Directional form of orc_adjoint: the derivative along `direction` (7 * n_materials doubles,
 * the same parameter layout: albedo 3m+c, roughness 3n+m, emission 4n+3m+c). */
int orc_adjoint_dir(const orc_scene* s, const lum_render_params* p, const double* dl_dimage,
                    const int32_t* light_material, int detach, int threads, const double* direction,
                    double* out);
void orc_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
/* xoshiro256++ outputs from a raw state, and the SplitMix64-expanded state of a u64 seed. */
void orc_xoshiro_from_state(const uint64_t state[4], uint32_t n, uint64_t* out);
void orc_seed_state(uint64_t seed, uint64_t out[4]);

#ifdef __cplusplus
}
#endif
#endif
