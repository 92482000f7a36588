/*
 * luminara_gpu.h -- C ABI of the B200 path-tracing core.
 *
 * This header is the drop-in boundary for the per-pixel sample loop of the Luminara
 * renderer.  Every type here is plain C: fixed-width integers, doubles, floats and
 * pointers.  No CUDA, C++ or Python type crosses the boundary, so the library can be
 * bound from Rust (`extern "C"`), ctypes, cgo or JNI alike.
 *
 * Reference interfaces replaced (paths are relative to the Luminara project root):
 *   render()            src/render.rs:1557-1562   pub fn render(config, camera, world, lights) -> RenderResult
 *   Hittable::hit       src/hit.rs:47-53          closest hit of one ray (here: lum_intersect on a ray set)
 *   SceneWorld          src/scene.rs:774-839      BVH of bounded objects + linear list of planes
 *   BvhNode::build      src/bvh.rs:16-58          (the library builds its own SAH BVH inside lum_scene_create)
 *   LightInfo           src/render.rs:16-39       NEE light records (lum_light)
 *   CameraConfig        src/camera.rs:17-41       (lum_camera)
 *   RenderConfig        src/render.rs:239-431     (lum_render_params: the fields the sample loop reads)
 *   Material / Texture  src/material.rs:15-28, src/texture.rs:4-50   (lum_material)
 *
 * Conventions
 *   - Every entry point returns a lum_status; LUM_OK is 0.  On failure, lum_last_error()
 *     returns a message for the calling thread.
 *   - Host buffers are owned by the caller.  Device buffers created by lum_scene_create
 *     are owned by the scene handle and freed by lum_scene_destroy.  They come from one
 *     stream-ordered memory pool per device, which keeps up to 4 GiB of freed memory for the
 *     next scenes (creating and destroying scenes then does not call the driver's allocator);
 *     other allocators of the process do not see that reserve.
 *   - A scene handle owns one CUDA stream; calls on one handle are serialised on it.
 *     Distinct handles may be used from distinct threads.
 *   - Geometry and material parameters are given in double precision (the reference is
 *     f64 throughout); the device computes in f32.
 *   - Output images are float32 linear RGB, row-major, top row first, W*H*3 values
 *     (src/render.rs:2610-2624 with exposure applied).
 */
#ifndef LUMINARA_GPU_H
#define LUMINARA_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LUM_ABI_VERSION 3

typedef int32_t lum_status;
enum {
    LUM_OK = 0,
    LUM_ERR_INVALID_ARGUMENT = 1, /* null pointer, bad index, bad size */
    LUM_ERR_UNSUPPORTED = 2,      /* a feature outside the GPU path (e.g. a transformed medium) */
    LUM_ERR_CUDA = 3,             /* a CUDA runtime call failed */
    LUM_ERR_OUT_OF_MEMORY = 4,    /* device allocation failed */
    LUM_ERR_NO_DEVICE = 5,        /* no CUDA device visible */
    LUM_ERR_KERNEL = 6,           /* a kernel reported an error flag (stack overflow, wait limit) */
    LUM_ERR_TOO_LARGE = 7         /* request exceeds a fixed capacity */
};

/* ------------------------------------------------------------------------------------
 * Scene description
 * ---------------------------------------------------------------------------------- */

/* Object kinds.  Parameter layout in lum_object.p[] is given per kind.
 * Each kind restates one reference Hittable. */
enum {
    LUM_OBJ_SPHERE = 1,        /* src/sphere.rs:7-68      p[0..2] center, p[3] radius */
    LUM_OBJ_MOVING_SPHERE = 2, /* src/sphere.rs:71-125    p[0..2] center0, p[3..5] center1, p[6] radius */
    LUM_OBJ_QUAD = 3,          /* src/quad.rs:7-72        p[0..2] Q, p[3..5] u, p[6..8] v */
    LUM_OBJ_RECT_XY = 4,       /* src/rect.rs:8-45        p[0] x0, p[1] x1, p[2] y0, p[3] y1, p[4] k (z=k) */
    LUM_OBJ_RECT_XZ = 5,       /* src/rect.rs:48-85       p[0] x0, p[1] x1, p[2] z0, p[3] z1, p[4] k (y=k) */
    LUM_OBJ_RECT_YZ = 6,       /* src/rect.rs:88-125      p[0] y0, p[1] y1, p[2] z0, p[3] z1, p[4] k (x=k) */
    LUM_OBJ_TRIANGLE = 7,      /* src/triangle.rs:7-70    p[0..2] v0, p[3..5] v1, p[6..8] v2 */
    LUM_OBJ_DISK = 8,          /* src/disk.rs:7-65        p[0..2] center, p[3..5] normal, p[6] radius */
    LUM_OBJ_PLANE = 9,         /* src/plane.rs:7-74       p[0..2] point, p[3..5] normal (unbounded) */
    LUM_OBJ_BOX = 10,          /* src/rect.rs:128-141 + src/scene.rs:1561-1600
                                  p[0..2] p_min, p[3..5] p_max: six axis rects.  With a
                                  transform the six rects form one composite object. */
    LUM_OBJ_FOG_SPHERE = 11,   /* src/constant_medium.rs:9-74 over a sphere boundary
                                  p[0..2] center, p[3] radius, p[4] density; material = ISOTROPIC */
    LUM_OBJ_FOG_BOX = 12       /* constant medium over a make_box boundary
                                  p[0..2] p_min, p[3..5] p_max, p[6] density; material = ISOTROPIC */
};

typedef struct lum_object {
    int32_t kind;      /* LUM_OBJ_* */
    int32_t material;  /* index into lum_scene_desc.materials */
    int32_t transform; /* -1, or index into lum_scene_desc.transforms */
    int32_t reserved;
    double p[12];
} lum_object;

/* Transform operations, applied in order (first op innermost), mirroring the wrapper
 * order of src/scene.rs:1573-1592 (scale, rotate_x, rotate_y, rotate_z, translate). */
enum {
    LUM_XF_TRANSLATE = 1, /* src/transform.rs:7-29    arg xyz */
    LUM_XF_ROTATE_X = 2,  /* src/transform.rs:108-179 arg[0] degrees */
    LUM_XF_ROTATE_Y = 3,  /* src/transform.rs:31-106  arg[0] degrees */
    LUM_XF_ROTATE_Z = 4,  /* src/transform.rs:181-256 arg[0] degrees */
    LUM_XF_SCALE = 5      /* src/transform.rs:258-284 arg[0] factor */
};
#define LUM_MAX_XF_OPS 6
typedef struct lum_transform {
    int32_t n_ops;
    int32_t op[LUM_MAX_XF_OPS];
    int32_t reserved;
    double arg[LUM_MAX_XF_OPS][3];
} lum_transform;

/* Triangle mesh: one reference MeshTriangle per triangle (src/obj.rs:250-320). */
typedef struct lum_mesh {
    const double* positions;      /* n_vertices * 3 */
    const double* normals;        /* n_vertices * 3, or NULL for flat normals */
    uint32_t n_vertices;
    uint32_t n_triangles;
    const uint32_t* indices;      /* n_triangles * 3 */
    const int32_t* tri_material;  /* n_triangles material indices, or NULL */
    int32_t material;             /* used when tri_material is NULL */
    int32_t reserved;
} lum_mesh;

enum {
    LUM_MAT_LAMBERTIAN = 1, /* src/material.rs:43-71 */
    LUM_MAT_METAL = 2,      /* src/material.rs:75-107 */
    LUM_MAT_DIELECTRIC = 3, /* src/material.rs:111-214 */
    LUM_MAT_EMISSIVE = 4,   /* src/material.rs:218-244 */
    LUM_MAT_MICROFACET = 5, /* src/material.rs:248-391 */
    LUM_MAT_ISOTROPIC = 6,  /* src/constant_medium.rs:77-89 */
    /* The other reference materials (src/material.rs:396-870).  Parameters beyond color /
     * color2 / ior / roughness are in lum_material.extra[]; the constructors' clamps are
     * applied by lum_scene_create. */
    LUM_MAT_BLEND = 7,       /* :396-421  sub[0] = mat_a, sub[1] = mat_b, extra[0] = ratio
                                (probability of mat_a).  Blends nest at most 4 deep. */
    LUM_MAT_TRANSPARENT = 8, /* :427-440  no parameters */
    LUM_MAT_IRIDESCENT = 9,  /* :447-528  color = base_color, extra[0] = thickness (nm),
                                ior = film_ior, roughness */
    LUM_MAT_TOON = 10,       /* :530-578  color, extra[0] = bands, extra[1] = specular */
    LUM_MAT_ANISOTROPIC = 11,/* :581-642  color, extra[0] = roughness_u, extra[1] = roughness_v,
                                extra[2] = tangent axis (0 x, 1 y, 2 z) */
    LUM_MAT_CLEARCOAT = 12,  /* :645-708  color = base_color, extra[0] = coat_gloss, ior = coat_ior */
    LUM_MAT_VELVET = 13,     /* :711-747  color, extra[0] = sheen */
    LUM_MAT_TRANSLUCENT = 14,/* :750-798  color, extra[0] = translucency, extra[1] = scatter_width */
    LUM_MAT_SUBSURFACE = 15  /* :801-865  color, extra[0] = mean_free_path, color2 = scatter_color */
};
enum {
    LUM_TEX_SOLID = 0,  /* src/texture.rs:9-23 */
    LUM_TEX_CHECKER = 1 /* src/texture.rs:26-50 */
};
typedef struct lum_material {
    int32_t kind;       /* LUM_MAT_* */
    int32_t texture;    /* LUM_TEX_* (albedo texture of Lambertian/Microfacet, colour of Emissive) */
    double color[3];    /* albedo, emission colour, or checker "even" colour */
    double color2[3];   /* checker "odd" colour */
    double tex_scale;   /* checker scale */
    double fuzz;        /* Metal (clamped to <= 1 as Metal::new does) */
    double ior;         /* Dielectric refraction index */
    double roughness;   /* Dielectric frost / Microfacet roughness (clamped to [0.01,1]) */
    double metallic;    /* Microfacet (clamped to [0,1]) */
    double intensity;   /* Emissive */
    double dispersion;  /* Dielectric */
    double tint[3];     /* Dielectric Beer tint; (1,1,1) = clear */
    int32_t sub[2];     /* Blend: the two blended materials */
    double extra[4];    /* per-kind parameters (LUM_MAT_* above) */
} lum_material;

enum {
    LUM_LIGHT_SPHERE = 1, /* p0 center, radius */
    LUM_LIGHT_RECT = 2,   /* p0 origin, u, v, normal */
    LUM_LIGHT_DISK = 3    /* p0 center, normal, radius */
};
/* One NEE light (src/render.rs:16-39).  The list is given explicitly: the reference's
 * scene loader harvests it from emissive objects (src/scene.rs:1180-1200, 1329-1344,
 * 1388-1412, 1503-1532, 1607-1619). */
typedef struct lum_light {
    int32_t kind;
    int32_t reserved;
    double p0[3];
    double u[3];
    double v[3];
    double normal[3];
    double radius;
    double emission[3];
} lum_light;

typedef struct lum_camera {
    double look_from[3];
    double look_at[3];
    double vup[3];
    double vfov_degrees;
    double aspect_ratio;
    double aperture;
    double focus_dist;
    int32_t panorama;   /* 1: equirectangular 360-degree camera (camera.rs:83-90): longitude
                           2 pi s - pi, latitude pi (1 - t) about forward = look_at - look_from,
                           right and up of the camera basis; unit directions, no lens */
    int32_t reserved;
} lum_camera;

typedef struct lum_scene_desc {
    const lum_object* objects;
    uint32_t n_objects;
    uint32_t n_meshes;
    const lum_mesh* meshes;
    const lum_material* materials;
    uint32_t n_materials;
    uint32_t n_transforms;
    const lum_transform* transforms;
    const lum_light* lights;
    uint32_t n_lights;
    uint32_t reserved;
    lum_camera camera;
} lum_scene_desc;

/* ------------------------------------------------------------------------------------
 * Render parameters (the RenderConfig fields the sample loop reads)
 * ---------------------------------------------------------------------------------- */
enum {
    LUM_BG_SKY = 0,      /* src/render.rs:75-79 */
    LUM_BG_SOLID = 1,    /* src/render.rs:80 */
    LUM_BG_GRADIENT = 2, /* src/render.rs:81-85 */
    LUM_BG_SUN = 3,      /* src/render.rs:152-169 */
    LUM_BG_STARFIELD = 4,/* src/render.rs:86-112: bg_star_density, bg_star_brightness */
    LUM_BG_ENVMAP = 5    /* src/render.rs:113-151: the scene's environment map
                            (lum_scene_set_envmap) times bg_intensity */
};
enum {
    LUM_FILTER_BOX = 0, /* src/render.rs:201-237 */
    LUM_FILTER_TRIANGLE = 1,
    LUM_FILTER_GAUSSIAN = 2,
    LUM_FILTER_MITCHELL = 3
};
typedef struct lum_render_params {
    uint32_t width;
    uint32_t height;
    uint32_t samples_per_pixel; /* rounded up to a square as src/render.rs:1589-1590 */
    uint32_t max_depth;
    uint64_t seed;
    int32_t background;         /* LUM_BG_* */
    int32_t pixel_filter;       /* LUM_FILTER_* */
    double bg_color[3];         /* SOLID colour, GRADIENT bottom, SUN sun colour */
    double bg_color2[3];        /* GRADIENT top, SUN sky colour */
    double bg_dir[3];           /* SUN direction */
    double bg_intensity;        /* SUN intensity */
    double exposure;            /* multiplies the f32 output (src/render.rs:2616-2618) */
    int32_t has_crop;
    uint32_t crop[4];           /* x, y, w, h  (src/render.rs:1575-1583) */
    uint32_t sample_begin;      /* first stratum index rendered (0 for a full render) */
    uint32_t sample_count;      /* strata rendered; 0 = all sqrt_spp^2 strata */
    int32_t adaptive;           /* 1 = adaptive sampling (src/render.rs:1592, 1628-1676): strata in
                                   order, a pixel stops once n >= max(spp/4, 16) and the standard
                                   error of its clamped luminance is below adaptive_threshold; the
                                   pixel is the plain mean (no pixel filter).  Needs all strata. */
    double adaptive_threshold;  /* the reference's default is 0.03 (src/render.rs:456) */
    double time_limit;          /* seconds; > 0: a tile that starts after the limit renders one
                                   sample per pixel at the pixel centre (src/render.rs:1601-1623,
                                   per row there); 0 = none */
    double bg_star_density;     /* STARFIELD */
    double bg_star_brightness;  /* STARFIELD */
} lum_render_params;

typedef struct lum_stats {
    uint64_t paths;        /* camera samples traced: the reference's "rays" count (src/main.rs:702) */
    uint64_t segments;     /* closest-hit rays traced */
    uint64_t shadow_rays;  /* NEE any-hit rays traced */
    double kernel_ms;      /* device time of the render kernel(s) */
    double total_ms;       /* host wall time of the call */
    uint32_t error_flags;  /* kernel-reported error bits (LUM_KERR_*) */
    uint32_t reserved;
} lum_stats;

enum {
    LUM_KERR_STACK_OVERFLOW = 1u << 0, /* traversal stack overflowed (ray treated as miss) */
    LUM_KERR_QUEUE_OVERFLOW = 1u << 1, /* wavefront queue overflow */
    LUM_KERR_ITERATION_CAP = 1u << 2   /* persistent loop hit its iteration cap */
};

/* One ray of a ray set; time is the motion-blur time (src/ray.rs). */
typedef struct lum_ray {
    float org[3];
    float tmin;
    float dir[3];
    float tmax;
    float time;
    float pad[3];
} lum_ray;

/* Closest-hit record (src/hit.rs:7-44).  prim_id < 0 means miss.  Primitive ids count
 * the expanded primitives in description order: one per object (six per LUM_OBJ_BOX,
 * in make_box order), then every mesh triangle in mesh order. */
typedef struct lum_hit {
    float t;
    float u;
    float v;
    float normal[3];   /* faces the ray */
    int32_t prim_id;
    int32_t front_face;
    int32_t material;
    int32_t reserved;
} lum_hit;

/* Test counts of one render from the counter build of the render kernel (same seeds, same
 * paths); used to turn kernel time into achieved flops/bytes of the counted tests. */
typedef struct lum_test_counts {
    uint64_t node_visits;     /* BVH node visits; each visit slab-tests two child boxes */
    uint64_t sphere_tests;
    uint64_t quad_tests;
    uint64_t triangle_tests;
    uint64_t disk_tests;
    uint64_t fog_tests;
    uint64_t plane_tests;
    uint64_t segments;
    uint64_t shadow_rays;
    uint64_t paths;
} lum_test_counts;

typedef struct lum_scene lum_scene; /* opaque */

/* ------------------------------------------------------------------------------------
 * Entry points
 * ---------------------------------------------------------------------------------- */

/* ABI version (LUM_ABI_VERSION). */
int32_t lum_abi_version(void);

/* Message of the last failed call on this thread ("" if none). */
const char* lum_last_error(void);

/* Replaces scene::load_scene's world construction + SceneWorld::from_list
 * (src/scene.rs:846-1645, 786-808): flattens transforms, builds the BVH on the host and
 * uploads structure-of-arrays device buffers.  An empty scene is valid (every ray misses).
 * Returns LUM_ERR_INVALID_ARGUMENT, naming the object, for a parameter that is not finite in
 * f32 (objects, mesh vertices and normals, transforms, materials, lights, camera), for a
 * degenerate quad or rect (u x v = 0) or disk (radius 0), and for a negative medium density;
 * no ray hits such a quad or disk in the reference, whose loader reads only finite numbers.
 * Zero-area sides of a box (a box flat along one axis) are left out, keeping their ids. */
lum_status lum_scene_create(const lum_scene_desc* desc, lum_scene** out_scene);

/* Frees the scene's device buffers (back to the device's pool) and stream.  Synchronises the
 * device first, as cudaFree would, so work that other streams still run on the scene
 * finishes before its memory is reused. */
lum_status lum_scene_destroy(lum_scene* scene);

/* Number of expanded primitives and BVH nodes (diagnostics). */
lum_status lum_scene_info(const lum_scene* scene, uint32_t* n_prims, uint32_t* n_nodes,
                          uint32_t* n_lights, uint64_t* device_bytes);

/* Replaces render::render (src/render.rs:1557-1731): renders into a caller-owned HOST
 * buffer of width*height*3 floats (crop size when has_crop).  Device output buffers are
 * owned by the scene.  The image is read back through pinned staging buffers shared per
 * device (4 MB chunks, copied into out_rgb by up to 8 host threads); a call that finds them
 * in use by another thread copies directly.  stats may be NULL. */
lum_status lum_render(lum_scene* scene, const lum_render_params* params, float* out_rgb,
                      lum_stats* stats);

/* Same as lum_render but writes a caller-owned DEVICE buffer on the caller's CUDA stream
 * (cudaStream_t passed as void*, NULL = the scene's stream); no host copies.  With stats, the
 * call waits for the render and reports the kernel's error flags; with stats NULL it only
 * enqueues the work and returns (back-to-back frames keep the GPU busy whatever the host is
 * doing; kernel error flags are then not reported).  Asynchronous calls on one scene must use
 * one stream: they share the scene's work counters. */
lum_status lum_render_device(lum_scene* scene, const lum_render_params* params,
                             float* d_out_rgb, void* stream, lum_stats* stats);

/* The render's raw per-pixel sums, before the division of render.rs:1705, into a caller-owned
 * DEVICE buffer of width*height*4 int64 values (crop size when has_crop) on `stream` (NULL =
 * the scene's stream): for each pixel the sums over its rendered strata of the filter-weighted,
 * luminance-clamped radiance (R, G, B) and of the filter weight (render.rs:1692-1704), in fixed
 * point with 2^-32 units, each path's value rounded once.  Sums of disjoint stratum ranges
 * (sample_begin / sample_count) add exactly, so a frame split across devices or calls combines
 * with one integer sum (an all-reduce) and lum_sums_finalize_device then gives the
 * single-device lum_render image bit for bit, for every pixel filter.  Adaptive sampling and
 * the time limit return LUM_ERR_UNSUPPORTED.  With stats the call waits and reports error flags;
 * with stats NULL it only enqueues. */
lum_status lum_render_sums_device(lum_scene* scene, const lum_render_params* params, int64_t* d_sums,
                                  void* stream, lum_stats* stats);

/* Pixels of raw sums (lum_render_sums_device, possibly summed over several calls): for each of
 * width*height pixels, rgb = (sum_rgb / sum_w) * exposure (sum_rgb itself where sum_w is 0), as
 * float32 linear RGB into a DEVICE buffer, on `stream` (NULL = the default stream).  Allocates
 * nothing; does not synchronise. */
lum_status lum_sums_finalize_device(const int64_t* d_sums, uint32_t width, uint32_t height, double exposure,
                                    float* d_rgb, void* stream);

/* Environment map of LUM_BG_ENVMAP (Background::EnvMap, src/render.rs:113-151): an
 * equirectangular linear RGB image, width*height*3 floats, top row first, copied to the
 * scene's device memory (replacing any previous map; rgb NULL removes it). */
lum_status lum_scene_set_envmap(lum_scene* scene, const float* rgb, uint32_t width, uint32_t height);

/* AOV passes (src/render.rs:3508-3568): one ray per pixel through the pixel centre, its
 * closest hit: depth = t (0 on a miss), W*H floats; normals = the hit normal facing the ray
 * mapped to bytes ((n * 0.5 + 0.5) * 255, clamped, truncated), W*H*3; albedo = the scatter
 * attenuation clamped to [0,1] * 255, or for a surface that does not scatter its emission
 * divided by max(max component, 1), W*H*3.  Any output may be NULL.  Caller-owned HOST
 * buffers (crop size when has_crop).  The lens and scatter draws come from the keyed RNG of
 * (pixel, stratum 0), not the reference's per-pixel stream. */
lum_status lum_render_aov(lum_scene* scene, const lum_render_params* params, float* depth,
                          uint8_t* normals, uint8_t* albedo);

/* Allocation-free render.  Same image as lum_render into the same caller-owned HOST buffer,
 * but it allocates no device memory, ever: the device image and the kernel's work counters
 * live in one fixed array of LUM_NOALLOC_MAX_PIXELS * 12 + 256 bytes (12 MiB), part of the
 * render kernels' module, which each device holds from the moment that module is loaded there
 * until the process exits.  It is for callers that cannot call cudaMalloc at render time --
 * services that reserve all device memory at start-up, or whose free memory is held by another
 * allocator's pool, where a render-time cudaMalloc would fail or stall on device-wide
 * synchronisation.  lum_render, by contrast, allocates its device image on first use and
 * whenever the image grows.
 *   - Images of more than LUM_NOALLOC_MAX_PIXELS pixels (after crop) are rejected with
 *     LUM_ERR_TOO_LARGE.
 *   - lum_scene_create loads the render kernels' module on its device and looks up the array's
 *     device address (cudaGetSymbolAddress) there, so a scene created before the caller
 *     reserves device memory is all the set-up a device needs.  (Under CUDA's lazy module
 *     loading the module would otherwise load -- and need 12 MiB -- at the first render.)  If
 *     that look-up failed, the first lum_render_noalloc call on the device repeats it; make
 *     that call before any stream capture.
 *   - The address is cached per device for the life of the process: after cudaDeviceReset
 *     (or anything else that destroys the device's primary context) do not call this entry
 *     point again in the same process.
 *   - All calls share the one array: calls that overlap on the GPU (e.g. from several host
 *     threads at once, on different scenes) race on it.  Calls on one scene handle are
 *     serialised like lum_render's.  Each call clears the counters it needs and overwrites the
 *     image region it returns.
 *   - Adaptive sampling and the time limit (params->adaptive, params->time_limit) are not
 *     available here: they return LUM_ERR_UNSUPPORTED.
 *   - stats->kernel_ms is 0 (no events are created); total_ms is the host wall time.
 * No counterpart in the reference. */
#define LUM_NOALLOC_MAX_PIXELS (1u << 20)
lum_status lum_render_noalloc(lum_scene* scene, const lum_render_params* params, float* out_rgb,
                              lum_stats* stats);

/* Diagnostics: runs the counter build of the render kernel for `params` (output discarded)
 * and returns its test counts.  No counterpart in the reference, which counts only paths
 * (src/render.rs:1704). */
lum_status lum_count_tests(lum_scene* scene, const lum_render_params* params, lum_test_counts* counts);

/* Replaces SceneWorld::hit (src/scene.rs:816-834) for a set of rays: closest hit of each
 * ray in [tmin, tmax].  rays/hits are HOST arrays of n entries. */
lum_status lum_intersect(lum_scene* scene, const lum_ray* rays, uint32_t n, lum_hit* hits);

/* Any-hit (shadow) query, src/render.rs:1457-1460: occluded[i] = 1 if world.hit(ray) is
 * Some.  HOST arrays. */
lum_status lum_occluded(lum_scene* scene, const lum_ray* rays, uint32_t n, int32_t* occluded);

/* ------------------------------------------------------------------------------------
 * Differentiable rendering: a forward/backward pair.  No counterpart in the reference (it
 * renders only); the estimator differentiated is the reference's (render.rs:1472-1537).
 * ---------------------------------------------------------------------------------- */

/* The forward render (same as lum_render). */
lum_status lum_forward(lum_scene* scene, const lum_render_params* params, float* out_rgb, lum_stats* stats);

/* Path-replay adjoint: given dL/d(image) (HOST, W*H*3 floats, the layout lum_forward
 * returns), writes dL/d(albedo) (3 per material: Lambertian/Metal/Microfacet colour),
 * dL/d(roughness) (1 per material: Microfacet) and dL/d(emission) (3 per material: the
 * Emissive colour * intensity) into HOST arrays sized by the scene's material count.
 * light_material[k] names the material whose emission light k carries (NEE), or -1; NULL =
 * none.  Each path is re-traced from its RNG key (no path storage).  Russian-roulette and
 * microfacet-lobe probabilities are held constant in the weights they divide, and the NEE term
 * (which the reference adds only on surviving paths, undivided by the survival probability)
 * carries a survival score term, so the gradient is an unbiased estimate of the derivative of
 * the expected image; visibility changes are not differentiated.  max_depth <= 16.  Pixels
 * whose dL/d(image) is zero are not replayed.  The call stages one chunk of replayed paths at
 * a time in device memory (at most 8 GiB or a quarter of the free memory, 48 + 64 * max_depth
 * bytes per path). */
lum_status lum_backward(lum_scene* scene, const lum_render_params* params, const float* dL_dimage,
                        const int32_t* light_material, float* d_albedo, float* d_roughness, float* d_emission,
                        lum_stats* stats);

/* ------------------------------------------------------------------------------------
 * Batched wavefront rendering: many scenes per launch sequence.
 *
 * The reference renders one scene per render() call (src/render.rs:1557); a batch is the
 * same as n independent render() calls (one lum_render_params per scene), traced together by
 * a persistent wavefront tracer with material-sorted queues under a captured CUDA graph.
 * Images equal lum_render's up to float rounding of the per-pixel sum (the batch sums in 64-bit
 * fixed point, independent of completion order).
 * ---------------------------------------------------------------------------------- */
enum {
    LUM_BATCH_WAVEFRONT = 0,  /* path pool, material-sorted queues, graph-captured iterations */
    LUM_BATCH_MEGAKERNEL = 1, /* one persistent megakernel whose tile queue spans all scenes */
    LUM_BATCH_STREAMS = 2     /* lum_render's megakernel once per scene, heaviest first, over 4
                                 streams: a scene's tail overlaps the next scene's start */
};
typedef struct lum_batch_config {
    uint32_t pool_paths;      /* wavefront: path slots in flight (1024 .. 2^24) */
    uint32_t block_threads;   /* wavefront: 128 or 256 */
    uint32_t sort_threshold;  /* wavefront: extend queues shorter than this shade in one generic kernel */
    uint32_t iters_per_graph; /* wavefront: iterations captured per CUDA graph launch (1 .. 64) */
    uint32_t mode;            /* LUM_BATCH_* */
    uint32_t reserved[3];
} lum_batch_config;

typedef struct lum_batch_stats {
    uint64_t paths;
    uint64_t segments;
    uint64_t shadow_rays;
    double device_ms;         /* CUDA-event time from the first kernel to the last */
    double total_ms;          /* host wall time of the call */
    uint32_t graph_launches;
    uint32_t iterations;
    uint32_t error_flags;     /* LUM_KERR_* */
    uint32_t reserved;
} lum_batch_stats;

typedef struct lum_batch lum_batch; /* opaque; references its scenes, which must outlive it */

lum_status lum_batch_default_config(lum_batch_config* cfg);
/* Times candidate configurations (mode; pool size, block size, sort threshold) on calibration
 * runs of the batch -- all of them on 1/8 of each scene's strata, the three fastest again on
 * 1/4 -- and returns the fastest of the second round (best_ms is its time); results are
 * cached per device and batch signature in $LUM_AUTOTUNE_CACHE (default
 * ~/.cache/luminara_b200_autotune.txt).  best_ms may be NULL; it is -1 on a cache hit. */
lum_status lum_batch_autotune(lum_scene* const* scenes, const lum_render_params* params, uint32_t n,
                              lum_batch_config* out, double* best_ms);
/* cfg NULL = autotuned.  Allocates the path pool, queues and accumulators and captures the
 * iteration graph. */
lum_status lum_batch_create(lum_scene* const* scenes, const lum_render_params* params, uint32_t n,
                            const lum_batch_config* cfg, lum_batch** out);
lum_status lum_batch_config_of(const lum_batch* batch, lum_batch_config* cfg);
/* Renders every scene into caller-owned HOST buffers outs[s] (W*H*3 floats each).
 * scene_done_ms (n entries, may be NULL) receives each scene's completion time from the start
 * of the batch. */
lum_status lum_batch_render(lum_batch* batch, float* const* outs, double* scene_done_ms, lum_batch_stats* stats);
/* Same into caller-owned DEVICE buffers. */
lum_status lum_batch_render_device(lum_batch* batch, float* const* d_outs, double* scene_done_ms,
                                   lum_batch_stats* stats);
lum_status lum_batch_destroy(lum_batch* batch);

/* ------------------------------------------------------------------------------------
 * LDR output: exposure, tone curve and sRGB on the GPU.
 *
 * Replaces the per-pixel colour pipeline of render::render (src/render.rs:2594-2625 for the
 * exposure and auto-exposure, 3100-3260 for the per-pixel chain, 3608-3658 for the tone
 * curves and gamma_correct): for each pixel of a linear HDR image, in this order,
 *   exposure (times 0.18 / log-average luminance when auto_exposure), vignette, white
 *   balance, hue shift, saturation, shadow/highlight grading, tone curve per channel,
 *   ordered dither, sRGB (gamma <= 0) or 1/gamma power to 8 bits, brightness, contrast,
 *   sepia, tint, colour balance, posterize;
 * output RGBA8 (alpha 255), rows top first.  Stylisation passes and spatial filters of the
 * reference (bloom, denoise, blur, edge effects, ...) are not part of this chain.
 * ---------------------------------------------------------------------------------- */
enum {
    LUM_TONEMAP_ACES = 0,      /* src/render.rs:3608-3617 (the reference's default) */
    LUM_TONEMAP_REINHARD = 1,  /* src/render.rs:3619-3622 */
    LUM_TONEMAP_FILMIC = 2,    /* src/render.rs:3626-3641 (Hable / Uncharted 2) */
    LUM_TONEMAP_NONE = 3       /* clamp to [0, 1] */
};

typedef struct lum_tonemap_params {  /* the RenderConfig fields of the pixel chain */
    int32_t tone_map;           /* LUM_TONEMAP_* */
    int32_t auto_exposure;      /* 0/1 */
    double exposure;            /* lum_tonemap_device only; lum_render_ldr uses the render's */
    double gamma;               /* <= 0: sRGB transfer function */
    int32_t dither;             /* 0/1: 4x4 Bayer dither before quantisation */
    int32_t posterize;          /* < 2: off */
    double vignette;            /* <= 0: off */
    double saturation;          /* 1: off */
    double white_balance;       /* 0: off */
    double hue_shift;           /* degrees, 0: off */
    double grade_shadows[3];    /* (1,1,1): off */
    double grade_highlights[3];
    double brightness;          /* 0: off */
    double contrast;            /* 1: off */
    double sepia;               /* <= 0: off */
    double tint[3];             /* (1,1,1): off */
    double color_balance[3];    /* (1,1,1): off */
    double reserved[4];
} lum_tonemap_params;

/* The reference's RenderConfig defaults for the chain (ACES, sRGB, everything else off). */
void lum_tonemap_default(lum_tonemap_params* out);

/* Device scratch that lum_tonemap_device needs when auto_exposure is set. */
#define LUM_TONEMAP_SCRATCH_BYTES 4096

/* Tone-maps a DEVICE linear image (width*height*3 floats, exposure not yet applied) into a
 * DEVICE RGBA8 buffer (width*height*4 bytes) on `stream` (cudaStream_t as void*, NULL = the
 * default stream).  d_scratch: LUM_TONEMAP_SCRATCH_BYTES of device memory, used only with
 * auto_exposure (may be NULL otherwise; 8-byte aligned).  d_hdr_rgb must be 4-byte aligned,
 * d_rgba may have any alignment (16-byte aligned buffers take the vectorised path).
 * Allocates nothing; does not synchronise, except that the first call on a device for a given
 * (tone_map, gamma) pair without optional steps computes that chain's byte-threshold table on
 * the host (a few milliseconds) and copies it synchronously into a fixed device table (16
 * pairs per device); make that first call outside stream capture. */
lum_status lum_tonemap_device(const float* d_hdr_rgb, uint32_t width, uint32_t height,
                              const lum_tonemap_params* tm, void* d_scratch, uint8_t* d_rgba,
                              void* stream);

/* Renders and tone-maps in one call: the HDR image stays in device memory (rendered at
 * exposure 1; the render's params->exposure is the chain's exposure, tm->exposure is ignored)
 * and only the RGBA8 image (width*height*4 bytes, crop size when has_crop) is copied to the
 * caller-owned HOST buffer.  Replaces render::render's LDR output path. */
lum_status lum_render_ldr(lum_scene* scene, const lum_render_params* params, const lum_tonemap_params* tm,
                          uint8_t* out_rgba, lum_stats* stats);

/* ------------------------------------------------------------------------------------
 * Diagnostics
 * ---------------------------------------------------------------------------------- */

/* L1 load throughput of the current device in GB/s, the roof of the megakernel's node and
 * primitive fetches (which L1 and L2 serve; DRAM sees almost none of them): 128-bit loads from
 * a 32 KiB table by every SM at full occupancy, independent loads only.  pattern 0: coalesced
 * (512 contiguous bytes per warp load); pattern 1: each lane one 64-byte record at a hashed
 * index, as a BVH node visit reads.  Allocates and frees its own small buffers and
 * synchronises the device.  No counterpart in the reference. */
lum_status lum_diag_l1_throughput(int32_t pattern, double* gbs);

#ifdef __cplusplus
}
#endif

#endif /* LUMINARA_GPU_H */
