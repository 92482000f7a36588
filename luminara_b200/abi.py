"""ctypes mirror of include/luminara_gpu.h.

The C header is the boundary; this module only restates its structs so Python callers
(tests, bench, examples) can fill a scene description and call the shared library.
Field order and types must stay identical to the header; ``tests/test_abi.py`` checks the
sizes against the compiled library.
"""
from __future__ import annotations

import ctypes as C

LUM_ABI_VERSION = 3

# status codes
LUM_OK = 0
LUM_ERR_INVALID_ARGUMENT = 1
LUM_ERR_UNSUPPORTED = 2
LUM_ERR_CUDA = 3
LUM_ERR_OUT_OF_MEMORY = 4
LUM_ERR_NO_DEVICE = 5
LUM_ERR_KERNEL = 6
LUM_ERR_TOO_LARGE = 7

# object kinds
OBJ_SPHERE = 1
OBJ_MOVING_SPHERE = 2
OBJ_QUAD = 3
OBJ_RECT_XY = 4
OBJ_RECT_XZ = 5
OBJ_RECT_YZ = 6
OBJ_TRIANGLE = 7
OBJ_DISK = 8
OBJ_PLANE = 9
OBJ_BOX = 10
OBJ_FOG_SPHERE = 11
OBJ_FOG_BOX = 12

XF_TRANSLATE = 1
XF_ROTATE_X = 2
XF_ROTATE_Y = 3
XF_ROTATE_Z = 4
XF_SCALE = 5
MAX_XF_OPS = 6

MAT_LAMBERTIAN = 1
MAT_METAL = 2
MAT_DIELECTRIC = 3
MAT_EMISSIVE = 4
MAT_MICROFACET = 5
MAT_ISOTROPIC = 6
MAT_BLEND = 7
MAT_TRANSPARENT = 8
MAT_IRIDESCENT = 9
MAT_TOON = 10
MAT_ANISOTROPIC = 11
MAT_CLEARCOAT = 12
MAT_VELVET = 13
MAT_TRANSLUCENT = 14
MAT_SUBSURFACE = 15

TEX_SOLID = 0
TEX_CHECKER = 1

LIGHT_SPHERE = 1
LIGHT_RECT = 2
LIGHT_DISK = 3

BG_SKY = 0
BG_SOLID = 1
BG_GRADIENT = 2
BG_SUN = 3
BG_STARFIELD = 4
BG_ENVMAP = 5

FILTER_BOX = 0
FILTER_TRIANGLE = 1
FILTER_GAUSSIAN = 2
FILTER_MITCHELL = 3

BATCH_WAVEFRONT = 0
BATCH_MEGAKERNEL = 1
BATCH_STREAMS = 2

KERR_STACK_OVERFLOW = 1 << 0
KERR_QUEUE_OVERFLOW = 1 << 1
KERR_ITERATION_CAP = 1 << 2

D3 = C.c_double * 3


class LumObject(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("material", C.c_int32),
        ("transform", C.c_int32),
        ("reserved", C.c_int32),
        ("p", C.c_double * 12),
    ]


class LumTransform(C.Structure):
    _fields_ = [
        ("n_ops", C.c_int32),
        ("op", C.c_int32 * MAX_XF_OPS),
        ("reserved", C.c_int32),
        ("arg", (C.c_double * 3) * MAX_XF_OPS),
    ]


class LumMesh(C.Structure):
    _fields_ = [
        ("positions", C.POINTER(C.c_double)),
        ("normals", C.POINTER(C.c_double)),
        ("n_vertices", C.c_uint32),
        ("n_triangles", C.c_uint32),
        ("indices", C.POINTER(C.c_uint32)),
        ("tri_material", C.POINTER(C.c_int32)),
        ("material", C.c_int32),
        ("reserved", C.c_int32),
    ]


class LumMaterial(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("texture", C.c_int32),
        ("color", D3),
        ("color2", D3),
        ("tex_scale", C.c_double),
        ("fuzz", C.c_double),
        ("ior", C.c_double),
        ("roughness", C.c_double),
        ("metallic", C.c_double),
        ("intensity", C.c_double),
        ("dispersion", C.c_double),
        ("tint", D3),
        ("sub", C.c_int32 * 2),
        ("extra", C.c_double * 4),
    ]


class LumLight(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("reserved", C.c_int32),
        ("p0", D3),
        ("u", D3),
        ("v", D3),
        ("normal", D3),
        ("radius", C.c_double),
        ("emission", D3),
    ]


class LumCamera(C.Structure):
    _fields_ = [
        ("look_from", D3),
        ("look_at", D3),
        ("vup", D3),
        ("vfov_degrees", C.c_double),
        ("aspect_ratio", C.c_double),
        ("aperture", C.c_double),
        ("focus_dist", C.c_double),
        ("panorama", C.c_int32),
        ("reserved", C.c_int32),
    ]


class LumSceneDesc(C.Structure):
    _fields_ = [
        ("objects", C.POINTER(LumObject)),
        ("n_objects", C.c_uint32),
        ("n_meshes", C.c_uint32),
        ("meshes", C.POINTER(LumMesh)),
        ("materials", C.POINTER(LumMaterial)),
        ("n_materials", C.c_uint32),
        ("n_transforms", C.c_uint32),
        ("transforms", C.POINTER(LumTransform)),
        ("lights", C.POINTER(LumLight)),
        ("n_lights", C.c_uint32),
        ("reserved", C.c_uint32),
        ("camera", LumCamera),
    ]


class LumRenderParams(C.Structure):
    _fields_ = [
        ("width", C.c_uint32),
        ("height", C.c_uint32),
        ("samples_per_pixel", C.c_uint32),
        ("max_depth", C.c_uint32),
        ("seed", C.c_uint64),
        ("background", C.c_int32),
        ("pixel_filter", C.c_int32),
        ("bg_color", D3),
        ("bg_color2", D3),
        ("bg_dir", D3),
        ("bg_intensity", C.c_double),
        ("exposure", C.c_double),
        ("has_crop", C.c_int32),
        ("crop", C.c_uint32 * 4),
        ("sample_begin", C.c_uint32),
        ("sample_count", C.c_uint32),
        ("adaptive", C.c_int32),
        ("adaptive_threshold", C.c_double),
        ("time_limit", C.c_double),
        ("bg_star_density", C.c_double),
        ("bg_star_brightness", C.c_double),
    ]


class LumStats(C.Structure):
    _fields_ = [
        ("paths", C.c_uint64),
        ("segments", C.c_uint64),
        ("shadow_rays", C.c_uint64),
        ("kernel_ms", C.c_double),
        ("total_ms", C.c_double),
        ("error_flags", C.c_uint32),
        ("reserved", C.c_uint32),
    ]


class LumRay(C.Structure):
    _fields_ = [
        ("org", C.c_float * 3),
        ("tmin", C.c_float),
        ("dir", C.c_float * 3),
        ("tmax", C.c_float),
        ("time", C.c_float),
        ("pad", C.c_float * 3),
    ]


class LumHit(C.Structure):
    _fields_ = [
        ("t", C.c_float),
        ("u", C.c_float),
        ("v", C.c_float),
        ("normal", C.c_float * 3),
        ("prim_id", C.c_int32),
        ("front_face", C.c_int32),
        ("material", C.c_int32),
        ("reserved", C.c_int32),
    ]


class LumTestCounts(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in ("node_visits", "sphere_tests", "quad_tests", "triangle_tests",
                                          "disk_tests", "fog_tests", "plane_tests", "segments", "shadow_rays",
                                          "paths")]


class LumBatchConfig(C.Structure):
    _fields_ = [
        ("pool_paths", C.c_uint32),
        ("block_threads", C.c_uint32),
        ("sort_threshold", C.c_uint32),
        ("iters_per_graph", C.c_uint32),
        ("mode", C.c_uint32),
        ("reserved", C.c_uint32 * 3),
    ]


class LumBatchStats(C.Structure):
    _fields_ = [
        ("paths", C.c_uint64),
        ("segments", C.c_uint64),
        ("shadow_rays", C.c_uint64),
        ("device_ms", C.c_double),
        ("total_ms", C.c_double),
        ("graph_launches", C.c_uint32),
        ("iterations", C.c_uint32),
        ("error_flags", C.c_uint32),
        ("reserved", C.c_uint32),
    ]


# numpy dtypes of the ray/hit records (for bulk arrays)
def ray_dtype():
    import numpy as np

    return np.dtype(
        [("org", "<f4", 3), ("tmin", "<f4"), ("dir", "<f4", 3), ("tmax", "<f4"), ("time", "<f4"), ("pad", "<f4", 3)]
    )


def hit_dtype():
    import numpy as np

    return np.dtype(
        [
            ("t", "<f4"),
            ("u", "<f4"),
            ("v", "<f4"),
            ("normal", "<f4", 3),
            ("prim_id", "<i4"),
            ("front_face", "<i4"),
            ("material", "<i4"),
            ("reserved", "<i4"),
        ]
    )


TONEMAP_ACES = 0
TONEMAP_REINHARD = 1
TONEMAP_FILMIC = 2
TONEMAP_NONE = 3
TONEMAP_SCRATCH_BYTES = 4096


class LumTonemapParams(C.Structure):
    _fields_ = [
        ("tone_map", C.c_int32),
        ("auto_exposure", C.c_int32),
        ("exposure", C.c_double),
        ("gamma", C.c_double),
        ("dither", C.c_int32),
        ("posterize", C.c_int32),
        ("vignette", C.c_double),
        ("saturation", C.c_double),
        ("white_balance", C.c_double),
        ("hue_shift", C.c_double),
        ("grade_shadows", C.c_double * 3),
        ("grade_highlights", C.c_double * 3),
        ("brightness", C.c_double),
        ("contrast", C.c_double),
        ("sepia", C.c_double),
        ("tint", C.c_double * 3),
        ("color_balance", C.c_double * 3),
        ("reserved", C.c_double * 4),
    ]


STRUCT_SIZES = {
    "lum_object": C.sizeof(LumObject),
    "lum_transform": C.sizeof(LumTransform),
    "lum_mesh": C.sizeof(LumMesh),
    "lum_material": C.sizeof(LumMaterial),
    "lum_light": C.sizeof(LumLight),
    "lum_camera": C.sizeof(LumCamera),
    "lum_scene_desc": C.sizeof(LumSceneDesc),
    "lum_render_params": C.sizeof(LumRenderParams),
    "lum_stats": C.sizeof(LumStats),
    "lum_ray": C.sizeof(LumRay),
    "lum_hit": C.sizeof(LumHit),
    "lum_test_counts": C.sizeof(LumTestCounts),
    "lum_batch_config": C.sizeof(LumBatchConfig),
    "lum_batch_stats": C.sizeof(LumBatchStats),
    "lum_tonemap_params": C.sizeof(LumTonemapParams),
}
