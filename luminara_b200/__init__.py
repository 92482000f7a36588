"""luminara_b200 -- B200 path-tracing core of the Luminara renderer.

The product is ``libluminara_b200.so`` (CUDA sm_100a kernels + C++ host library) behind the
C ABI in ``include/luminara_gpu.h``.  This package binds that ABI with ctypes and mirrors
the reference's Rust entry point ``render(config, camera, world, lights) -> RenderResult``
(src/render.rs:1557-1562) for Python callers.  There is no CPU fallback: if the shared
library is missing or no CUDA device is visible, calls raise.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import time
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import abi
from .scene import (  # noqa: F401  (re-exported reference names)
    Anisotropic, Blend, CameraConfig, Checker, Clearcoat, ConstantMedium, Dielectric, Disk, Emissive, Iridescent,
    Isotropic, Lambertian, LightInfo, Mesh, Metal, Microfacet, MovingSphere, Plane, Quad, RenderConfig, RotateX,
    RotateY, RotateZ, Scale, SolidColor, Sphere, Subsurface, ToneMapConfig, Toon, Translate, Translucent,
    Transparent, Triangle, Velvet, World, XyRect, XzRect, YzRect, make_box,
)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libluminara_b200.so")
CSRC = os.path.join(HERE, "csrc")


class LuminaraError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"luminara status {status}: {message}")
        self.status = status


def build(force: bool = False) -> str:
    """Compiles libluminara_b200.so for sm_100a with the committed Makefile."""
    if force:
        subprocess.run(["make", "-s", "-C", CSRC, "clean"], check=True)
    subprocess.run(["make", "-s", "-C", CSRC], check=True)
    return LIB_PATH


_lib = None


def lib():
    """Loads the shared library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing; build it with luminara_b200.build() or `make -C {CSRC}`")
    L = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    L.lum_abi_version.restype = C.c_int32
    L.lum_last_error.restype = C.c_char_p
    L.lum_scene_create.argtypes = [C.POINTER(abi.LumSceneDesc), C.POINTER(vp)]
    L.lum_scene_destroy.argtypes = [vp]
    L.lum_scene_info.argtypes = [vp, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                 C.POINTER(C.c_uint64)]
    L.lum_render.argtypes = [vp, C.POINTER(abi.LumRenderParams), vp, C.POINTER(abi.LumStats)]
    L.lum_render_device.argtypes = [vp, C.POINTER(abi.LumRenderParams), vp, vp, C.POINTER(abi.LumStats)]
    L.lum_count_tests.argtypes = [vp, C.POINTER(abi.LumRenderParams), C.POINTER(abi.LumTestCounts)]
    L.lum_tonemap_default.argtypes = [C.POINTER(abi.LumTonemapParams)]
    L.lum_tonemap_default.restype = None
    L.lum_tonemap_device.argtypes = [vp, C.c_uint32, C.c_uint32, C.POINTER(abi.LumTonemapParams), vp, vp, vp]
    L.lum_render_ldr.argtypes = [vp, C.POINTER(abi.LumRenderParams), C.POINTER(abi.LumTonemapParams), vp,
                                 C.POINTER(abi.LumStats)]
    L.lum_forward.argtypes = [vp, C.POINTER(abi.LumRenderParams), vp, C.POINTER(abi.LumStats)]
    L.lum_backward.argtypes = [vp, C.POINTER(abi.LumRenderParams), vp, vp, vp, vp, vp, C.POINTER(abi.LumStats)]
    L.lum_scene_set_envmap.argtypes = [vp, vp, C.c_uint32, C.c_uint32]
    L.lum_render_aov.argtypes = [vp, C.POINTER(abi.LumRenderParams), vp, vp, vp]
    L.lum_intersect.argtypes = [vp, vp, C.c_uint32, vp]
    L.lum_occluded.argtypes = [vp, vp, C.c_uint32, vp]
    PP = C.POINTER(C.c_void_p)
    L.lum_batch_default_config.argtypes = [C.POINTER(abi.LumBatchConfig)]
    L.lum_batch_autotune.argtypes = [PP, C.POINTER(abi.LumRenderParams), C.c_uint32, C.POINTER(abi.LumBatchConfig),
                                     C.POINTER(C.c_double)]
    L.lum_batch_create.argtypes = [PP, C.POINTER(abi.LumRenderParams), C.c_uint32, C.POINTER(abi.LumBatchConfig),
                                   C.POINTER(vp)]
    L.lum_batch_config_of.argtypes = [vp, C.POINTER(abi.LumBatchConfig)]
    L.lum_batch_render.argtypes = [vp, PP, C.POINTER(C.c_double), C.POINTER(abi.LumBatchStats)]
    L.lum_batch_render_device.argtypes = [vp, PP, C.POINTER(C.c_double), C.POINTER(abi.LumBatchStats)]
    L.lum_batch_destroy.argtypes = [vp]
    for name in ("lum_scene_create", "lum_scene_destroy", "lum_scene_info", "lum_render", "lum_render_device",
                 "lum_count_tests", "lum_intersect", "lum_occluded", "lum_forward", "lum_backward",
                 "lum_tonemap_device", "lum_render_ldr", "lum_scene_set_envmap", "lum_render_aov",
                 "lum_batch_default_config",
                 "lum_batch_autotune", "lum_batch_create", "lum_batch_config_of", "lum_batch_render",
                 "lum_batch_render_device", "lum_batch_destroy", "lum_diag_l1_throughput",
                 "lum_render_sums_device", "lum_sums_finalize_device"):
        getattr(L, name).restype = C.c_int32
    if L.lum_abi_version() != abi.LUM_ABI_VERSION:
        raise ImportError("libluminara_b200.so ABI version mismatch")
    _lib = L
    return L


def check(status: int) -> None:
    if status != abi.LUM_OK:
        raise LuminaraError(status, lib().lum_last_error().decode(errors="replace"))


class GpuScene:
    """A scene uploaded to the device (lum_scene_create)."""

    def __init__(self, world: World):
        self.desc = world.desc()
        h = C.c_void_p()
        check(lib().lum_scene_create(self.desc.ref(), C.byref(h)))
        self.h = h
        self._lib = lib()          # kept for close(): module globals may be gone at exit
        if getattr(world, "env_map", None) is not None:
            self.set_envmap(world.env_map)

    def close(self):
        if getattr(self, "h", None):
            self._lib.lum_scene_destroy(self.h)
            self.h = None

    __del__ = close

    def info(self):
        n_p, n_n, n_l = C.c_uint32(), C.c_uint32(), C.c_uint32()
        nb = C.c_uint64()
        check(lib().lum_scene_info(self.h, C.byref(n_p), C.byref(n_n), C.byref(n_l), C.byref(nb)))
        return {"prims": n_p.value, "nodes": n_n.value, "lights": n_l.value, "device_bytes": nb.value}

    def render(self, cfg: RenderConfig, out: Optional[np.ndarray] = None):
        """Renders into a host float32 array (H, W, 3); returns (image, lum_stats)."""
        p = cfg.to_c()
        shape = cfg.out_shape()
        if out is None:
            out = np.empty(shape, dtype=np.float32)
        assert out.dtype == np.float32 and out.flags.c_contiguous and out.shape == shape
        st = abi.LumStats()
        check(lib().lum_render(self.h, C.byref(p), out.ctypes.data, C.byref(st)))
        return out, st

    def render_device(self, cfg: RenderConfig, d_out: int, stream: int = 0, wait: bool = True):
        """Renders into a caller-owned device buffer (pointer as int) on `stream`.  wait=False
        only enqueues the render (no stats, no synchronisation) and returns None."""
        p = cfg.to_c()
        if not wait:
            check(lib().lum_render_device(self.h, C.byref(p), C.c_void_p(d_out), C.c_void_p(stream), None))
            return None
        st = abi.LumStats()
        check(lib().lum_render_device(self.h, C.byref(p), C.c_void_p(d_out), C.c_void_p(stream), C.byref(st)))
        return st

    def render_sums_device(self, cfg: RenderConfig, d_sums: int, stream: int = 0):
        """lum_render_sums_device: the raw per-pixel fixed-point sums (H, W, 4) int64 into a
        caller-owned device buffer (pointer as int); waits and returns the stats."""
        p = cfg.to_c()
        st = abi.LumStats()
        check(lib().lum_render_sums_device(self.h, C.byref(p), C.c_void_p(d_sums), C.c_void_p(stream),
                                           C.byref(st)))
        return st

    def set_envmap(self, rgb: Optional[np.ndarray]):
        """lum_scene_set_envmap: an (H, W, 3) float32 equirectangular map (None removes it)."""
        if rgb is None:
            check(lib().lum_scene_set_envmap(self.h, None, 0, 0))
            return
        rgb = np.ascontiguousarray(rgb, dtype=np.float32)
        assert rgb.ndim == 3 and rgb.shape[2] == 3
        check(lib().lum_scene_set_envmap(self.h, rgb.ctypes.data, rgb.shape[1], rgb.shape[0]))

    def render_aov(self, cfg: RenderConfig):
        """lum_render_aov: (depth (H, W) float32, normals (H, W, 3) uint8, albedo (H, W, 3) uint8)."""
        h, w, _ = cfg.out_shape()
        p = cfg.to_c()
        depth = np.empty((h, w), dtype=np.float32)
        normals = np.empty((h, w, 3), dtype=np.uint8)
        albedo = np.empty((h, w, 3), dtype=np.uint8)
        check(lib().lum_render_aov(self.h, C.byref(p), depth.ctypes.data, normals.ctypes.data, albedo.ctypes.data))
        return depth, normals, albedo

    def render_ldr(self, cfg: RenderConfig, tm: Optional["ToneMapConfig"] = None):
        """lum_render_ldr: (H, W, 4) uint8 RGBA through the LDR colour chain, and stats.  The
        render's exposure is the chain's exposure (tm.exposure is ignored)."""
        p = cfg.to_c()
        t = (tm or ToneMapConfig()).to_c()
        h, w, _ = cfg.out_shape()
        out = np.empty((h, w, 4), dtype=np.uint8)
        st = abi.LumStats()
        check(lib().lum_render_ldr(self.h, C.byref(p), C.byref(t), out.ctypes.data, C.byref(st)))
        return out, st

    def forward(self, cfg: RenderConfig):
        """lum_forward: the image (H, W, 3) and stats."""
        p = cfg.to_c()
        out = np.empty(cfg.out_shape(), dtype=np.float32)
        st = abi.LumStats()
        check(lib().lum_forward(self.h, C.byref(p), out.ctypes.data, C.byref(st)))
        return out, st

    def backward(self, cfg: RenderConfig, dl_dimage: np.ndarray, light_material=None):
        """lum_backward: gradients of the loss w.r.t. per-material albedo (n, 3), roughness
        (n,) and emission (n, 3), given dL/d(image) of shape (H, W, 3)."""
        p = cfg.to_c()
        g = np.ascontiguousarray(dl_dimage, dtype=np.float32)
        assert g.shape == cfg.out_shape()
        n = self.desc.n_materials
        da = np.zeros((n, 3), np.float32)
        dr = np.zeros(n, np.float32)
        de = np.zeros((n, 3), np.float32)
        lm = None
        if light_material is not None:
            lm = np.ascontiguousarray(light_material, dtype=np.int32)
        st = abi.LumStats()
        check(lib().lum_backward(self.h, C.byref(p), g.ctypes.data, lm.ctypes.data if lm is not None else None,
                                 da.ctypes.data, dr.ctypes.data, de.ctypes.data, C.byref(st)))
        return da, dr, de, st

    def count_tests(self, cfg: RenderConfig) -> abi.LumTestCounts:
        """Node/primitive test counts of this render (counter build of the render kernel)."""
        p = cfg.to_c()
        c = abi.LumTestCounts()
        check(lib().lum_count_tests(self.h, C.byref(p), C.byref(c)))
        return c

    def intersect(self, rays: np.ndarray) -> np.ndarray:
        rays = np.ascontiguousarray(rays, dtype=abi.ray_dtype())
        hits = np.zeros(rays.shape[0], dtype=abi.hit_dtype())
        check(lib().lum_intersect(self.h, rays.ctypes.data, rays.shape[0], hits.ctypes.data))
        return hits

    def occluded(self, rays: np.ndarray) -> np.ndarray:
        rays = np.ascontiguousarray(rays, dtype=abi.ray_dtype())
        occ = np.zeros(rays.shape[0], dtype=np.int32)
        check(lib().lum_occluded(self.h, rays.ctypes.data, rays.shape[0], occ.ctypes.data))
        return occ


class Batch:
    """Many scenes rendered together by the persistent wavefront tracer (lum_batch_*).

    `scenes` are GpuScene objects (kept alive by the batch), `configs` one RenderConfig per
    scene.  `config` is None (autotuned, cached per device and batch), "default", or a dict
    with pool_paths / block_threads / sort_threshold / iters_per_graph."""

    def __init__(self, scenes, configs, config=None):
        self.scenes = list(scenes)
        self.configs = list(configs)
        n = len(self.scenes)
        self._handles = (C.c_void_p * n)(*[s.h.value for s in self.scenes])
        self._params = (abi.LumRenderParams * n)(*[c.to_c() for c in self.configs])
        cfg_ptr = None
        if config is not None:
            cfg = abi.LumBatchConfig()
            check(lib().lum_batch_default_config(C.byref(cfg)))
            if isinstance(config, dict):
                for k, v in config.items():
                    setattr(cfg, k, int(v))
            cfg_ptr = C.byref(cfg)
        h = C.c_void_p()
        check(lib().lum_batch_create(C.cast(self._handles, C.POINTER(C.c_void_p)), self._params, n, cfg_ptr,
                                     C.byref(h)))
        self.h = h
        self._lib = lib()

    def config(self):
        c = abi.LumBatchConfig()
        check(lib().lum_batch_config_of(self.h, C.byref(c)))
        return {"pool_paths": c.pool_paths, "block_threads": c.block_threads, "sort_threshold": c.sort_threshold,
                "iters_per_graph": c.iters_per_graph, "mode": c.mode}

    def render(self):
        """Returns (images, per-scene completion ms, lum_batch_stats)."""
        n = len(self.scenes)
        imgs = [np.empty(c.out_shape(), dtype=np.float32) for c in self.configs]
        ptrs = (C.c_void_p * n)(*[im.ctypes.data for im in imgs])
        done = (C.c_double * n)()
        st = abi.LumBatchStats()
        check(lib().lum_batch_render(self.h, C.cast(ptrs, C.POINTER(C.c_void_p)), done, C.byref(st)))
        return imgs, list(done), st

    def render_device(self, d_ptrs):
        n = len(self.scenes)
        ptrs = (C.c_void_p * n)(*d_ptrs)
        done = (C.c_double * n)()
        st = abi.LumBatchStats()
        check(lib().lum_batch_render_device(self.h, C.cast(ptrs, C.POINTER(C.c_void_p)), done, C.byref(st)))
        return list(done), st

    def close(self):
        if getattr(self, "h", None):
            self._lib.lum_batch_destroy(self.h)
            self.h = None

    __del__ = close


def sums_finalize_device(d_sums: int, width: int, height: int, exposure: float, d_rgb: int, stream: int = 0):
    """lum_sums_finalize_device: pixels of (summed) raw sums, device to device."""
    check(lib().lum_sums_finalize_device(C.c_void_p(d_sums), int(width), int(height), C.c_double(exposure),
                                         C.c_void_p(d_rgb), C.c_void_p(stream)))


def diag_l1_throughput(pattern: int = 0) -> float:
    """lum_diag_l1_throughput: the device's L1 load throughput in GB/s (pattern 0 coalesced,
    1 gather of 64-byte records), the roof of the megakernel's node and primitive fetches."""
    v = C.c_double()
    check(lib().lum_diag_l1_throughput(int(pattern), C.byref(v)))
    return v.value


def autotune(scenes, configs):
    """Runs (or reads from cache) the batch autotuner; returns (config dict, best ms or -1)."""
    n = len(scenes)
    handles = (C.c_void_p * n)(*[s.h.value for s in scenes])
    params = (abi.LumRenderParams * n)(*[c.to_c() for c in configs])
    cfg = abi.LumBatchConfig()
    ms = C.c_double()
    check(lib().lum_batch_autotune(C.cast(handles, C.POINTER(C.c_void_p)), params, n, C.byref(cfg), C.byref(ms)))
    return ({"pool_paths": cfg.pool_paths, "block_threads": cfg.block_threads, "sort_threshold": cfg.sort_threshold,
             "iters_per_graph": cfg.iters_per_graph, "mode": cfg.mode}, ms.value)


@dataclass
class RenderResult:
    """src/render.rs:1540-1554 (the HDR part: linear f32 RGB with exposure applied)."""
    hdr_data: np.ndarray
    total_rays: int
    render_time_secs: float
    stats: abi.LumStats


def render(config: RenderConfig, camera: CameraConfig, world: World, lights=None) -> RenderResult:
    """Drop-in for render::render (src/render.rs:1557): uploads the scene, renders on the
    GPU, returns the f32 linear image.  `lights` replaces world.lights when given."""
    t0 = time.perf_counter()
    world.camera = camera
    if lights is not None:
        world.lights = list(lights)
    sc = GpuScene(world)
    try:
        img, st = sc.render(config)
    finally:
        sc.close()
    return RenderResult(img, int(st.paths), time.perf_counter() - t0, st)


def make_rays(org, dir, tmin=0.001, tmax=np.inf, time_=0.0) -> np.ndarray:
    org = np.atleast_2d(np.asarray(org, dtype=np.float32))
    dir = np.atleast_2d(np.asarray(dir, dtype=np.float32))
    n = max(org.shape[0], dir.shape[0])
    r = np.zeros(n, dtype=abi.ray_dtype())
    r["org"] = org
    r["dir"] = dir
    r["tmin"] = tmin
    r["tmax"] = tmax
    r["time"] = time_
    return r


from .toml_scene import UnsupportedSceneError, load_scene, load_scene_file, tonemap_config  # noqa: E402,F401


def tonemap_device(d_hdr: int, width: int, height: int, tm=None, d_scratch: int = 0, d_rgba: int = 0,
                   stream: int = 0) -> None:
    """lum_tonemap_device on device pointers (e.g. torch tensors' data_ptr())."""
    t = (tm or ToneMapConfig()).to_c()
    check(lib().lum_tonemap_device(d_hdr or None, width, height, C.byref(t), d_scratch or None, d_rgba or None,
                                   stream or None))
