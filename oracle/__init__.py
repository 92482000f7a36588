"""ctypes binding of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE: imported only by tests/, __graft_entry__.smoke() and bench.py's CPU
baseline leg, as the checker.  The product package never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from luminara_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

MODE_STREAM = 0
MODE_KEYED = 1


class OrcStats(C.Structure):
    _fields_ = [
        ("paths", C.c_uint64),
        ("segments", C.c_uint64),
        ("shadow_rays", C.c_uint64),
        ("seconds", C.c_double),
        ("threads", C.c_int32),
        ("reserved", C.c_int32),
    ]


ORC_RAY = np.dtype([("org", "<f8", 3), ("tmin", "<f8"), ("dir", "<f8", 3), ("tmax", "<f8"), ("time", "<f8"),
                    ("pad", "<f8")])
ORC_HIT = np.dtype([("t", "<f8"), ("u", "<f8"), ("v", "<f8"), ("point", "<f8", 3), ("normal", "<f8", 3),
                    ("prim_id", "<i4"), ("front_face", "<i4"), ("material", "<i4"), ("reserved", "<i4")])

_lib = None


def build(force: bool = False) -> str:
    """Compiles liboracle.so with the committed Makefile."""
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < max(
            os.path.getmtime(os.path.join(HERE, f)) for f in ("oracle.cpp", "oracle.h", "Makefile")):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB_PATH)
        vp = C.c_void_p
        dp = C.POINTER(C.c_double)
        L.orc_scene_create.argtypes = [C.POINTER(abi.LumSceneDesc), C.POINTER(vp)]
        L.orc_scene_destroy.argtypes = [vp]
        L.orc_intersect.argtypes = [vp, vp, C.c_uint32, vp]
        L.orc_occluded.argtypes = [vp, vp, C.c_uint32, vp]
        L.orc_tie_count.argtypes = [vp, vp, C.c_uint32, C.c_double, C.c_double, vp]
        L.orc_render.argtypes = [vp, C.POINTER(abi.LumRenderParams), C.c_int, C.c_int, dp, C.POINTER(OrcStats)]
        L.orc_render_expired.argtypes = L.orc_render.argtypes
        L.orc_scene_set_envmap.argtypes = [vp, vp, C.c_uint32, C.c_uint32]
        L.orc_render_aov.argtypes = [vp, C.POINTER(abi.LumRenderParams), C.c_int, vp, vp, vp]
        L.orc_render_rows.argtypes = [vp, C.POINTER(abi.LumRenderParams), C.c_int, C.c_int, C.c_uint32,
                                      C.c_uint32, dp, C.POINTER(OrcStats)]
        L.orc_render_sums.argtypes = [vp, C.POINTER(abi.LumRenderParams), C.c_int, C.c_int, dp, C.POINTER(OrcStats)]
        L.orc_render_row_list.argtypes = [vp, C.POINTER(abi.LumRenderParams), C.c_int, C.c_int, vp, C.c_uint32,
                                          dp, C.POINTER(OrcStats)]
        L.orc_adjoint.argtypes = [vp, C.POINTER(abi.LumRenderParams), dp, vp, C.c_int, C.c_int, dp, dp, dp, dp]
        L.orc_adjoint_dir.argtypes = [vp, C.POINTER(abi.LumRenderParams), dp, vp, C.c_int, C.c_int, dp, dp]
        L.orc_scatter.argtypes = [C.POINTER(abi.LumMaterial), dp, dp, dp, C.c_double, C.c_double, C.c_double,
                                  C.c_uint64, C.c_int, dp]
        L.orc_scatter_in.argtypes = [C.POINTER(abi.LumMaterial), C.c_uint32, C.c_uint32, dp, dp, dp, C.c_double,
                                     C.c_double, C.c_double, C.c_uint64, C.c_int, dp]
        L.orc_emitted.argtypes = [C.POINTER(abi.LumMaterial), C.c_uint32, C.c_uint32, C.c_double, C.c_double, dp]
        L.orc_emitted.restype = C.c_double
        L.orc_is_specular.argtypes = [C.POINTER(abi.LumMaterial)]
        L.orc_thin_film.argtypes = [C.c_double, C.c_double, C.c_double, C.c_int]
        L.orc_thin_film.restype = C.c_double
        L.orc_schlick.argtypes = [C.c_double, C.c_double]
        L.orc_schlick.restype = C.c_double
        L.orc_ggx_d.argtypes = [C.c_double, C.c_double]
        L.orc_ggx_d.restype = C.c_double
        L.orc_camera_ray.argtypes = [C.POINTER(abi.LumCamera), C.c_double, C.c_double, C.c_uint64, dp]
        L.orc_filter_weight.argtypes = [C.c_int, C.c_double, C.c_double]
        L.orc_filter_weight.restype = C.c_double
        L.orc_sample_direct_light.argtypes = [vp, dp, dp, dp, C.c_uint64, C.c_int, dp]
        L.orc_aabb_hit.argtypes = [dp, dp, dp, C.c_double, C.c_double]
        L.orc_scene_bbox.argtypes = [vp, C.c_int32, dp]
        L.orc_bvh_stats.argtypes = [vp, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
        L.orc_refract.argtypes = [dp, dp, C.c_double, dp]
        L.orc_reflect.argtypes = [dp, dp, dp]
        L.orc_stream_u64.argtypes = [C.c_uint64, C.c_uint32, C.POINTER(C.c_uint64)]
        L.orc_stream_f64.argtypes = [C.c_uint64, C.c_uint32, dp]
        L.orc_philox.argtypes = [C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
        L.orc_xoshiro_from_state.argtypes = [C.POINTER(C.c_uint64), C.c_uint32, C.POINTER(C.c_uint64)]
        L.orc_seed_state.argtypes = [C.c_uint64, C.POINTER(C.c_uint64)]
        _lib = L
    return _lib


def _d(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(C.POINTER(C.c_double))


class OracleScene:
    """An oracle SceneWorld built from a luminara_b200.scene.World."""

    def __init__(self, world):
        self.desc = world.desc()
        h = C.c_void_p()
        rc = lib().orc_scene_create(self.desc.ref(), C.byref(h))
        if rc != 0:
            raise RuntimeError(f"orc_scene_create failed: {rc}")
        self.h = h
        if getattr(world, "env_map", None) is not None:
            self.set_envmap(world.env_map)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_scene_destroy(self.h)
            self.h = None

    def intersect(self, rays: np.ndarray) -> np.ndarray:
        rays = np.ascontiguousarray(rays, dtype=ORC_RAY)
        hits = np.zeros(rays.shape[0], dtype=ORC_HIT)
        lib().orc_intersect(self.h, rays.ctypes.data, rays.shape[0], hits.ctypes.data)
        return hits

    def tie_count(self, rays: np.ndarray, rel=1e-6, abs_eps=1e-6) -> np.ndarray:
        rays = np.ascontiguousarray(rays, dtype=ORC_RAY)
        c = np.zeros(rays.shape[0], dtype=np.int32)
        lib().orc_tie_count(self.h, rays.ctypes.data, rays.shape[0], rel, abs_eps, c.ctypes.data)
        return c

    def occluded(self, rays: np.ndarray) -> np.ndarray:
        rays = np.ascontiguousarray(rays, dtype=ORC_RAY)
        occ = np.zeros(rays.shape[0], dtype=np.int32)
        lib().orc_occluded(self.h, rays.ctypes.data, rays.shape[0], occ.ctypes.data)
        return occ

    def render(self, cfg, mode=MODE_STREAM, threads=0, rows=None, expired=False):
        """expired=True renders as if every row started after the time limit."""
        p = cfg.to_c()
        shape = cfg.out_shape()
        out = np.zeros(shape, dtype=np.float64)
        st = OrcStats()
        if expired:
            rc = lib().orc_render_expired(self.h, C.byref(p), mode, threads,
                                          out.ctypes.data_as(C.POINTER(C.c_double)), C.byref(st))
        elif rows is None:
            rc = lib().orc_render(self.h, C.byref(p), mode, threads,
                                  out.ctypes.data_as(C.POINTER(C.c_double)), C.byref(st))
        else:
            rc = lib().orc_render_rows(self.h, C.byref(p), mode, threads, rows[0], rows[1],
                                       out.ctypes.data_as(C.POINTER(C.c_double)), C.byref(st))
        if rc != 0:
            raise RuntimeError(f"orc_render failed: {rc}")
        return out, st

    def render_sums(self, cfg, mode=MODE_KEYED, threads=0):
        """Per-pixel sums before the division (H, W, 4): filter-weighted clamped R, G, B and the
        filter weight (render.rs:1692-1704)."""
        p = cfg.to_c()
        h, w, _ = cfg.out_shape()
        out = np.zeros((h, w, 4), dtype=np.float64)
        st = OrcStats()
        rc = lib().orc_render_sums(self.h, C.byref(p), mode, threads, out.ctypes.data_as(C.POINTER(C.c_double)),
                                   C.byref(st))
        if rc != 0:
            raise RuntimeError(f"orc_render_sums failed: {rc}")
        return out, st

    def render_row_list(self, cfg, rows, mode=MODE_STREAM, threads=0):
        """Renders the image rows `rows` (OpenMP over the list); returns (array (len(rows), W, 3)
        with row k = image row rows[k], stats)."""
        p = cfg.to_c()
        r = np.ascontiguousarray(rows, dtype=np.uint32)
        w = cfg.out_shape()[1]
        out = np.zeros((len(r), w, 3), dtype=np.float64)
        st = OrcStats()
        rc = lib().orc_render_row_list(self.h, C.byref(p), mode, threads, r.ctypes.data, len(r),
                                       out.ctypes.data_as(C.POINTER(C.c_double)), C.byref(st))
        if rc != 0:
            raise RuntimeError(f"orc_render_row_list failed: {rc}")
        return out, st

    def set_envmap(self, rgb):
        if rgb is None:
            lib().orc_scene_set_envmap(self.h, None, 0, 0)
            return
        self._env = np.ascontiguousarray(rgb, dtype=np.float32)
        lib().orc_scene_set_envmap(self.h, self._env.ctypes.data, self._env.shape[1], self._env.shape[0])

    def render_aov(self, cfg, mode=MODE_KEYED):
        """(depth (H, W) f64 holding f32 values, normals (H, W, 3) u8, albedo (H, W, 3) u8)."""
        h, w, _ = cfg.out_shape()
        p = cfg.to_c()
        depth = np.zeros((h, w), dtype=np.float64)
        normals = np.zeros((h, w, 3), dtype=np.uint8)
        albedo = np.zeros((h, w, 3), dtype=np.uint8)
        rc = lib().orc_render_aov(self.h, C.byref(p), mode, depth.ctypes.data, normals.ctypes.data,
                                  albedo.ctypes.data)
        if rc != 0:
            raise RuntimeError(f"orc_render_aov failed: {rc}")
        return depth, normals, albedo

    def adjoint(self, cfg, dl_dimage, light_material=None, detach=True, threads=0):
        """f64 adjoint of the keyed estimator: (d_albedo (n,3), d_roughness (n,), d_emission (n,3),
        primal image)."""
        p = cfg.to_c()
        g = np.ascontiguousarray(dl_dimage, dtype=np.float64)
        assert g.shape == cfg.out_shape()
        n = self.desc.n_materials
        da, dr, de = np.zeros((n, 3)), np.zeros(n), np.zeros((n, 3))
        img = np.zeros(cfg.out_shape())
        lm = None if light_material is None else np.ascontiguousarray(light_material, dtype=np.int32)
        dp_ = C.POINTER(C.c_double)
        rc = lib().orc_adjoint(self.h, C.byref(p), g.ctypes.data_as(dp_), lm.ctypes.data if lm is not None else None,
                               int(detach), threads, da.ctypes.data_as(dp_), dr.ctypes.data_as(dp_),
                               de.ctypes.data_as(dp_), img.ctypes.data_as(dp_))
        if rc != 0:
            raise RuntimeError(f"orc_adjoint failed: {rc}")
        return da, dr, de, img

    def adjoint_dir(self, cfg, dl_dimage, direction, light_material=None, detach=True, threads=0):
        """Directional derivative of sum(dl_dimage * image) along `direction` (7n parameters).
        detach: 0/False plain, 1/True probabilities held with the survival score term, 2 held
        without it."""
        p = cfg.to_c()
        g = np.ascontiguousarray(dl_dimage, dtype=np.float64)
        d = np.ascontiguousarray(direction, dtype=np.float64)
        assert d.shape == (7 * self.desc.n_materials,)
        lm = None if light_material is None else np.ascontiguousarray(light_material, dtype=np.int32)
        out = C.c_double()
        dp_ = C.POINTER(C.c_double)
        rc = lib().orc_adjoint_dir(self.h, C.byref(p), g.ctypes.data_as(dp_), lm.ctypes.data if lm is not None else None,
                                   int(detach), threads, d.ctypes.data_as(dp_), C.byref(out))
        if rc != 0:
            raise RuntimeError(f"orc_adjoint_dir failed: {rc}")
        return out.value

    def sample_direct_light(self, p, n, albedo, seed, n_iter):
        out = np.zeros((n_iter, 3))
        pa, pp = _d(p)
        na, nn = _d(n)
        aa, ap = _d(albedo)
        lib().orc_sample_direct_light(self.h, pp, nn, ap, seed, n_iter, out.ctypes.data_as(C.POINTER(C.c_double)))
        return out

    def object_bbox(self, i):
        out = np.zeros(6)
        rc = lib().orc_scene_bbox(self.h, i, out.ctypes.data_as(C.POINTER(C.c_double)))
        return None if rc else out

    def bvh_stats(self):
        n = C.c_uint32()
        d = C.c_uint32()
        lib().orc_bvh_stats(self.h, C.byref(n), C.byref(d))
        return n.value, d.value


def make_rays(org, dir, tmin=0.001, tmax=np.inf, time=0.0) -> np.ndarray:
    org = np.atleast_2d(np.asarray(org, dtype=np.float64))
    dir = np.atleast_2d(np.asarray(dir, dtype=np.float64))
    n = max(org.shape[0], dir.shape[0])
    r = np.zeros(n, dtype=ORC_RAY)
    r["org"] = org
    r["dir"] = dir
    r["tmin"] = tmin
    r["tmax"] = tmax
    r["time"] = time
    return r


def _material_array(material):
    """lum_material records of `material` (index 0) and every Blend child below it."""
    order = []

    def visit(m):
        if any(m is x for x in order):
            return
        order.append(m)
        for c in (m.children or ()):
            visit(c)

    visit(material)

    def index_of(m):
        return next(i for i, x in enumerate(order) if x is m)

    return (abi.LumMaterial * len(order))(*[m.to_c(index_of) for m in order]), len(order)


def scatter(material, ray_o, ray_d, point, outward_normal, t=1.0, u=0.5, v=0.5, seed=42, n_iter=1, time=0.0,
            origin=False):
    """Material::scatter n_iter times from one stream (stream mode): rows of ok, dir[3], att[3],
    front_face (and origin[3] with origin=True)."""
    arr, n = _material_array(material)
    ray = np.array([*ray_o, *ray_d, time], dtype=np.float64)
    out = np.zeros((n_iter, 11))
    p = np.asarray(point, dtype=np.float64)
    nrm = np.asarray(outward_normal, dtype=np.float64)
    dp = C.POINTER(C.c_double)
    rc = lib().orc_scatter_in(arr, n, 0, ray.ctypes.data_as(dp), p.ctypes.data_as(dp), nrm.ctypes.data_as(dp),
                              t, u, v, seed, n_iter, out.ctypes.data_as(dp))
    if rc != 0:
        raise RuntimeError(f"orc_scatter_in failed: {rc}")
    return out if origin else out[:, :8]


def emitted_sum(material, u=0.5, v=0.5, p=(0.0, 0.0, 0.0)):
    arr, n = _material_array(material)
    q = np.asarray(p, dtype=np.float64)
    return lib().orc_emitted(arr, n, 0, u, v, q.ctypes.data_as(C.POINTER(C.c_double)))


def is_specular(material):
    m = material.to_c(lambda _m: 0)
    return bool(lib().orc_is_specular(C.byref(m)))


def thin_film(cos_theta, thickness, film_ior):
    return np.array([lib().orc_thin_film(cos_theta, thickness, film_ior, c) for c in range(3)])


def schlick(cosine, ref_idx):
    return lib().orc_schlick(cosine, ref_idx)


def ggx_d(n_dot_h, alpha):
    return lib().orc_ggx_d(n_dot_h, alpha)


def camera_ray(cam_cfg, s, t, seed=0):
    c = cam_cfg.to_c()
    out = np.zeros(7)
    lib().orc_camera_ray(C.byref(c), s, t, seed, out.ctypes.data_as(C.POINTER(C.c_double)))
    return out[:3], out[3:6], out[6]


def filter_weight(f, dx, dy):
    return lib().orc_filter_weight(f, dx, dy)


def aabb_hit(mn, mx, o, d, tmin=0.001, tmax=np.inf):
    mn = np.asarray(mn, dtype=np.float64)
    mx = np.asarray(mx, dtype=np.float64)
    ray = np.array([*o, *d, 0.0], dtype=np.float64)
    P = C.POINTER(C.c_double)
    return bool(lib().orc_aabb_hit(mn.ctypes.data_as(P), mx.ctypes.data_as(P), ray.ctypes.data_as(P), tmin, tmax))


def refract(v, n, eta):
    v = np.asarray(v, dtype=np.float64)
    n = np.asarray(n, dtype=np.float64)
    out = np.zeros(3)
    P = C.POINTER(C.c_double)
    lib().orc_refract(v.ctypes.data_as(P), n.ctypes.data_as(P), eta, out.ctypes.data_as(P))
    return out


def reflect(v, n):
    v = np.asarray(v, dtype=np.float64)
    n = np.asarray(n, dtype=np.float64)
    out = np.zeros(3)
    P = C.POINTER(C.c_double)
    lib().orc_reflect(v.ctypes.data_as(P), n.ctypes.data_as(P), out.ctypes.data_as(P))
    return out


def stream_u64(seed, n):
    out = (C.c_uint64 * n)()
    lib().orc_stream_u64(seed, n, out)
    return [int(x) for x in out]


def stream_f64(seed, n):
    out = np.zeros(n)
    lib().orc_stream_f64(seed, n, out.ctypes.data_as(C.POINTER(C.c_double)))
    return out


def philox(ctr, key):
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    lib().orc_philox(c, k, o)
    return [int(x) for x in o]


def xoshiro_from_state(state, n):
    st = (C.c_uint64 * 4)(*state)
    out = (C.c_uint64 * n)()
    lib().orc_xoshiro_from_state(st, n, out)
    return [int(x) for x in out]


def seed_state(seed):
    out = (C.c_uint64 * 4)()
    lib().orc_seed_state(seed, out)
    return [int(x) for x in out]
