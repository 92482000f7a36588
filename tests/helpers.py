"""Shared test helpers: seeded ray sets, the oracle robustness filter, image statistics."""
from __future__ import annotations

import numpy as np

import oracle as O
from luminara_b200 import abi


def f32(x):
    return np.asarray(x, dtype=np.float32)


def random_rays(rng, n, lo, hi, tmin=0.001, tmax=np.inf):
    """Rays with origins uniform in the box [lo, hi] and isotropic directions, as float32
    values (the same numbers go to the device and, widened, to the f64 oracle)."""
    lo, hi = np.asarray(lo, float), np.asarray(hi, float)
    o = f32(lo + (hi - lo) * rng.random((n, 3)))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    d *= rng.uniform(0.5, 2.0, (n, 1))           # unnormalised, as the reference's rays are
    return o, f32(d), tmin, tmax


def camera_rays(world, cfg, rng, n):
    cam = world.camera
    lf = np.asarray(cam.look_from, float)
    la = np.asarray(cam.look_at, float)
    vup = np.asarray(cam.vup, float)
    th = np.radians(cam.vfov_degrees)
    h = np.tan(th / 2)
    vh, vw = 2 * h, cam.aspect_ratio * 2 * h
    w = (lf - la) / np.linalg.norm(lf - la)
    u = np.cross(vup, w)
    u /= np.linalg.norm(u)
    v = np.cross(w, u)
    hor, ver = u * vw * cam.focus_dist, v * vh * cam.focus_dist
    llc = lf - hor / 2 - ver / 2 - w * cam.focus_dist
    s = rng.random((n, 1))
    t = rng.random((n, 1))
    d = llc + s * hor + t * ver - lf
    o = np.tile(lf, (n, 1))
    return f32(o), f32(d), 0.001, np.inf


def to_gpu_rays(o, d, tmin, tmax, time=0.0):
    r = np.zeros(o.shape[0], dtype=abi.ray_dtype())
    r["org"] = o
    r["dir"] = d
    r["tmin"] = tmin
    r["tmax"] = tmax
    r["time"] = time
    return r


def to_orc_rays(o, d, tmin, tmax, time=0.0):
    r = np.zeros(o.shape[0], dtype=O.ORC_RAY)
    r["org"] = o.astype(np.float64)
    r["dir"] = d.astype(np.float64)
    r["tmin"] = np.float64(np.float32(tmin))
    r["tmax"] = np.float64(np.float32(tmax)) if np.isfinite(tmax) else np.inf
    r["time"] = np.float64(np.float32(time))
    return r


def robust_mask(orc_scene, o, d, tmin, tmax, rng, scale, rel=1e-5, n_perturb=6, normals=None, robust_scene=None):
    """True where the oracle's (hit?, prim id) is unchanged under small perturbations of
    the ray, i.e. the ray is away from edges, grazing angles and near-ties.

    Directions move by `rel` relative.  Origins move by rel*scale; for rays that start on
    a surface (`normals` given) the move is tangential plus a normal offset of a few f32
    ulps of the coordinates, so the test flags self-intersection-sensitive rays without
    pushing origins through their surface.  `robust_scene` (default: the scene itself)
    is the world used for the perturbed queries, e.g. the scene without its fog, whose
    hash-based free-flight distance is re-drawn by any change of the ray."""
    base = orc_scene.intersect(to_orc_rays(o, d, tmin, tmax))
    rs = robust_scene or orc_scene
    ref = base if robust_scene is None else rs.intersect(to_orc_rays(o, d, tmin, tmax))
    ok = np.ones(o.shape[0], dtype=bool)
    o64, d64 = o.astype(np.float64), d.astype(np.float64)
    for _ in range(n_perturb):
        noise = rng.normal(size=o.shape)
        if normals is not None:
            n = np.asarray(normals, np.float64)
            tang = noise - (noise * n).sum(1, keepdims=True) * n
            ulp = 4.0 * np.finfo(np.float32).eps * np.abs(o64).max(axis=1, keepdims=True)
            po = o64 + rel * scale * tang + ulp * rng.normal(size=(o.shape[0], 1)) * n
        else:
            po = o64 + rel * scale * noise
        pd = d64 * (1.0 + rel * rng.normal(size=d.shape))
        r = np.zeros(o.shape[0], dtype=O.ORC_RAY)
        r["org"], r["dir"], r["tmin"], r["tmax"] = po, pd, tmin, tmax
        h = rs.intersect(r)
        ok &= h["prim_id"] == ref["prim_id"]
    # exact ties (coplanar coincident faces, e.g. a box bottom on the floor): the winner
    # depends on traversal order, so such rays are not comparable
    if orc_scene.desc.n_prims <= 20000:
        ok &= orc_scene.tie_count(to_orc_rays(o, d, tmin, tmax)) <= 1
    return base, ok


def secondary_rays(orc_scene, o, d, tmin, tmax, rng):
    """Rays starting on surfaces: the hit points of a first set with new directions
    n + unit vector (the Lambertian rule).  Returns (o, d, tmin, tmax, normals)."""
    h = orc_scene.intersect(to_orc_rays(o, d, tmin, tmax))
    m = h["prim_id"] >= 0
    p = f32(h["point"][m])
    n = h["normal"][m]
    dd = rng.normal(size=p.shape)
    dd /= np.linalg.norm(dd, axis=1, keepdims=True)
    dd = dd + n
    return p, f32(dd), tmin, tmax, n


def luminance(img):
    return 0.2126 * img[..., 0] + 0.7152 * img[..., 1] + 0.0722 * img[..., 2]


def rmse(a, b):
    return float(np.sqrt(np.mean((np.asarray(a, float) - np.asarray(b, float)) ** 2)))


def t_tolerance(t_ref, d, n_ref, scale):
    """Allowed |t_gpu - t_ref|: 2e-4 relative, plus f32 coordinate quantization (4e-7 of
    the scene scale, ~4 ulps) measured along the normal and divided by the incidence."""
    dl = np.linalg.norm(d, axis=1)
    cos = np.abs((n_ref * d).sum(1)) / dl
    return 2e-4 * np.maximum(1.0, t_ref) + 4e-7 * scale / (np.maximum(cos, 1e-2) * dl)


def dump(name, **arrays):
    """Saves arrays for offline diagnosis when LUM_TEST_DUMP_DIR is set."""
    import os

    d = os.environ.get("LUM_TEST_DUMP_DIR")
    if d:
        os.makedirs(d, exist_ok=True)
        np.savez_compressed(os.path.join(d, name + ".npz"), **arrays)
