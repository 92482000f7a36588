"""GPU parity of the intersection kernels against the f64 oracle.

Tolerances (f32 device vs f64 oracle on the same f32-representable rays):
  - hit/miss and primitive id: exact on rays the oracle finds robust (unchanged under
    1e-5 relative perturbations of origin and direction, and not an exact tie between
    coincident surfaces); at least 98% of primary rays are robust.
  - t: |t_gpu - t_ref| <= 2e-4 * max(1, t_ref) + 4e-7 * scale / (|cos| * |d|), i.e. relative
    2e-4 plus ~4 f32 ulps of the scene's coordinates along the normal (helpers.t_tolerance),
    for hits with incidence |cos| >= 0.01; at grazing incidence t is ill-conditioned (a ray
    tangent to a sphere moves its root by sqrt of the rounding), so those hits are checked
    for hit/miss and primitive id only
  - normal: |n_gpu - n_ref| <= 2e-3 (unit vectors, facing the ray), front_face exact
"""
import numpy as np
import pytest

import luminara_b200 as L
import oracle as O
from luminara_b200 import scene as S
from luminara_b200 import workloads as W
from tests import helpers as H

pytestmark = pytest.mark.gpu

T_TOL = 2e-4
N_TOL = 2e-3
GRAY = (0.5, 0.5, 0.5)


def gpu_hit1(world, o, d, tmin=0.001, tmax=np.inf):
    sc = L.GpuScene(world)
    h = sc.intersect(L.make_rays(o, d, tmin, tmax))[0]
    return h if h["prim_id"] >= 0 else None


# ---------------------------------------------------------------- reference known answers
def test_kat_quad_center():                                 # quad.rs:85-101
    w = S.World()
    w.add(S.Quad((0, 0, 0), (1, 0, 0), (0, 0, 1), S.Lambertian(GRAY)))
    h = gpu_hit1(w, (0.5, 1.0, 0.5), (0, -1, 0))
    assert h is not None
    assert abs(h["t"] - 1.0) < 1e-6 and abs(h["u"] - 0.5) < 1e-6 and abs(h["v"] - 0.5) < 1e-6
    assert gpu_hit1(w, (2.0, 1.0, 0.5), (0, -1, 0)) is None
    assert gpu_hit1(w, (0.5, 1.0, 0.5), (1, 0, 0)) is None


def test_kat_plane_t5():                                    # plane.rs:86-93
    w = S.World()
    w.add(S.Plane((0, 0, 0), (0, 1, 0), S.Lambertian(GRAY)))
    h = gpu_hit1(w, (0, 5, 0), (0, -1, 0))
    assert h is not None and abs(h["t"] - 5.0) < 1e-6
    assert gpu_hit1(w, (0, 1, 0), (1, 0, 0)) is None


def test_kat_transforms():                                  # transform.rs:365-422
    w = S.World()
    w.add(S.Translate(S.Sphere((0, 0, 0), 1.0, S.Lambertian(GRAY)), (5, 0, 0)))
    assert gpu_hit1(w, (5, 0, -5), (0, 0, 1)) is not None
    assert gpu_hit1(w, (0, 0, -5), (0, 0, 1)) is None
    for rot, c, o, d in [(S.RotateY, (2, 0, 0), (0, 0, -5), (0, 0, 1)), (S.RotateX, (0, 2, 0), (0, 0, -5), (0, 0, 1)),
                         (S.RotateZ, (2, 0, 0), (0, 5, 0), (0, -1, 0))]:
        w = S.World()
        w.add(rot(S.Sphere(c, 0.5, S.Lambertian(GRAY)), 90.0))
        assert gpu_hit1(w, o, d) is not None


def test_kat_primitives_and_bvh():
    w = S.World()
    for i in range(50):                                     # bvh.rs:199-218
        w.add(S.Sphere((i * 2.0, 0, 0), 0.5, S.Lambertian(GRAY)))
    h = gpu_hit1(w, (0, 0, -2), (0, 0, 1))
    assert h is not None and h["prim_id"] == 0
    assert gpu_hit1(w, (0, 5, 0), (0, 0, 1)) is None
    w = S.World()
    w.add(S.Triangle((0, 0, 0), (1, 0, 0), (0, 1, 0), S.Lambertian(GRAY)))
    assert gpu_hit1(w, (0.2, 0.2, -1), (0, 0, 1)) is not None
    assert gpu_hit1(w, (2, 2, -1), (0, 0, 1)) is None
    w = S.World()
    w.add(S.Disk((0, 0, 0), (0, 1, 0), 1.0, S.Lambertian(GRAY)))
    assert gpu_hit1(w, (0, 1, 0), (0, -1, 0)) is not None
    assert gpu_hit1(w, (5, 1, 0), (0, -1, 0)) is None
    w = S.World()
    w.add(S.MovingSphere((0, 0, 0), (10, 0, 0), 1.0, S.Lambertian(GRAY)))
    sc = L.GpuScene(w)
    assert sc.intersect(L.make_rays((10, 0, -5), (0, 0, 1), time_=1.0))[0]["prim_id"] == 0
    assert sc.intersect(L.make_rays((0, 0, -5), (0, 0, 1), time_=1.0))[0]["prim_id"] == -1
    w = S.World()                                           # constant_medium.rs:126-137
    w.add(S.ConstantMedium(S.Sphere((0, 0, 0), 5.0, None), 100.0, (1, 1, 1)))
    assert gpu_hit1(w, (0, 0, -10), (0, 0, 1)) is not None


def test_empty_scene_misses():
    sc = L.GpuScene(S.World())
    h = sc.intersect(L.make_rays((0, 0, 0), (0, 0, 1)))
    assert h["prim_id"][0] == -1


# ---------------------------------------------------------------- seeded ray sets vs oracle
def compare_sets(world, o, d, tmin, tmax, scale, rng, min_robust=0.98, normals=None, robust_world=None):
    orc = O.OracleScene(world)
    gpu = L.GpuScene(world)
    rs = O.OracleScene(robust_world) if robust_world is not None else None
    base, ok = H.robust_mask(orc, o, d, tmin, tmax, rng, scale, normals=normals, robust_scene=rs)
    g = gpu.intersect(H.to_gpu_rays(o, d, tmin, tmax))
    assert ok.mean() >= min_robust, f"only {ok.mean():.4f} of rays are robust"
    bad = ok & (g["prim_id"] != base["prim_id"])
    d64 = d.astype(np.float64)
    cos = np.abs((base["normal"] * d64).sum(1)) / np.linalg.norm(d64, axis=1)
    hit = ok & (base["prim_id"] >= 0) & (cos >= 0.01)
    t_ref = base["t"][hit]
    t_tol = H.t_tolerance(t_ref, d[hit].astype(np.float64), base["normal"][hit], scale)
    t_bad = np.abs(g["t"][hit] - t_ref) > t_tol
    if bad.any() or t_bad.any():
        H.dump(f"intersect_fail_{len(o)}_{int(scale)}", o=o, d=d, gpu_prim=g["prim_id"], gpu_t=g["t"],
               ref_prim=base["prim_id"], ref_t=base["t"], ok=ok)
    assert bad.sum() == 0, f"{bad.sum()} robust rays disagree on prim id (of {ok.sum()})"
    assert not t_bad.any(), f"{t_bad.sum()} t errors above tolerance, worst excess {(np.abs(g['t'][hit] - t_ref) / t_tol).max()}"
    n_err = np.abs(g["normal"][hit] - base["normal"][hit]).max(axis=1)
    assert n_err.max(initial=0) <= N_TOL, f"max normal error {n_err.max()}"
    assert (g["front_face"][hit] == base["front_face"][hit]).all()
    assert (g["material"][hit] == base["material"][hit]).all()
    # occlusion queries with the same rays, tmax = 0.5 * closest t (or 10 on misses)
    tm = np.where(base["prim_id"] >= 0, 0.5 * base["t"], 10.0).astype(np.float32)
    orc_occ = orc.occluded(_occ_rays(o, d, tmin, tm))
    gpu_occ = gpu.occluded(_gpu_occ_rays(o, d, tmin, tm))
    assert (orc_occ[ok] == gpu_occ[ok]).mean() >= 0.999
    return ok.mean(), hit.sum()


def _occ_rays(o, d, tmin, tm):
    r = H.to_orc_rays(o, d, tmin, np.inf)
    r["tmax"] = tm.astype(np.float64)
    return r


def _gpu_occ_rays(o, d, tmin, tm):
    r = H.to_gpu_rays(o, d, tmin, np.inf)
    r["tmax"] = tm
    return r


@pytest.mark.parametrize("name", ["box_room", "random_spheres", "diff_quads"])
def test_ray_sets_match_oracle(name):
    rng = np.random.default_rng(123)
    world, cfg = W.CONFIGS[name]()
    bounds = {"box_room": ((1, 1, 1), (554, 554, 554), 555.0),
              "random_spheres": ((-11, 0.01, -11), (11, 3, 11), 22.0),
              "diff_quads": ((-5, -5, -5), (5, 5, 5), 10.0)}[name]
    n = 20000
    o, d, tmin, tmax = H.random_rays(rng, n, bounds[0], bounds[1])
    compare_sets(world, o, d, tmin, tmax, bounds[2], rng)
    o, d, tmin, tmax = H.camera_rays(world, cfg, rng, n)
    compare_sets(world, o, d, tmin, tmax, bounds[2], rng)
    o2, d2, tmin, tmax, n2 = H.secondary_rays(O.OracleScene(world), o, d, tmin, tmax, rng)
    compare_sets(world, o2, d2, tmin, tmax, bounds[2], rng, min_robust=0.8, normals=n2)


def test_ray_sets_dense_mesh_match_oracle():
    # 81,920 triangles + plane, disks and the fog box.  Geometric robustness is judged on
    # the fog-free world; fog decisions (the reference's hash of the exact ray) must match.
    rng = np.random.default_rng(7)
    world, cfg = W.dense_mesh(level=6)
    clear, _ = W.dense_mesh(level=6, fog=False)
    o, d, tmin, tmax = H.camera_rays(world, cfg, rng, 20000)
    compare_sets(world, o, d, tmin, tmax, 2.0, rng, robust_world=clear)
    o, d, tmin, tmax = H.random_rays(rng, 20000, (-2, -1, -2), (2, 2, 2))
    compare_sets(world, o, d, tmin, tmax, 2.0, rng, min_robust=0.97, robust_world=clear)


def test_transformed_boxes_prim_ids():
    # box_room: the two rotated boxes are prims 0..11; camera rays that hit them agree
    rng = np.random.default_rng(5)
    world, cfg = W.box_room()
    o, d, tmin, tmax = H.camera_rays(world, cfg, rng, 20000)
    orc = O.OracleScene(world)
    base, ok = H.robust_mask(orc, o, d, tmin, tmax, rng, 555.0)
    g = L.GpuScene(world).intersect(H.to_gpu_rays(o, d, tmin, tmax))
    box_hits = ok & (base["prim_id"] < 12) & (base["prim_id"] >= 0)
    assert box_hits.sum() > 1000
    assert (g["prim_id"][box_hits] == base["prim_id"][box_hits]).all()
    np.testing.assert_allclose(g["u"][box_hits], base["u"][box_hits], atol=1e-3)
    np.testing.assert_allclose(g["v"][box_hits], base["v"][box_hits], atol=1e-3)
