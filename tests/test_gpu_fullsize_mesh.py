"""The dense-mesh workload at its full size: the level-8 displaced icosphere (1,310,720
triangles, GGX per 1k-triangle patch), ground plane, three disk lights and the fog box, at
1920x1080, 128 spp (144 strata), depth 8.

* Intersection: 20,000 camera rays and 20,000 interior rays against the f64 oracle with the
  rules of test_gpu_intersect (hit/miss and primitive id exact on robust rays, t and normal
  within tolerance), on the real 1.31 M-triangle BVH (reference traversal: bvh.rs:52-68;
  triangle test: triangle.rs:21-64).
* Rendering: three full-width rows of the full frame against the reference estimator (oracle
  stream mode, the reference's per-row SmallRng sample loop) in mean luminance, within 4
  standard errors of the per-pixel difference, as test_gpu_fullsize does for the headline frame.
"""
import numpy as np
import pytest

import luminara_b200 as L
import oracle as O
from luminara_b200 import workloads as W
from tests import helpers as H
from tests.test_gpu_intersect import compare_sets

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mesh():
    world, cfg = W.dense_mesh()
    clear, _ = W.dense_mesh(fog=False)
    return world, cfg, clear


def test_full_mesh_ray_sets_match_oracle(mesh):
    world, cfg, clear = mesh
    assert world.n_prims() > 1_300_000
    rng = np.random.default_rng(17)
    o, d, tmin, tmax = H.camera_rays(world, cfg, rng, 20000)
    compare_sets(world, o, d, tmin, tmax, 2.0, rng, robust_world=clear)
    o, d, tmin, tmax = H.random_rays(rng, 20000, (-2, -1, -2), (2, 2, 2))
    compare_sets(world, o, d, tmin, tmax, 2.0, rng, min_robust=0.97, robust_world=clear)


def test_full_mesh_rows_match_reference_estimator(mesh):
    world, cfg, _ = mesh
    sc = L.GpuScene(world)
    img, st = sc.render(cfg)
    assert img.shape == (1080, 1920, 3) and np.isfinite(img).all()
    assert st.paths == 1920 * 1080 * 144 and st.error_flags == 0
    rows = [300, 700, 1000]
    ref, _ = O.OracleScene(world).render_row_list(cfg, rows, mode=O.MODE_STREAM)
    for k, row in enumerate(rows):
        lg, lr = H.luminance(img[row]), H.luminance(ref[k])
        d = lg - lr
        se = d.std() / np.sqrt(d.size)
        assert abs(d.mean()) <= 4.0 * se + 1e-3 * abs(lr.mean()), (row, d.mean(), se)
