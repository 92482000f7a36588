"""The headline frame at its full size (random spheres 1920x1080, 256 spp, depth 16) through
properties that do not need a full oracle render: the frame is deterministic, the two halves
of its stratum range combine to it (linearity of the estimator), and sampled rows agree with
the reference estimator (oracle stream mode) within their standard error."""
import numpy as np
import pytest

import luminara_b200 as L
import oracle as O
from luminara_b200 import workloads as W
from tests import helpers as H

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def headline():
    world, cfg = W.random_spheres()
    sc = L.GpuScene(world)
    img, st = sc.render(cfg)
    return world, cfg, sc, img, st


def test_full_frame_is_deterministic(headline):
    world, cfg, sc, img, st = headline
    assert img.shape == (1080, 1920, 3) and np.isfinite(img).all()
    assert st.paths == 1920 * 1080 * 256 and st.error_flags == 0
    again, st2 = sc.render(cfg)
    assert np.array_equal(again, img) and st2.segments == st.segments


def test_full_frame_stratum_halves_combine(headline):
    world, cfg, sc, img, st = headline
    cfg.sample_begin, cfg.sample_count = 0, 128
    a, sa = sc.render(cfg)
    cfg.sample_begin, cfg.sample_count = 128, 128
    b, sb = sc.render(cfg)
    cfg.sample_begin, cfg.sample_count = 0, 0
    assert sa.paths + sb.paths == st.paths and sa.segments + sb.segments == st.segments
    np.testing.assert_allclose(0.5 * (a + b), img, rtol=1e-4, atol=1e-6)


@pytest.mark.parametrize("row", [300, 700, 1000])
def test_full_frame_rows_match_reference_estimator(headline, row):
    world, cfg, sc, img, st = headline
    ref, _ = O.OracleScene(world).render(cfg, mode=O.MODE_STREAM, rows=(row, row + 1))
    lg, lr = H.luminance(img[row]), H.luminance(ref[row])
    d = lg - lr
    se = d.std() / np.sqrt(d.size)
    assert abs(d.mean()) <= 4.0 * se + 1e-3 * abs(lr.mean()), (row, d.mean(), se)
