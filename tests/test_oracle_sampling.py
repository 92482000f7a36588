"""The oracle's adaptive sampling and time limit (render.rs:1592-1678) on the CPU.

The adaptive loop is pinned against a pure-Python restatement of the reference's stopping
rule run on the oracle's own per-stratum samples: in keyed mode a render of the single stratum
k with the box filter is that stratum's clamped sample, so the Python loop sees exactly the
values the oracle's loop sees.
"""
import math

import numpy as np
import pytest

import oracle as O
from luminara_b200 import RenderConfig
from luminara_b200 import workloads as W


def scene(name, w, h, spp):
    world, cfg = W.CONFIGS[name]()
    cfg.width, cfg.height, cfg.samples_per_pixel = w, h, spp
    world.camera.aspect_ratio = w / h
    return world, cfg


def with_(cfg, **kw):
    return RenderConfig(**{**cfg.__dict__, **kw})


def welford_pixel(samples, min_samples, threshold):
    """render.rs:1628-1676 for one pixel: (mean colour, samples used)."""
    mean = np.zeros(3)
    mean_lum = m2 = 0.0
    n = 0
    for c in samples:
        n += 1
        lum = 0.2126 * c[0] + 0.7152 * c[1] + 0.0722 * c[2]
        d1 = lum - mean_lum
        mean_lum += d1 / n
        m2 += d1 * (lum - mean_lum)
        mean = mean + (c - mean) / n
        if n >= min_samples and n > 1 and math.sqrt(m2 / (n - 1) / n) < threshold:
            break
    return mean, n


@pytest.mark.parametrize("name,thr", [("box_room", 0.01), ("random_spheres", 0.03), ("diff_quads", 0.03)])
def test_adaptive_matches_python_restatement(name, thr):
    world, cfg = scene(name, 12, 8, 64)
    sc = O.OracleScene(world)
    total = 64
    per = np.stack([sc.render(with_(cfg, sample_begin=k, sample_count=1), mode=O.MODE_KEYED)[0]
                    for k in range(total)], axis=2)                     # (h, w, strata, 3)
    got, st = sc.render(with_(cfg, adaptive=True, adaptive_threshold=thr), mode=O.MODE_KEYED)
    min_samples = max(total // 4, 16)
    used = 0
    for j in range(cfg.height):
        for i in range(cfg.width):
            mean, n = welford_pixel(per[j, i], min_samples, thr)
            used += n
            np.testing.assert_allclose(got[j, i], mean, rtol=1e-12, atol=1e-15)
    assert st.paths == used
    assert 12 * 8 * 16 <= used < 12 * 8 * 64          # some pixels stopped early, not all at once


def test_adaptive_limits():
    world, cfg = scene("box_room", 16, 12, 64)
    sc = O.OracleScene(world)
    full, st_full = sc.render(cfg, mode=O.MODE_KEYED)
    # threshold 0: the test never passes; the pixel is the plain mean of all strata
    never, st = sc.render(with_(cfg, adaptive=True, adaptive_threshold=0.0), mode=O.MODE_KEYED)
    np.testing.assert_allclose(never, full, rtol=1e-12, atol=1e-15)
    assert st.paths == st_full.paths
    # a huge threshold stops every pixel at max(spp/4, 16) = 16 strata, taken in order
    first, _ = sc.render(with_(cfg, sample_count=16), mode=O.MODE_KEYED)
    early, st = sc.render(with_(cfg, adaptive=True, adaptive_threshold=1e30), mode=O.MODE_KEYED)
    np.testing.assert_allclose(early, first, rtol=1e-12, atol=1e-15)
    assert st.paths == 16 * 12 * 16
    # fewer strata than the minimum: never stops early (10 spp -> 16 strata, min 16)
    _, st = sc.render(with_(cfg, samples_per_pixel=4, adaptive=True, adaptive_threshold=1e30), mode=O.MODE_KEYED)
    assert st.paths == 16 * 12 * 4
    # the reference's own estimator (stream mode) takes the same branch
    _, st = sc.render(with_(cfg, adaptive=True, adaptive_threshold=1e30), mode=O.MODE_STREAM)
    assert st.paths == 16 * 12 * 16


def test_adaptive_needs_all_strata():
    world, cfg = scene("box_room", 8, 8, 16)
    with pytest.raises(RuntimeError):
        O.OracleScene(world).render(with_(cfg, adaptive=True, sample_begin=4), mode=O.MODE_KEYED)


@pytest.mark.parametrize("mode", [O.MODE_KEYED, O.MODE_STREAM])
def test_time_limit(mode):
    world, cfg = scene("box_room", 16, 12, 16)
    sc = O.OracleScene(world)
    full, st_full = sc.render(cfg, mode=mode)
    expired, st = sc.render(cfg, mode=mode, expired=True)
    assert st.paths == 16 * 12
    assert np.isfinite(expired).all() and expired.mean() > 0
    # a limit that has passed before the first row starts: every row expired
    tiny, st = sc.render(with_(cfg, time_limit=1e-12), mode=mode)
    np.testing.assert_array_equal(tiny, expired)
    assert st.paths == 16 * 12
    # a limit far away: the plain render
    far, st = sc.render(with_(cfg, time_limit=1e6), mode=mode)
    np.testing.assert_array_equal(far, full)
    assert st.paths == st_full.paths


def test_expired_sample_is_the_pixel_centre():
    # a pinhole camera through an empty scene: the centre sample of pixel (i, j) is the sky
    # at u = (i + 0.5) / (W - 1), v = (H - 1 - j + 0.5) / (H - 1) (render.rs:1612-1616)
    from luminara_b200 import scene as S
    world = S.World()
    world.camera.aspect_ratio = 8 / 6
    cfg = S.RenderConfig(width=8, height=6, samples_per_pixel=4, max_depth=4)
    sc = O.OracleScene(world)
    img, _ = sc.render(cfg, mode=O.MODE_KEYED, expired=True)
    # the sky gradient lerp(white, (0.5, 0.7, 1), (y + 1) / 2) only depends on the ray's unit
    # y, which rises with v: its red falls from the bottom row to the top row
    col = img[:, 3, 0]
    assert np.all(np.diff(col) > 0) and np.all(img[..., 2] == 1.0)
    rng_free, _ = sc.render(cfg, mode=O.MODE_STREAM, expired=True)
    np.testing.assert_allclose(img, rng_free, rtol=1e-12)   # no jitter: both RNGs give the same image


def test_render_config_fields_reach_the_abi():
    c = RenderConfig(adaptive=True, adaptive_threshold=0.5, time_limit=2.5)
    p = c.to_c()
    assert p.adaptive == 1 and p.adaptive_threshold == 0.5 and p.time_limit == 2.5
    assert RenderConfig().to_c().adaptive_threshold == 0.03
