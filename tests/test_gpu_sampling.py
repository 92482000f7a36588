"""GPU adaptive sampling and time limit (k_render_sampled) against the oracle.

The device and the oracle's keyed mode trace the same paths, so an adaptive pixel stops at
the same sample count on both unless an f32/f64 difference moves its standard error across
the threshold at the stopping sample: sample totals agree within 1%, and >= 97% of pixels
agree within the keyed tolerance of the plain render (2e-3 * (1 + |ref|) per channel).
"""
import numpy as np
import pytest

import luminara_b200 as L
import oracle as O
from luminara_b200 import RenderConfig
from luminara_b200 import workloads as W

pytestmark = pytest.mark.gpu


def scene(name, w, h, spp):
    world, cfg = W.CONFIGS[name]()
    cfg.width, cfg.height, cfg.samples_per_pixel = w, h, spp
    world.camera.aspect_ratio = w / h
    return world, cfg


def with_(cfg, **kw):
    return RenderConfig(**{**cfg.__dict__, **kw})


def close_frac(img, ref):
    return (np.abs(img - ref) <= 2e-3 * (1.0 + np.abs(ref))).all(axis=2).mean()


@pytest.mark.parametrize("name,w,h,spp,thr", [("box_room", 48, 32, 64, 0.01), ("random_spheres", 64, 36, 64, 0.03),
                                              ("diff_quads", 40, 40, 36, 0.03), ("box_room", 37, 29, 10, 0.003)])
def test_adaptive_matches_oracle(name, w, h, spp, thr):
    world, cfg = scene(name, w, h, spp)
    cfg = with_(cfg, adaptive=True, adaptive_threshold=thr)
    img, st = L.GpuScene(world).render(cfg)
    ref, ost = O.OracleScene(world).render(cfg, mode=O.MODE_KEYED)
    assert st.error_flags == 0
    assert abs(st.paths - ost.paths) <= 0.01 * ost.paths, (st.paths, ost.paths)
    assert close_frac(img, ref) >= 0.97


def test_adaptive_limits_on_the_device():
    world, cfg = scene("box_room", 40, 24, 64)
    sc = L.GpuScene(world)
    full, st_full = sc.render(cfg)
    # threshold 0 never stops: the plain mean of all strata (box filter)
    never, st = sc.render(with_(cfg, adaptive=True, adaptive_threshold=0.0))
    np.testing.assert_allclose(never, full, rtol=2e-6, atol=1e-7)
    assert st.paths == st_full.paths
    # a huge threshold stops every pixel at 16 strata, taken in order
    first, _ = sc.render(with_(cfg, sample_count=16))
    early, st = sc.render(with_(cfg, adaptive=True, adaptive_threshold=1e30))
    np.testing.assert_allclose(early, first, rtol=2e-6, atol=1e-7)
    assert st.paths == 40 * 24 * 16
    assert st.segments < st_full.segments / 2


def test_time_limit_far_away_is_the_plain_render_bit_for_bit():
    world, cfg = scene("box_room", 40, 24, 16)
    sc = L.GpuScene(world)
    full, st_full = sc.render(cfg)
    far, st = sc.render(with_(cfg, time_limit=1e6))
    np.testing.assert_array_equal(far, full)
    assert st.paths == st_full.paths


def tiles_equal(img, ref):
    """Per pixel: whether the pixel's 8x4 tile equals ref's bit for bit."""
    h, w, _ = img.shape
    out = np.zeros((h, w), bool)
    for y0 in range(0, h, 4):
        for x0 in range(0, w, 8):
            t = (slice(y0, y0 + 4), slice(x0, x0 + 8))
            out[t] = np.array_equal(img[t], ref[t])
    return out


@pytest.mark.parametrize("adaptive", [False, True])
def test_time_limit_expired_tiles_take_one_centre_sample(adaptive):
    # A 1 ns limit.  %globaltimer ticks coarsely, so tiles of the first wave may still read
    # the start stamp and start "in time"; a frame with more tiles (64 x 64) than resident
    # warps has later tiles that start after the first ones finish, certainly expired.  A
    # tile that started in time equals the render without the limit bit for bit.
    world, cfg = scene("box_room", 512, 256, 16)
    cfg = with_(cfg, adaptive=adaptive, adaptive_threshold=0.01)
    sc = L.GpuScene(world)
    full, _ = sc.render(cfg)
    img, st = sc.render(with_(cfg, time_limit=1e-9))
    assert st.error_flags == 0
    ref, _ = O.OracleScene(world).render(cfg, mode=O.MODE_KEYED, expired=True)
    # tiles equal to the plain render: those that started in time, and expired tiles whose
    # pixels are constant either way (black outside the room, the light's clamped emission)
    maybe_started = tiles_equal(img, full)
    close = (np.abs(img - ref) <= 2e-3 * (1.0 + np.abs(ref))).all(axis=2)
    assert close[~maybe_started].mean() >= 0.97
    if not adaptive:
        n = 512 * 256
        started_px, rem = divmod(st.paths - n, 15)           # 16 samples per started pixel, 1 per expired
        assert rem == 0 and started_px % 32 == 0
        assert started_px <= maybe_started.sum() and started_px <= 0.8 * n


def test_adaptive_crop_and_ldr():
    world, cfg = scene("random_spheres", 64, 36, 16)
    cfg = with_(cfg, adaptive=True, adaptive_threshold=0.03)
    sc = L.GpuScene(world)
    img, _ = sc.render(cfg)
    crop, st = sc.render(with_(cfg, crop=(8, 4, 24, 20)))
    np.testing.assert_array_equal(crop, img[4:24, 8:32])
    ldr, _ = sc.render_ldr(cfg, L.ToneMapConfig())
    assert ldr.shape == (36, 64, 4) and ldr[..., :3].max() > 100


def test_zero_spp_and_depth_zero():
    world, cfg = scene("box_room", 16, 8, 0)
    sc = L.GpuScene(world)
    img, st = sc.render(with_(cfg, adaptive=True))
    assert not img.any() and st.paths == 0
    img, st = sc.render(with_(cfg, samples_per_pixel=16, max_depth=0, adaptive=True))
    assert not img.any()
    # the time limit's centre sample does not depend on spp (render.rs:1612-1622): expired
    # tiles trace one path per pixel, tiles that started in time none
    world, cfg = scene("box_room", 512, 256, 0)
    img, st = L.GpuScene(world).render(with_(cfg, time_limit=1e-9))
    black = tiles_equal(img, np.zeros_like(img))     # started in time (or an all-black expired tile)
    assert 0 < (~black).sum() <= st.paths <= 512 * 256 and st.paths % 32 == 0


def test_sampled_renders_reject_partial_strata_and_other_entry_points():
    world, cfg = scene("box_room", 16, 8, 16)
    sc = L.GpuScene(world)
    with pytest.raises(L.LuminaraError):
        sc.render(with_(cfg, adaptive=True, sample_begin=4))
    with pytest.raises(L.LuminaraError):
        sc.render(with_(cfg, time_limit=1.0, sample_count=4))
    with pytest.raises(L.LuminaraError):
        L.Batch([sc], [with_(cfg, adaptive=True)], config="default")
    with pytest.raises(L.LuminaraError):
        sc.forward(with_(cfg, time_limit=1.0))
