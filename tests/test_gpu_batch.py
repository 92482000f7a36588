"""GPU tests of the batched tracer (lum_batch_*), both modes.

Every path is traced from the same RNG key by the same device functions, and every kernel adds
finished paths to 64-bit fixed-point pixel sums (integer sums do not depend on the order in
which paths finish), so each scene's image must equal lum_render's bit for bit.
"""
import numpy as np
import pytest

import luminara_b200 as L
from luminara_b200 import abi
from luminara_b200 import workloads as W

pytestmark = pytest.mark.gpu


def small_batch():
    rng = np.random.default_rng(11)
    items = [W.uneven_scene(rng, n, w, h, spp) for n, w, h, spp in
             [(12, 32, 24, 4), (300, 48, 32, 16), (2000, 40, 40, 9), (50, 24, 24, 64)]]
    w, c = W.box_room(width=40, height=40, spp=16)
    items.append((w, c))
    w, c = W.random_spheres(width=48, height=27, spp=16)
    w.camera.aspect_ratio = 48 / 27
    items.append((w, c))
    w, c = W.dense_mesh(level=4, width=32, height=18, spp=4)
    w.camera.aspect_ratio = 32 / 18
    items.append((w, c))
    return items


def compare(img, ref):
    np.testing.assert_array_equal(img, ref)


@pytest.mark.parametrize("sort_threshold", [0, 1 << 16, 0xFFFFFFFF])
def test_batch_matches_megakernel(sort_threshold):
    items = small_batch()
    scenes = [L.GpuScene(w) for w, _ in items]
    cfgs = [c for _, c in items]
    refs = [s.render(c)[0] for s, c in zip(scenes, cfgs)]
    b = L.Batch(scenes, cfgs, config={"pool_paths": 1 << 16, "block_threads": 128,
                                      "sort_threshold": sort_threshold, "iters_per_graph": 4})
    imgs, done, st = b.render()
    assert st.error_flags == 0
    assert st.paths == sum(int(np.prod(c.out_shape()[:2])) * int(np.ceil(np.sqrt(c.samples_per_pixel))) ** 2
                           for c in cfgs)
    for img, ref in zip(imgs, refs):
        compare(img, ref)
    assert all(0 < t <= st.device_ms + 1e-3 for t in done)
    b.close()


def test_batch_is_deterministic_and_refills_a_small_pool():
    items = small_batch()
    scenes = [L.GpuScene(w) for w, _ in items]
    cfgs = [c for _, c in items]
    b = L.Batch(scenes, cfgs, config={"pool_paths": 4096, "block_threads": 256, "sort_threshold": 1024,
                                      "iters_per_graph": 8})
    a, _, st1 = b.render()
    c, _, st2 = b.render()
    for x, y in zip(a, c):
        assert np.array_equal(x, y)
    assert st1.iterations > 20 and st1.graph_launches >= 3
    assert st1.segments == st2.segments
    refs = [s.render(cf)[0] for s, cf in zip(scenes, cfgs)]
    for img, ref in zip(a, refs):
        compare(img, ref)


@pytest.mark.parametrize("mode", [abi.BATCH_MEGAKERNEL, abi.BATCH_STREAMS])
def test_megakernel_modes_equal_lum_render(mode):
    items = small_batch()
    scenes = [L.GpuScene(w) for w, _ in items]
    cfgs = [c for _, c in items]
    refs = [s.render(c)[0] for s, c in zip(scenes, cfgs)]
    b = L.Batch(scenes, cfgs, config={"mode": mode})
    imgs, done, st = b.render()
    assert st.error_flags == 0 and st.segments > 0
    for img, ref in zip(imgs, refs):
        compare(img, ref)
    assert all(0 < t <= st.device_ms + 1e-3 for t in done)


@pytest.mark.parametrize("mode,pixel_filter", [(abi.BATCH_WAVEFRONT, abi.FILTER_GAUSSIAN),
                                               (abi.BATCH_WAVEFRONT, abi.FILTER_MITCHELL),
                                               (abi.BATCH_MEGAKERNEL, abi.FILTER_TRIANGLE),
                                               (abi.BATCH_STREAMS, abi.FILTER_GAUSSIAN)])
def test_batch_device_outputs_and_filters(mode, pixel_filter):
    import torch
    items = small_batch()[:3]
    for _, c in items:
        c.pixel_filter = pixel_filter
        c.exposure = 0.5
    scenes = [L.GpuScene(w) for w, _ in items]
    cfgs = [c for _, c in items]
    refs = [s.render(c)[0] for s, c in zip(scenes, cfgs)]
    outs = [torch.empty(c.out_shape(), dtype=torch.float32, device="cuda") for c in cfgs]
    b = L.Batch(scenes, cfgs, config={"mode": mode})
    b.render_device([o.data_ptr() for o in outs])
    for o, ref in zip(outs, refs):
        compare(o.cpu().numpy(), ref)


def test_autotuner_picks_and_caches(tmp_path, monkeypatch):
    monkeypatch.setenv("LUM_AUTOTUNE_CACHE", str(tmp_path / "tune.txt"))
    items = small_batch()[:4]
    scenes = [L.GpuScene(w) for w, _ in items]
    cfgs = [c for _, c in items]
    cfg, ms = L.autotune(scenes, cfgs)
    assert ms > 0 and cfg["mode"] in (abi.BATCH_WAVEFRONT, abi.BATCH_MEGAKERNEL, abi.BATCH_STREAMS)
    assert cfg["mode"] != abi.BATCH_WAVEFRONT or cfg["pool_paths"] in (1 << 19, 1 << 20, 1 << 21)
    cfg2, ms2 = L.autotune(scenes, cfgs)
    assert cfg2 == cfg and ms2 == -1.0
    b = L.Batch(scenes, cfgs)            # autotuned (cache hit)
    assert b.config() == cfg
    imgs, _, st = b.render()
    assert st.error_flags == 0


def _benchmark_scenes(n=6):
    """n scenes of the 64-scene benchmark batch (workloads.batched()), smallest to largest
    primitive count, at their own resolutions."""
    items = W.batched()
    counts = [w.n_prims() for w, _ in items]
    order = np.argsort(counts)
    return [items[int(order[k])] for k in np.linspace(0, len(order) - 1, n).round().astype(int)]


@pytest.mark.parametrize("mode", [abi.BATCH_WAVEFRONT, abi.BATCH_MEGAKERNEL, abi.BATCH_STREAMS])
def test_benchmark_batch_scenes_match_keyed_oracle(mode):
    """Scenes of the 64-scene benchmark batch itself (uneven primitive counts, resolutions and
    materials -- spheres, quads and triangles, Lambertian / Metal / Dielectric / GGX, sphere and
    rect lights) rendered through the batch API and compared with the oracle's keyed mode, not
    with another device kernel: six scenes from 15 to 36,259 primitives, 128^2 to 1024^2, one
    stratum per pixel, so a pixel differs only where its one path took another discrete decision
    (f32 against f64: a hit, a Russian-roulette or lobe choice flipping).  Tolerance of the keyed
    render tests: >= 97% of pixels within 2e-3 * (1 + |ref|) per channel, image means within
    0.5%, traced segments within 1%.  In the densest scene (36,259 small interpenetrating
    primitives) about 1.7% of the paths take another decision, so at several strata per pixel the
    share of pixels touched by one grows past 3% (4 strata: 94%); the converged check below
    covers that scene's statistics."""
    import oracle as O

    picked = _benchmark_scenes()
    worlds = [w for w, _ in picked]
    cfgs = [c for _, c in picked]
    for c in cfgs:
        c.samples_per_pixel = 1
    scenes = [L.GpuScene(w) for w in worlds]
    b = L.Batch(scenes, cfgs, config={"mode": mode, "pool_paths": 1 << 18})
    imgs, _, st = b.render()
    assert st.error_flags == 0
    for w, c, img in zip(worlds, cfgs, imgs):
        ref, ost = O.OracleScene(w).render(c, mode=O.MODE_KEYED)
        close = np.abs(img - ref) <= 2e-3 * (1.0 + np.abs(ref))
        frac = close.all(axis=2).mean()
        assert frac >= 0.97, (w.n_prims(), c.width, frac)
        m_g, m_r = img.mean(axis=(0, 1)), ref.mean(axis=(0, 1))
        assert np.all(np.abs(m_g - m_r) <= 5e-3 * np.maximum(m_r, 1e-3)), (w.n_prims(), m_g, m_r)
    b.close()


def test_densest_benchmark_batch_scene_converges_to_reference_estimator():
    """The densest scene of the benchmark batch (36,259 primitives, 512^2): the batch's image at
    256 spp against the reference estimator (oracle stream mode) at 64 spp must have an RMSE no
    larger than 1.15x that of a second, independent 64-spp reference render, and a mean-luminance
    bias within 4 standard errors."""
    import oracle as O
    from tests import helpers as H

    w, c = _benchmark_scenes()[-1]
    assert w.n_prims() > 30000
    c.samples_per_pixel = 256
    b = L.Batch([L.GpuScene(w)], [c], config={"mode": abi.BATCH_WAVEFRONT, "pool_paths": 1 << 20})
    g = b.render()[0][0]
    b.close()
    c.samples_per_pixel = 64
    r1, _ = O.OracleScene(w).render(c, mode=O.MODE_STREAM)
    c.seed += 17
    r2, _ = O.OracleScene(w).render(c, mode=O.MODE_STREAM)
    assert H.rmse(g, r1) <= 1.15 * H.rmse(r2, r1), (H.rmse(g, r1), H.rmse(r2, r1))
    d = (H.luminance(g) - H.luminance(r1)).ravel()
    assert abs(d.mean()) <= 4.0 * d.std() / np.sqrt(d.size)
