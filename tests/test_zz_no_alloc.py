"""GPU test of lum_render_noalloc, the allocation-free render entry point.

Some callers cannot call cudaMalloc while rendering: services that reserve the device's
memory at start-up, or whose free memory is held by another allocator's pool, where a
render-time allocation would fail or stall on device-wide synchronisation.  For them
lum_render_noalloc keeps the device image and the kernel's counters in one fixed array
(LUM_NOALLOC_MAX_PIXELS pixels) instead of allocating.  This file checks, through the C ABI,
that two calls in a row return the same image as lum_render, bit for bit (same kernel and
seeds; pixel sums in 64-bit fixed point do not depend on path order), that the shared array is
reused cleanly by a call with another scene and size, that renders leave the device's free
memory unchanged, and that images beyond the maximum and the adaptive / time-limited sample
loop are rejected.  It is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

import luminara_b200 as L
from luminara_b200 import abi
from luminara_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _noalloc():
    f = L.lib().lum_render_noalloc
    f.argtypes = [C.c_void_p, C.POINTER(abi.LumRenderParams), C.c_void_p, C.POINTER(abi.LumStats)]
    f.restype = C.c_int32
    return f


def _call(scene, cfg):
    p = cfg.to_c()
    out = np.full(cfg.out_shape(), np.nan, dtype=np.float32)
    st = abi.LumStats()
    rc = _noalloc()(scene.h, C.byref(p), out.ctypes.data, C.byref(st))
    return rc, out, st


def test_noalloc_matches_render_on_two_calls_in_a_row():
    world, cfg = W.box_room(width=96, height=64, spp=16)
    world.camera.aspect_ratio = 96 / 64
    sc = L.GpuScene(world)
    ref, ref_st = sc.render(cfg)
    for _ in range(2):
        rc, out, st = _call(sc, cfg)
        assert rc == abi.LUM_OK, L.lib().lum_last_error()
        # lum_render splits this small frame's strata into groups, the allocation-free path does
        # not; both add the same paths in 64-bit fixed point, so the images are identical
        np.testing.assert_array_equal(out, ref)
        assert st.paths == ref_st.paths == 96 * 64 * 16
        assert st.segments == ref_st.segments and st.error_flags == 0


def test_noalloc_reuses_the_shared_array_across_scenes_and_sizes():
    world, cfg = W.random_spheres(width=128, height=72, spp=4)
    world.camera.aspect_ratio = 128 / 72
    sc = L.GpuScene(world)
    ref, _ = sc.render(cfg)
    rc, out, _ = _call(sc, cfg)
    assert rc == abi.LUM_OK, L.lib().lum_last_error()
    np.testing.assert_array_equal(out, ref)
    cfg.crop = (10, 5, 40, 30)                 # smaller region after a larger one
    ref2, _ = sc.render(cfg)
    rc, out2, _ = _call(sc, cfg)
    assert rc == abi.LUM_OK, L.lib().lum_last_error()
    np.testing.assert_array_equal(out2, ref2)


def test_noalloc_rejects_images_beyond_the_maximum():
    world, cfg = W.box_room(width=2048, height=1024, spp=1)   # 2^21 pixels > 2^20
    sc = L.GpuScene(world)
    rc, _, _ = _call(sc, cfg)
    assert rc == abi.LUM_ERR_TOO_LARGE
    assert b"maximum" in L.lib().lum_last_error()


def test_noalloc_allocates_no_device_memory():
    """The property the entry point exists for: once a device is set up (scenes created, which
    loads the module holding the fixed array), renders of other scenes and sizes leave the
    device's free memory unchanged.  Both scenes render once first, so each kernel build has
    been launched (a first launch may grow the driver's per-context local-memory reserve)."""
    import torch

    w1, c1 = W.box_room(width=64, height=64, spp=4)
    w2, c2 = W.random_spheres(width=96, height=54, spp=4)
    s1, s2 = L.GpuScene(w1), L.GpuScene(w2)
    for sc, cfg in ((s1, c1), (s2, c2)):
        rc, _, _ = _call(sc, cfg)
        assert rc == abi.LUM_OK, L.lib().lum_last_error()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    c1.width, c1.height, c1.samples_per_pixel = 512, 384, 9
    w1.camera.aspect_ratio = 512 / 384
    c2.width, c2.height = 1024, 1024                     # the maximum size
    c2.crop = None
    for sc, cfg in ((s1, c1), (s2, c2), (s1, c1)):
        rc, out, st = _call(sc, cfg)
        assert rc == abi.LUM_OK, L.lib().lum_last_error()
        assert np.isfinite(out).all() and st.error_flags == 0
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, f"free device memory moved by {free0 - free1} bytes"


def test_noalloc_rejects_adaptive_sampling_and_time_limit():
    world, cfg = W.box_room(width=32, height=32, spp=16)
    sc = L.GpuScene(world)
    cfg.adaptive = True
    rc, _, _ = _call(sc, cfg)
    assert rc == abi.LUM_ERR_UNSUPPORTED
    cfg.adaptive = False
    cfg.time_limit = 1.0
    rc, _, _ = _call(sc, cfg)
    assert rc == abi.LUM_ERR_UNSUPPORTED
