"""GPU tests of the kernels' error paths: each failure is provoked on the host side, by a
diagnostic limit, so no GPU faults, traps or hangs.

* Traversal stack overflow.  LUM_STACK_BUDGET (read by lum_scene_create) caps the traversal
  stack below the depth the scene's BVH needs.  The push is bounds-checked against that cap:
  an overflowing push sets LUM_KERR_STACK_OVERFLOW and drops the far subtree, the kernel runs
  to its end, and the entry point returns LUM_ERR_KERNEL with the flag in lum_stats.
* Wavefront iteration cap.  LUM_BATCH_MAX_LAUNCHES caps the host's graph relaunch loop below
  what the batch needs; the batch returns LUM_ERR_KERNEL with LUM_KERR_ITERATION_CAP, and the
  next render of the same batch (without the cap) is complete and equal to lum_render's.

The reference has no counterpart on the GPU; its renderer is infallible (render.rs:1563-1569
clamps its inputs) and its scene loader returns Err(String) (scene.rs:846).
"""
import ctypes as C

import numpy as np
import pytest

import luminara_b200 as L
from luminara_b200 import abi
from luminara_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _render_raw(sc, cfg):
    p = cfg.to_c()
    out = np.empty(cfg.out_shape(), dtype=np.float32)
    st = abi.LumStats()
    rc = L.lib().lum_render(sc.h, C.byref(p), out.ctypes.data, C.byref(st))
    return rc, out, st


def test_stack_overflow_reaches_the_caller(monkeypatch):
    world, cfg = W.random_spheres(width=64, height=36, spp=4)
    ok_scene = L.GpuScene(world)
    ref, ref_st = ok_scene.render(cfg)
    assert ref_st.error_flags == 0
    monkeypatch.setenv("LUM_STACK_BUDGET", "2")
    small = L.GpuScene(world)                 # the budget is read when the scene is created
    monkeypatch.delenv("LUM_STACK_BUDGET")
    rc, out, st = _render_raw(small, cfg)
    assert rc == abi.LUM_ERR_KERNEL, L.lib().lum_last_error()
    assert st.error_flags & abi.KERR_STACK_OVERFLOW
    assert b"error flags" in L.lib().lum_last_error()
    # the kernel finished every path (skipped subtrees read as misses): the frame is complete
    # and finite, and differs from the full traversal's
    assert st.paths == ref_st.paths and np.isfinite(out).all()
    assert not np.array_equal(out, ref)
    # the ray-set entry point reports the same flag
    rays = L.make_rays(np.tile(world.camera.look_from, (256, 1)),
                       np.random.default_rng(3).normal(size=(256, 3)) + np.array([0.0, 0.0, -2.0]))
    with pytest.raises(L.LuminaraError) as e:
        small.intersect(rays)
    assert e.value.status == abi.LUM_ERR_KERNEL
    # the context stays usable: the scene without the cap renders its exact image again
    img, st2 = ok_scene.render(cfg)
    assert st2.error_flags == 0
    np.testing.assert_array_equal(img, ref)
    small.close()
    ok_scene.close()


def test_wavefront_iteration_cap_reaches_the_caller(monkeypatch):
    items = W.batched(n_scenes=4, res_choices=(64,), seed=11)
    scenes = [L.GpuScene(w) for w, _ in items]
    cfgs = [c for _, c in items]
    refs = [s.render(c)[0] for s, c in zip(scenes, cfgs)]
    batch = L.Batch(scenes, cfgs, config={"mode": abi.BATCH_WAVEFRONT, "pool_paths": 4096,
                                          "iters_per_graph": 1})
    n = len(scenes)
    imgs = [np.zeros(c.out_shape(), dtype=np.float32) for c in cfgs]
    ptrs = (C.c_void_p * n)(*[im.ctypes.data for im in imgs])
    done = (C.c_double * n)()
    st = abi.LumBatchStats()
    monkeypatch.setenv("LUM_BATCH_MAX_LAUNCHES", "2")
    rc = L.lib().lum_batch_render(batch.h, C.cast(ptrs, C.POINTER(C.c_void_p)), done, C.byref(st))
    monkeypatch.delenv("LUM_BATCH_MAX_LAUNCHES")
    assert rc == abi.LUM_ERR_KERNEL, L.lib().lum_last_error()
    assert st.error_flags & abi.KERR_ITERATION_CAP
    assert st.graph_launches == 2
    assert b"0x4" in L.lib().lum_last_error()
    # without the cap the same batch completes and equals lum_render bit for bit
    out, _, st2 = batch.render()
    assert st2.error_flags == 0
    for a, b in zip(out, refs):
        np.testing.assert_array_equal(a, b)
    batch.close()
    for s in scenes:
        s.close()
