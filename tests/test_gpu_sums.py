"""GPU tests of the raw per-pixel sums (lum_render_sums_device / lum_sums_finalize_device) that
split frames combine through.

The reference's pixel is the ratio of two per-pixel sums over its samples (render.rs:1692-1705).
Stratum shards rendered as raw 64-bit fixed-point sums and added as integers must give
lum_render's full frame bit for bit, for every pixel filter; the sums must also equal the
oracle's f64 sums (keyed mode) within the keyed tolerance.  The multi-rank helper
(distributed.render_frame_sharded) is run as one NCCL rank on this GPU.
"""
import os
import socket

import numpy as np
import pytest
import torch

import luminara_b200 as L
import oracle as O
from luminara_b200 import distributed as D
from luminara_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _frame(flt, w=72, h=40, spp=16):
    world, cfg = W.box_room(width=w, height=h, spp=spp)
    world.camera.aspect_ratio = w / h
    cfg.pixel_filter = flt
    return world, cfg


@pytest.mark.parametrize("flt", [0, 1, 2, 3])
def test_stratum_shard_sums_combine_to_the_full_frame(flt):
    world, cfg = _frame(flt)
    sc = L.GpuScene(world)
    full, _ = sc.render(cfg)
    h, w, _ = cfg.out_shape()
    total = torch.zeros((h, w, 4), dtype=torch.int64, device="cuda")
    part = torch.empty_like(total)
    for r in range(3):                                  # three uneven shards: 6 + 5 + 5 strata
        pc, _ = D.shard_config(cfg, r, 3)
        st = sc.render_sums_device(pc, part.data_ptr())
        assert st.error_flags == 0 and st.paths == h * w * pc.sample_count
        total += part
    out = torch.empty((h, w, 3), dtype=torch.float32, device="cuda")
    L.sums_finalize_device(total.data_ptr(), w, h, cfg.exposure, out.data_ptr())
    torch.cuda.synchronize()
    np.testing.assert_array_equal(out.cpu().numpy(), full)
    # against the oracle's f64 sums of the same keyed paths
    ref, _ = O.OracleScene(world).render_sums(cfg, mode=O.MODE_KEYED)
    got = total.cpu().numpy().astype(np.float64) / 2.0 ** 32
    close = np.abs(got - ref) <= 2e-3 * (1.0 + np.abs(ref)) * cfg.samples_per_pixel
    assert close.all(axis=2).mean() >= 0.97
    np.testing.assert_allclose(got[..., 3], ref[..., 3], rtol=1e-5)      # filter weights: jitter only


def test_sharded_helper_as_one_nccl_rank():
    import torch.distributed as dist

    world, cfg = _frame(3)
    sc = L.GpuScene(world)
    full, _ = sc.render(cfg)
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("nccl", rank=0, world_size=1, device_id=torch.device("cuda", 0))
    try:
        out = D.render_frame_sharded(sc, cfg, 0, 1)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(out.cpu().numpy(), full)
    finally:
        dist.destroy_process_group()
