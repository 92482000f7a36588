"""Multi-process (gloo, world size 2, CPU) test of stratum sharding and the frame combine.

Each rank renders the raw per-pixel sums of its stratum range of a small keyed frame with the
oracle (the device's estimator in f64; the sharding logic is the same code the GPU ranks use),
the ranks add them with one all-reduce, and the ratio of the summed sums (render.rs:1705) must
equal the single-process full frame for every pixel filter.  A count-weighted mean of the
shards' pixels, shown beside it, equals the frame only for the box filter.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from luminara_b200 import distributed as D


def test_strata_shards_cover_the_range_once():
    for n in (1, 4, 9, 16, 144, 256):
        for ws in (1, 2, 3, 8):
            got = [D.strata_shard(n, r, ws) for r in range(ws)]
            assert sum(c for _, c in got) == n
            assert got[0][0] == 0
            for (b0, c0), (b1, _) in zip(got, got[1:]):
                assert b0 + c0 == b1
            assert max(c for _, c in got) - min(c for _, c in got) <= 1
    with pytest.raises(ValueError):
        D.strata_shard(16, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


FILTERS = (0, 1, 2, 3)          # box, triangle, Gaussian, Mitchell


def _frame_cfg(flt):
    from luminara_b200 import workloads as W

    world_, cfg = W.box_room(width=24, height=16, spp=9)
    world_.camera.aspect_ratio = 24 / 16
    cfg.pixel_filter = flt
    return world_, cfg


def _worker(rank, world, port, out_path):
    import torch
    import torch.distributed as dist

    import oracle as O

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    results = {}
    for flt in FILTERS:
        world_, cfg = _frame_cfg(flt)
        part_cfg, count = D.shard_config(cfg, rank, world)
        sc = O.OracleScene(world_)
        sums, _ = sc.render_sums(part_cfg, mode=O.MODE_KEYED, threads=1)
        t = torch.from_numpy(sums.copy())
        D.combine_sums(t)
        # the naive combine: this shard's pixels weighted by its stratum count
        img, _ = sc.render(part_cfg, mode=O.MODE_KEYED, threads=1)
        naive = torch.from_numpy(img * count)
        dist.all_reduce(naive)
        results[f"sums{flt}"] = t.numpy()
        results[f"naive{flt}"] = naive.numpy() / cfg.samples_per_pixel
    if rank == 0:
        np.savez(out_path, **results)
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_stratum_split_equals_full_frame(tmp_path):
    import oracle as O

    out = str(tmp_path / "combined.npz")
    mp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
    got = np.load(out)
    for flt in FILTERS:
        world_, cfg = _frame_cfg(flt)
        full, _ = O.OracleScene(world_).render(cfg, mode=O.MODE_KEYED, threads=1)
        s = got[f"sums{flt}"]
        w = s[..., 3:4]
        combined = np.where(w > 0, s[..., :3] / np.where(w > 0, w, 1.0), s[..., :3]) * cfg.exposure
        np.testing.assert_allclose(combined, full, rtol=1e-10, atol=1e-12, err_msg=f"filter {flt}")
        naive_err = np.abs(got[f"naive{flt}"] - full).max()
        if flt == 0:
            assert naive_err < 1e-10
        else:
            assert naive_err > 1e-6, f"filter {flt}: shards happened to weigh alike"
