"""Multi-process (gloo, world size 2, CPU) test of stratum sharding and the frame combine.

Each rank renders its stratum range of a small keyed frame with the oracle (the device's
estimator in f64; the sharding logic is the same code the GPU ranks use), the ranks combine
with one all-reduce, and the result must equal the single-process full frame.
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


def _worker(rank, world, port, out_path):
    import torch
    import torch.distributed as dist

    import oracle as O
    from luminara_b200 import workloads as W

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    world_, cfg = W.box_room(width=24, height=16, spp=9)
    world_.camera.aspect_ratio = 24 / 16
    part_cfg, count = D.shard_config(cfg, rank, world)
    img, _ = O.OracleScene(world_).render(part_cfg, mode=O.MODE_KEYED, threads=1)
    t = torch.from_numpy(img.copy())
    D.combine_frames(t, count)
    if rank == 0:
        np.save(out_path, t.numpy())
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_stratum_split_equals_full_frame(tmp_path):
    import oracle as O
    from luminara_b200 import workloads as W

    out = str(tmp_path / "combined.npy")
    mp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
    combined = np.load(out)
    world_, cfg = W.box_room(width=24, height=16, spp=9)
    world_.camera.aspect_ratio = 24 / 16
    full, _ = O.OracleScene(world_).render(cfg, mode=O.MODE_KEYED, threads=1)
    np.testing.assert_allclose(combined, full, rtol=1e-10, atol=1e-12)
