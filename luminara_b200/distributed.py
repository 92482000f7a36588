"""Splitting one frame's samples across ranks (one process per GPU).

Pixels and strata are independent (src/render.rs:1598 renders rows in parallel; each stratum
is its own path), so a frame shards by stratum ranges with no exchange until the end: rank r
renders strata [begin_r, begin_r + count_r) of every pixel (lum_render_params.sample_begin /
sample_count), and the partial images combine as a count-weighted mean, which equals the
single-device image up to float rounding (box filter; other filters weigh strata by their
jitter and combine the same way with per-stratum weights summed per shard).

The exchange is one all-reduce of count-weighted frames (NCCL over NVLink on GPUs, gloo in
the CPU tests).
"""
from __future__ import annotations

import math
from typing import Tuple


def total_strata(samples_per_pixel: int) -> int:
    n = math.ceil(math.sqrt(samples_per_pixel))
    return n * n


def strata_shard(n_strata: int, rank: int, world_size: int) -> Tuple[int, int]:
    """Contiguous, balanced stratum range (begin, count) of `rank` (counts differ by <= 1)."""
    if world_size <= 0 or not 0 <= rank < world_size:
        raise ValueError("bad rank/world_size")
    base, extra = divmod(n_strata, world_size)
    begin = rank * base + min(rank, extra)
    count = base + (1 if rank < extra else 0)
    return begin, count


def shard_config(cfg, rank: int, world_size: int):
    """Copy of a RenderConfig restricted to this rank's stratum range."""
    import copy

    c = copy.copy(cfg)
    begin, count = strata_shard(total_strata(cfg.samples_per_pixel), rank, world_size)
    c.sample_begin, c.sample_count = begin, count
    return c, count


def combine_frames(frame, count: int, group=None):
    """All-reduces count-weighted partial frames (torch tensors, in place) into the full-frame
    mean.  Returns the tensor.  `frame` holds this rank's mean over its `count` strata."""
    import torch
    import torch.distributed as dist

    weight = torch.tensor([float(count)], dtype=torch.float64, device=frame.device)
    frame.mul_(float(count))
    dist.all_reduce(frame, group=group)
    dist.all_reduce(weight, group=group)
    total = float(weight.item())
    if total > 0:
        frame.div_(total)
    return frame
