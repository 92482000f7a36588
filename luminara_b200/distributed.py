"""Splitting one frame's samples across ranks (one process per GPU).

Pixels and strata are independent (src/render.rs:1598 renders rows in parallel; each stratum
is its own path), so a frame shards by stratum ranges with no exchange until the end: rank r
renders strata [begin_r, begin_r + count_r) of every pixel (lum_render_params.sample_begin /
sample_count).

The reference's pixel is a ratio of two sums over the pixel's samples (src/render.rs:1692-1705):
the filter-weighted, luminance-clamped radiance and the filter weight.  With the box filter
every stratum weighs 1, but the triangle, Gaussian and Mitchell filters weigh each stratum by
its jitter, so the weight sums differ from shard to shard and a count-weighted mean of the
shards' pixels is not the frame's pixel.  The shards therefore exchange the two sums
themselves: each rank renders its raw sums (lum_render_sums_device: 64-bit fixed point, each
path's value rounded once), one integer all-reduce adds them -- integer addition is exact and
order-free -- and lum_sums_finalize_device divides, giving the single-device image bit for bit
for every filter.

The exchange is one all-reduce of W*H*4 int64 values (NCCL over NVLink on GPUs; the CPU tests
all-reduce the oracle's f64 sums over gloo).
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


def combine_sums(sums, group=None):
    """All-reduces (sum) the ranks' raw per-pixel sums in place: an (H, W, 4) tensor, int64
    fixed point on GPUs (exact), or float64 sums in the CPU tests.  Returns the tensor."""
    import torch.distributed as dist

    dist.all_reduce(sums, op=dist.ReduceOp.SUM, group=group)
    return sums


def render_frame_sharded(scene, cfg, rank: int, world_size: int, group=None, stream: int = 0):
    """Renders this rank's stratum shard of `cfg` on the current GPU, all-reduces the raw sums
    and returns the full frame (H, W, 3) float32 on the device -- the same image, bit for bit,
    as scene.render(cfg) on one device."""
    import torch

    from . import sums_finalize_device

    part, _ = shard_config(cfg, rank, world_size)
    h, w, _ = cfg.out_shape()
    sums = torch.empty((h, w, 4), dtype=torch.int64, device="cuda")
    scene.render_sums_device(part, sums.data_ptr(), stream)
    combine_sums(sums, group)
    out = torch.empty((h, w, 3), dtype=torch.float32, device="cuda")
    sums_finalize_device(sums.data_ptr(), w, h, cfg.exposure, out.data_ptr(), stream)
    return out
