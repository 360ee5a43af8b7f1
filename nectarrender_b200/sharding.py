"""Sample-index sharding of a render across ranks (one process per GPU).

The path tracer is embarrassingly parallel over (pixel, sample index): every
sample index s draws from its own counter-based random stream (subsequence
pixel + s*W*H), so any rank can render any subset of sample indices of the
full image and produce exactly the samples the single-GPU render would. Each
rank keeps FP64 sums of its samples; one sum all-reduce (NCCL over NVLink on
GPUs, gloo in the CPU tests) and a division by the total sample count give the
converged image. Nothing crosses ranks while rendering.
"""
from __future__ import annotations

from dataclasses import dataclass


@dataclass(frozen=True)
class Shard:
    rank: int
    world: int
    first: int   # first sample index of this rank
    count: int   # number of consecutive sample indices


def shard_samples(first: int, count: int, world: int, rank: int) -> Shard:
    """Contiguous split of sample indices [first, first+count) over `world`
    ranks; the first `count % world` ranks take one extra index."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    base, extra = divmod(count, world)
    start = first + rank * base + min(rank, extra)
    n = base + (1 if rank < extra else 0)
    return Shard(rank, world, start, n)


def combine_sums(local_sum, total_count: int, all_reduce) -> object:
    """Mean image from per-rank sums: all_reduce(sum) / total_count.
    `all_reduce` sums a tensor in place across ranks (torch.distributed)."""
    all_reduce(local_sum)
    return local_sum / float(total_count)


def render_shard(render, first: int, count: int, world: int, rank: int):
    """Renders this rank's shard of the sample indices [first, first+count)
    with `render` (a capi.Render created with fp64_accumulate=1, nothing
    rendered since its last reset) and returns (FP64 sum image, number of
    samples in it): the rank's term of the sum over ranks."""
    sh = shard_samples(first, count, world, rank)
    if sh.count:
        render.samples(sh.first, sh.count)
    return render.beauty_fp64_sum()
