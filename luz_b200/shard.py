"""Sample-range sharding of one frame across ranks (one process per GPU).

The Sampler is stateless and keyed on (seed, x, y, sample), so rendering
samples [offset, offset + count) on one GPU and summing the per-pixel sample
sums over ranks reproduces the single-GPU film. The only exchange is one sum
all-reduce of the FP32 film per frame (torch.distributed: NCCL on GPUs, gloo in
the CPU tests).
"""
from __future__ import annotations

from typing import Callable, Tuple


def sample_range(spp: int, rank: int, world: int) -> Tuple[int, int]:
    """Contiguous split of spp samples over world ranks: (offset, count); counts differ by <= 1."""
    if spp <= 0 or world <= 0 or not (0 <= rank < world):
        raise ValueError("sample_range needs spp > 0 and 0 <= rank < world")
    base, extra = divmod(spp, world)
    count = base + (1 if rank < extra else 0)
    offset = rank * base + min(rank, extra)
    return offset, count


def render_sharded(render_mean: Callable, spp: int, rank: int, world: int, all_reduce_sum: Callable):
    """Strong scaling over samples: render_mean(offset, count) returns this rank's per-pixel mean film
    (a torch tensor); returns the frame's mean film, identical on every rank."""
    offset, count = sample_range(spp, rank, world)
    if count > 0:
        film = render_mean(offset, count) * float(count)
    else:
        film = render_mean(0, 0)
        film.zero_()
    all_reduce_sum(film)
    return film / float(spp)
