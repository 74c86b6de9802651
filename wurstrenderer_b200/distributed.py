"""Multi-GPU plumbing: sample-split replicas with one FP64 film reduction.

The NEE+MIS estimator is a mean over independent camera samples
(src/renderer/pathnextevent.h:152-191), so N GPUs each render the whole image
with their own random streams and the final image is the mean of the N films:
one reduction per render, no other exchange. Every rank holds a full scene
replica. With the NCCL backend the reduction runs over NVLink; the same code
runs with gloo on CPU tensors (tests).
"""
from __future__ import annotations

GOLDEN_RATIO32 = 0x9E3779B9


def rank_seed(base_seed: int, rank: int) -> int:
    """Seed of `rank`'s random streams: distinct per rank, reproducible."""
    return (int(base_seed) + int(rank) * GOLDEN_RATIO32) & 0xFFFFFFFF


def combine_films(film, world_size: int, dist, dst: int = 0, average: bool = True):
    """Sums the per-rank films onto `dst` (one reduce) and, when `average`, divides by the
    number of ranks there, so that the result is the image of world_size x spp samples.
    `film` is an FP64 tensor (CUDA for nccl, CPU for gloo); returns it (valid on dst)."""
    if world_size > 1:
        dist.reduce(film, dst=dst, op=dist.ReduceOp.SUM)
        if average and dist.get_rank() == dst:
            film /= world_size
    return film


def max_over_ranks(value: float, world_size: int, dist, device=None) -> float:
    """Largest value over all ranks (per-rank device times -> job time)."""
    if world_size <= 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
