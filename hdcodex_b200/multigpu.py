"""Host logic of multi-GPU rendering: one process per GPU, scene replicated.

Every (pixel, sample, wavelength lane) is independent, so N GPUs render
disjoint sample ranges of the same frame (or disjoint jobs of a batch) with no
exchange on the data path. The only collectives are the ones a caller needs to
combine results: the FP64 CIE XYZ sums of a frame split by samples (one
all-reduce of width*height*3 doubles), and the max over ranks of a device
time. They run through torch.distributed: NCCL between GPUs, gloo on CPU.
"""
from __future__ import annotations

from typing import List, Sequence

import numpy as np


def sample_range(step: int, world: int, rank: int, spp: int) -> int:
    """First sample index of `rank`'s share of step `step` when every rank
    renders `spp` samples per step: the ranks' ranges are disjoint and,
    step after step, cover 0, 1, 2, ... without gaps."""
    return (step * world + rank) * spp


def job_shard(count: int, world: int, rank: int) -> List[int]:
    """Indices of the jobs of a `count`-job batch that `rank` renders (dealt
    round-robin, so ranks get equal numbers of jobs to within one)."""
    return list(range(rank, count, world))


def combine_xyz_sums(xyz_sum: np.ndarray, samples: int, group=None):
    """All-reduces per-rank FP64 XYZ sums (h, w, 3) and sample counts; returns
    (summed xyz, total samples). With a sample-range split this is the
    frame's XYZ sum over all ranks' samples; the mean is sum / samples."""
    import torch
    import torch.distributed as dist
    device = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.from_numpy(np.ascontiguousarray(xyz_sum, dtype=np.float64)).to(device)
    n = torch.tensor([float(samples)], dtype=torch.float64, device=device)
    dist.all_reduce(t, group=group)
    dist.all_reduce(n, group=group)
    return t.cpu().numpy(), int(n.item())


def max_over_ranks(value: float, group=None) -> float:
    """The largest `value` over the ranks (device times are reported as the
    slowest rank's)."""
    import torch
    import torch.distributed as dist
    device = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def covered_samples(steps: int, world: int, spp: int) -> Sequence[int]:
    """All sample indices the ranks render in `steps` steps (for checks)."""
    out = []
    for step in range(steps):
        for rank in range(world):
            s0 = sample_range(step, world, rank, spp)
            out.extend(range(s0, s0 + spp))
    return out
