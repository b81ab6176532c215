"""Multi-GPU partitioning of a frame's samples (one process per GPU, torch.distributed).

Camera paths are independent, so ranks split the sample space of a frame: rank r renders the
frame with its own block of frame seeds, and the ranks' radiance images are summed into rank 0
(the one exchange).  Timings are the maximum over ranks; ray counts are summed.
"""
from __future__ import annotations


def frame_seed(step: int, rank: int, world: int, spp: int) -> int:
    """First frame seed of `rank`'s samples in `step`; blocks of `spp` seeds never overlap."""
    return (step * world + rank) * spp


def combine_images(img, world: int, dist=None):
    """Sums the ranks' images (device or CPU tensors) into rank 0 in place; returns the
    per-sample mean on rank 0 when each rank's image is a mean over its own samples."""
    if world > 1:
        dist.reduce(img, dst=0)
        if dist.get_rank() == 0:
            img /= world
    return img


def job_time_and_totals(ms: float, counts: list[float], world: int, dist=None, device=None):
    """Whole-job time (max over ranks) and summed counters."""
    if world == 1:
        return ms, list(counts)
    import torch
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    c = torch.tensor(counts, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(c, op=dist.ReduceOp.SUM)
    return float(t[0]), [float(x) for x in c]
