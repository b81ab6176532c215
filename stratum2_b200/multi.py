"""Multi-GPU partitioning (one process per GPU, torch.distributed).

Camera paths are independent, so ranks split the work without any exchange inside the path:
* a single view: ranks split the sample space of a frame, rank r rendering the frame with its
  own block of frame seeds; the ranks' radiance images are summed into rank 0 (the one exchange);
* the batched form (many views per call): ranks split the views, balanced by pixel count; each
  rank renders its views with one s2_render_views call, and the images are gathered into rank 0
  by point-to-point sends (the one exchange).
Timings are the maximum over ranks; ray counts are summed.
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


def partition_views(pixel_counts, world: int) -> list[list[int]]:
    """View indices per rank: largest views first, each to the rank with the fewest pixels so far
    (ties to the lower rank), each rank's list in view order.  Deterministic, so every rank
    computes the same partition."""
    load = [0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for v in sorted(range(len(pixel_counts)), key=lambda k: (-int(pixel_counts[k]), k)):
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(v)
        load[r] += int(pixel_counts[v])
    return [sorted(p) for p in parts]


def gather_views(local: dict, shapes, parts, dist=None, device=None):
    """Collects every view's image on rank 0: `local` maps this rank's view indices to image tensors,
    `shapes` gives every view's image shape, `parts` the partition (partition_views).  Rank 0
    returns the list of all views' images; the other ranks send theirs and return None.  Sends and
    receives run in view order on every rank, so they pair up."""
    if dist is None or dist.get_world_size() == 1:
        return [local[v] for v in range(len(shapes))]
    import torch
    rank = dist.get_rank()
    owner = {v: r for r, vs in enumerate(parts) for v in vs}
    out = [None] * len(shapes) if rank == 0 else None
    for v in range(len(shapes)):
        r = owner[v]
        if rank == 0:
            if r == 0:
                out[v] = local[v]
            else:
                buf = torch.empty(shapes[v], dtype=torch.float32, device=device)
                dist.recv(buf, src=r)
                out[v] = buf
        elif rank == r:
            dist.send(local[v].contiguous(), dst=0)
    return out
