"""World-size-2 gloo ranks on CPU: the sample partition and the image/timing combination used by
bench.py's multi-GPU path (no GPU needed)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from stratum2_b200.multi import combine_images, frame_seed, job_time_and_totals


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        spp = 4
        seeds = [frame_seed(step, rank, world, spp) for step in range(3)]
        # stand-in for a rendered image: the mean over this rank's seeds of a seed-dependent value
        img = torch.full((2, 3, 4), float(np.mean([s + np.arange(spp) for s in seeds[:1]])), dtype=torch.float64)
        combine_images(img, world, dist)
        ms, (rays,) = job_time_and_totals(10.0 + rank, [100.0 * (rank + 1)], world, dist)
        out[rank] = (seeds, float(img[0, 0, 0]), ms, rays)
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_gloo_ranks_partition_and_combine():
    world = 2
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(world, port, out), nprocs=world, join=True, start_method="spawn")
    s0, img0, ms0, rays0 = out[0]
    s1, _, ms1, rays1 = out[1]
    # seed blocks are disjoint across ranks and steps
    blocks = {(s, s + 4) for s in s0 + s1}
    starts = sorted(s for s, _ in blocks)
    assert len(starts) == 6 and all(b - a >= 4 for a, b in zip(starts, starts[1:]))
    # rank 0 holds the mean over both ranks' samples
    expected = np.mean([np.mean(frame_seed(0, r, world, 4) + np.arange(4)) for r in range(world)])
    assert img0 == pytest.approx(expected)
    # job time is the max over ranks, counts are summed, on every rank
    assert ms0 == ms1 == 11.0
    assert rays0 == rays1 == 300.0


def test_single_rank_is_identity():
    img = torch.ones(3)
    assert combine_images(img, 1) is img
    assert job_time_and_totals(5.0, [1.0, 2.0], 1) == (5.0, [1.0, 2.0])
