"""World-size-2 gloo ranks on CPU: the sample partition and the image/timing combination used by
bench.py's multi-GPU path, and the view partition of the batched form (no GPU needed)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from stratum2_b200.multi import combine_images, frame_seed, gather_views, job_time_and_totals, partition_views


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


def _render_worker(rank, world, port, out):
    """Each rank renders its own block of frame seeds of the same small frame with the CPU oracle
    (the multi-GPU path's sample partition, with the oracle standing in for a GPU), and the images
    are combined into rank 0."""
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle_lib import OracleScene, default_render_params
        from stratum2_b200.scenegen import box_scene
        wl = box_scene(seed=1, n_random=50, width=12, height=10)
        spp = 4
        p = default_render_params()
        p.spp, p.min_path_length, p.max_path_length = spp, 2, 5
        p.frame_seed = frame_seed(0, rank, world, spp)
        r = OracleScene(wl.scene, 2).render(wl.view, p, wl.width, wl.height, precision=32, threads=1)
        img = torch.from_numpy(r["mean"].copy())
        combine_images(img, world, dist)
        if rank == 0:
            out[0] = img.numpy().tolist()
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_two_gloo_ranks_render_sample_blocks_that_combine_to_one_render():
    from oracle_lib import OracleScene, default_render_params
    from stratum2_b200.scenegen import box_scene
    world = 2
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_render_worker, args=(world, port, out), nprocs=world, join=True, start_method="spawn")
    wl = box_scene(seed=1, n_random=50, width=12, height=10)
    p = default_render_params()
    p.spp, p.min_path_length, p.max_path_length, p.frame_seed = 4 * world, 2, 5, frame_seed(0, 0, world, 4)
    ref = OracleScene(wl.scene, 2).render(wl.view, p, wl.width, wl.height, precision=32, threads=1)["mean"]
    np.testing.assert_allclose(np.array(out[0]), ref, rtol=1e-12, atol=1e-12)


def _dropout_worker(rank, world, port, out):
    """Rank 1 leaves between steps, before the step's collective; rank 0 learns of it from the
    collective's error (short process-group timeout), not by hanging."""
    import datetime
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=10))
    job_time_and_totals(1.0, [1.0], world, dist)  # step 0: both ranks
    if rank == 1:
        os._exit(0)  # leaves without its kernels or collectives in flight
    try:
        job_time_and_totals(1.0, [1.0], world, dist)  # step 1: the peer is gone
        out[0] = "no error"
    except Exception as e:  # noqa: BLE001 -- the failure is the point
        out[0] = type(e).__name__


@pytest.mark.timeout(120)
def test_a_rank_leaving_between_steps_ends_the_next_collective_with_an_error():
    world = 2
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    ctx = mp.start_processes(_dropout_worker, args=(world, port, out), nprocs=world, join=False, start_method="spawn")
    for p in ctx.processes:
        p.join(60)
    assert all(not p.is_alive() for p in ctx.processes)
    assert out.get(0) not in (None, "no error"), out.get(0)


def test_view_partition_balances_pixels_and_covers_every_view():
    counts = [1920 * 1080, 256 * 256, 640 * 480, 1280 * 720, 300 * 200, 800 * 800, 512 * 512]
    for world in (1, 2, 3, 4, 8):
        parts = partition_views(counts, world)
        assert sorted(v for p in parts for v in p) == list(range(len(counts)))
        loads = [sum(counts[v] for v in p) for p in parts]
        # greedy largest-first: no rank exceeds the mean load by more than the largest view
        assert max(loads) <= sum(counts) / world + max(counts)
        assert parts == partition_views(counts, world)  # every rank computes the same partition
    assert partition_views(counts, 2)[0][0] == 0 and len(partition_views([5], 3)[2]) == 0


_VIEWS = [(12, 10, (0.0, 0.0, 3.0)), (8, 6, (0.3, 0.1, 2.8)), (10, 10, (-0.2, 0.0, 3.1)), (6, 4, (0.0, 0.4, 2.6))]


def _view_worker(rank, world, port, out):
    """Each rank renders its share of four views of different extents with the CPU oracle (the
    batched form's view partition, the oracle standing in for a GPU); rank 0 gathers all views."""
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle_lib import OracleScene, default_render_params
        from stratum2_b200.scene import make_view
        from stratum2_b200.scenegen import box_scene
        wl = box_scene(seed=1, n_random=50, width=12, height=10)
        osc = OracleScene(wl.scene, 2)
        p = default_render_params()
        p.spp, p.min_path_length, p.max_path_length, p.frame_seed = 2, 2, 5, 5
        parts = partition_views([w * h for w, h, _ in _VIEWS], world)
        local = {}
        for v in parts[rank]:
            w, h, pos = _VIEWS[v]
            r = osc.render(make_view(pos, w, h, 40.0), p, w, h, precision=32, threads=1)
            local[v] = torch.from_numpy(r["mean"].astype(np.float32))
        imgs = gather_views(local, [(h, w, 3) for w, h, _ in _VIEWS], parts, dist)
        if rank == 0:
            out[0] = [im.numpy().tolist() for im in imgs]
        else:
            out[rank] = imgs is None
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_two_gloo_ranks_render_their_views_and_gather_them():
    from oracle_lib import OracleScene, default_render_params
    from stratum2_b200.scene import make_view
    from stratum2_b200.scenegen import box_scene
    world = 2
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_view_worker, args=(world, port, out), nprocs=world, join=True, start_method="spawn")
    assert out[1] is True
    wl = box_scene(seed=1, n_random=50, width=12, height=10)
    osc = OracleScene(wl.scene, 2)
    p = default_render_params()
    p.spp, p.min_path_length, p.max_path_length, p.frame_seed = 2, 2, 5, 5
    for v, (w, h, pos) in enumerate(_VIEWS):
        ref = osc.render(make_view(pos, w, h, 40.0), p, w, h, precision=32, threads=1)["mean"].astype(np.float32)
        np.testing.assert_array_equal(np.array(out[0][v], dtype=np.float32), ref)
