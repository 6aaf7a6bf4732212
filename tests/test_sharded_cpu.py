"""Row-band sharding of one render job over several ranks (tpt_dist), on CPU
with the gloo backend.

* pixel_band: the bands tile the image (disjoint, in order, every pixel once),
  differ by one row at most, and ranks past the last row get empty bands.
* gather_bands: three gloo ranks each render their band of a 12x7 Cornell
  image with the oracle (uneven bands: 2, 2, 3 rows); the all-gathered image
  equals the oracle's one-process render bit for bit on every rank.
* sum_gradients: the same ranks each run the oracle adjoint with dLoss/dimage
  restricted to their band; the all-reduced FP64 gradient equals the
  whole-image adjoint to 1e-12 relative (only the order of the sums differs).
* balanced_bands (the cost-weighted partition): bands tile the rows, each
  band's cost is within two rows' cost of total/world, uniform or zero costs
  give the equal-row bands; three gloo ranks gather uneven cost-weighted bands
  (1, 2, 4 rows) into the oracle's image bit for bit.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import tpt_dist

W, H, SPP, DEPTH = 12, 7, 16, 6


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


@pytest.mark.parametrize("world,width,height", [(1, 5, 4), (2, 9, 7), (3, 9, 7), (4, 3, 2), (8, 16, 16)])
def test_pixel_band_tiles_the_image(world, width, height):
    bands = [tpt_dist.pixel_band(r, world, width, height) for r in range(world)]
    pos = 0
    for first, n in bands:
        assert first == pos and n % width == 0
        pos += n
    assert pos == width * height
    rows = [n // width for _, n in bands]
    assert max(rows) - min(rows) <= 1
    with pytest.raises(ValueError):
        tpt_dist.pixel_band(world, world, width, height)


def _scene():
    import oracle as orc
    import tpt
    import tpt_scenes

    sc = tpt_scenes.cornell_patches()
    return sc, orc.RenderScene(sc, tpt.build_light_tree(sc))


def _rank_main(rank, world, port, out):
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "toy-path-tracing_b200"))
    from datetime import timedelta

    import torch
    import torch.distributed as dist

    import tpt_dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        sc, rs = _scene()
        first, n = tpt_dist.pixel_band(rank, world, W, H)
        band = rs.render(sc["camera"], W, H, SPP, DEPTH, pixels=(first, first + n), nthreads=1)
        image = tpt_dist.gather_bands(torch.from_numpy(band).reshape(-1), W, H)
        d_image = np.random.default_rng(3).uniform(0.5, 1.5, W * H * 3).astype(np.float32)
        d_band = np.zeros_like(d_image)
        d_band[first * 3:(first + n) * 3] = d_image[first * 3:(first + n) * 3]
        g = rs.adjoint(sc["camera"], W, H, SPP, DEPTH, d_band, nthreads=1)
        g = tpt_dist.sum_gradients(torch.from_numpy(g))
        out[rank] = (n, image.numpy().copy(), g.numpy().copy())
    finally:
        dist.destroy_process_group()


def test_three_gloo_ranks_gather_and_sum():
    world = 3
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.start_processes(_rank_main, args=(world, port, out), nprocs=world, join=True, start_method="spawn")
        res = dict(out)
    sc, rs = _scene()
    full = rs.render(sc["camera"], W, H, SPP, DEPTH, nthreads=1).reshape(H, W, 3)
    d_image = np.random.default_rng(3).uniform(0.5, 1.5, W * H * 3).astype(np.float32)
    g_full = rs.adjoint(sc["camera"], W, H, SPP, DEPTH, d_image, nthreads=1)
    assert sorted(res[r][0] // W for r in range(world)) == [2, 2, 3]
    assert np.abs(g_full).max() > 0
    for r in range(world):
        _, image, g = res[r]
        assert np.array_equal(image, full)
        assert np.linalg.norm(g - g_full) <= 1e-12 * np.linalg.norm(g_full)


def test_balanced_bands_follow_the_cost():
    rng = np.random.default_rng(11)
    for world in (1, 2, 3, 5, 8):
        for height in (1, 7, 64, 301):
            cost = rng.exponential(1.0, height) * np.where(np.arange(height) < height // 3, 10.0, 1.0)
            bands = tpt_dist.balanced_bands(cost, world)
            assert len(bands) == world
            pos = 0
            for r0, rows in bands:
                assert r0 == pos and rows >= 0
                pos += rows
            assert pos == height
            share = [cost[r0:r0 + rows].sum() for r0, rows in bands]
            # each boundary is within one row of its ideal place
            assert max(share) - cost.sum() / world <= 2 * cost.max() + 1e-9
    # uniform costs give the equal-row bands; zero costs fall back to them
    for world, height in ((3, 9), (4, 17), (8, 16)):
        eq = [(tpt_dist.pixel_band(r, world, 1, height)[0], tpt_dist.pixel_band(r, world, 1, height)[1])
              for r in range(world)]
        assert tpt_dist.balanced_bands(np.zeros(height), world) == eq
    assert tpt_dist.balanced_bands(np.ones(12), 4) == [(0, 3), (3, 3), (6, 3), (9, 3)]
    # a single expensive row gets a band of its own; some bands stay empty
    b = tpt_dist.balanced_bands([100.0, 1, 1, 1], 4)
    assert (0, 1) in b and sum(k for _, k in b) == 4 and any(k == 0 for _, k in b)
    with pytest.raises(ValueError):
        tpt_dist.balanced_bands([1.0, -1.0], 2)


def _rank_weighted(rank, world, port, out):
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "toy-path-tracing_b200"))
    from datetime import timedelta

    import torch
    import torch.distributed as dist

    import tpt_dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        sc, rs = _scene()
        bands = tpt_dist.balanced_bands([5.0, 1, 1, 1, 1, 1, 1], world)  # rows 1, 2, 4
        r0, rows = bands[rank]
        band = rs.render(sc["camera"], W, H, SPP, DEPTH, pixels=(r0 * W, (r0 + rows) * W), nthreads=1)
        image = tpt_dist.gather_bands(torch.from_numpy(band).reshape(-1), W, H, bands=bands)
        out[rank] = (bands, image.numpy().copy())
    finally:
        dist.destroy_process_group()


def test_three_gloo_ranks_weighted_bands():
    world = 3
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.start_processes(_rank_weighted, args=(world, port, out), nprocs=world, join=True, start_method="spawn")
        res = dict(out)
    sc, rs = _scene()
    full = rs.render(sc["camera"], W, H, SPP, DEPTH, nthreads=1).reshape(H, W, 3)
    for r in range(world):
        bands, image = res[r]
        assert [k for _, k in bands] == [1, 2, 4]
        assert np.array_equal(image, full)


def test_partition_jobs_balances_batches():
    rng = np.random.default_rng(12)
    for world in (1, 2, 3, 8):
        for n_jobs in (0, 1, 5, 64):
            costs = rng.choice([16, 64, 256], n_jobs) * rng.choice([128 * 128, 640 * 480, 1024 * 768], n_jobs)
            parts = tpt_dist.partition_jobs(costs, world)
            assert len(parts) == world
            assert sorted(j for p in parts for j in p) == list(range(n_jobs))
            assert all(p == sorted(p) for p in parts)
            if n_jobs:
                load = [sum(costs[j] for j in p) for p in parts]
                # the LPT bound: no rank exceeds the mean by more than its largest job
                assert max(load) <= costs.sum() / world + costs.max()
            assert tpt_dist.partition_jobs(costs, world) == parts  # deterministic
    assert tpt_dist.partition_jobs([5, 4, 3, 3, 3], 2) == [[0, 3], [1, 2, 4]]
    with pytest.raises(ValueError):
        tpt_dist.partition_jobs([1.0, float("nan")], 2)
