"""Batched rendering (tpt_render_batch_device): many jobs of different scenes,
cameras, resolutions, spp and depths through one wavefront launch sequence.

Bar: every job's image equals tpt_render_device's for the same job bit for bit
(the per-path arithmetic and the in-order per-pixel accumulation are the same),
with the default capacity and with a small capacity that splits jobs across
chunks and puts several jobs in one chunk.
"""
import numpy as np
import pytest

import tpt
import tpt_scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mixed(ctx):
    scenes = []
    for sc in (tpt_scenes.cornell_box(1, tpt_scenes.LAMBERT), tpt_scenes.cornell_box(2, tpt_scenes.OPENPBR),
               tpt_scenes.grid_scene(seed=7, n_side=6, tris_per_object=200, n_materials=12, n_emissive_tris=40)):
        scenes.append((sc, tpt.Scene(ctx, sc["meshes"], sc["instances"], materials=sc["materials"])))
    shapes = [(0, 40, 30, 8, 8), (1, 33, 17, 4, 5), (2, 64, 48, 16, 12), (0, 16, 16, 1, 3), (2, 25, 31, 3, 16),
              (1, 48, 48, 32, 8)]
    jobs = [scenes[i][1].job(scenes[i][0]["camera"], w, h, spp, depth) for i, w, h, spp, depth in shapes]
    yield jobs
    for _, s in scenes:
        s.close()


def _render_each(ctx, jobs):
    import torch

    outs = []
    st = torch.cuda.current_stream().cuda_stream
    for j in jobs:
        img = torch.empty(j.width * j.height * 3, device="cuda")
        tpt.lib().tpt_render_device(ctx.h, tpt.C.byref(j), tpt.C.c_void_p(img.data_ptr()), tpt.C.c_void_p(st))
        outs.append(img)
    torch.cuda.synchronize()
    return [o.cpu().numpy() for o in outs]


def _render_batch(ctx, jobs):
    import torch

    outs = [torch.full((j.width * j.height * 3,), -1.0, device="cuda") for j in jobs]
    ctx.render_batch_device(jobs, [o.data_ptr() for o in outs], torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return [o.cpu().numpy() for o in outs]


@pytest.mark.parametrize("capacity,block", [(0, 256), (4096, 256), (0, 128)],
                         ids=["default", "small_chunks", "shade_block_128"])
def test_batch_equals_single_jobs(ctx, mixed, capacity, block):
    ctx.wavefront_capacity = 0
    ref = _render_each(ctx, mixed)
    ctx.wavefront_capacity = capacity
    ctx.set_shade_block(block)
    try:
        got = _render_batch(ctx, mixed)
    finally:
        ctx.wavefront_capacity = 0
        ctx.set_shade_block(256)
    for a, b in zip(got, ref):
        assert np.all(np.isfinite(a)) and b.max() > 0
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_capacity_does_not_change_single_renders(ctx, mixed):
    ref = _render_each(ctx, mixed[:3])
    ctx.wavefront_capacity = 2048
    try:
        got = _render_each(ctx, mixed[:3])
    finally:
        ctx.wavefront_capacity = 0
    for a, b in zip(got, ref):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    with pytest.raises(tpt.TptError):
        ctx.wavefront_capacity = 100


def test_graph_replay_equals_direct_launches(ctx, mixed):
    """Bounces replayed from captured graphs give the same bits as direct launches,
    on the legacy default stream, on a side stream, and batched."""
    import torch

    ctx.set_graphs(False)
    try:
        direct = _render_each(ctx, mixed)
        direct_b = _render_batch(ctx, mixed)
    finally:
        ctx.set_graphs(True)
    for _ in range(2):  # the first pass captures, the second replays
        graphs = _render_each(ctx, mixed)
        graphs_b = _render_batch(ctx, mixed)
    side = torch.cuda.Stream()
    with torch.cuda.stream(side):
        graphs_s = _render_each(ctx, mixed)
    for a, b, c, d, e in zip(direct, graphs, direct_b, graphs_b, graphs_s):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
        assert np.array_equal(c.view(np.uint32), d.view(np.uint32))
        assert np.array_equal(a.view(np.uint32), e.view(np.uint32))


def test_autotune_applies_a_setting_that_renders_the_same(ctx, mixed):
    import torch

    ref = _render_each(ctx, mixed)
    try:
        r = ctx.autotune(mixed)
        assert r["execution"] in (tpt.EXEC_WAVEFRONT, tpt.EXEC_MEGAKERNEL)
        assert r["ms"] > 0 and r["ms"] <= r["ms_megakernel"] * 1.0001
        assert r["pilot_paths"] == sum(j.width * j.height * j.spp for j in mixed)  # small: the whole workload
        # every reported time is from the one (here: first) pilot, the other shade block included
        assert r["stage"] == 1 and r["candidates"] >= 3 and r["shade_block"] in (128, 256)
        auto = [tpt.RenderJob(j.scene, j.camera, j.width, j.height, j.spp, j.max_depth, j.integrator, tpt.EXEC_AUTO, j.seed)
                for j in mixed]
        got = _render_each(ctx, auto)
        for a, b in zip(got, ref):
            assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
        # the batch entry point under the tuned choice (one launch sequence or job by job)
        assert r["batched"] in (0, 1)
        outs = [torch.empty(j.width * j.height * 3, dtype=torch.float32, device="cuda") for j in mixed]
        ctx.render_batch_device(mixed, [o.data_ptr() for o in outs], torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        for o, b in zip(outs, ref):
            assert np.array_equal(o.cpu().numpy().view(np.uint32), np.asarray(b).reshape(-1).view(np.uint32))
    finally:
        ctx.wavefront_capacity = 0
        ctx.set_graphs(True)
        ctx.set_shade_block(256)


def test_host_render_of_several_jobs_is_batched_and_equal(ctx, mixed):
    """tpt_render with several wavefront jobs takes the batched path; images equal the single renders."""
    import ctypes as C

    ref = _render_each(ctx, mixed)
    outs = [np.empty(j.width * j.height * 3, np.float32) for j in mixed]
    arr = (tpt.RenderJob * len(mixed))(*mixed)
    ptrs = (C.c_void_p * len(mixed))(*[o.ctypes.data for o in outs])
    assert tpt.lib().tpt_render(ctx.h, arr, len(mixed), ptrs) == 0
    for a, b in zip(outs, ref):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_seeded_jobs_in_a_batch_equal_their_single_renders(ctx, mixed):
    """Sample-stream seeds travel with each batched job: a batch mixing seeds
    gives every job its own seeded single render, and a seed changes the image."""
    seeded = [tpt.RenderJob(j.scene, j.camera, j.width, j.height, j.spp, j.max_depth, j.integrator, j.execution,
                            (7919 * (k + 1)) if k % 2 == 0 else 0) for k, j in enumerate(mixed)]
    ctx.wavefront_capacity = 0
    ref = _render_each(ctx, seeded)
    plain = _render_each(ctx, mixed)
    got = _render_batch(ctx, seeded)
    for k, (a, b, p) in enumerate(zip(got, ref, plain)):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
        assert np.array_equal(b, p) == (k % 2 == 1)
