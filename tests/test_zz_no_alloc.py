"""tpt_render_device_noalloc: the allocation-free render entry point.

It exists for callers that cannot call cudaMalloc while they render (work
recorded inside a CUDA stream capture, hosts whose device memory belongs to
another allocator with a fixed budget, latency-critical loops): it keeps its
per-sample scratch and its work counter in fixed arrays inside the library.
This test calls it through the C ABI twice in a row, with different jobs, and
checks each image against the existing entry point tpt_render_device: both run
the same megakernel over the same paths with the same accumulation, so the
images must be equal bit for bit.  It also checks that the calls leave the
device's free memory unchanged and that no device-side check fired.  The file
name sorts last so a failing run stops only after every other test ran; it
also passes when run alone.
"""
import ctypes as C

import numpy as np
import pytest

import tpt
import tpt_scenes

pytestmark = pytest.mark.gpu

# cudaStreamLegacy: the legacy default stream, which torch's current stream is
# in a fresh process; passing it keeps the call ordered after the reference
# render that torch's stream already holds (NULL would mean the context's own
# stream instead)
LEGACY_STREAM = C.c_void_p(1)


def test_noalloc_matches_render_device(ctx):
    import torch

    sc = tpt_scenes.cornell_box(4, tpt_scenes.LAMBERT)
    scene = tpt.Scene(ctx, sc["meshes"], sc["instances"], materials=sc["materials"])
    lib = tpt.lib()
    stream = torch.cuda.current_stream()
    assert stream.cuda_stream == 0  # torch's default stream: the legacy stream above
    cam2 = dict(sc["camera"], eye=(0.4, 1.2, 6.0))
    jobs = [scene.job(sc["camera"], 64, 48, 16, 8, execution=tpt.EXEC_MEGAKERNEL),
            scene.job(cam2, 40, 40, 8, 5, execution=tpt.EXEC_MEGAKERNEL)]
    refs, outs = [], []
    for job in jobs:
        ref = torch.empty(job.width * job.height * 3, device="cuda")
        scene.render_device(job, ref.data_ptr(), stream.cuda_stream)
        refs.append(ref)
        outs.append(torch.full((job.width * job.height * 3,), -1.0, device="cuda"))
    # the first call on a device looks up the fixed arrays (and loads the code
    # that holds them): do it once before measuring free memory
    warm = torch.empty(jobs[1].width * jobs[1].height * 3, device="cuda")
    assert lib.tpt_render_device_noalloc(ctx.h, C.byref(jobs[1]), C.c_void_p(warm.data_ptr()), LEGACY_STREAM) == 0
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    for job, out in zip(jobs, outs):  # two calls in a row
        st = lib.tpt_render_device_noalloc(ctx.h, C.byref(job), C.c_void_p(out.data_ptr()), LEGACY_STREAM)
        assert st == 0, lib.tpt_last_error(ctx.h)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free_before
    ctx.check(0)
    for out, ref in zip(outs, refs):
        a, b = out.cpu().numpy(), ref.cpu().numpy()
        assert b.mean() > 0
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_noalloc_rejects_jobs_beyond_its_scratch(ctx):
    import torch

    sc = tpt_scenes.cornell_box(4, tpt_scenes.LAMBERT)
    scene = tpt.Scene(ctx, sc["meshes"], sc["instances"], materials=sc["materials"])
    job = scene.job(sc["camera"], 1024, 1024, 2, 4)  # 2^21 paths > 2^20
    out = torch.empty(1024 * 1024 * 3, device="cuda")  # a full-size image buffer all the same
    st = tpt.lib().tpt_render_device_noalloc(ctx.h, C.byref(job), C.c_void_p(out.data_ptr()), None)
    assert st == 4  # TPT_ERR_CAPACITY, before any device work
    assert b"exceeds its fixed scratch" in tpt.lib().tpt_last_error(ctx.h)
