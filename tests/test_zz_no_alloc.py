"""tpt_render_device_noalloc: the allocation-free render entry point.

It exists for callers that cannot call cudaMalloc while they render (work
recorded inside a CUDA stream capture, hosts whose device memory belongs to
another allocator with a fixed budget, latency-critical loops): it keeps its
per-sample scratch in a fixed array inside the library.  This test calls it
through the C ABI twice in a row, with different jobs, and checks each image
against the existing entry point tpt_render_device (same megakernel) within the
render tests' tolerance.  The file name sorts last so a failing run stops only
after every other test ran; it also passes when run alone.
"""
import ctypes as C

import numpy as np
import pytest

import tpt
import tpt_scenes

pytestmark = pytest.mark.gpu

REL_RMSE_TOL = 1e-4


def rel_rmse(a, b):
    return float(np.sqrt(np.mean((a.astype(np.float64) - b) ** 2)) / np.sqrt(np.mean(b.astype(np.float64) ** 2)))


def test_noalloc_matches_render_device(ctx):
    import torch

    sc = tpt_scenes.cornell_box(4, tpt_scenes.LAMBERT)
    scene = tpt.Scene(ctx, sc["meshes"], sc["instances"], materials=sc["materials"])
    lib = tpt.lib()
    stream = torch.cuda.current_stream().cuda_stream
    cam2 = dict(sc["camera"], eye=(0.4, 1.2, 6.0))
    for cam, (w, h, spp, depth) in [(sc["camera"], (64, 48, 16, 8)), (cam2, (40, 40, 8, 5))]:
        job = scene.job(cam, w, h, spp, depth, execution=tpt.EXEC_MEGAKERNEL)
        ref = torch.empty(w * h * 3, device="cuda")
        scene.render_device(job, ref.data_ptr(), stream)
        out = torch.full((w * h * 3,), -1.0, device="cuda")
        st = lib.tpt_render_device_noalloc(ctx.h, C.byref(job), C.c_void_p(out.data_ptr()), C.c_void_p(1))
        assert st == 0, lib.tpt_last_error(ctx.h)
        torch.cuda.synchronize()
        a, b = out.cpu().numpy(), ref.cpu().numpy()
        assert np.all(np.isfinite(a)) and b.mean() > 0
        assert rel_rmse(a, b) <= REL_RMSE_TOL


def test_noalloc_rejects_jobs_beyond_its_scratch(ctx):
    import torch

    sc = tpt_scenes.cornell_box(4, tpt_scenes.LAMBERT)
    scene = tpt.Scene(ctx, sc["meshes"], sc["instances"], materials=sc["materials"])
    job = scene.job(sc["camera"], 1024, 1024, 2, 4)  # 2^21 paths > 2^20
    out = torch.empty(1024 * 1024 * 3, device="cuda")  # a full-size image buffer all the same
    st = tpt.lib().tpt_render_device_noalloc(ctx.h, C.byref(job), C.c_void_p(out.data_ptr()), None)
    assert st == 4  # TPT_ERR_CAPACITY, before any device work
    assert b"exceeds its fixed scratch" in tpt.lib().tpt_last_error(ctx.h)
