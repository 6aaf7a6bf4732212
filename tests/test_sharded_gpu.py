"""Pixel ranges of one job on the device: the per-rank units of a sharded render.

* tpt_render_pixels_device: the bands of 3 ranks (uneven rows) rendered one
  by one and laid end to end equal tpt_render_device's image bit for bit, for
  the MIS wavefront, MIS megakernel, NEE and BDPT paths, on the Cornell box
  with area, point, spot and directional lights plus the environment.
* tpt_dist.render_sharded with one rank is tpt_render_device's image.
* The adjoint over the bands (tpt_adjoint_desc.first_pixel/num_pixels, each
  band's dLoss/dimage only) sums to the whole-image gradient within 1e-12
  relative (FP64 atomics: the sums' order differs); the host-buffer entry
  point gives the same band gradient.
* Ranges past the image end are rejected.
* The cost-weighted partition from the device-timed pilot renders the same
  image.
* A batch split by job (render_batch_sharded) renders each job as its
  single-job render.
"""
import numpy as np
import pytest

import tpt
import tpt_dist
import tpt_scenes

pytestmark = pytest.mark.gpu

W, H = 40, 29


def _stream():
    import torch

    return torch.cuda.current_stream().cuda_stream


@pytest.fixture(scope="module")
def lit(ctx):
    sc = tpt_scenes.cornell_environment(7, tpt_scenes.OPENPBR)
    lights = tpt_scenes.cornell_lights(7, tpt_scenes.OPENPBR)
    for k in ("point_lights", "spot_lights", "directional_lights"):
        sc[k] = lights[k]
    scene = tpt.Scene(ctx, sc["meshes"], sc["instances"], materials=sc["materials"], lights=sc)
    yield sc, scene
    scene.close()


@pytest.mark.parametrize("integrator,execution", [(tpt.INTEGRATOR_MIS, tpt.EXEC_WAVEFRONT),
                                                  (tpt.INTEGRATOR_MIS, tpt.EXEC_MEGAKERNEL),
                                                  (tpt.INTEGRATOR_NEE, tpt.EXEC_WAVEFRONT),
                                                  (tpt.INTEGRATOR_BDPT, tpt.EXEC_WAVEFRONT)],
                         ids=["mis-wavefront", "mis-megakernel", "nee", "bdpt"])
def test_bands_equal_whole_image(lit, integrator, execution):
    import torch

    sc, scene = lit
    job = scene.job(sc["camera"], W, H, 16, 5, integrator, execution)
    full = torch.empty(W * H * 3, device="cuda")
    scene.render_device(job, full.data_ptr(), _stream())
    parts = []
    for r in range(3):
        first, n = tpt_dist.pixel_band(r, 3, W, H)
        band = torch.empty(n * 3, device="cuda")
        scene.render_pixels_device(job, first, n, band.data_ptr(), _stream())
        parts.append(band)
    torch.cuda.synchronize()
    assert full.abs().sum() > 0
    assert torch.equal(torch.cat(parts), full)
    one = tpt_dist.render_sharded(scene, job)
    assert torch.equal(one.view(-1), full)


def test_band_adjoints_sum_to_whole(ctx):
    import torch

    sc = tpt_scenes.cornell_patches()
    scene = tpt.Scene(ctx, sc["meshes"], sc["instances"], materials=sc["materials"])
    try:
        job = scene.job(sc["camera"], W, H, 16, 6)
        d = torch.from_numpy(np.random.default_rng(5).uniform(0.5, 1.5, W * H * 3).astype(np.float32)).cuda()
        g_full = torch.zeros(scene.n_materials * tpt.GRAD_PARAMS, dtype=torch.float64, device="cuda")
        scene.adjoint_device(job, d.data_ptr(), g_full.data_ptr(), stream=_stream())
        g_sum = torch.zeros_like(g_full)
        host_band = None
        for r in range(3):
            first, n = tpt_dist.pixel_band(r, 3, W, H)
            band = d[first * 3:(first + n) * 3].contiguous()
            g = torch.zeros_like(g_full)
            scene.adjoint_device(job, band.data_ptr(), g.data_ptr(), stream=_stream(), first_pixel=first,
                                 num_pixels=n)
            g_sum += g
            if r == 1:
                torch.cuda.synchronize()
                host_band = (g.cpu().numpy(), scene.adjoint(job, band.cpu().numpy(), first_pixel=first,
                                                            num_pixels=n))
        torch.cuda.synchronize()
        a, b = g_sum.cpu().numpy(), g_full.cpu().numpy()
        assert np.abs(b).max() > 0
        assert np.linalg.norm(a - b) <= 1e-12 * np.linalg.norm(b)
        gd, gh = host_band
        assert np.abs(gd).max() > 0
        assert np.linalg.norm(gh.reshape(-1) - gd) <= 1e-12 * np.linalg.norm(gd)
        one = tpt_dist.adjoint_sharded(scene, job, d.view(H, W, 3))
        assert np.linalg.norm(one.cpu().numpy().reshape(-1) - b) <= 1e-12 * np.linalg.norm(b)
    finally:
        scene.close()


def test_pixel_range_bounds(lit):
    import torch

    sc, scene = lit
    job = scene.job(sc["camera"], W, H, 4, 3)
    out = torch.empty(W * 3, device="cuda")
    with pytest.raises(tpt.TptError):
        scene.render_pixels_device(job, W * H - W + 1, W, out.data_ptr(), _stream())
    g = torch.zeros(scene.n_materials * tpt.GRAD_PARAMS, dtype=torch.float64, device="cuda")
    with pytest.raises(tpt.TptError):
        scene.adjoint_device(job, out.data_ptr(), g.data_ptr(), stream=_stream(), first_pixel=W * H, num_pixels=1)
    scene.render_pixels_device(job, W * H, 0, out.data_ptr(), _stream())  # empty range: nothing to do
    torch.cuda.synchronize()


def test_pilot_cost_partition(lit):
    """estimate_row_cost (1-sample pilot, device-timed slabs) gives a finite,
    positive per-row cost; the 3-rank cost-weighted bands it yields, rendered
    one by one, equal the whole image bit for bit."""
    import torch

    sc, scene = lit
    job = scene.job(sc["camera"], W, H, 16, 5)
    cost = tpt_dist.estimate_row_cost(scene, job, slabs=8)
    assert cost.shape == (H,) and np.all(np.isfinite(cost)) and np.all(cost > 0)
    bands = tpt_dist.balanced_bands(cost, 3)
    full = torch.empty(W * H * 3, device="cuda")
    scene.render_device(job, full.data_ptr(), _stream())
    parts = []
    for r0, rows in bands:
        band = torch.empty(rows * W * 3, device="cuda")
        if rows:
            scene.render_pixels_device(job, r0 * W, rows * W, band.data_ptr(), _stream())
        parts.append(band)
    torch.cuda.synchronize()
    assert torch.equal(torch.cat(parts), full)
    one = tpt_dist.render_sharded(scene, job, bands=[(0, H)])
    assert torch.equal(one.view(-1), full)
    side = torch.cuda.Stream()  # a caller's stream: ordered against torch's current one
    two = tpt_dist.render_sharded(scene, job, stream=side.cuda_stream)
    assert torch.equal(two.view(-1), full)


def test_batch_sharded_one_rank(ctx, lit):
    """render_batch_sharded with one rank renders every job of the batch, each
    image equal to its single-job render bit for bit."""
    import torch

    sc, scene = lit
    jobs = [scene.job(sc["camera"], w, h, spp, 5) for w, h, spp in ((32, 24, 16), (17, 9, 64), (40, 29, 4))]
    images = tpt_dist.render_batch_sharded(ctx, jobs)
    assert sorted(images) == [0, 1, 2]
    for j, job in enumerate(jobs):
        ref = torch.empty(job.width * job.height * 3, device="cuda")
        scene.render_device(job, ref.data_ptr(), _stream())
        torch.cuda.synchronize()
        assert torch.equal(images[j].view(-1), ref)
