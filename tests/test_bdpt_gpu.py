"""Device BDPT (integrator/bdpt.rs) against the oracle restatement.

The wavefront execution (subpaths, connection queue, visibility rays through
the persistent traversal kernel, MIS, in-order per-sample sums) and the
one-kernel execution give the same samples bit for bit.

Same bar as the MIS render tests: with the reference's per-pixel sample streams
replayed, >= 99% of the per-sample radiances agree to 1e-5 relative and >= 99.5%
to 1e-3 (libm last-bit differences compound through the MIS weights' products
of pdf ratios), and images agree to 1e-4 relative RMSE.
"""
import numpy as np
import pytest

import oracle as orc
import tpt
import tpt_scenes

pytestmark = pytest.mark.gpu

REL_RMSE_TOL = 1e-4


def rel_rmse(a, b):
    return float(np.sqrt(np.mean((a.astype(np.float64) - b) ** 2)) / np.sqrt(np.mean(b.astype(np.float64) ** 2)))


def bdpt_samples(dev, sc, w, h, spp, depth, execution=tpt.EXEC_WAVEFRONT):
    import torch

    n = w * h * spp
    out = torch.empty(n * 3, dtype=torch.float32, device="cuda")
    job = dev.job(sc["camera"], w, h, spp, depth, integrator=tpt.INTEGRATOR_BDPT, execution=execution)
    dev.render_samples_device(job, 0, n, out.data_ptr(), stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return out.cpu().numpy().reshape(n, 3)


def scene_pair(ctx, sc):
    dev = tpt.Scene(ctx, sc["meshes"], sc["instances"], materials=sc["materials"])
    return dev, orc.RenderScene(sc, dev.light_tree())


MIXED = [
    {"kind": tpt.OPENPBR, "base_color": [0.9, 0.6, 0.3], "base_metalness": 1.0, "specular_roughness": 0.4},
    {"kind": tpt.OPENPBR, "base_color": [0.2, 0.7, 0.3], "specular_roughness": 0.3, "coat_weight": 0.7,
     "coat_roughness": 0.2},
    {"kind": tpt.OPENPBR, "base_color": [0.8, 0.2, 0.2], "specular_roughness": 0.02, "coat_weight": 1.0},
    {"kind": tpt.LAMBERT, "rho": np.array([0.6, 0.5, 0.4], np.float32)},
]


@pytest.mark.parametrize("kind", ["lambert", "openpbr", "mixed"])
def test_bdpt_samples_match_oracle(ctx, kind):
    sc = tpt_scenes.cornell_box(2, tpt_scenes.LAMBERT if kind == "lambert" else tpt_scenes.OPENPBR)
    if kind == "mixed":
        for k, m in enumerate(MIXED):
            sc["materials"][3 + k] = m
    dev, ref = scene_pair(ctx, sc)
    w = h = 24
    spp, depth = 8, 6
    d = bdpt_samples(dev, sc, w, h, spp, depth)
    r = ref.samples(sc["camera"], w, h, spp, depth, 0, w * h * spp, integrator=1)
    rel = np.abs(d - r).max(1) / np.maximum(np.abs(r).max(1), 1e-30)
    assert np.all(np.isfinite(d))
    assert (rel <= 1e-5).mean() >= 0.99, (rel <= 1e-5).mean()
    assert (rel <= 1e-3).mean() >= 0.995, (rel <= 1e-3).mean()
    assert r.mean() > 0


def test_bdpt_image_matches_oracle(ctx):
    sc = tpt_scenes.cornell_box(1, tpt_scenes.OPENPBR)
    dev, ref = scene_pair(ctx, sc)
    w, h, spp, depth = 48, 48, 8, 8
    img = dev.render(sc["camera"], w, h, spp, depth, integrator=tpt.INTEGRATOR_BDPT)
    oimg = ref.render(sc["camera"], w, h, spp, depth, integrator=1).reshape(h, w, 3)
    assert rel_rmse(img, oimg) <= REL_RMSE_TOL
    assert img.mean() > 0.001


def test_bdpt_execution_field_is_ignored(ctx):
    sc = tpt_scenes.cornell_box(1, tpt_scenes.LAMBERT)
    dev = tpt.Scene(ctx, sc["meshes"], sc["instances"], materials=sc["materials"])
    a = dev.render(sc["camera"], 16, 16, 4, 5, integrator=tpt.INTEGRATOR_BDPT, execution=tpt.EXEC_WAVEFRONT)
    b = dev.render(sc["camera"], 16, 16, 4, 5, integrator=tpt.INTEGRATOR_BDPT, execution=tpt.EXEC_MEGAKERNEL)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_bdpt_depth_limit(ctx):
    sc = tpt_scenes.cornell_box(1, tpt_scenes.LAMBERT)
    dev = tpt.Scene(ctx, sc["meshes"], sc["instances"], materials=sc["materials"])
    with pytest.raises(tpt.TptError):
        dev.render(sc["camera"], 8, 8, 1, 17, integrator=tpt.INTEGRATOR_BDPT)
    img = dev.render(sc["camera"], 8, 8, 1, 16, integrator=tpt.INTEGRATOR_BDPT)
    assert np.all(np.isfinite(img))


@pytest.mark.parametrize("kind", ["openpbr", "mixed"])
def test_bdpt_wavefront_equals_single_kernel(ctx, kind):
    sc = tpt_scenes.cornell_box(3, tpt_scenes.OPENPBR)
    if kind == "mixed":
        for k, m in enumerate(MIXED):
            sc["materials"][3 + k] = m
    dev, _ = scene_pair(ctx, sc)
    a = bdpt_samples(dev, sc, 40, 24, 8, 10, tpt.EXEC_WAVEFRONT)
    b = bdpt_samples(dev, sc, 40, 24, 8, 10, tpt.EXEC_MEGAKERNEL)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    ia = dev.render(sc["camera"], 32, 32, 4, 7, integrator=tpt.INTEGRATOR_BDPT, execution=tpt.EXEC_WAVEFRONT)
    ib = dev.render(sc["camera"], 32, 32, 4, 7, integrator=tpt.INTEGRATOR_BDPT, execution=tpt.EXEC_MEGAKERNEL)
    assert np.array_equal(ia.view(np.uint32), ib.view(np.uint32))
    dev.close()
