"""Point, spot and directional lights on the device MIS renderer.

Parity with the oracle on the Cornell box lit by a point light, a spot light
and a directional light, with and without the ceiling area light and with a
directional light alone (a scene without a light tree): per sample >= 99%
agree to 1e-5 relative and >= 99.9% to 1e-3 (the tolerance of the area-light
parity tests: last-bit differences between CUDA's and glibc's transcendental
functions compound over bounces); the wavefront and the megakernel agree bit
for bit.  BDPT (wavefront and one-kernel, equal bit for bit) matches the
oracle's BDPT with the same lights.  The adjoint, whose light samples
at OpenPBR vertices come from directional lights, matches the oracle's adjoint
and the base-colour identity of a BSDF linear in base_color.
"""
import numpy as np
import pytest

import oracle as orc
import tpt
import tpt_scenes

pytestmark = pytest.mark.gpu

NO_TREE = (np.zeros(0, tpt.LIGHT_NODE_DTYPE), 0xFFFFFFFF)


def upload(ctx, sc):
    return tpt.Scene(ctx, sc["meshes"], sc["instances"], materials=sc["materials"], lights=sc)


def directional_only():
    sc = tpt_scenes.cornell_lights(3, area=False)
    sc["point_lights"] = []
    sc["spot_lights"] = []
    return sc


SCENES = {
    "all_lights": lambda: tpt_scenes.cornell_lights(1),
    "no_area": lambda: tpt_scenes.cornell_lights(2, tpt_scenes.OPENPBR, area=False),
    "directional_only": directional_only,
}


@pytest.fixture(scope="module", params=list(SCENES))
def lit(ctx, request):
    sc = SCENES[request.param]()
    dev = upload(ctx, sc)
    nodes, root = dev.light_tree()
    ref = orc.RenderScene(sc, (nodes, root) if len(nodes) else NO_TREE)
    return sc, dev, ref


def device_samples(dev, sc, w, h, spp, depth, execution):
    import torch

    n = w * h * spp
    out = torch.empty(n * 3, dtype=torch.float32, device="cuda")
    job = dev.job(sc["camera"], w, h, spp, depth, execution=execution)
    dev.render_samples_device(job, 0, n, out.data_ptr(), stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return out.cpu().numpy().reshape(n, 3)


@pytest.mark.parametrize("execution", [tpt.EXEC_WAVEFRONT, tpt.EXEC_MEGAKERNEL], ids=["wavefront", "megakernel"])
def test_samples_match_oracle(lit, execution):
    sc, dev, ref = lit
    w, h, spp, depth = 32, 32, 8, 8
    d = device_samples(dev, sc, w, h, spp, depth, execution)
    r = ref.samples(sc["camera"], w, h, spp, depth, 0, w * h * spp)
    rel = np.abs(d - r).max(1) / np.maximum(np.abs(r).max(1), 1e-30)
    assert (rel <= 1e-5).mean() >= 0.99, (rel <= 1e-5).mean()
    assert (rel <= 1e-3).mean() >= 0.999, (rel <= 1e-3).mean()
    assert np.all(np.isfinite(d)) and r.mean() > 0.005


def test_wavefront_equals_megakernel(lit):
    sc, dev, _ = lit
    a = device_samples(dev, sc, 32, 24, 16, 8, tpt.EXEC_WAVEFRONT)
    b = device_samples(dev, sc, 32, 24, 16, 8, tpt.EXEC_MEGAKERNEL)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def bdpt_samples(dev, sc, w, h, spp, depth, execution):
    import torch

    n = w * h * spp
    out = torch.empty(n * 3, dtype=torch.float32, device="cuda")
    job = dev.job(sc["camera"], w, h, spp, depth, integrator=tpt.INTEGRATOR_BDPT, execution=execution)
    dev.render_samples_device(job, 0, n, out.data_ptr(), stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return out.cpu().numpy().reshape(n, 3)


def test_bdpt_matches_oracle(lit):
    # light subpaths from the area lights; each camera vertex takes a light
    # sample that skips area lights (bdpt.rs:207-221, 396-464); the bar of the
    # area-light BDPT tests
    sc, dev, ref = lit
    w, h, spp, depth = 24, 24, 8, 6
    d = bdpt_samples(dev, sc, w, h, spp, depth, tpt.EXEC_WAVEFRONT)
    r = ref.samples(sc["camera"], w, h, spp, depth, 0, w * h * spp, integrator=1)
    rel = np.abs(d - r).max(1) / np.maximum(np.abs(r).max(1), 1e-30)
    assert np.all(np.isfinite(d)) and r.mean() > 0.005
    assert (rel <= 1e-5).mean() >= 0.99, (rel <= 1e-5).mean()
    assert (rel <= 1e-3).mean() >= 0.995, (rel <= 1e-3).mean()
    one = bdpt_samples(dev, sc, w, h, spp, depth, tpt.EXEC_MEGAKERNEL)
    assert np.array_equal(d.view(np.uint32), one.view(np.uint32))


SUN = {"direction": (-0.35, -0.45, -1.0), "color": (1.0, 0.95, 0.9), "intensity": 1.5}


def _adjoint(scene, sc, W, spp, depth, d_image, mask=0):
    import torch

    job = scene.job(sc["camera"], W, W, spp, depth)
    d = torch.from_numpy(np.ascontiguousarray(d_image, np.float32)).cuda()
    g = torch.zeros(scene.n_materials * tpt.GRAD_PARAMS, dtype=torch.float64, device="cuda")
    scene.adjoint_device(job, d.data_ptr(), g.data_ptr(), mask, 0.0, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return g.cpu().numpy().reshape(scene.n_materials, tpt.GRAD_PARAMS)


def test_adjoint_with_lights_matches_oracle(ctx):
    # the 64-patch box (OpenPBR) with point, spot and directional lights: the
    # directional light's samples at OpenPBR vertices carry f at the light
    # direction, which the adjoint differentiates too
    sc = tpt_scenes.cornell_patches()
    lit = tpt_scenes.cornell_lights(1)
    for k in ("point_lights", "spot_lights"):
        sc[k] = lit[k]
    sc["directional_lights"] = [SUN]
    scene = upload(ctx, sc)
    W, spp, depth = 32, 16, 6
    d_image = np.random.default_rng(1).uniform(0.5, 1.5, W * W * 3).astype(np.float32)
    gd = _adjoint(scene, sc, W, spp, depth, d_image)
    ref = orc.RenderScene(sc, scene.light_tree())
    go = ref.adjoint(sc["camera"], W, W, spp, depth, d_image)
    assert np.abs(go).max() > 0
    assert np.linalg.norm(gd - go) / np.linalg.norm(go) <= 1e-4
    # without the light samples' own term the gradients are measurably different
    sc_nodir = dict(sc, directional_lights=[])
    go_nodir = orc.RenderScene(sc_nodir, scene.light_tree()).adjoint(sc["camera"], W, W, spp, depth, d_image)
    assert np.linalg.norm(go_nodir - go) / np.linalg.norm(go) > 0.05
    scene.close()


def test_adjoint_identity_with_directional_light(ctx):
    # BSDF linear in base_color (specular_weight 0, metalness 0), one bounce:
    # sum_m bc[m] * grad[m] = image(depth 1) - image(depth 0), the light
    # samples of the first vertex included
    sc = tpt_scenes.cornell_patches()
    for m in sc["materials"][:64]:
        m["specular_weight"] = 0.0
        m["base_metalness"] = 0.0
    sc["directional_lights"] = [SUN]
    scene = upload(ctx, sc)
    W, spp = 64, 16
    g = _adjoint(scene, sc, W, spp, 1, np.ones(W * W * 3, np.float32), mask=tpt.GRAD_MASK_BASE_COLOR)
    img1 = scene.render(sc["camera"], W, W, spp, 1).astype(np.float64).reshape(-1, 3).sum(0)
    img0 = scene.render(sc["camera"], W, W, spp, 0).astype(np.float64).reshape(-1, 3).sum(0)
    bc = np.array([m["base_color"] for m in sc["materials"][:64]], np.float64)
    lhs = (g[:64, :3] * bc).sum(0)
    np.testing.assert_allclose(lhs, img1 - img0, rtol=2e-4)
    scene.close()
