"""The environment light on the device MIS renderer.

Parity with the oracle on the Cornell box (open at the front) under a
procedural sky with a sun, Lambert and OpenPBR, with and without the ceiling
light, and with a directional light beside the map: per sample >= 99% agree to
1e-5 relative and >= 99.9% to 1e-3 (as for the area-light parity tests:
CUDA's and glibc's transcendental functions differ in the last bits, and here
also in the map lookups' acos/atan2); the wavefront and the megakernel agree
bit for bit.  A lone diffuse floor under a uniform map renders albedo x
radiance in every sample.  BDPT (wavefront and one-kernel, equal bit for
bit) matches the oracle's BDPT under the map.  The adjoint
matches the oracle's with the map lighting OpenPBR vertices, and the
base-colour identity holds.
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


def with_sun_and_directional():
    sc = tpt_scenes.cornell_environment(4, tpt_scenes.OPENPBR, area=False)
    sc["directional_lights"] = [{"direction": (-0.35, -0.45, -1.0), "color": (1.0, 0.95, 0.9), "intensity": 1.5}]
    return sc


SCENES = {
    "lambert_area": lambda: tpt_scenes.cornell_environment(1, tpt_scenes.LAMBERT),
    "openpbr_area": lambda: tpt_scenes.cornell_environment(2, tpt_scenes.OPENPBR),
    "lambert_env_only": lambda: tpt_scenes.cornell_environment(3, tpt_scenes.LAMBERT, area=False),
    "openpbr_env_directional": with_sun_and_directional,
}


@pytest.fixture(scope="module", params=list(SCENES))
def lit(ctx, request):
    sc = SCENES[request.param]()
    dev = upload(ctx, sc)
    nodes, root = dev.light_tree()
    ref = orc.RenderScene(sc, (nodes, root) if len(nodes) else NO_TREE)
    return sc, dev, ref


def device_samples(dev, sc, w, h, spp, depth, execution, camera=None):
    import torch

    n = w * h * spp
    out = torch.empty(n * 3, dtype=torch.float32, device="cuda")
    job = dev.job(camera or sc["camera"], w, h, spp, depth, execution=execution)
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
    assert np.all(np.isfinite(d)) and r.mean() > 0.01


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


def test_floor_under_uniform_environment(ctx):
    sc = {"meshes": [{"positions": np.array([[-50, 0, -50], [50, 0, -50], [50, 0, 50], [-50, 0, 50]], np.float32),
                      "normals": np.array([[0, 1, 0]] * 4, np.float32),
                      "indices": np.array([0, 2, 1, 0, 3, 2], np.uint32)}],
          "materials": [{"kind": tpt_scenes.LAMBERT, "rho": np.full(3, 0.8, np.float32)}],
          "instances": [tpt_scenes.identity_instance(0, 0)],
          "environment": {"pixels": np.full((16, 32, 3), 2.0, np.float32)}}
    dev = upload(ctx, sc)
    cam = {"eye": (0.0, 3.0, 0.0), "look_at": (0.0, 0.0, 0.5), "up": (0.0, 1.0, 0.0), "fov_y": 0.5}
    for ex in (tpt.EXEC_WAVEFRONT, tpt.EXEC_MEGAKERNEL):
        smp = device_samples(dev, sc, 16, 16, 4, 5, ex, camera=cam)
        assert np.allclose(smp, np.float32(0.8) * np.float32(2.0), rtol=1e-6)
    sky = {"eye": (0.0, 1.0, 0.0), "look_at": (0.0, 5.0, 0.1), "up": (0.0, 0.0, 1.0), "fov_y": 0.2}
    assert np.all(device_samples(dev, sc, 4, 4, 2, 4, tpt.EXEC_WAVEFRONT, camera=sky) == np.float32(2.0))
    dev.close()


def _adjoint(scene, sc, W, spp, depth, d_image, mask=0):
    import torch

    job = scene.job(sc["camera"], W, W, spp, depth)
    d = torch.from_numpy(np.ascontiguousarray(d_image, np.float32)).cuda()
    g = torch.zeros(scene.n_materials * tpt.GRAD_PARAMS, dtype=torch.float64, device="cuda")
    scene.adjoint_device(job, d.data_ptr(), g.data_ptr(), mask, 0.0, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return g.cpu().numpy().reshape(scene.n_materials, tpt.GRAD_PARAMS)


def test_adjoint_with_environment_matches_oracle(ctx):
    sc = tpt_scenes.cornell_patches()
    sc["environment"] = tpt_scenes.sky_environment(rotate_y=0.35)
    scene = upload(ctx, sc)
    W, spp, depth = 32, 16, 6
    d_image = np.random.default_rng(2).uniform(0.5, 1.5, W * W * 3).astype(np.float32)
    gd = _adjoint(scene, sc, W, spp, depth, d_image)
    go = orc.RenderScene(sc, scene.light_tree()).adjoint(sc["camera"], W, W, spp, depth, d_image)
    assert np.abs(go).max() > 0
    assert np.linalg.norm(gd - go) / np.linalg.norm(go) <= 1e-4
    scene.close()


def test_adjoint_identity_with_environment(ctx):
    sc = tpt_scenes.cornell_patches()
    for m in sc["materials"][:64]:
        m["specular_weight"] = 0.0
        m["base_metalness"] = 0.0
    sc["environment"] = tpt_scenes.sky_environment(rotate_y=0.35)
    scene = upload(ctx, sc)
    W, spp = 64, 16
    g = _adjoint(scene, sc, W, spp, 1, np.ones(W * W * 3, np.float32), mask=tpt.GRAD_MASK_BASE_COLOR)
    img1 = scene.render(sc["camera"], W, W, spp, 1).astype(np.float64).reshape(-1, 3).sum(0)
    img0 = scene.render(sc["camera"], W, W, spp, 0).astype(np.float64).reshape(-1, 3).sum(0)
    bc = np.array([m["base_color"] for m in sc["materials"][:64]], np.float64)
    lhs = (g[:64, :3] * bc).sum(0)
    np.testing.assert_allclose(lhs, img1 - img0, rtol=2e-4)
    scene.close()
