"""OpenPBR emission on the device renderers against the oracle.

The Cornell box lit by OpenPBR emitters (a ceiling quad of luminance 15 and a
glowing short box): plain, under a tinted coat and a fuzz layer, and
thin-walled (emitting from both faces).  Emission enters at camera and bounce
hits (with the MIS weight of the light tree's pdf), at NEE light samples (the
light's shading vertex seen from the receiver decides the face and the exit
tint) and at BDPT light endpoints (the tint toward the emitted direction).
Bars of the other render parity tests: per sample >= 99% within 1e-5
relative and >= 99.5% within 1e-3, the wavefront and the megakernel equal bit
for bit, BDPT's two executions equal bit for bit.  The adjoint replays
the emission the forward pass added and matches the oracle's gradients; coat
gradients of a coated emitter are refused (the replay differentiates the
BSDF, not the exit tint), and tpt_scene_set_openpbr refuses to change the
emission the light tree was built from.
"""
import numpy as np
import pytest

import oracle as orc
import tpt
import tpt_scenes

pytestmark = pytest.mark.gpu

VARIANTS = {
    "plain": dict(),
    "coat_fuzz": dict(coat=0.7, fuzz=0.4),
    "thin_coat": dict(coat=0.5, thin_walled=True),
}


@pytest.fixture(scope="module", params=list(VARIANTS))
def lit(ctx, request):
    sc = tpt_scenes.cornell_openpbr_emitter(2, **VARIANTS[request.param])
    dev = tpt.Scene(ctx, sc["meshes"], sc["instances"], materials=sc["materials"])
    ref = orc.RenderScene(sc, dev.light_tree())
    yield sc, dev, ref
    dev.close()


def device_samples(dev, sc, w, h, spp, depth, execution, integrator=tpt.INTEGRATOR_MIS):
    import torch

    n = w * h * spp
    out = torch.empty(n * 3, dtype=torch.float32, device="cuda")
    job = dev.job(sc["camera"], w, h, spp, depth, integrator=integrator, execution=execution)
    dev.render_samples_device(job, 0, n, out.data_ptr(), stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return out.cpu().numpy().reshape(n, 3)


def check(d, r, label):
    rel = np.abs(d - r).max(1) / np.maximum(np.abs(r).max(1), 1e-30)
    print(f"{label}: within 1e-5 {(rel <= 1e-5).mean():.5f}, within 1e-3 {(rel <= 1e-3).mean():.5f}")
    assert np.all(np.isfinite(d)) and r.mean() > 0.005
    assert (rel <= 1e-5).mean() >= 0.99, (rel <= 1e-5).mean()
    assert (rel <= 1e-3).mean() >= 0.995, (rel <= 1e-3).mean()


@pytest.mark.parametrize("integrator", [tpt.INTEGRATOR_MIS, tpt.INTEGRATOR_NEE, tpt.INTEGRATOR_PT],
                         ids=["mis", "nee", "pt"])
def test_unidirectional_matches_oracle(lit, integrator):
    sc, dev, ref = lit
    w = h = 32
    spp, depth = 8, 8
    outs = [device_samples(dev, sc, w, h, spp, depth, e, integrator) for e in (tpt.EXEC_WAVEFRONT,
                                                                             tpt.EXEC_MEGAKERNEL)]
    assert np.array_equal(outs[0].view(np.uint32), outs[1].view(np.uint32))
    r = ref.samples(sc["camera"], w, h, spp, depth, 0, w * h * spp, integrator=integrator)
    check(outs[0], r, f"integrator {integrator}")


def test_bdpt_matches_oracle(lit):
    sc, dev, ref = lit
    w = h = 24
    spp, depth = 8, 6
    d = device_samples(dev, sc, w, h, spp, depth, tpt.EXEC_WAVEFRONT, tpt.INTEGRATOR_BDPT)
    r = ref.samples(sc["camera"], w, h, spp, depth, 0, w * h * spp, integrator=tpt.INTEGRATOR_BDPT)
    check(d, r, "bdpt")
    one = device_samples(dev, sc, w, h, spp, depth, tpt.EXEC_MEGAKERNEL, tpt.INTEGRATOR_BDPT)
    assert np.array_equal(d.view(np.uint32), one.view(np.uint32))


def test_back_faces_do_not_emit_unless_thin_walled(ctx):
    """Seen from above, the ceiling emitter's back face is dark unless thin-walled."""
    for thin in (False, True):
        sc = tpt_scenes.cornell_openpbr_emitter(2, thin_walled=thin)
        sc["camera"] = {"eye": (0.0, 3.6, 0.0), "look_at": (0.0, 2.0, 0.0), "up": (0.0, 0.0, -1.0),
                        "fov_y": float(np.float32(np.radians(8.0))), "exposure": 1.0}
        # only the emitter quad and the floor, so nothing occludes it from above
        keep = [0, 7]
        sc["instances"] = [sc["instances"][k] for k in keep]
        dev = tpt.Scene(ctx, sc["meshes"], sc["instances"], materials=sc["materials"])
        img = dev.render(sc["camera"], 8, 8, 1, 1)
        ref = orc.RenderScene(sc, dev.light_tree()).render(sc["camera"], 8, 8, 1, 1).reshape(8, 8, 3)
        np.testing.assert_allclose(img, ref, rtol=1e-5, atol=1e-6)
        centre = img[3:5, 3:5].mean()
        if thin:
            assert centre > 5.0
        else:
            assert centre < 1e-6
        dev.close()


def test_adjoint_with_emitters_matches_oracle(ctx):
    import torch

    sc = tpt_scenes.cornell_openpbr_emitter(3)
    dev = tpt.Scene(ctx, sc["meshes"], sc["instances"], materials=sc["materials"])
    W, spp, depth = 32, 8, 6
    d_image = np.random.default_rng(2).uniform(0.5, 1.5, W * W * 3).astype(np.float32)
    job = dev.job(sc["camera"], W, W, spp, depth)
    d = torch.from_numpy(d_image).cuda()
    g = torch.zeros(dev.n_materials * tpt.GRAD_PARAMS, dtype=torch.float64, device="cuda")
    dev.adjoint_device(job, d.data_ptr(), g.data_ptr(), 0, 0.0, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    gd = g.cpu().numpy().reshape(dev.n_materials, tpt.GRAD_PARAMS)
    go = orc.RenderScene(sc, dev.light_tree()).adjoint(sc["camera"], W, W, spp, depth, d_image)
    assert np.abs(go).max() > 0
    assert np.linalg.norm(gd - go) / np.linalg.norm(go) <= 1e-4
    dev.close()


def test_coated_emitter_refuses_coat_gradients_and_emission_changes(ctx):
    sc = tpt_scenes.cornell_openpbr_emitter(3, coat=0.5)
    dev = tpt.Scene(ctx, sc["meshes"], sc["instances"], materials=sc["materials"])
    job = dev.job(sc["camera"], 8, 8, 1, 2)
    d_image = np.ones(8 * 8 * 3, np.float32)
    with pytest.raises(tpt.TptError, match="coated OpenPBR emitter"):
        dev.adjoint(job, d_image)
    g = dev.adjoint(job, d_image, mask=tpt.GRAD_ALL & ~tpt.GRAD_MASK_COAT)
    assert np.all(np.isfinite(g))
    m = dict(sc["materials"][7])
    m["emission_luminance"] = 20.0
    with pytest.raises(tpt.TptError, match="emission differs"):
        dev.set_openpbr([7], [m])
    m = dict(sc["materials"][7])
    m["base_color"] = np.array([0.2, 0.3, 0.4], np.float32)
    dev.set_openpbr([7], [m])  # same emission: accepted
    dev.close()
