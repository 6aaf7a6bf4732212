"""Alpha-tested materials on the device against the oracle.

A material with opacity < 1 (NormalizedLambert / Emissive `opacity`, OpenPBR
geometry_opacity) has an alpha test: Scene::closest_hit keeps a candidate hit
on it iff a draw from the path's AuxRng is below the opacity
(scene/mod.rs:360-377, 686-723), the draws taken in the candidates' test
order.  The traversal query with AuxRng states must equal the oracle's hit for
hit and leave the same states; renders must follow each integrator's AuxRng
order (mis.rs, nee.rs, pt.rs, bdpt.rs) to match the oracle sample for sample,
with the wavefront equal to the megakernel bit for bit.
"""
import numpy as np
import pytest

import oracle as orc
import tpt
import tpt_scenes

pytestmark = pytest.mark.gpu


def cutout_cornell(seed=2):
    """The Cornell box with a 40 %-opaque Lambert short box and a 60 %-opaque
    OpenPBR tall box (both walls' colours, cut-outs by the alpha test), lifted
    off the floor: rays inside a box would otherwise meet its bottom and the
    floor in one plane, whose tie decides the number of AuxRng draws."""
    sc = tpt_scenes.lift_boxes(tpt_scenes.cornell_box(seed, tpt_scenes.LAMBERT))
    sc["materials"][5] = {"kind": tpt.OPENPBR, "base_color": np.array([0.7, 0.6, 0.5], np.float32),
                          "specular_roughness": 0.4, "geometry_opacity": 0.6}
    sc["materials"][6] = dict(sc["materials"][6], opacity=0.4)
    return sc


def test_alpha_query_matches_oracle(ctx):
    import torch

    sc = cutout_cornell()
    dev = tpt.Scene(ctx, sc["meshes"], sc["instances"], materials=sc["materials"])
    ref = orc.RenderScene(sc, dev.light_tree())
    rng = np.random.default_rng(5)
    n = 20000
    o = np.stack([rng.uniform(-1.4, 1.4, n), rng.uniform(0.05, 2.9, n), rng.uniform(-1.4, 4.0, n)], 1)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays6 = np.concatenate([o, d], 1).astype(np.float32)
    aux0 = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
    planes = np.zeros((7, n), np.float32)
    planes[:6] = rays6.T
    planes[6] = np.inf
    t_rays = torch.from_numpy(planes).cuda()
    t_aux = torch.from_numpy(aux0.view(np.int32)).cuda()
    prim = torch.empty(n, dtype=torch.int32, device="cuda")
    inst = torch.empty(n, dtype=torch.int32, device="cuda")
    tt = torch.empty(n, dtype=torch.float32, device="cuda")
    dev.traverse_alpha_device(t_rays.data_ptr(), n, t_aux.data_ptr(), prim.data_ptr(), tt.data_ptr(),
                              inst.data_ptr(), stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    ri, rt, rtt, raux = ref.closest_alpha(rays6, aux0)
    assert np.array_equal(prim.cpu().numpy(), rt)
    assert np.array_equal(inst.cpu().numpy(), ri)
    assert np.array_equal(tt.cpu().numpy().view(np.uint32), rtt.view(np.uint32))
    assert np.array_equal(t_aux.cpu().numpy().view(np.uint32), raux)
    drew = raux != aux0
    assert 0.05 < drew.mean() < 0.95  # some rays met the cut-outs
    dev.close()


def device_samples(dev, sc, w, h, spp, depth, execution, integrator):
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
def test_cutout_renders_match_oracle(ctx, integrator):
    sc = cutout_cornell()
    dev = tpt.Scene(ctx, sc["meshes"], sc["instances"], materials=sc["materials"])
    ref = orc.RenderScene(sc, dev.light_tree())
    w = h = 32
    spp, depth = 8, 8
    a = device_samples(dev, sc, w, h, spp, depth, tpt.EXEC_WAVEFRONT, integrator)
    b = device_samples(dev, sc, w, h, spp, depth, tpt.EXEC_MEGAKERNEL, integrator)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    r = ref.samples(sc["camera"], w, h, spp, depth, 0, w * h * spp, integrator=integrator)
    check(a, r, f"cut-out integrator {integrator}")
    dev.close()


def test_cutout_bdpt_matches_oracle(ctx):
    sc = cutout_cornell(3)
    dev = tpt.Scene(ctx, sc["meshes"], sc["instances"], materials=sc["materials"])
    ref = orc.RenderScene(sc, dev.light_tree())
    w = h = 24
    spp, depth = 4, 6
    # the wavefront execution renders alpha-tested scenes with the one-kernel BDPT
    a = device_samples(dev, sc, w, h, spp, depth, tpt.EXEC_WAVEFRONT, tpt.INTEGRATOR_BDPT)
    b = device_samples(dev, sc, w, h, spp, depth, tpt.EXEC_MEGAKERNEL, tpt.INTEGRATOR_BDPT)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    r = ref.samples(sc["camera"], w, h, spp, depth, 0, w * h * spp, integrator=tpt.INTEGRATOR_BDPT)
    check(a, r, "cut-out BDPT")
    dev.close()


def test_cutout_in_a_batch_equals_its_single_render(ctx):
    sc = cutout_cornell(4)
    dev = tpt.Scene(ctx, sc["meshes"], sc["instances"], materials=sc["materials"])
    plain = tpt_scenes.cornell_box(4)
    dev2 = tpt.Scene(ctx, plain["meshes"], plain["instances"], materials=plain["materials"])
    import torch

    jobs = [dev.job(sc["camera"], 32, 32, 4, 6), dev2.job(plain["camera"], 24, 24, 4, 6)]
    outs = [torch.empty(j.width * j.height * 3, dtype=torch.float32, device="cuda") for j in jobs]
    ctx.render_batch_device(jobs, [o.data_ptr() for o in outs], torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    single = [dev.render(sc["camera"], 32, 32, 4, 6), dev2.render(plain["camera"], 24, 24, 4, 6)]
    for a, b in zip(outs, single):
        assert np.array_equal(a.cpu().numpy().view(np.uint32), np.asarray(b).reshape(-1).view(np.uint32))
    dev.close()
    dev2.close()
