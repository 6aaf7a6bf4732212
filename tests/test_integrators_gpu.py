"""The NEE and PT integrators (integrator/nee.rs, pt.rs) on the device.

Per-sample parity with the oracle (>= 99% of the samples within 1e-5
relative, >= 99.9% within 1e-3, the MIS render bar) on area-lit, delta-lit
and sky-lit Cornell boxes; the wavefront and the megakernel agree bit for bit;
a batch mixing MIS, NEE and PT jobs gives each job's single render bit for bit.
"""
import numpy as np
import pytest

import oracle as orc
import tpt
import tpt_scenes

pytestmark = pytest.mark.gpu

NO_TREE = (np.zeros(0, tpt.LIGHT_NODE_DTYPE), 0xFFFFFFFF)

SCENES = {
    "area_lambert": lambda: tpt_scenes.cornell_box(1, tpt_scenes.LAMBERT),
    "lights": lambda: tpt_scenes.cornell_lights(2),
    "sky_openpbr": lambda: tpt_scenes.cornell_environment(3, tpt_scenes.OPENPBR),
}


@pytest.fixture(scope="module", params=list(SCENES))
def lit(ctx, request):
    sc = SCENES[request.param]()
    dev = tpt.Scene(ctx, sc["meshes"], sc["instances"], materials=sc["materials"], lights=sc)
    nodes, root = dev.light_tree()
    ref = orc.RenderScene(sc, (nodes, root) if len(nodes) else NO_TREE)
    return sc, dev, ref


def samples(dev, sc, w, h, spp, depth, integrator, execution):
    import torch

    n = w * h * spp
    out = torch.empty(n * 3, dtype=torch.float32, device="cuda")
    job = dev.job(sc["camera"], w, h, spp, depth, integrator=integrator, execution=execution)
    dev.render_samples_device(job, 0, n, out.data_ptr(), stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return out.cpu().numpy().reshape(n, 3)


@pytest.mark.parametrize("integrator", [tpt.INTEGRATOR_NEE, tpt.INTEGRATOR_PT], ids=["nee", "pt"])
def test_matches_oracle_and_executions_agree(lit, integrator):
    sc, dev, ref = lit
    w, h, spp, depth = 32, 32, 8, 8
    d = samples(dev, sc, w, h, spp, depth, integrator, tpt.EXEC_WAVEFRONT)
    r = ref.samples(sc["camera"], w, h, spp, depth, 0, w * h * spp, integrator=integrator)
    rel = np.abs(d - r).max(1) / np.maximum(np.abs(r).max(1), 1e-30)
    assert np.all(np.isfinite(d)) and r.mean() > 0.001
    assert (rel <= 1e-5).mean() >= 0.99, (rel <= 1e-5).mean()
    assert (rel <= 1e-3).mean() >= 0.999, (rel <= 1e-3).mean()
    mk = samples(dev, sc, w, h, spp, depth, integrator, tpt.EXEC_MEGAKERNEL)
    assert np.array_equal(d.view(np.uint32), mk.view(np.uint32))


def test_batch_mixing_integrators_equals_single_renders(ctx, lit):
    import torch

    sc, dev, _ = lit
    specs = [(tpt.INTEGRATOR_MIS, 40, 24, 4, 6), (tpt.INTEGRATOR_NEE, 24, 40, 8, 5), (tpt.INTEGRATOR_PT, 32, 32, 2, 8)]
    jobs = [dev.job(sc["camera"], w, h, spp, depth, integrator=integ) for integ, w, h, spp, depth in specs]
    outs = [torch.empty(w * h * 3, device="cuda") for _, w, h, _, _ in specs]
    st = torch.cuda.current_stream().cuda_stream
    ctx.render_batch_device(jobs, [o.data_ptr() for o in outs], st)
    torch.cuda.synchronize()
    for (integ, w, h, spp, depth), o in zip(specs, outs):
        single = dev.render(sc["camera"], w, h, spp, depth, integrator=integ)
        assert np.array_equal(o.cpu().numpy().reshape(h, w, 3).view(np.uint32), single.view(np.uint32)), integ


@pytest.mark.parametrize("integrator", [tpt.INTEGRATOR_MIS, tpt.INTEGRATOR_BDPT, tpt.INTEGRATOR_NEE,
                                        tpt.INTEGRATOR_PT], ids=["mis", "bdpt", "nee", "pt"])
def test_seeded_streams_match_oracle(ctx, integrator):
    """A job with a sample-stream seed other than 0 renders the oracle's
    samples of the same seed (wavefront and megakernel bit for bit), and they
    differ from seed 0's."""
    import torch

    sc = tpt_scenes.cornell_box(1, tpt_scenes.LAMBERT)
    dev = tpt.Scene(ctx, sc["meshes"], sc["instances"], materials=sc["materials"])
    ref = orc.RenderScene(sc, dev.light_tree())
    w = h = 24
    spp, depth, seed = 4, 6, 0xC0FFEE
    n = w * h * spp
    outs = []
    for execution in (tpt.EXEC_WAVEFRONT, tpt.EXEC_MEGAKERNEL):
        out = torch.empty(n * 3, dtype=torch.float32, device="cuda")
        job = dev.job(sc["camera"], w, h, spp, depth, integrator=integrator, execution=execution, seed=seed)
        dev.render_samples_device(job, 0, n, out.data_ptr(), stream=torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        outs.append(out.cpu().numpy().reshape(n, 3))
    assert np.array_equal(outs[0].view(np.uint32), outs[1].view(np.uint32))
    r = ref.samples(sc["camera"], w, h, spp, depth, 0, n, integrator=integrator, seed=seed)
    r0 = ref.samples(sc["camera"], w, h, spp, depth, 0, n, integrator=integrator)
    assert not np.array_equal(r, r0)
    rel = np.abs(outs[0] - r).max(1) / np.maximum(np.abs(r).max(1), 1e-30)
    assert (rel <= 1e-5).mean() >= 0.99, (rel <= 1e-5).mean()
    assert (rel <= 1e-3).mean() >= 0.995, (rel <= 1e-3).mean()
    dev.close()
