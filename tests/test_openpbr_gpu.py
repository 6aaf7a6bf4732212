"""Device OpenPBR against the oracle: tables, BSDF queries and full renders.

* The three lookup tables are built on the GPU and must equal the oracle's CPU
  build bit for bit (the sample directions' trigonometry is host-computed on
  both sides; everything else is correctly rounded arithmetic).
* BSDF eval / pdf / sample of lowered materials: >= 99% of the values agree to
  1e-5 relative and all to 1e-3 (CUDA's atan2f / expf / powf / sinf / cosf
  differ from glibc's in the last bit); sampled lobes (flags) agree for
  >= 99.9% of the queries.
* Renders of the OpenPBR Cornell box: per-sample and image tolerances of the
  Lambert render tests; wavefront and megakernel are bit-identical.
"""
import numpy as np
import pytest

import oracle as orc
import tpt
import tpt_scenes

pytestmark = pytest.mark.gpu

REL_RMSE_TOL = 1e-4

MATERIALS = [
    {"base_color": [0.5, 0.4, 0.3], "base_diffuse_roughness": 1.0, "specular_roughness": 1.0},
    {"base_color": [0.9, 0.6, 0.3], "base_metalness": 1.0, "specular_roughness": 0.4},
    {"base_color": [0.2, 0.7, 0.3], "specular_roughness": 0.3, "coat_weight": 0.7, "coat_roughness": 0.2},
    {"base_color": [0.6, 0.6, 0.6], "specular_roughness": 0.5, "fuzz_weight": 0.6, "fuzz_roughness": 0.5,
     "coat_weight": 0.3, "coat_roughness": 0.1, "specular_roughness_anisotropy": 0.5, "base_metalness": 0.3},
    {"base_color": [0.8, 0.2, 0.2], "specular_roughness": 0.02, "coat_weight": 1.0, "coat_roughness": 0.0},
    {"base_color": [0.3, 0.3, 0.9], "specular_roughness": 0.05, "base_metalness": 1.0},
    {"base_color": [0.4, 0.5, 0.6], "specular_weight": 0.3, "specular_ior": 1.8, "specular_roughness": 0.7,
     "coat_weight": 0.5, "coat_ior": 1.4, "coat_roughness": 0.25, "coat_color": [0.9, 0.7, 0.5]},
]


def rel_rmse(a, b):
    return float(np.sqrt(np.mean((a.astype(np.float64) - b) ** 2)) / np.sqrt(np.mean(b.astype(np.float64) ** 2)))


def rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b) / np.maximum(np.abs(b), 1e-30)


@pytest.fixture(scope="module")
def bsdf_scene(ctx):
    quad = tpt_scenes._quad((-1, 0, 1), (1, 0, 1), (1, 0, -1), (-1, 0, -1), (0, 1, 0))
    mats = [dict(m, kind=tpt.OPENPBR) for m in MATERIALS]
    return tpt.Scene(ctx, [quad], [tpt_scenes.identity_instance(0, 0)], materials=mats)


def test_tables_match_oracle(ctx):
    e, e_avg = ctx.lut_conductor_ec()
    oe, oe_avg = orc.lut_conductor_ec()
    assert np.array_equal(e.view(np.uint32), oe.view(np.uint32))
    assert np.array_equal(e_avg.view(np.uint32), oe_avg.view(np.uint32))
    e, e_avg = ctx.lut_dielectric_ec()
    oe, oe_avg = orc.lut_dielectric_ec()
    assert np.array_equal(e.view(np.uint32), oe.view(np.uint32))
    assert np.array_equal(e_avg.view(np.uint32), oe_avg.view(np.uint32))
    for eta in (1.5, 1.6):
        da = ctx.lut_dielectric_albedo(eta)
        assert np.array_equal(da.view(np.uint32), orc.lut_dielectric_albedo(eta).view(np.uint32)), eta


def _dirs(rng, n, below=0.0):
    v = rng.normal(size=(n, 3)).astype(np.float32)
    v[:, 2] = np.abs(v[:, 2]) + 0.05
    if below:
        flip = rng.random(n) < below
        v[flip, 2] *= -1
    return (v / np.linalg.norm(v, axis=1, keepdims=True)).astype(np.float32)


def _assert_close(dev, ref, what):
    r = rel_err(dev, ref)
    ok5 = (r <= 1e-5) | (np.abs(np.asarray(dev, np.float64) - ref) <= 1e-9)
    assert ok5.mean() >= 0.99, (what, ok5.mean())
    assert np.all((r <= 1e-3) | (np.abs(np.asarray(dev, np.float64) - ref) <= 1e-7)), (what, r.max())


@pytest.mark.parametrize("mode", [0, 1], ids=["radiance", "importance"])
@pytest.mark.parametrize("mi", range(len(MATERIALS)))
def test_bsdf_eval_pdf_match_oracle(bsdf_scene, mi, mode):
    import torch

    rng = np.random.default_rng(100 + mi + 50 * mode)
    n = 2000
    wo = _dirs(rng, n)
    wi = _dirs(rng, n, below=0.1)
    front = (rng.random(n) < 0.7).astype(np.uint32)
    t = {k: torch.from_numpy(v).cuda() for k, v in (("wo", wo), ("wi", wi), ("front", front.view(np.int32)))}
    f = torch.empty((n, 3), dtype=torch.float32, device="cuda")
    pdf = torch.empty(n, dtype=torch.float32, device="cuda")
    bsdf_scene.bsdf_eval_device(mi, n, t["wo"].data_ptr(), t["wi"].data_ptr(), t["front"].data_ptr(), f.data_ptr(),
                                pdf.data_ptr(), stream=torch.cuda.current_stream().cuda_stream, mode=mode)
    torch.cuda.synchronize()
    f, pdf = f.cpu().numpy(), pdf.cpu().numpy()
    m = orc.OpenPbrMaterial(MATERIALS[mi])
    rf = np.array([m.eval(wo[k], wi[k], front=bool(front[k]), mode=mode) for k in range(n)])
    rp = np.array([m.pdf(wo[k], wi[k], front=bool(front[k])) for k in range(n)], np.float32)
    assert np.all(np.isfinite(f)) and np.all(np.isfinite(pdf))
    assert (rp > 0).mean() > 0.5 and (rf.max(1) > 0).mean() > 0.5
    _assert_close(f, rf, "f")
    _assert_close(pdf, rp, "pdf")


@pytest.mark.parametrize("mode", [0, 1], ids=["radiance", "importance"])
@pytest.mark.parametrize("mi", range(len(MATERIALS)))
def test_bsdf_sample_matches_oracle(bsdf_scene, mi, mode):
    import torch

    rng = np.random.default_rng(200 + mi + 50 * mode)
    n = 2000
    wo = _dirs(rng, n)
    u = rng.random((n, 3)).astype(np.float32)
    front = (rng.random(n) < 0.7).astype(np.uint32)
    tw, tu, tf = (torch.from_numpy(a).cuda() for a in (wo, u, front.view(np.int32)))
    out = torch.empty((n, 9), dtype=torch.float32, device="cuda")
    bsdf_scene.bsdf_sample_device(mi, n, tw.data_ptr(), tu.data_ptr(), tf.data_ptr(), out.data_ptr(),
                                  stream=torch.cuda.current_stream().cuda_stream, mode=mode)
    torch.cuda.synchronize()
    out = out.cpu().numpy()
    flags = out[:, 8].view(np.uint32)
    m = orc.OpenPbrMaterial(MATERIALS[mi])
    ref = [m.sample(wo[k], u[k, 0], u[k, 1:], front=bool(front[k]), mode=mode) for k in range(n)]
    rflags = np.array([0 if s is None else s["flags"] for s in ref], np.uint32)
    assert (flags == rflags).mean() >= 0.999
    both = np.nonzero((flags == rflags) & (rflags != 0))[0]
    assert len(both) > n // 2
    rw = np.array([ref[k]["weight"] for k in both])
    rwi = np.array([ref[k]["wi"] for k in both])
    rpdf = np.array([ref[k]["pdf"] for k in both], np.float32)
    rrev = np.array([ref[k]["pdf_rev"] for k in both], np.float32)
    _assert_close(out[both, 0:3], rw, "weight")
    _assert_close(out[both, 3:6], rwi, "wi")
    _assert_close(out[both, 6], rpdf, "pdf")
    _assert_close(out[both, 7], rrev, "pdf_rev")


@pytest.fixture(scope="module")
def cornell_openpbr(ctx):
    sc = tpt_scenes.cornell_box(1, tpt_scenes.OPENPBR)
    dev = tpt.Scene(ctx, sc["meshes"], sc["instances"], materials=sc["materials"])
    ref = orc.RenderScene(sc, dev.light_tree())
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
def test_openpbr_samples_match_oracle(cornell_openpbr, execution):
    sc, dev, ref = cornell_openpbr
    w = h = 40
    spp, depth = 8, 8
    d = device_samples(dev, sc, w, h, spp, depth, execution)
    r = ref.samples(sc["camera"], w, h, spp, depth, 0, w * h * spp)
    rel = np.abs(d - r).max(1) / np.maximum(np.abs(r).max(1), 1e-30)
    assert np.all(np.isfinite(d))
    assert (rel <= 1e-5).mean() >= 0.99, (rel <= 1e-5).mean()
    assert (rel <= 1e-3).mean() >= 0.999, (rel <= 1e-3).mean()


def test_openpbr_wavefront_equals_megakernel(cornell_openpbr):
    sc, dev, _ = cornell_openpbr
    a = device_samples(dev, sc, 32, 24, 16, 8, tpt.EXEC_WAVEFRONT)
    b = device_samples(dev, sc, 32, 24, 16, 8, tpt.EXEC_MEGAKERNEL)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


@pytest.mark.parametrize("execution", [tpt.EXEC_WAVEFRONT, tpt.EXEC_MEGAKERNEL], ids=["wavefront", "megakernel"])
def test_openpbr_image_matches_oracle(cornell_openpbr, execution):
    sc, dev, ref = cornell_openpbr
    w, h, spp, depth = 64, 64, 16, 8
    img = dev.render(sc["camera"], w, h, spp, depth, execution=execution)
    oimg = ref.render(sc["camera"], w, h, spp, depth).reshape(h, w, 3)
    assert rel_rmse(img, oimg) <= REL_RMSE_TOL
    assert img.mean() > 0.001


def test_mixed_lobes_render_matches_oracle(ctx):
    """Cornell box whose walls and boxes use the metal / coat / fuzz /
    anisotropic / smooth materials above next to Lambert walls (NEE there)."""
    sc = tpt_scenes.cornell_box(3, tpt_scenes.OPENPBR)
    for k, m in enumerate(MATERIALS):
        sc["materials"][k] = dict(m, kind=tpt.OPENPBR)
    sc["materials"][6] = {"kind": tpt.LAMBERT, "rho": np.array([0.6, 0.5, 0.4], np.float32)}
    dev = tpt.Scene(ctx, sc["meshes"], sc["instances"], materials=sc["materials"])
    ref = orc.RenderScene(sc, dev.light_tree())
    w = h = 32
    spp, depth = 8, 8
    for execution in (tpt.EXEC_WAVEFRONT, tpt.EXEC_MEGAKERNEL):
        d = device_samples(dev, sc, w, h, spp, depth, execution)
        r = ref.samples(sc["camera"], w, h, spp, depth, 0, w * h * spp)
        rel = np.abs(d - r).max(1) / np.maximum(np.abs(r).max(1), 1e-30)
        assert np.all(np.isfinite(d))
        assert (rel <= 1e-5).mean() >= 0.99, (rel <= 1e-5).mean()
        assert (rel <= 1e-3).mean() >= 0.995, (rel <= 1e-3).mean()
    img = dev.render(sc["camera"], 48, 48, 16, 8)
    oimg = ref.render(sc["camera"], 48, 48, 16, 8).reshape(48, 48, 3)
    assert rel_rmse(img, oimg) <= REL_RMSE_TOL


def test_every_openpbr_parameter_reaches_the_device(ctx):
    """Nothing of an untextured OpenPBR material is refused any more: a tall box
    combining a cut-out (geometry_opacity), emission, dispersive transmission,
    coat, fuzz and thin film renders on the device as in the oracle."""
    sc = tpt_scenes.lift_boxes(tpt_scenes.cornell_box(6, tpt_scenes.OPENPBR))  # no floor/box-bottom ties
    sc["materials"][5] = {"kind": tpt.OPENPBR, "base_color": np.array([0.7, 0.6, 0.5], np.float32),
                          "specular_roughness": 0.3, "transmission_weight": 0.6,
                          "transmission_dispersion_scale": 1.0, "coat_weight": 0.4, "coat_roughness": 0.2,
                          "fuzz_weight": 0.3, "thin_film_weight": 0.5, "thin_film_thickness": 0.4,
                          "geometry_opacity": 0.7, "emission_luminance": 0.5,
                          "emission_color": np.array([1.0, 0.8, 0.6], np.float32)}
    dev = tpt.Scene(ctx, sc["meshes"], sc["instances"], materials=sc["materials"])
    ref = orc.RenderScene(sc, dev.light_tree())
    w = h = 24
    spp, depth = 4, 6
    a = device_samples(dev, sc, w, h, spp, depth, tpt.EXEC_WAVEFRONT)
    b = device_samples(dev, sc, w, h, spp, depth, tpt.EXEC_MEGAKERNEL)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    r = ref.samples(sc["camera"], w, h, spp, depth, 0, w * h * spp)
    rel = np.abs(a - r).max(1) / np.maximum(np.abs(r).max(1), 1e-30)
    assert np.all(np.isfinite(a)) and r.mean() > 0.005
    assert (rel <= 1e-5).mean() >= 0.99, (rel <= 1e-5).mean()
    assert (rel <= 1e-3).mean() >= 0.995, (rel <= 1e-3).mean()
    dev.close()
