"""Device OpenPBR specular transmission, thin-walled surfaces and thin film against the oracle.

The lobes are bsdf/open_pbr.rs's: the GGX BTDF with its multiple-scattering
term (eval_spec_btdf, pdf_specular_btdf, sample_spec_btdf at 1024-1222 and
1670-1836), smooth refraction, and for thin-walled materials the two-interface
slab (thin_wall_coefficients 931-979) reflecting through the specular lobe and
transmitting through the mirrored thin-wall GGX lobe (1053-1072); thin film
(bsdf/thin_film.rs) on the specular, metal and transmission Fresnel terms.
Dispersion is off (the untextured parameter set has no dispersion scale).

Bars as for the other OpenPBR tests: BSDF eval / pdf / sample values >= 99%
within 1e-5 relative and all within 1e-3, sampled lobes equal for >= 99.9%
of the queries; renders of Cornell boxes with glass boxes >= 99% of samples
within 1e-5 relative and image relative RMSE <= 1e-4; wavefront and
megakernel equal bit for bit.
"""
import numpy as np
import pytest

import oracle as orc
import tpt
import tpt_scenes

pytestmark = pytest.mark.gpu

REL_RMSE_TOL = 1e-4

MATERIALS = [
    {"base_color": [0.8, 0.8, 0.8], "specular_roughness": 0.3, "transmission_weight": 1.0},
    {"base_color": [0.5, 0.7, 0.2], "specular_roughness": 0.6, "transmission_weight": 0.7,
     "transmission_color": [0.9, 0.6, 0.3], "coat_weight": 0.4, "coat_roughness": 0.2},
    {"base_color": [0.6, 0.5, 0.4], "specular_roughness": 0.0, "transmission_weight": 0.6},
    {"base_color": [0.4, 0.5, 0.6], "specular_roughness": 0.4, "transmission_weight": 0.8,
     "geometry_thin_walled": 1, "transmission_color": [0.7, 0.8, 0.9]},
    {"base_color": [0.5, 0.5, 0.5], "specular_roughness": 0.0, "transmission_weight": 0.6,
     "geometry_thin_walled": 1},
    {"base_color": [0.3, 0.6, 0.8], "specular_roughness": 0.5, "specular_ior": 2.2, "transmission_weight": 0.9,
     "specular_roughness_anisotropy": 0.6, "fuzz_weight": 0.3},
    # thin film (bsdf/thin_film.rs) over glass, a metal, a coated dielectric and a thin-walled sheet
    {"base_color": [0.7, 0.7, 0.7], "specular_roughness": 0.3, "transmission_weight": 0.8, "thin_film_weight": 1.0,
     "thin_film_thickness": 0.4, "thin_film_ior": 1.45},
    {"base_color": [0.9, 0.6, 0.3], "base_metalness": 1.0, "specular_roughness": 0.35, "thin_film_weight": 0.7,
     "thin_film_thickness": 0.3, "thin_film_ior": 1.8},
    {"base_color": [0.2, 0.5, 0.3], "specular_roughness": 0.4, "coat_weight": 0.6, "coat_roughness": 0.2,
     "thin_film_weight": 1.0, "thin_film_thickness": 0.55},
    {"base_color": [0.5, 0.5, 0.6], "specular_roughness": 0.3, "transmission_weight": 0.7, "geometry_thin_walled": 1,
     "thin_film_weight": 0.8, "thin_film_thickness": 0.3},
]


def rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b) / np.maximum(np.abs(b), 1e-30)


def rel_rmse(a, b):
    return float(np.sqrt(np.mean((a.astype(np.float64) - b) ** 2)) / np.sqrt(np.mean(b.astype(np.float64) ** 2)))


def _assert_close(dev, ref, what):
    r = rel_err(dev, ref)
    ok5 = (r <= 1e-5) | (np.abs(np.asarray(dev, np.float64) - ref) <= 1e-9)
    assert ok5.mean() >= 0.99, (what, ok5.mean())
    assert np.all((r <= 1e-3) | (np.abs(np.asarray(dev, np.float64) - ref) <= 1e-7)), (what, r.max())


def _dirs(rng, n, below=0.0):
    v = rng.normal(size=(n, 3)).astype(np.float32)
    v[:, 2] = np.abs(v[:, 2]) + 0.05
    if below:
        flip = rng.random(n) < below
        v[flip, 2] *= -1
    return (v / np.linalg.norm(v, axis=1, keepdims=True)).astype(np.float32)


@pytest.fixture(scope="module")
def bsdf_scene(ctx):
    quad = tpt_scenes._quad((-1, 0, 1), (1, 0, 1), (1, 0, -1), (-1, 0, -1), (0, 1, 0))
    mats = [dict(m, kind=tpt.OPENPBR) for m in MATERIALS]
    return tpt.Scene(ctx, [quad], [tpt_scenes.identity_instance(0, 0)], materials=mats)


@pytest.mark.parametrize("mode", [0, 1], ids=["radiance", "importance"])
@pytest.mark.parametrize("mi", range(len(MATERIALS)))
def test_transmission_eval_pdf_match_oracle(bsdf_scene, mi, mode):
    import torch

    rng = np.random.default_rng(300 + mi + 50 * mode)
    n = 4000
    wo = _dirs(rng, n)
    wi = _dirs(rng, n, below=0.5)
    front = (rng.random(n) < 0.6).astype(np.uint32)
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
    below = wi[:, 2] < 0
    rough = MATERIALS[mi]["specular_roughness"] > 0
    if MATERIALS[mi].get("transmission_weight", 0) == 0:
        assert np.all(rf[below] == 0)
    elif rough:  # the BTDF is non-zero below the surface
        assert (rf[below].max(1) > 0).mean() > 0.3 and (rp[below] > 0).mean() > 0.3
    else:
        assert np.all(rf[below] == 0) and np.all(rp[below] == 0)
    _assert_close(f, rf, "f")
    _assert_close(pdf, rp, "pdf")


@pytest.mark.parametrize("mode", [0, 1], ids=["radiance", "importance"])
@pytest.mark.parametrize("mi", range(len(MATERIALS)))
def test_transmission_sample_matches_oracle(bsdf_scene, mi, mode):
    import torch

    rng = np.random.default_rng(400 + mi + 50 * mode)
    n = 4000
    wo = _dirs(rng, n)
    u = rng.random((n, 3)).astype(np.float32)
    front = (rng.random(n) < 0.6).astype(np.uint32)
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
    if MATERIALS[mi].get("transmission_weight", 0) > 0:
        assert ((rflags & 2) != 0).mean() > 0.1  # transmission samples are drawn
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
    # transmitted directions leave below the surface
    tr = both[(rflags[both] & 2) != 0]
    assert np.all(out[tr, 5] < 0)


def device_samples(dev, sc, w, h, spp, depth, execution, integrator=tpt.INTEGRATOR_MIS):
    import torch

    n = w * h * spp
    out = torch.empty(n * 3, dtype=torch.float32, device="cuda")
    job = dev.job(sc["camera"], w, h, spp, depth, integrator=integrator, execution=execution)
    dev.render_samples_device(job, 0, n, out.data_ptr(), stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return out.cpu().numpy().reshape(n, 3)


@pytest.mark.parametrize("thin", [False, True], ids=["solid_glass", "thin_walled"])
def test_glass_cornell_renders_match_oracle(ctx, thin):
    sc = tpt_scenes.cornell_glass(2, thin_walled=thin)
    dev = tpt.Scene(ctx, sc["meshes"], sc["instances"], materials=sc["materials"])
    ref = orc.RenderScene(sc, dev.light_tree())
    w = h = 48
    spp, depth = 8, 10
    outs = []
    for execution in (tpt.EXEC_WAVEFRONT, tpt.EXEC_MEGAKERNEL):
        d = device_samples(dev, sc, w, h, spp, depth, execution)
        outs.append(d)
    assert np.array_equal(outs[0].view(np.uint32), outs[1].view(np.uint32))
    r = ref.samples(sc["camera"], w, h, spp, depth, 0, w * h * spp)
    d = outs[0]
    rel = np.abs(d - r).max(1) / np.maximum(np.abs(r).max(1), 1e-30)
    print(f"thin={thin}: within 1e-5 {(rel <= 1e-5).mean():.5f}, within 1e-3 {(rel <= 1e-3).mean():.5f}")
    assert np.all(np.isfinite(d))
    assert (rel <= 1e-5).mean() >= 0.99, (rel <= 1e-5).mean()
    assert (rel <= 1e-3).mean() >= 0.995, (rel <= 1e-3).mean()
    img = dev.render(sc["camera"], 64, 64, 16, depth)
    oimg = ref.render(sc["camera"], 64, 64, 16, depth).reshape(64, 64, 3)
    err = rel_rmse(img, oimg)
    print(f"thin={thin}: image rel RMSE {err:.3g}")
    assert err <= REL_RMSE_TOL
    dev.close()


def test_glass_cornell_bdpt_matches_oracle(ctx):
    """BDPT through the glass boxes: light and camera subpaths refract (importance
    transport on the light side), connections evaluate the BTDF."""
    sc = tpt_scenes.cornell_glass(4)
    dev = tpt.Scene(ctx, sc["meshes"], sc["instances"], materials=sc["materials"])
    ref = orc.RenderScene(sc, dev.light_tree())
    w = h = 32
    spp, depth = 4, 8
    d = device_samples(dev, sc, w, h, spp, depth, tpt.EXEC_WAVEFRONT, integrator=tpt.INTEGRATOR_BDPT)
    r = ref.samples(sc["camera"], w, h, spp, depth, 0, w * h * spp, integrator=tpt.INTEGRATOR_BDPT)
    rel = np.abs(d - r).max(1) / np.maximum(np.abs(r).max(1), 1e-30)
    print(f"BDPT glass: within 1e-5 {(rel <= 1e-5).mean():.5f}")
    assert np.all(np.isfinite(d))
    assert (rel <= 1e-5).mean() >= 0.99, (rel <= 1e-5).mean()
    assert (rel <= 1e-3).mean() >= 0.995, (rel <= 1e-3).mean()
    dev.close()
