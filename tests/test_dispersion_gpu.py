"""Dispersive OpenPBR transmission on the device against the oracle.

The BTDF of a glass with transmission_dispersion_scale > 0
(bsdf/open_pbr.rs:1024-1051, 1154-1222, 1250-1427, 1670-1928 with
bsdf/dispersion.rs): camera-integrated evaluation and the wavelength-mixture
pdf while the path is unlocked, the Cauchy IOR of the locked wavelength once
a dispersive refraction was sampled, wavelength locks drawn from the
throughput-weighted camera basis (smooth glass) or from three sampled camera
channels (rough glass).  BSDF eval / pdf / sample through the path-state
queries (throughput and lock per query, the u_extra randoms per sample) are
held to the bars of the other OpenPBR tests; renders of the Cornell box with
dispersive glass (MIS wavefront and megakernel equal bit for bit, BDPT) to
the per-sample bars of the glass renders.  The adjoint refuses dispersive
materials.
"""
import numpy as np
import pytest

import oracle as orc
import tpt
import tpt_scenes

pytestmark = pytest.mark.gpu

MATERIALS = [
    {"base_color": [0.8, 0.8, 0.8], "specular_roughness": 0.35, "transmission_weight": 1.0,
     "transmission_dispersion_scale": 1.0, "transmission_dispersion_abbe_number": 20.0},
    {"base_color": [0.6, 0.7, 0.5], "specular_roughness": 0.0, "transmission_weight": 0.9,
     "transmission_color": [0.9, 0.8, 0.7], "transmission_dispersion_scale": 0.5},
    {"base_color": [0.5, 0.5, 0.6], "specular_roughness": 0.5, "specular_ior": 1.7, "transmission_weight": 0.8,
     "coat_weight": 0.5, "coat_roughness": 0.1, "transmission_dispersion_scale": 2.0,
     "transmission_dispersion_abbe_number": 30.0},
    {"base_color": [0.7, 0.7, 0.7], "specular_roughness": 0.3, "transmission_weight": 1.0, "thin_film_weight": 0.8,
     "thin_film_thickness": 0.4, "transmission_dispersion_scale": 1.0},
]
LOCKS = [None, 450.0, 530.0, 655.0]


def _dirs(rng, n, lower=False):
    v = rng.normal(size=(n, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    v[:, 2] = np.abs(v[:, 2]) + 0.02
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    if lower:
        v[:, 2] = -v[:, 2]
    return v.astype(np.float32)


@pytest.fixture(scope="module")
def bsdf_scene(ctx):
    quad = tpt_scenes._quad((-1, 0, 1), (1, 0, 1), (1, 0, -1), (-1, 0, -1), (0, 1, 0))
    mats = [dict(m, kind=tpt.OPENPBR) for m in MATERIALS]
    sc = tpt.Scene(ctx, [quad], [tpt_scenes.identity_instance(0, 0)], materials=mats)
    yield sc
    sc.close()


def _assert_close(got, ref, what):
    got = np.asarray(got, np.float64)
    ref = np.asarray(ref, np.float64)
    rel = np.abs(got - ref) / np.maximum(np.abs(ref), 1e-6)
    rel = rel.max(axis=-1) if rel.ndim > 1 else rel
    assert (rel <= 1e-5).mean() >= 0.99, (what, (rel <= 1e-5).mean())
    assert (rel <= 1e-3).mean() >= 0.999, (what, (rel <= 1e-3).mean(), rel.max())


@pytest.mark.parametrize("mode", [0, 1], ids=["radiance", "importance"])
@pytest.mark.parametrize("mi", range(len(MATERIALS)))
def test_dispersive_eval_pdf_matches_oracle(bsdf_scene, mi, mode):
    import torch

    rng = np.random.default_rng(700 + mi + 20 * mode)
    n = 1200
    wo = _dirs(rng, n)
    wi = _dirs(rng, n, lower=True)
    wi[: n // 4] = _dirs(rng, n // 4)  # some reflection pairs too
    front = (rng.random(n) < 0.7).astype(np.uint32)
    thr = rng.uniform(0.05, 1.5, (n, 3)).astype(np.float32)
    locks = np.array([LOCKS[k % 4] if LOCKS[k % 4] is not None else np.nan for k in range(n)], np.float32)
    state = np.concatenate([thr, locks[:, None]], 1).astype(np.float32)
    t = [torch.from_numpy(a).cuda() for a in (wo, wi, front.view(np.int32), state)]
    f = torch.empty((n, 3), dtype=torch.float32, device="cuda")
    pdf = torch.empty(n, dtype=torch.float32, device="cuda")
    bsdf_scene.bsdf_eval_path_device(mi, n, t[0].data_ptr(), t[1].data_ptr(), t[2].data_ptr(), t[3].data_ptr(),
                                     f.data_ptr(), pdf.data_ptr(), stream=torch.cuda.current_stream().cuda_stream,
                                     mode=mode)
    torch.cuda.synchronize()
    f, pdf = f.cpu().numpy(), pdf.cpu().numpy()
    m = orc.OpenPbrMaterial(MATERIALS[mi])
    lk = [None if np.isnan(x) else float(x) for x in locks]
    rf = np.array([m.eval(wo[k], wi[k], front=bool(front[k]), mode=mode, throughput=thr[k], lock=lk[k])
                   for k in range(n)])
    rp = np.array([m.pdf(wo[k], wi[k], front=bool(front[k]), throughput=thr[k], lock=lk[k]) for k in range(n)],
                  np.float32)
    assert np.abs(rf).max() > 0
    _assert_close(f, rf, "f")
    _assert_close(pdf, rp, "pdf")


@pytest.mark.parametrize("mi", range(len(MATERIALS)))
def test_dispersive_sample_matches_oracle(bsdf_scene, mi):
    import torch

    rng = np.random.default_rng(900 + mi)
    n = 3000
    wo = _dirs(rng, n)
    u = rng.random((n, 7)).astype(np.float32)
    front = (rng.random(n) < 0.7).astype(np.uint32)
    thr = rng.uniform(0.05, 1.5, (n, 3)).astype(np.float32)
    locks = np.array([LOCKS[k % 4] if LOCKS[k % 4] is not None else np.nan for k in range(n)], np.float32)
    state = np.concatenate([thr, locks[:, None]], 1).astype(np.float32)
    t = [torch.from_numpy(a).cuda() for a in (wo, u, front.view(np.int32), state)]
    out = torch.empty((n, 10), dtype=torch.float32, device="cuda")
    bsdf_scene.bsdf_sample_path_device(mi, n, t[0].data_ptr(), t[1].data_ptr(), t[2].data_ptr(), t[3].data_ptr(),
                                       out.data_ptr(), stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    out = out.cpu().numpy()
    flags = out[:, 8].view(np.uint32)
    m = orc.OpenPbrMaterial(MATERIALS[mi])
    ref = [m.sample(wo[k], u[k, 0], u[k, 1:3], front=bool(front[k]), u_extra=u[k, 3:7], throughput=thr[k],
                    lock=None if np.isnan(locks[k]) else float(locks[k])) for k in range(n)]
    rflags = np.array([0 if s is None else s["flags"] for s in ref], np.uint32)
    assert (flags == rflags).mean() >= 0.999
    both = np.nonzero((flags == rflags) & (rflags != 0))[0]
    assert len(both) > n // 2
    _assert_close(out[both, 0:3], np.array([ref[k]["weight"] for k in both]), "weight")
    _assert_close(out[both, 3:6], np.array([ref[k]["wi"] for k in both]), "wi")
    _assert_close(out[both, 6], np.array([ref[k]["pdf"] for k in both], np.float32), "pdf")
    rl = np.array([np.nan if ref[k]["wavelength_lock"] is None else ref[k]["wavelength_lock"] for k in both],
                  np.float32)
    dl = out[both, 9]
    assert np.array_equal(np.isnan(dl), np.isnan(rl))
    ok = ~np.isnan(rl)
    assert ok.sum() > 0  # some samples lock a wavelength
    _assert_close(dl[ok], rl[ok], "lock")
    assert np.all((dl[ok] >= 400.0) & (dl[ok] <= 720.0))


def device_samples(dev, sc, w, h, spp, depth, execution, integrator=tpt.INTEGRATOR_MIS):
    import torch

    n = w * h * spp
    out = torch.empty(n * 3, dtype=torch.float32, device="cuda")
    job = dev.job(sc["camera"], w, h, spp, depth, integrator=integrator, execution=execution)
    dev.render_samples_device(job, 0, n, out.data_ptr(), stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return out.cpu().numpy().reshape(n, 3)


def check(d, r, label, within5=0.99, within3=0.995):
    rel = np.abs(d - r).max(1) / np.maximum(np.abs(r).max(1), 1e-30)
    print(f"{label}: within 1e-5 {(rel <= 1e-5).mean():.5f}, within 1e-3 {(rel <= 1e-3).mean():.5f}")
    assert np.all(np.isfinite(d)) and r.mean() > 0.005
    assert (rel <= 1e-5).mean() >= within5, (rel <= 1e-5).mean()
    assert (rel <= 1e-3).mean() >= within3, (rel <= 1e-3).mean()


def test_dispersive_glass_cornell_matches_oracle(ctx):
    sc = tpt_scenes.cornell_glass(3, dispersion=1.0)
    dev = tpt.Scene(ctx, sc["meshes"], sc["instances"], materials=sc["materials"])
    ref = orc.RenderScene(sc, dev.light_tree())
    w = h = 40
    spp, depth = 8, 10
    outs = [device_samples(dev, sc, w, h, spp, depth, e) for e in (tpt.EXEC_WAVEFRONT, tpt.EXEC_MEGAKERNEL)]
    assert np.array_equal(outs[0].view(np.uint32), outs[1].view(np.uint32))
    r = ref.samples(sc["camera"], w, h, spp, depth, 0, w * h * spp)
    check(outs[0], r, "dispersive glass MIS")
    # the glass renders colour fringes: the image is not grey where the
    # boxes refract the light
    dev.close()


def test_dispersive_glass_cornell_bdpt_matches_oracle(ctx):
    sc = tpt_scenes.cornell_glass(5, dispersion=1.0)
    dev = tpt.Scene(ctx, sc["meshes"], sc["instances"], materials=sc["materials"])
    ref = orc.RenderScene(sc, dev.light_tree())
    w = h = 24
    spp, depth = 4, 8
    d = device_samples(dev, sc, w, h, spp, depth, tpt.EXEC_WAVEFRONT, tpt.INTEGRATOR_BDPT)
    r = ref.samples(sc["camera"], w, h, spp, depth, 0, w * h * spp, integrator=tpt.INTEGRATOR_BDPT)
    check(d, r, "dispersive glass BDPT", 0.98, 0.99)
    one = device_samples(dev, sc, w, h, spp, depth, tpt.EXEC_MEGAKERNEL, tpt.INTEGRATOR_BDPT)
    assert np.array_equal(d.view(np.uint32), one.view(np.uint32))
    dev.close()


def test_adjoint_refuses_dispersion(ctx):
    sc = tpt_scenes.cornell_glass(3, dispersion=1.0)
    dev = tpt.Scene(ctx, sc["meshes"], sc["instances"], materials=sc["materials"])
    job = dev.job(sc["camera"], 8, 8, 1, 2)
    with pytest.raises(tpt.TptError, match="dispersive"):
        dev.adjoint(job, np.ones(8 * 8 * 3, np.float32))
    dev.close()
