"""Pins the oracle's OpenPBR restatement to the reference's own unit tests.

Ported (same inputs, same bounds) from crates/renderer/src/bsdf/eon.rs:206-360,
bsdf/open_pbr.rs:2297-2560 and bsdf/directional_albedo.rs:1025-1056, plus
consistency properties of the material-level lowering (sample weight equals
f * cos / pdf, sample pdf equals the pdf query).
"""
import numpy as np
import pytest

import oracle as orc


def unit(v):
    v = np.asarray(v, np.float32)
    return (v / np.float32(np.sqrt(np.float32(np.dot(v, v))))).astype(np.float32)


# ---- bsdf/eon.rs tests -------------------------------------------------------
def test_eon_lambert_reduction_when_roughness_zero():
    wo, wi = unit([0.2, 0.3, 0.9327379]), unit([-0.1, 0.4, 0.910])
    f, _ = orc.eon_eval_pdf_batch([0.7] * 3, 0.0, wo, wi[None])
    np.testing.assert_allclose(f[0], np.full(3, 0.7 / np.pi), atol=1e-5)


def test_eon_upper_hemisphere_only():
    f, pdf = orc.eon_eval_pdf_batch([1, 1, 1], 0.5, [0, 0, 1], np.array([[0, 0, -1]], np.float32))
    assert np.all(f == 0) and pdf[0] == 0
    f, _ = orc.eon_eval_pdf_batch([1, 1, 1], 0.5, [0, 0, -1], np.array([[0, 0, 1]], np.float32))
    assert np.all(f == 0)
    assert orc.eon_sample([1, 1, 1], 0.5, [0, 0, -1], (0.5, 0.5)) is None


def test_eon_reciprocity():
    rho = [0.6, 0.4, 0.2]
    pairs = [([0, 0, 1], [0.3, -0.4, 0.866]), ([0.5, 0, 0.866], [-0.5, 0.2, 0.84]),
             ([0.7, 0, 0.71414], [0, 0.7, 0.71414])]
    for r in (0.2, 0.5, 0.9, 1.0):
        for a, b in pairs:
            wo, wi = unit(a), unit(b)
            fa, _ = orc.eon_eval_pdf_batch(rho, r, wo, wi[None])
            fb, _ = orc.eon_eval_pdf_batch(rho, r, wi, wo[None])
            np.testing.assert_allclose(fa, fb, atol=1e-5)


def test_eon_sample_weight_matches_eval_cos_over_pdf():
    rho, wo = [0.7, 0.5, 0.3], unit([0.2, -0.1, 0.9746794])
    for us in [(0.01, 0.42), (0.37, 0.82), (0.6, 0.1), (0.95, 0.5)]:
        s = orc.eon_sample(rho, 0.6, wo, us)
        assert s is not None
        f, _ = orc.eon_eval_pdf_batch(rho, 0.6, wo, s["wi"][None])
        np.testing.assert_allclose(s["weight"], f[0] * (s["wi"][2] / s["pdf"]), atol=1e-4)


def test_eon_sample_pdf_matches_pdf_query():
    wo = unit([0.3, -0.2, 0.932])
    for us in [(0.05, 0.3), (0.5, 0.7), (0.85, 0.15)]:
        s = orc.eon_sample([1, 1, 1], 0.4, wo, us)
        _, pdf = orc.eon_eval_pdf_batch([1, 1, 1], 0.4, wo, s["wi"][None])
        assert abs(s["pdf"] - pdf[0]) / max(s["pdf"], 1e-6) < 1e-4


def test_eon_pdf_integrates_to_one():
    wis, dA = orc.hemisphere_grid(256, 256)
    for wo in ([0, 0, 1], unit([0.4, 0, 0.9165151]), unit([0, 0.8, 0.6])):
        _, pdf = orc.eon_eval_pdf_batch([1, 1, 1], 0.6, wo, wis)
        assert abs(float(pdf.astype(np.float64).sum()) * dA - 1.0) < 0.005


@pytest.mark.parametrize("wo,tol", [([0, 0, 1], 0.01), ([0.6, 0, 0.8], 0.02)])
def test_eon_white_furnace(wo, tol):
    wis, dA = orc.hemisphere_grid(256, 256)
    f, _ = orc.eon_eval_pdf_batch([1, 1, 1], 1.0, wo, wis)
    e = (f.astype(np.float64) * wis[:, 2:3]).sum(0) * dA
    assert np.all(np.abs(e - 1.0) < tol), e


# ---- bsdf/open_pbr.rs tests ------------------------------------------------------
def default_params():
    return dict(base_color=[0.8, 0.6, 0.4], base=0.8, specular=1.0, specular_color=[1, 1, 1],
                specular_alpha_x=0.04, specular_alpha_y=0.04, specular_eta=1.5, transmission_eta=1.5,
                metalness=0.0, coat=0.0, coat_color=[1, 1, 1], coat_darkening=[1, 1, 1], coat_alpha_x=0.01,
                coat_alpha_y=0.01, coat_eta=1.5, fuzz=0.0, fuzz_color=[1, 1, 1], fuzz_roughness=0.3,
                transmission=0.0, transmission_color=[1, 1, 1], diffuse_roughness=0.0, subsurface=0.0,
                subsurface_color=[1, 1, 1], front_face=1)


def modulated_eta(eta, w):
    f0 = np.float32(((eta - 1.0) / (eta + 1.0)) ** 2)
    eps = np.sqrt(np.clip(np.float32(w) * f0, 0.0, 0.99999)) * np.sign(eta - 1.0)
    return float(max((1.0 + eps) / max(1.0 - eps, 1e-6), 1e-4))


WO = unit([0.25, -0.15, 0.956556])


def energy(bsdf, wo=WO):
    wis, dA = orc.hemisphere_grid(128, 128)
    f, _ = bsdf.eval_pdf_batch(wo, wis)
    return (f.astype(np.float64) * wis[:, 2:3]).sum(0) * dA


def test_default_diffuse_dominant_evaluates_finite():
    b = orc.OpenPbrParamsBsdf(default_params(), luts="const")
    assert np.all(np.isfinite(b.eval([0, 0, 1], unit([0.2, 0.3, 0.9327379]))))


@pytest.mark.parametrize("roughness", [0.35, 0.65, 0.88, 1.0])
def test_rough_dielectric_specular_within_white_furnace(roughness):
    p = default_params()
    p.update(base=0.0, base_color=[0, 0, 0])
    p["specular_alpha_x"] = p["specular_alpha_y"] = np.float32(roughness) * np.float32(roughness)
    e = energy(orc.OpenPbrParamsBsdf(p))
    assert np.all(np.isfinite(e)) and e.max() <= 1.0 + 1e-2, e


@pytest.mark.parametrize("roughness", [0.35, 0.65, 0.88, 1.0])
def test_rough_diffuse_plus_specular_does_not_gain_energy(roughness):
    p = default_params()
    p.update(base=1.0, base_color=[1, 1, 1], diffuse_roughness=1.0)
    p["specular_alpha_x"] = p["specular_alpha_y"] = np.float32(roughness) * np.float32(roughness)
    e = energy(orc.OpenPbrParamsBsdf(p))
    assert np.all(np.isfinite(e)) and e.max() <= 1.0 + 1e-2, e


def test_nonmetal_rough_specular_stays_near_dielectric_reflectance():
    p = default_params()
    a = np.float32(0.88) * np.float32(0.88)
    p.update(base=0.0, base_color=[0, 0, 0], diffuse_roughness=1.0, specular_alpha_x=a, specular_alpha_y=a)
    spec = energy(orc.OpenPbrParamsBsdf(p))
    p.update(base=1.0, base_color=[0.28, 0.04, 0.1])
    total = energy(orc.OpenPbrParamsBsdf(p))
    assert 0.005 <= spec[0] <= 0.06 and np.allclose(spec, spec[0], atol=1e-5), spec
    assert total.max() <= 1.0 + 1e-2, total


def test_low_weight_nonmetal_rough_specular_remains_low_energy():
    p = default_params()
    a = np.float32(0.88) * np.float32(0.88)
    eta = modulated_eta(1.5, 0.01)
    p.update(base=0.0, base_color=[0, 0, 0], diffuse_roughness=1.0, specular_alpha_x=a, specular_alpha_y=a,
             specular_eta=eta, transmission_eta=eta)
    spec = energy(orc.OpenPbrParamsBsdf(p, spec_eta=eta))
    assert spec.max() <= 0.004, spec


def test_zero_weight_nonmetal_rough_specular_vanishes():
    p = default_params()
    a = np.float32(0.88) * np.float32(0.88)
    eta = modulated_eta(1.5, 0.0)
    p.update(base=0.0, base_color=[0, 0, 0], specular=0.0, specular_alpha_x=a, specular_alpha_y=a,
             specular_eta=eta, transmission_eta=eta)
    spec = energy(orc.OpenPbrParamsBsdf(p, spec_eta=eta))
    assert spec.max() <= 1e-4, spec


@pytest.mark.parametrize("roughness", [0.35, 0.65, 0.88, 1.0])
def test_rough_metal_within_white_furnace(roughness):
    p = default_params()
    p.update(base=1.0, base_color=[1, 1, 1], metalness=1.0)
    p["specular_alpha_x"] = p["specular_alpha_y"] = np.float32(roughness) * np.float32(roughness)
    e = energy(orc.OpenPbrParamsBsdf(p))
    assert np.all(np.isfinite(e)) and e.max() <= 1.0 + 1.5e-2, e


def test_pure_metallic_returns_specular_lobe():
    p = default_params()
    p.update(metalness=1.0, specular_alpha_x=0.2, specular_alpha_y=0.2)
    b = orc.OpenPbrParamsBsdf(p, luts="const")
    wo = unit([0.2, -0.1, 0.9746794])
    for u in [(0.1, (0.3, 0.7)), (0.5, (0.9, 0.2)), (0.9, (0.5, 0.5))]:
        s = b.sample(wo, u[0], u[1])
        assert s is not None and s["flags"] & 1  # REFLECTION


# ---- bsdf/directional_albedo.rs tests ---------------------------------------
def test_conductor_ec_lookup_returns_cell_center_values():
    e, _ = orc.lut_conductor_ec()
    for ci, ri in [(0, 0), (7, 5), (31, 23), (63, 63)]:
        sqrt_cos = (np.float32(ci) + np.float32(0.5)) / np.float32(64)
        cos_t = sqrt_cos * sqrt_cos
        r = (np.float32(ri) + np.float32(0.5)) / np.float32(64)
        got = orc.lib().orc_lut_conductor_lookup_e(float(cos_t), float(r))
        assert abs(got - e[ri * 64 + ci]) < 1e-5


def test_conductor_ec_lookup_stays_in_bounds():
    for c in (0.0, 0.1, 0.5, 0.9, 1.0):
        for r in (0.0, 0.05, 0.25, 0.75, 1.0):
            assert 0.0 <= orc.lib().orc_lut_conductor_lookup_e(c, r) <= 1.0


def test_tables_are_albedos():
    e, e_avg = orc.lut_conductor_ec()
    assert np.all((e >= 0) & (e <= 1)) and np.all((e_avg >= 0) & (e_avg <= 1))
    # white-Fresnel GGX: the smoothest row keeps (nearly) all energy, roughness loses it
    assert e_avg[0] > 0.999 and e_avg[-1] < e_avg[0]
    de, de_avg = orc.lut_dielectric_ec()
    assert np.all((de >= 0) & (de <= 1)) and np.all((de_avg >= 0) & (de_avg <= 1))
    da = orc.lut_dielectric_albedo(1.5).reshape(64, 16, 64, 16)
    assert np.all((da >= 0) & (da <= 1))
    # near-smooth cells equal the Fresnel reflectance (4 % at normal incidence for
    # eta 1.5); rough cells lose energy to masking and rise towards grazing
    assert abs(da[-1, 0, 0, 8] - 0.04) < 1e-3
    assert 0.01 < da[-1, 0, 48, 8] < 0.04 and da[0, 0, 48, 8] > da[-1, 0, 48, 8]


# ---- material-level consistency -------------------------------------------------
MATERIALS = [
    {"base_color": [0.5, 0.4, 0.3], "base_diffuse_roughness": 1.0, "specular_roughness": 1.0},
    {"base_color": [0.9, 0.6, 0.3], "base_metalness": 1.0, "specular_roughness": 0.4},
    {"base_color": [0.2, 0.7, 0.3], "specular_roughness": 0.3, "coat_weight": 0.7, "coat_roughness": 0.2},
    {"base_color": [0.6, 0.6, 0.6], "specular_roughness": 0.5, "fuzz_weight": 0.6, "fuzz_roughness": 0.5,
     "coat_weight": 0.3, "coat_roughness": 0.1, "specular_roughness_anisotropy": 0.5, "base_metalness": 0.3},
    # rough glass, frosted glass with a tint, and a thin-walled sheet
    {"base_color": [0.8, 0.8, 0.8], "specular_roughness": 0.3, "transmission_weight": 1.0},
    {"base_color": [0.5, 0.7, 0.2], "specular_roughness": 0.6, "transmission_weight": 0.7,
     "transmission_color": [0.9, 0.6, 0.3], "coat_weight": 0.4, "coat_roughness": 0.2},
    {"base_color": [0.4, 0.5, 0.6], "specular_roughness": 0.4, "transmission_weight": 0.8,
     "geometry_thin_walled": 1, "transmission_color": [0.7, 0.8, 0.9]},
]


@pytest.mark.parametrize("mi", range(len(MATERIALS)))
def test_material_sample_consistent_with_eval_and_pdf(mi):
    m = orc.OpenPbrMaterial(MATERIALS[mi])
    rng = np.random.default_rng(mi)
    n_ok = 0
    for _ in range(200):
        wo = unit(rng.normal(size=3) * [1, 1, 0.3] + [0, 0, 1.0])
        if wo[2] <= 0.05:
            continue
        front = bool(rng.integers(2))
        u = rng.random(3).astype(np.float32)
        s = m.sample(wo, u[0], (u[1], u[2]), front=front)
        if s is None:
            continue
        n_ok += 1
        if s["flags"] & 16:  # delta
            continue
        f = m.eval(wo, s["wi"], front=front)
        pdf = m.pdf(wo, s["wi"], front=front)
        assert abs(pdf - s["pdf"]) <= 1e-6 * max(pdf, 1.0)
        np.testing.assert_allclose(s["weight"], f * (abs(s["wi"][2]) / pdf), rtol=1e-5, atol=1e-7)
    assert n_ok > 150


def test_every_untextured_parameter_is_supported():
    orc.OpenPbrMaterial({"geometry_opacity": 0.5})
    orc.OpenPbrMaterial({"emission_luminance": 2.0})
    orc.OpenPbrMaterial({"transmission_weight": 0.5})
    orc.OpenPbrMaterial({"geometry_thin_walled": 1})
    orc.OpenPbrMaterial({"thin_film_weight": 1.0})


# ---- thin film (bsdf/thin_film.rs:264-297) ----------------------------------------
def test_thin_film_zero_thickness_returns_finite_rgb():
    f = orc.thin_film_dielectric(0.7, 1.0, 1.5, 1.5, 0.0)
    assert np.all(np.isfinite(f)) and np.all(f >= 0)


def test_thin_film_dielectric_changes_response_with_thickness():
    f0 = orc.thin_film_dielectric(0.85, 1.0, 2.4, 1.5, 0.0)
    f250 = orc.thin_film_dielectric(0.85, 1.0, 2.4, 1.5, 250.0)
    f500 = orc.thin_film_dielectric(0.85, 1.0, 2.4, 1.5, 500.0)
    assert np.abs(f0 - f250).max() > 1e-3 or np.abs(f250 - f500).max() > 1e-3


def test_thin_film_conductor_returns_finite_rgb():
    f = orc.thin_film_conductor(0.7, 1.0, 2.0, [0.18, 0.42, 1.37], [3.42, 2.35, 1.77], 300.0)
    assert np.all(np.isfinite(f)) and np.all((f >= 0) & (f <= 1))


def test_thin_film_materials_sample_consistently():
    """Filmed dielectric, metal, coated and thin-walled materials: sample
    weight = f |cos| / pdf and pdf = the pdf query (finalize_rough_sample)."""
    for m in ({"specular_roughness": 0.3, "thin_film_weight": 1.0, "thin_film_thickness": 0.4},
              {"base_metalness": 1.0, "specular_roughness": 0.35, "thin_film_weight": 0.7, "thin_film_ior": 1.8},
              {"specular_roughness": 0.4, "coat_weight": 0.6, "coat_roughness": 0.2, "thin_film_weight": 1.0},
              {"specular_roughness": 0.3, "transmission_weight": 0.8, "geometry_thin_walled": 1,
               "thin_film_weight": 0.8, "thin_film_thickness": 0.3}):
        mat = orc.OpenPbrMaterial(m)
        rng = np.random.default_rng(7)
        n_ok = 0
        for _ in range(150):
            wo = unit(rng.normal(size=3) * [1, 1, 0.3] + [0, 0, 1.0])
            u = rng.random(3).astype(np.float32)
            s = mat.sample(wo, u[0], (u[1], u[2]))
            if s is None or s["flags"] & 16:
                continue
            n_ok += 1
            f = mat.eval(wo, s["wi"])
            pdf = mat.pdf(wo, s["wi"])
            assert abs(pdf - s["pdf"]) <= 1e-5 * max(pdf, 1.0)
            np.testing.assert_allclose(s["weight"], f * (abs(s["wi"][2]) / pdf), rtol=1e-4, atol=1e-7)
        assert n_ok > 80


# ---- transmission (bsdf/open_pbr.rs:2561-2643) ----------------------------------
def test_thin_walled_specular_btdf_yields_pass_through():
    """open_pbr.rs:2561-2584: a smooth thin-walled sheet transmits straight
    through (wi = -wo)."""
    p = default_params()
    p.update(thin_walled=1, transmission=1.0, transmission_alpha_x=0.0, transmission_alpha_y=0.0, specular=0.0,
             base=0.0)
    b = orc.OpenPbrParamsBsdf(p, luts="const")
    wo = unit([0.2, -0.3, 0.9327379])
    rng = np.random.default_rng(0)
    got = False
    for _ in range(32):
        u = rng.random(3)
        s = b.sample(wo, u[0], (u[1], u[2]))
        if s is not None and s["flags"] & 2:
            np.testing.assert_allclose(s["wi"], -wo, atol=1e-5)
            got = True
            break
    assert got


def refract(wo, eta):  # math/mod.rs:83-100
    sin2_t = eta * eta * max(1.0 - wo[2] * wo[2], 0.0)
    cos_t = np.sqrt(max(1.0 - sin2_t, 0.0))
    return unit([-eta * wo[0], -eta * wo[1], -cos_t])


def test_smooth_transmission_eta_controls_refraction_direction():
    """open_pbr.rs:2619-2642: the smooth BTDF refracts with the transmission
    eta (1.5), not the specular one (1.0)."""
    p = default_params()
    p.update(base=0.0, specular=0.0, transmission=1.0, transmission_alpha_x=0.0, transmission_alpha_y=0.0,
             specular_eta=1.0, transmission_eta=1.5)
    b = orc.OpenPbrParamsBsdf(p, luts="const")
    wo = unit([0.35, 0.0, 0.93675])
    s = b.sample(wo, 0.999, (0.0, 0.0))  # the last non-empty lobe: the BTDF
    assert s is not None and s["flags"] & 2 and s["flags"] & 16
    np.testing.assert_allclose(s["wi"], refract(wo, 1.0 / 1.5), atol=1e-5)


def test_rough_transmission_pdf_and_weight_consistent():
    """Rough BTDF samples (both faces): weight = f |cos| / pdf and pdf = the
    pdf query, the identities finalize_rough_sample (open_pbr.rs:1997-2027)
    builds them from; the pdf over the lower hemisphere integrates below 1."""
    for front in (1, 0):
        p = default_params()
        p.update(base=0.0, transmission=1.0, specular_alpha_x=0.2, specular_alpha_y=0.2, transmission_alpha_x=0.2,
                 transmission_alpha_y=0.2, front_face=front)
        b = orc.OpenPbrParamsBsdf(p, luts="real")
        rng = np.random.default_rng(front)
        n_t = 0
        for _ in range(300):
            wo = unit(rng.normal(size=3) * [1, 1, 0.3] + [0, 0, 1.0])
            u = rng.random(3)
            s = b.sample(wo, u[0], (u[1], u[2]))
            if s is None or not (s["flags"] & 2):
                continue
            n_t += 1
            assert s["wi"][2] < 0
            f = b.eval(wo, s["wi"])
            pdf = b.pdf(wo, s["wi"])
            assert abs(pdf - s["pdf"]) <= 1e-5 * max(pdf, 1.0)
            np.testing.assert_allclose(s["weight"], f * (abs(s["wi"][2]) / pdf), rtol=1e-4, atol=1e-7)
        assert n_t > 50
        wis, dA = orc.hemisphere_grid(256, 256)
        wis = wis * [1, 1, -1]
        _, pdf = b.eval_pdf_batch(WO, wis)
        assert 0.3 < float(pdf.astype(np.float64).sum() * dA) <= 1.0 + 1e-2
