"""Dispersion in the oracle (CPU only): bsdf/dispersion.rs and the dispersive
OpenPBR BTDF (bsdf/open_pbr.rs:1024-1051, 1154-1222, 1250-1427, 1670-1928).

The reference's own unit tests are restated first (dispersion.rs:221-292:
the Cauchy IOR at the d line, disabled at Abbe 0, red below blue; the camera
basis over uniform and throughput-weighted wavelength samples integrating to
white; sampled wavelengths inside the camera table; open_pbr.rs:2587-2616:
a rough dispersive BTDF sample locks a wavelength with positive weight in all
channels; material/open_pbr.rs:987-994: the dispersion scale maps to the Abbe
number).  Then properties of the restatement itself: the camera-integrated
evaluation is the basis-weighted sum of locked evaluations at the interval
midpoints, the camera-mixture pdf integrates to one over the sphere, and a
locked path refracts as a non-dispersive glass of the Cauchy IOR.
"""
import numpy as np
import pytest

import oracle as orc

from test_oracle_openpbr import default_params


def test_cauchy_returns_n_d_at_d_line():
    assert abs(orc.cauchy_ior(587.56, 1.5, 50.0) - 1.5) < 1e-4


def test_cauchy_disabled_at_zero_abbe_returns_n_d():
    assert abs(orc.cauchy_ior(450.0, 1.5, 0.0) - 1.5) < 1e-6


def test_cauchy_red_lower_than_blue():
    assert orc.cauchy_ior(656.0, 1.5, 30.0) < orc.cauchy_ior(486.0, 1.5, 30.0)


@pytest.mark.parametrize("throughput", [(1.0, 1.0, 1.0), (0.8, 0.35, 0.1)], ids=["uniform", "weighted"])
def test_dispersion_basis_integrates_to_white(throughput):
    n = 200_000
    acc = np.zeros(3, np.float64)
    for i in range(0, n, 7):  # every 7th of the reference's 200k midpoints
        _, basis = orc.sample_dispersion_wavelength((i + 0.5) / n, throughput)
        acc += basis
    avg = acc / len(range(0, n, 7))
    assert np.all(np.abs(avg - 1.0) < 5e-3), avg


def test_dispersion_wavelength_stays_in_camera_table_range():
    n = 4096
    for i in range(n):
        lam, basis = orc.sample_dispersion_wavelength((i + 0.5) / n)
        assert 400.0 <= lam <= 720.0
        assert np.all(basis >= 0.0)


def test_camera_channel_wavelengths_stay_in_table_range():
    n = 4096
    for ch in range(3):
        for i in range(0, n, 3):
            assert 400.0 <= orc.sample_camera_channel_wavelength(ch, (i + 0.5) / n) <= 720.0


def test_rough_dispersion_sample_uses_camera_channel_wavelengths():
    p = default_params()
    p.update(base=0.0, specular=0.0, transmission=1.0, transmission_alpha_x=0.45, transmission_alpha_y=0.45,
             transmission_dispersion_abbe=20.0, path_throughput=[0.8, 0.5, 0.3])
    b = orc.OpenPbrParamsBsdf(p, luts="const")
    # the reference calls sample_spec_btdf with p_lobe = 1; through sample()
    # u_lobe near 1 picks the transmission lobe (the last one with weight)
    s = b.sample((0.0, 0.0, 1.0), 0.999, (0.37, 0.82), u_extra=(0.41, 0.17, 0.53, 0.91))
    assert s is not None and s["flags"] & 2  # transmission
    assert s["wavelength_lock"] is not None and 400.0 <= s["wavelength_lock"] <= 720.0
    assert np.all(s["weight"] > 0.0)


def glass(**kw):
    m = {"base_color": [0.8, 0.8, 0.8], "specular_roughness": 0.35, "transmission_weight": 1.0,
         "transmission_dispersion_scale": 1.0, "transmission_dispersion_abbe_number": 20.0}
    m.update(kw)
    return orc.OpenPbrMaterial(m)


def test_dispersion_scale_maps_to_abbe_number():
    """scale 0.25 with Abbe number 20 is Abbe 80 (80 / 1.0 exactly); scale 0
    turns dispersion off, so a lock changes nothing."""
    wo, wi = (0.3, 0.1, 0.948683), (-0.2, 0.05, -0.978286)
    a = glass(transmission_dispersion_scale=0.25, transmission_dispersion_abbe_number=20.0)
    b = glass(transmission_dispersion_scale=1.0, transmission_dispersion_abbe_number=80.0)
    for lock in (None, 450.0, 650.0):
        np.testing.assert_array_equal(a.eval(wo, wi, lock=lock), b.eval(wo, wi, lock=lock))
    off = glass(transmission_dispersion_scale=0.0)
    np.testing.assert_array_equal(off.eval(wo, wi, lock=450.0), off.eval(wo, wi))
    on = glass()
    assert not np.array_equal(on.eval(wo, wi, lock=450.0), on.eval(wo, wi, lock=650.0))


def test_camera_integrated_eval_is_basis_weighted_sum_of_locked_evals():
    """Where every wavelength has a refraction half vector (elsewhere the
    locked evaluation drops its multiple-scattering term with the single-
    scattering one, open_pbr.rs:1034-1037, while the integrated one keeps it,
    1272-1286)."""
    m = glass()
    wo = np.float32([0.3, 0.1, 0.948683])
    rng = np.random.default_rng(3)
    checked = 0
    for _ in range(24):
        wi = rng.normal(size=3)
        wi[2] = -abs(wi[2]) - 0.2
        wi /= np.linalg.norm(wi)
        lams = 400.0 + 10.0 * (np.arange(32) + 0.5)
        # one wavelength's value is grey (no film, colourless glass)
        locked = [m.eval(wo, wi, lock=lam).astype(np.float64) for lam in lams]
        if any(v.max() == 0.0 for v in locked):
            continue
        ref = sum(orc.camera_rgb_basis_at(lam) * v * 10.0 for lam, v in zip(lams, locked))
        np.testing.assert_allclose(m.eval(wo, wi), ref, rtol=2e-4)
        checked += 1
    assert checked >= 8


def test_camera_mixture_pdf_integrates_to_one():
    """The unlocked pdf mixes the 32 per-wavelength pdfs with the throughput-
    weighted wavelength pdf, so it is still a density over the sphere."""
    m = glass(base_color=[0.8, 0.8, 0.8])
    wo = (0.3, 0.1, 0.948683)
    n_z, n_phi = 192, 192
    z = (np.arange(n_z) + 0.5) / n_z
    phi = (np.arange(n_phi) + 0.5) / n_phi * 2 * np.pi
    total = 0.0
    for sign in (1.0, -1.0):
        for zz in z:
            r = np.sqrt(1 - zz * zz)
            for pp in phi[::4]:
                total += m.pdf(wo, (r * np.cos(pp), r * np.sin(pp), sign * zz), throughput=(0.8, 0.5, 0.3))
    total *= (1.0 / n_z) * (2 * np.pi / n_phi) * 4
    assert abs(total - 1.0) < 0.03, total


def test_locked_smooth_glass_refracts_with_cauchy_ior():
    m = glass(specular_roughness=0.0)
    wo = np.float32([0.5, 0.0, np.sqrt(0.75)])
    for lam in (420.0, 550.0, 700.0):
        eta = orc.cauchy_ior(lam, 1.5, 20.0)
        s = None
        for u in np.linspace(0.05, 0.95, 19):
            t = m.sample(wo, u, (0.5, 0.5), lock=lam)
            if t is not None and t["flags"] & 2:
                s = t
                break
        assert s is not None and s["wavelength_lock"] is None  # already locked: no new lock
        sin_t = np.hypot(s["wi"][0], s["wi"][1])
        assert abs(sin_t - 0.5 / eta) < 1e-5
