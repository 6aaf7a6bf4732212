"""OpenPBR emission in the oracle and the host light-tree builder (CPU only).

OpenPbrMaterial::le (material/open_pbr.rs:351-375) radiates emission_color *
emission_luminance from the front face (both faces when thin-walled), tinted
by emission_exit_tint (608-638): the coat colour over the refracted exit path
lerped by the coat weight, times lerp(1, 1 - E_fuzz(cos), fuzz weight).
may_emit / max_emission (377-391) put such a surface in the light tree with
flux max(emission_color) * luminance * area (light_tree/builder.rs:141-148).
The reference's own unit test (open_pbr.rs:1036-1054,
emission_is_under_coat_and_fuzz) is restated first.
"""
import numpy as np
import pytest

import oracle as orc
import tpt
import tpt_scenes


def mat(**kw):
    return orc.OpenPbrMaterial(kw)


def test_emission_is_under_coat_and_fuzz():
    base = {"emission_luminance": 10.0, "emission_color": [1.0, 1.0, 1.0]}
    up = (0.0, 0.0, 1.0)
    plain = mat(**base).le(up)
    coated = mat(**base, coat_weight=1.0, coat_color=[0.25, 0.25, 0.25]).le(up)
    assert coated.max() < plain.max()
    fuzzed = mat(**base, fuzz_weight=1.0, fuzz_roughness=0.5).le(up)
    assert fuzzed.max() < plain.max()


def test_plain_emission_is_colour_times_luminance_front_face_only():
    m = mat(emission_luminance=3.0, emission_color=[0.2, 0.5, 1.0])
    rng = np.random.default_rng(3)
    for _ in range(16):
        wo = rng.normal(size=3)
        wo[2] = abs(wo[2]) + 0.05
        wo /= np.linalg.norm(wo)
        le = m.le(wo)
        np.testing.assert_array_equal(le, np.float32([0.2, 0.5, 1.0]) * np.float32(3.0))
        assert m.le(wo, front=False) is None
    thin = mat(emission_luminance=3.0, emission_color=[0.2, 0.5, 1.0], geometry_thin_walled=1)
    assert thin.le((0.0, 0.0, 1.0), front=False) is not None
    assert mat(emission_luminance=0.0).le((0.0, 0.0, 1.0)) is None


def test_coat_tint_follows_refracted_exit_path():
    """At normal exit the coat passes coat_color^1 (mu_t = 1); at grazing
    exit the refracted cosine is smaller, so the tint is darker."""
    c = np.float32([0.6, 0.75, 0.9])
    m = mat(emission_luminance=1.0, coat_weight=1.0, coat_color=c.tolist(), coat_ior=1.5)
    le0 = m.le((0.0, 0.0, 1.0))
    np.testing.assert_allclose(le0, c, rtol=1e-6)
    s = np.sin(np.radians(80.0))
    le80 = m.le((s, 0.0, np.cos(np.radians(80.0))))
    mu_t = np.sqrt(1.0 - s * s / 1.5 ** 2)
    np.testing.assert_allclose(le80, c ** (1.0 / mu_t), rtol=1e-5)
    assert np.all(le80 < le0)
    half = mat(emission_luminance=1.0, coat_weight=0.5, coat_color=c.tolist()).le((0.0, 0.0, 1.0))
    np.testing.assert_allclose(half, 1.0 + (c - 1.0) * 0.5, rtol=1e-6)


def test_light_tree_holds_openpbr_emitters_with_their_flux():
    sc = tpt_scenes.cornell_openpbr_emitter(2)
    nodes, root = tpt.build_light_tree(sc)
    leaves = nodes[nodes["left"] == 0xFFFFFFFF] if "left" in nodes.dtype.names else None
    assert leaves is not None and len(leaves) > 0
    # ceiling quad (instance 7) and the short box (instance 6): 2 + 12 triangles
    insts = sorted(set(int(i) for i in leaves["leaf_instance"]))
    assert insts == [6, 7]
    assert len(leaves) == 14
    for lf in leaves:
        m = sc["materials"][int(lf["leaf_instance"])]
        expect = np.float32(max(m["emission_color"])) * np.float32(m["emission_luminance"]) * lf["area"]
        np.testing.assert_allclose(lf["flux"], expect, rtol=1e-6)


@pytest.mark.parametrize("variant", [dict(), dict(coat=0.7, fuzz=0.4), dict(coat=0.5, thin_walled=True)],
                         ids=["plain", "coat_fuzz", "thin_coat"])
def test_oracle_emitter_render_is_finite_and_lit(variant):
    sc = tpt_scenes.cornell_openpbr_emitter(2, **variant)
    ref = orc.RenderScene(sc, tpt.build_light_tree(sc))
    img = ref.render(sc["camera"], 16, 16, 4, 6).reshape(16, 16, 3)
    assert np.all(np.isfinite(img))
    assert img.mean() > 0.01
