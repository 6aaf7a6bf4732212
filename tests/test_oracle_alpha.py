"""The alpha-test filter of Scene::closest_hit in the oracle (CPU only).

closest_mesh_hit_with_filter (scene/mod.rs:686-723) keeps a candidate hit of
an instance whose material has an alpha test (opacity < 1:
normalized_lambert.rs:85-107, emissive.rs:96-118, material/open_pbr.rs:
321-343) only if u < opacity, u drawn from the path's AuxRng
(aux_rng.rs:15-29) per candidate in traversal order.  The reference's own
test (scene/mod.rs:1213-1240, a zero-opacity quad in front of an opaque one)
is restated first; then the draw count, the hit statistics of a half-
transparent quad, and renders through a cut-out material.
"""
import numpy as np

import oracle as orc
import tpt
import tpt_scenes


def pcg_transition(s):
    return (int(s) * 747796405 + 2891336453) & 0xFFFFFFFF


def two_quads(front_material, back_material=None):
    front = tpt_scenes._quad((-1, -1, 0), (1, -1, 0), (1, 1, 0), (-1, 1, 0), (0, 0, 1))
    back = tpt_scenes._quad((-1, -1, -1), (1, -1, -1), (1, 1, -1), (-1, 1, -1), (0, 0, 1))
    mats = [front_material, back_material or {"kind": tpt.LAMBERT, "rho": np.full(3, 0.5, np.float32)}]
    return {"meshes": [front, back], "instances": [tpt_scenes.identity_instance(0, 0),
                                                   tpt_scenes.identity_instance(1, 1)],
            "materials": mats}


NO_TREE = (np.zeros(0, tpt.LIGHT_NODE_DTYPE), 0xFFFFFFFF)


def test_closest_hit_skips_zero_opacity_material_and_returns_geometry_behind_it():
    sc = two_quads({"kind": tpt.LAMBERT, "rho": np.ones(3, np.float32), "opacity": 0.0})
    ref = orc.RenderScene(sc, NO_TREE)
    inst, tri, t, aux = ref.closest_alpha([[0.25, 0.25, 2.0, 0.0, 0.0, -1.0]], [pcg_transition(0)])
    assert inst[0] == 1 and abs(t[0] - 3.0) < 1e-6


def test_one_draw_per_alpha_tested_candidate():
    # opaque front: no draw; the draw happens only for the alpha-tested quad
    for opacity, draws in ((1.0, 0), (0.5, 1), (0.0, 1)):
        sc = two_quads({"kind": tpt.LAMBERT, "rho": np.ones(3, np.float32), "opacity": opacity})
        ref = orc.RenderScene(sc, NO_TREE)
        s0 = pcg_transition(12345)
        _, _, _, aux = ref.closest_alpha([[0.3, 0.1, 2.0, 0.0, 0.0, -1.0]], [s0])  # off the diagonal
        s = s0
        for _ in range(draws):
            s = pcg_transition(s)
        assert int(aux[0]) == s


def test_half_opacity_passes_half_the_rays():
    sc = two_quads({"kind": tpt.OPENPBR, "base_color": np.full(3, 0.5, np.float32), "geometry_opacity": 0.5})
    ref = orc.RenderScene(sc, NO_TREE)
    n = 4000
    rng = np.random.default_rng(1)
    rays = np.zeros((n, 6), np.float32)
    rays[:, 0:2] = rng.uniform(-0.9, 0.9, (n, 2))
    rays[:, 2] = 2.0
    rays[:, 5] = -1.0
    seeds = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
    inst, _, t, _ = ref.closest_alpha(rays, seeds)
    front = (inst == 0).mean()
    assert abs(front - 0.5) < 0.04, front
    assert np.all(np.isin(inst, [0, 1]))


def test_render_through_cutout_is_finite_and_between_the_opaque_extremes():
    """A Cornell box whose short box is a 40 %-opaque cut-out: the image lies
    between the opaque box's and the box-less one's (pixel-mean sense)."""
    def img(opacity):
        sc = tpt_scenes.cornell_box(2, tpt_scenes.LAMBERT)
        sc["materials"][6]["opacity"] = opacity
        ref = orc.RenderScene(sc, tpt.build_light_tree(sc))
        return ref.render(sc["camera"], 16, 16, 8, 5).reshape(16, 16, 3)
    a, b, c = img(1.0), img(0.4), img(0.0)
    assert np.all(np.isfinite(b))
    assert not np.array_equal(a, b) and not np.array_equal(b, c)
