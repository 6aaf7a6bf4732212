"""CPU tests of the render path's host parts and the oracle's MIS integrator.

* Known answers of the reference integrator tests (integrator/mis.rs:388-434)
  on its floor + area-light fixture (integrator/mod.rs:451-523), run on the
  oracle with the light tree built by the library's host builder;
* light-tree builder invariants (light_tree/builder.rs tests);
* oracle image sanity on the Cornell-box scene.
"""
import math

import numpy as np
import pytest

import oracle as orc
import tpt
import tpt_scenes

PI = math.pi


def unit_mesh(z):
    return {"positions": np.array([[0, 0, z], [1, 0, z], [0, 1, z]], np.float32),
            "normals": np.array([[0, 0, 1]] * 3, np.float32),
            "uvs": np.array([[0, 0], [1, 0], [0, 1]], np.float32),
            "indices": np.array([0, 1, 2], np.uint32)}


def floor_with_area_light(albedo, strength):
    """integrator/mod.rs:451-460: unit triangle floor at z=0, emissive unit triangle at z=1."""
    return {
        "meshes": [unit_mesh(0.0), unit_mesh(1.0)],
        "materials": [{"kind": tpt_scenes.LAMBERT, "rho": np.full(3, albedo, np.float32)},
                      {"kind": tpt_scenes.EMISSIVE, "color": np.ones(3, np.float32), "strength": strength}],
        "instances": [tpt_scenes.identity_instance(0, 0), tpt_scenes.identity_instance(1, 1)],
    }


@pytest.fixture(scope="module")
def floor_scene():
    sc = floor_with_area_light(0.8, 10.0)
    return orc.RenderScene(sc, tpt.build_light_tree(sc))


def test_direct_light_balance_heuristic_known_answer(floor_scene):
    # mis.rs:388-408: floor vertex at bary (0.5, 0.25, 0.25) seen along -z,
    # u_tree 0, us (0.25, 0.5) -> (4/pi) * (2 / (2 + 1/pi))
    r = floor_scene.direct_light(0, 0, (0.5, 0.25, 0.25), (0, 0, -1), 0.0, (0.25, 0.5))
    expected = (4.0 / PI) * (2.0 / (2.0 + 1.0 / PI))
    assert np.allclose(r, expected, atol=1e-3), (r, expected)


def test_emitted_balance_heuristic_known_answer(floor_scene):
    # mis.rs:410-434: BSDF-sampled hit of the light vertex -> 8 * ((1/pi) / (2 + 1/pi))
    bsdf_pdf = floor_scene.material_pdf(0, 0, (0.5, 0.25, 0.25), (0, 0, -1), (0, 0, 1))
    assert abs(bsdf_pdf - 1.0 / PI) < 1e-6
    r = floor_scene.emitted(0, 0, (0.5, 0.25, 0.25), (0, 0, -1), 1, 0, (0.5, 0.25, 0.25), (0, 0, 1),
                            (0.8, 0.8, 0.8), bsdf_pdf)
    expected = 8.0 * ((1.0 / PI) / (2.0 + 1.0 / PI))
    assert np.allclose(r, expected, atol=1e-3), (r, expected)
    # mis.rs:436+: a delta BSDF sample takes the full emitted radiance
    r = floor_scene.emitted(0, 0, (0.5, 0.25, 0.25), (0, 0, -1), 1, 0, (0.5, 0.25, 0.25), (0, 0, 1),
                            (0.8, 0.8, 0.8), bsdf_pdf, delta=True)
    assert np.allclose(r, 8.0, atol=1e-4)


def test_light_tree_single_emitter():
    sc = floor_with_area_light(0.8, 10.0)
    nodes, root = tpt.build_light_tree(sc)
    assert len(nodes) == 1 and root == 0
    n = nodes[0]
    assert n["leaf_instance"] == 1 and n["leaf_triangle"] == 0
    assert abs(n["flux"] - 10.0 * 0.5) < 1e-6  # max_emission * area
    assert abs(n["area"] - 0.5) < 1e-7
    assert n["parent"] == 0xFFFFFFFF
    assert abs(n["lambda"] - 0.5 * (3 - 0.25) / 0.75) < 1e-5  # nu_bar = 0.5 n_geom


def test_light_tree_invariants_cornell_and_grid():
    sc = tpt_scenes.cornell_box(3, tpt_scenes.LAMBERT)
    # add a grid of 64 extra emitters to get a real tree
    rng = np.random.default_rng(0)
    grid = {"positions": [], "indices": []}
    for k in range(64):
        c = rng.uniform(-1.2, 1.2, 3).astype(np.float32)
        c[1] = 2.5
        base = len(grid["positions"])
        grid["positions"] += [c, c + [0.05, 0, 0], c + [0, 0, 0.05]]
        grid["indices"] += [base, base + 1, base + 2]
    sc["meshes"].append({"positions": np.array(grid["positions"], np.float32),
                         "indices": np.array(grid["indices"], np.uint32)})
    sc["materials"].append({"kind": tpt_scenes.EMISSIVE, "color": np.array([1, 0.5, 0.25], np.float32),
                            "strength": 3.0})
    sc["instances"].append(tpt_scenes.identity_instance(len(sc["meshes"]) - 1, len(sc["materials"]) - 1))
    nodes, root = tpt.build_light_tree(sc)
    leaves = nodes[nodes["leaf_instance"] != 0xFFFFFFFF]
    assert len(leaves) == 2 + 64 and len(nodes) == 2 * len(leaves) - 1
    inner = nodes[nodes["leaf_instance"] == 0xFFFFFFFF]
    # flux of an interior node is the sum of its children's (merge_cluster_params)
    for i, n in enumerate(nodes):
        if n["leaf_instance"] == 0xFFFFFFFF:
            l, r = nodes[n["left"]], nodes[n["right"]]
            assert abs(n["flux"] - (l["flux"] + r["flux"])) <= 1e-5 * n["flux"]
            assert nodes[n["left"]]["parent"] == i and nodes[n["right"]]["parent"] == i
    assert abs(nodes[root]["flux"] - leaves["flux"].sum()) <= 1e-4 * leaves["flux"].sum()
    assert np.all(inner["lambda"] >= 0)
    assert set(zip(leaves["leaf_instance"].tolist(), leaves["leaf_triangle"].tolist())) == \
        {(7, 0), (7, 1)} | {(8, k) for k in range(64)}


def test_no_emitter_is_an_error():
    sc = floor_with_area_light(0.8, 10.0)
    sc["materials"][1] = {"kind": tpt_scenes.LAMBERT, "rho": np.full(3, 0.5, np.float32)}
    with pytest.raises(tpt.TptError):
        tpt.build_light_tree(sc)


def test_oracle_cornell_render_is_finite_and_lit():
    sc = tpt_scenes.cornell_box(1, tpt_scenes.LAMBERT)
    r = orc.RenderScene(sc, tpt.build_light_tree(sc))
    img = r.render(sc["camera"], 32, 32, 4, 8)
    assert np.all(np.isfinite(img)) and np.all(img >= 0)
    assert img.mean() > 0.01
