"""CPU tests of point, spot and directional lights: the host light-tree builder
and the oracle's direct-light estimator.

* Known answers of the reference's MIS integrator tests (integrator/mis.rs:
  507-625) on its floor fixtures (integrator/mod.rs:462-515): a unit triangle
  floor of albedo 0.8, the shading vertex at barycentrics (0.5, 0.25, 0.25),
  i.e. (0.25, 0.25, 0), seen along -z;
* the spot cone's smoothstep falloff (light/spot.rs:91-135) and directional
  blocking (integrator/nee.rs:437-462), through the same estimator;
* the light-sampler categories (light/mod.rs:537-560): one per directional
  light, picked in proportion to luminance(color) * irradiance;
* light-tree leaves for point and spot lights (light_tree/builder.rs:848-887).
"""
import math

import numpy as np
import pytest

import oracle as orc
import tpt
import tpt_scenes

PI = math.pi
VTX = (0.5, 0.25, 0.25)  # barycentrics of (0.25, 0.25, 0) on the floor triangle
NO_TREE = (np.zeros(0, tpt.LIGHT_NODE_DTYPE), 0xFFFFFFFF)


def unit_mesh(z):
    return {"positions": np.array([[0, 0, z], [1, 0, z], [0, 1, z]], np.float32),
            "normals": np.array([[0, 0, 1]] * 3, np.float32),
            "uvs": np.array([[0, 0], [1, 0], [0, 1]], np.float32),
            "indices": np.array([0, 1, 2], np.uint32)}


def floor(albedo=0.8, blocker=False):
    sc = {"meshes": [unit_mesh(0.0)], "materials": [{"kind": tpt_scenes.LAMBERT, "rho": np.full(3, albedo, np.float32)}],
          "instances": [tpt_scenes.identity_instance(0, 0)]}
    if blocker:  # mis.rs:528-553: a Lambert unit triangle at z = 1 between the floor and the light
        sc["meshes"].append(unit_mesh(1.0))
        sc["materials"].append({"kind": tpt_scenes.LAMBERT, "rho": np.full(3, 0.5, np.float32)})
        sc["instances"].append(tpt_scenes.identity_instance(1, 1))
    return sc


def point(power, pos=(0.25, 0.25, 2.0), color=(1.0, 1.0, 1.0)):
    return {"position": pos, "color": color, "intensity": power}


def spot(power, total_deg, start_deg, direction, pos=(0.25, 0.25, 2.0)):
    return {"position": pos, "direction": direction, "color": (1.0, 1.0, 1.0), "intensity": power,
            "total_width": math.radians(total_deg), "falloff_start": math.radians(start_deg)}


def oracle_scene(sc):
    has_tree = sc.get("point_lights") or sc.get("spot_lights")
    return orc.RenderScene(sc, tpt.build_light_tree(sc) if has_tree else NO_TREE)


def direct(sc, u_category=0.0):
    return oracle_scene(sc).direct_light(0, 0, VTX, (0, 0, -1), 0.0, (0.0, 0.0), u_category)


def test_point_light_full_weight_known_answer():
    # mis.rs:507-526: power 16 pi at distance 2 -> Li = 1; 0.8/pi * cos 1 / pmf 1
    sc = floor()
    sc["point_lights"] = [point(16.0 * PI)]
    assert np.allclose(direct(sc), 0.8 / PI, atol=1e-3)


def test_point_light_occluded_is_zero():
    sc = floor(blocker=True)
    sc["point_lights"] = [point(16.0 * PI)]
    assert np.array_equal(direct(sc), np.zeros(3, np.float32))


def test_directional_light_full_weight_known_answer():
    # mis.rs:555-574: irradiance 2 along -z -> 2 * 0.8/pi
    sc = floor()
    sc["directional_lights"] = [{"direction": (0, 0, -1), "color": (1, 1, 1), "intensity": 2.0}]
    assert np.allclose(direct(sc), 1.6 / PI, atol=1e-3)


def test_directional_light_blocked_is_zero():
    # nee.rs:437-462
    sc = floor(blocker=True)
    sc["directional_lights"] = [{"direction": (0, 0, -1), "color": (1, 1, 1), "intensity": 2.0}]
    assert np.array_equal(direct(sc), np.zeros(3, np.float32))


def test_spot_light_inside_cone_known_answer():
    # mis.rs:576-600: on the axis the falloff is 1 and the spot is a point light
    sc = floor()
    sc["spot_lights"] = [spot(16.0 * PI, 30.0, 20.0, (0, 0, -1))]
    assert np.allclose(direct(sc), 0.8 / PI, atol=1e-3)


def test_spot_light_outside_cone_is_zero():
    # mis.rs:602-625: a 10/5 degree spot pointing along +x misses the floor point
    sc = floor()
    sc["spot_lights"] = [spot(16.0 * PI, 10.0, 5.0, (1, 0, 0))]
    assert np.array_equal(direct(sc), np.zeros(3, np.float32))


def test_spot_light_smoothstep_midpoint():
    # spot.rs:120-135: halfway (in cosine) between the two cone angles the
    # falloff is 0.5.  The light sits above and to the side of the floor point
    # so that the point lies on that cosine.
    total, start = math.radians(30.0), math.radians(20.0)
    mid_cos = 0.5 * (math.cos(total) + math.cos(start))
    theta = math.acos(mid_cos)
    h = 2.0
    off = h * math.tan(theta)
    sc = floor()
    sc["spot_lights"] = [spot(16.0 * PI, 30.0, 20.0, (0, 0, -1), pos=(0.25 - off, 0.25, h))]
    d2 = h * h + off * off
    cos_surface = h / math.sqrt(d2)
    expected = 0.8 / PI * 4.0 * 0.5 / d2 * cos_surface  # intensity 16 pi / 4 pi = 4
    assert np.allclose(direct(sc), expected, rtol=2e-3), (direct(sc), expected)


def test_directional_categories_pick_by_irradiance():
    # light/mod.rs:537-560: each directional light is its own category, pmf in
    # proportion to luminance * irradiance (1 : 3 here)
    sc = floor()
    d1 = np.array([1.0, 0.0, -1.0]) / math.sqrt(2.0)
    sc["directional_lights"] = [{"direction": (0, 0, -1), "color": (1, 1, 1), "intensity": 1.0},
                                {"direction": tuple(d1), "color": (1, 1, 1), "intensity": 3.0}]
    r0 = direct(sc, u_category=0.1)
    r1 = direct(sc, u_category=0.9)
    assert np.allclose(r0, 1.0 * 0.8 / PI / 0.25, rtol=1e-4)
    assert np.allclose(r1, 3.0 * 0.8 / PI * (1.0 / math.sqrt(2.0)) / 0.75, rtol=1e-4)


def test_tree_and_directional_share_the_sampler():
    # the tree category weight is the root flux (luminance * power for a
    # point light); with a directional light of the same weight both pmfs are 1/2
    sc = floor()
    sc["point_lights"] = [point(16.0 * PI)]
    sc["directional_lights"] = [{"direction": (0, 0, -1), "color": (1, 1, 1), "intensity": 16.0 * PI}]
    nodes, root = tpt.build_light_tree(sc)
    lum = 0.2126 + 0.7152 + 0.0722
    assert abs(nodes[root]["flux"] - np.float32(lum) * np.float32(16.0 * PI)) <= 1e-5 * nodes[root]["flux"]
    r_tree = direct(sc, u_category=0.25)
    r_dir = direct(sc, u_category=0.75)
    w_tree, w_dir = float(nodes[root]["flux"]), lum * 16.0 * PI
    p_tree = w_tree / (w_tree + w_dir)
    assert np.allclose(r_tree, 0.8 / PI / p_tree, rtol=1e-3)
    assert np.allclose(r_dir, 16.0 * PI * 0.8 / PI / (1.0 - p_tree), rtol=1e-3)


def test_point_light_only_tree():
    # builder.rs:848-861: one leaf, lambda ~ 0 (an undirected emitter)
    sc = floor()
    sc["point_lights"] = [point(10.0, pos=(1.0, 2.0, 3.0))]
    nodes, root = tpt.build_light_tree(sc)
    assert len(nodes) == 1 and root == 0
    n = nodes[0]
    assert n["leaf_instance"] == tpt.LIGHT_LEAF_POINT and n["leaf_triangle"] == 0
    assert abs(n["lambda"]) < 1e-5
    assert np.allclose(n["mu"], (1.0, 2.0, 3.0))


def test_spot_lambda_grows_with_narrower_cone():
    # builder.rs:863-887
    def lam(total, start):
        sc = floor()
        sc["spot_lights"] = [spot(1.0, total, start, (0, 0, -1), pos=(0, 0, 0))]
        nodes, root = tpt.build_light_tree(sc)
        assert nodes[root]["leaf_instance"] == tpt.LIGHT_LEAF_SPOT
        return float(nodes[root]["lambda"])
    assert lam(5.0, 3.0) > lam(60.0, 30.0)


def test_mixed_tree_leaf_order_and_flux():
    # leaves: the emissive triangles in instance order, then point, then spot lights
    sc = tpt_scenes.cornell_lights(2)
    nodes, root = tpt.build_light_tree(sc)
    leaves = nodes[nodes["leaf_instance"] != 0xFFFFFFFF]
    kinds = sorted(leaves["leaf_instance"].tolist())
    assert kinds.count(tpt.LIGHT_LEAF_POINT) == 1 and kinds.count(tpt.LIGHT_LEAF_SPOT) == 1
    assert len(leaves) == 4 and len(nodes) == 7  # two ceiling triangles + point + spot
    assert abs(nodes[root]["flux"] - leaves["flux"].sum()) <= 1e-5 * leaves["flux"].sum()


def test_zero_power_lights_are_skipped():
    sc = floor()
    sc["point_lights"] = [point(0.0)]
    with pytest.raises(tpt.TptError):
        tpt.build_light_tree(sc)


def test_oracle_render_with_lights_is_finite_and_lit():
    for area in (True, False):
        sc = tpt_scenes.cornell_lights(1, area=area)
        r = orc.RenderScene(sc, tpt.build_light_tree(sc))
        for integrator in (0, 1):  # MIS, BDPT
            img = r.render(sc["camera"], 24, 24, 4, 6, integrator=integrator)
            assert np.all(np.isfinite(img)) and np.all(img >= 0)
            assert img.mean() > 0.01
