"""CPU tests of the oracle's BDPT with lights that are not emissive triangles.

The reference's BDPT (integrator/bdpt.rs) keeps light subpaths on area lights
and adds, at every camera vertex of a scene with point, spot, directional or
environment lights, a light sample that skips area lights
(direct_non_area_light_contribution, :396-464), and the environment's radiance
to camera rays that leave the scene (emitted_radiance_from_infinite_hit,
:466-486).  Known answers of its tests (:853-1120) on the reference's floor
fixtures (integrator/mod.rs:451-515).
"""
import math

import numpy as np
import pytest

import oracle as orc
import tpt
import tpt_scenes
from test_oracle_lights import VTX, floor, point, spot

PI = math.pi
NO_TREE = (np.zeros(0, tpt.LIGHT_NODE_DTYPE), 0xFFFFFFFF)


def oracle_scene(sc):
    has_tree = sc.get("point_lights") or sc.get("spot_lights") or len(sc["materials"]) > 1 and any(
        m["kind"] == tpt_scenes.EMISSIVE for m in sc["materials"])
    return orc.RenderScene(sc, tpt.build_light_tree(sc) if has_tree else NO_TREE)


def non_area(sc, us=(0.0, 0.0), u_category=0.0):
    return oracle_scene(sc).direct_light(0, 0, VTX, (0, 0, -1), 0.0, us, u_category, non_area_only=True)


def test_skips_area_light_samples():
    # bdpt.rs:853-871: the floor + area light fixture gives zero
    sc = floor()
    sc["meshes"].append({"positions": np.array([[0, 0, 1], [1, 0, 1], [0, 1, 1]], np.float32),
                         "normals": np.array([[0, 0, 1]] * 3, np.float32),
                         "indices": np.array([0, 1, 2], np.uint32)})
    sc["materials"].append({"kind": tpt_scenes.EMISSIVE, "color": np.ones(3, np.float32), "strength": 10.0})
    sc["instances"].append(tpt_scenes.identity_instance(1, 1))
    r = oracle_scene(sc)
    assert np.array_equal(r.direct_light(0, 0, VTX, (0, 0, -1), 0.0, (0.25, 0.5), 0.0, non_area_only=True),
                          np.zeros(3, np.float32))
    # the MIS estimator does sample it
    assert r.direct_light(0, 0, VTX, (0, 0, -1), 0.0, (0.25, 0.5), 0.0).max() > 0.0


def test_point_light_estimator():
    sc = floor()
    sc["point_lights"] = [point(16.0 * PI)]
    assert np.allclose(non_area(sc, (0.5, 0.5)), 0.8 / PI, atol=1e-3)


def test_directional_light_estimator():
    sc = floor()
    sc["directional_lights"] = [{"direction": (0, 0, -1), "color": (1, 1, 1), "intensity": 2.0}]
    assert np.allclose(non_area(sc), 1.6 / PI, atol=1e-3)


def test_spot_light_estimator():
    sc = floor()
    sc["spot_lights"] = [spot(16.0 * PI, 30.0, 20.0, (0, 0, -1))]
    assert np.allclose(non_area(sc), 0.8 / PI, atol=1e-3)


def test_zero_when_delta_light_is_occluded():
    sc = floor(blocker=True)
    sc["point_lights"] = [point(16.0 * PI)]
    assert np.array_equal(non_area(sc), np.zeros(3, np.float32))


def test_includes_environment_light():
    # bdpt.rs:941-1004 with a vertex facing the map's bright texel: the
    # floor's normal is +z, so the bright texel is put where +z-facing
    # directions sample it
    px = np.zeros((2, 4, 3), np.float32)
    px[0, 0] = 4.0  # u in [0, 1/4), upper half: phi near +z, theta < 90 degrees
    sc = floor()
    sc["environment"] = {"pixels": px}
    env = orc.Environment(px)
    s = env.sample(0.5, 0.5, compensated=True)
    assert s is not None and s["radiance"][0] > 0.0
    r = non_area(sc, (0.5, 0.5))
    if s["direction"][2] > 0.0:
        assert np.all(r > 0.0)
    else:
        assert np.all(r == 0.0)
    # directly: at least one sample position lights the +z-facing floor
    assert max(non_area(sc, (u, v))[0] for u in (0.1, 0.5, 0.9) for v in (0.1, 0.5, 0.9)) > 0.0


def test_emitted_radiance_from_infinite_hit():
    # bdpt.rs:1034-1073: full weight for primary and delta samples, MIS otherwise
    sc = floor()
    sc["environment"] = {"pixels": np.tile(np.array([0.2, 0.4, 0.8], np.float32), (8, 16, 1))}
    r = oracle_scene(sc)
    assert np.allclose(r.env_escape((0, 1, 0), (1, 1, 1), 0.0, delta=True), [0.2, 0.4, 0.8], atol=1e-5)
    sc["environment"] = {"pixels": np.full((8, 16, 3), 2.0, np.float32)}
    r = oracle_scene(sc)
    assert np.array_equal(r.env_escape((0, 1, 0), (1, 1, 1), 0.0), np.zeros(3, np.float32))
    assert r.env_escape((0, 1, 0), (1, 1, 1), 1000.0)[0] > 2.0 * 0.9


def test_camera_ray_escape_reads_environment():
    # bdpt.rs:1085-1104
    sc = floor()
    sc["environment"] = {"pixels": np.tile(np.array([0.1, 0.4, 0.9], np.float32), (8, 16, 1))}
    r = oracle_scene(sc)
    cam = {"eye": (0.25, 0.25, 1.0), "look_at": (0.25, 0.25, 5.0), "up": (0.0, 1.0, 0.0), "fov_y": 0.2}
    smp = r.samples(cam, 4, 4, 2, 4, 0, 32, integrator=1)
    assert np.allclose(smp, [0.1, 0.4, 0.9], atol=1e-6)


def test_positive_delta_light_contribution():
    # bdpt.rs:1106-1118: the camera looks down at the floor under the point light
    sc = floor()
    sc["point_lights"] = [point(16.0 * PI)]
    r = oracle_scene(sc)
    cam = {"eye": (0.25, 0.25, 1.0), "look_at": (0.25, 0.25, 0.0), "up": (0.0, 1.0, 0.0), "fov_y": 0.05}
    smp = r.samples(cam, 2, 2, 1, 1, 0, 4, integrator=1)
    assert np.all(smp > 0.0)
    # depth 1: only the light sample of the first vertex, Li f cos / pmf (pmf 1)
    mis = r.samples(cam, 2, 2, 1, 1, 0, 4, integrator=0)
    assert np.array_equal(smp, mis)


def test_bdpt_under_uniform_environment_is_albedo_times_radiance():
    # no area lights: no light subpaths; the camera path's escaping ray takes
    # full weight (a uniform map has no compensated samples), as in MIS
    from test_oracle_environment import floor_scene
    sc = floor_scene(0.8)
    sc["environment"] = {"pixels": np.full((16, 32, 3), 2.0, np.float32)}
    r = orc.RenderScene(sc, NO_TREE)
    cam = {"eye": (0.0, 3.0, 0.0), "look_at": (0.0, 0.0, 0.5), "up": (0.0, 1.0, 0.0), "fov_y": 0.5}
    smp = r.samples(cam, 8, 8, 4, 5, 0, 256, integrator=1)
    assert np.allclose(smp, np.float32(0.8) * np.float32(2.0), rtol=1e-6)
