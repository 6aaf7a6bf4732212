"""CPU tests of the oracle's NEE and PT integrators (integrator/nee.rs, pt.rs).

* Known answers of the reference's NEE tests (nee.rs:284-435) on its floor
  fixtures: the light-sampling estimator without MIS (area light 4/pi, point,
  directional and spot lights as for MIS), zero when occluded;
* the environment through the NEE integrator's plain distribution (a uniform
  map has samples there, none in the MIS-compensated one);
* PT and NEE camera rays that escape read the map (pt.rs:96-113); a diffuse
  floor under a uniform map is albedo x radiance in every PT sample;
* MIS, NEE, PT and BDPT estimate the same image under area and environment
  light: their means agree within their standard errors.
"""
import math

import numpy as np
import pytest

import oracle as orc
import tpt
import tpt_scenes
from test_oracle_lights import VTX, floor, point, spot
from test_oracle_render import floor_with_area_light

PI = math.pi
NO_TREE = (np.zeros(0, tpt.LIGHT_NODE_DTYPE), 0xFFFFFFFF)
MIS, BDPT, NEE, PT = 0, 1, 2, 3


def scene_of(sc):
    try:
        tree = tpt.build_light_tree(sc)
    except tpt.TptError:
        tree = NO_TREE
    return orc.RenderScene(sc, tree)


def nee_direct(sc, us=(0.0, 0.0), u_tree=0.0):
    return scene_of(sc).direct_light(0, 0, VTX, (0, 0, -1), u_tree, us, 0.0, nee=True)


def test_nee_area_light_estimator():
    # nee.rs:284-302: one area light (pmf 1): the classic estimator 4/pi
    sc = floor_with_area_light(0.8, 10.0)
    assert np.allclose(nee_direct(sc, (0.25, 0.5)), 4.0 / PI, atol=1e-3)


def test_nee_zero_when_occluded():
    # nee.rs:305-331: a blocker at z = 0.5
    sc = floor_with_area_light(0.8, 10.0)
    sc["meshes"].append({"positions": np.array([[0, 0, 0.5], [1, 0, 0.5], [0, 1, 0.5]], np.float32),
                         "normals": np.array([[0, 0, 1]] * 3, np.float32),
                         "indices": np.array([0, 1, 2], np.uint32)})
    sc["materials"].append({"kind": tpt_scenes.LAMBERT, "rho": np.full(3, 0.5, np.float32)})
    sc["instances"].append(tpt_scenes.identity_instance(2, 2))
    assert np.array_equal(nee_direct(sc, (0.25, 0.5)), np.zeros(3, np.float32))


@pytest.mark.parametrize("light,expected", [("point", 0.8 / PI), ("directional", 1.6 / PI), ("spot", 0.8 / PI)])
def test_nee_delta_light_estimators(light, expected):
    # nee.rs:371-435
    sc = floor()
    if light == "point":
        sc["point_lights"] = [point(16.0 * PI)]
    elif light == "directional":
        sc["directional_lights"] = [{"direction": (0, 0, -1), "color": (1, 1, 1), "intensity": 2.0}]
    else:
        sc["spot_lights"] = [spot(16.0 * PI, 30.0, 20.0, (0, 0, -1))]
    assert np.allclose(nee_direct(sc), expected, atol=1e-3)


def test_nee_samples_uniform_environment():
    # the plain distribution of a uniform map: pdf 1/(4 pi), no MIS weight
    sc = floor()
    sc["environment"] = {"pixels": np.full((8, 16, 3), 2.0, np.float32)}
    r = scene_of(sc)
    env = orc.Environment(sc["environment"]["pixels"])
    hits = 0
    for us in [(0.1, 0.2), (0.3, 0.3), (0.6, 0.45), (0.9, 0.1)]:
        s = env.sample(*us)
        got = r.direct_light(0, 0, VTX, (0, 0, -1), 0.0, us, 0.0, nee=True)
        if s["direction"][2] <= 0.0:
            assert np.all(got == 0.0)
            continue
        expected = s["radiance"] * (0.8 / PI) * s["direction"][2] / s["pdf"]
        assert np.allclose(got, expected, rtol=1e-4), (got, expected)
        hits += 1
        assert np.all(r.direct_light(0, 0, VTX, (0, 0, -1), 0.0, us, 0.0) == 0.0)  # MIS: no compensated sample
    assert hits >= 1


@pytest.mark.parametrize("integrator", [NEE, PT])
def test_camera_ray_escape_reads_environment(integrator):
    from test_oracle_environment import floor_scene
    sc = floor_scene()
    sc["environment"] = {"pixels": np.tile(np.array([0.2, 0.4, 0.8], np.float32), (8, 16, 1))}
    r = orc.RenderScene(sc, NO_TREE)
    cam = {"eye": (0.0, 1.0, 0.0), "look_at": (0.0, 5.0, 0.1), "up": (0.0, 0.0, 1.0), "fov_y": 0.2}
    assert np.allclose(r.samples(cam, 4, 4, 2, 4, 0, 32, integrator=integrator), [0.2, 0.4, 0.8], atol=1e-6)


def test_pt_floor_under_uniform_environment():
    from test_oracle_environment import floor_scene
    sc = floor_scene(0.8)
    sc["environment"] = {"pixels": np.full((16, 32, 3), 2.0, np.float32)}
    r = orc.RenderScene(sc, NO_TREE)
    cam = {"eye": (0.0, 3.0, 0.0), "look_at": (0.0, 0.0, 0.5), "up": (0.0, 1.0, 0.0), "fov_y": 0.5}
    assert np.allclose(r.samples(cam, 8, 8, 4, 5, 0, 256, integrator=PT), np.float32(1.6), rtol=1e-6)


def test_integrators_agree_in_the_mean():
    # unbiased estimators of the same image (area light and environment; PT
    # cannot see delta lights, as in the reference): the image means agree
    # within their standard errors
    sc = tpt_scenes.cornell_environment(1, tpt_scenes.LAMBERT)
    r = orc.RenderScene(sc, tpt.build_light_tree(sc))
    w = h = 16
    spp, depth = 64, 6
    means = {}
    for integ in (MIS, NEE, PT, BDPT):
        smp = r.samples(sc["camera"], w, h, spp, depth, 0, w * h * spp, integrator=integ).astype(np.float64)
        means[integ] = (smp.mean(0), smp.std(0) / math.sqrt(len(smp)))
    m0, e0 = means[MIS]
    for integ in (NEE, PT, BDPT):
        m, e = means[integ]
        assert np.all(np.abs(m - m0) <= 5.0 * np.sqrt(e * e + e0 * e0)), (integ, m, m0, e, e0)
