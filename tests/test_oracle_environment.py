"""CPU tests of the environment light (light/environment.rs) on the oracle.

* The reference's unit tests of EnvironmentLight (environment.rs:535-846):
  uv mapping round trips, uniform maps with pdf 1/(4 pi), sample/pdf
  consistency, zero maps, peaked maps, the MIS-compensated distribution, the
  pyramid layout, non-power-of-two maps and rotation about +y;
* its use by the MIS integrator (integrator/mis.rs:461-506, 627-654,
  nee.rs:334-368): camera rays that escape read the map, a lone diffuse floor
  under a uniform map returns albedo x radiance for every sample (a uniform map
  has no MIS-compensated samples, so escaping BSDF samples take full weight),
  the NEE estimator against its closed form, and a mixed area + environment
  render.
"""
import math

import numpy as np
import pytest

import oracle as orc
import tpt
import tpt_scenes

PI = math.pi
NO_TREE = (np.zeros(0, tpt.LIGHT_NODE_DTYPE), 0xFFFFFFFF)


def uniform(width, height, radiance):
    return orc.Environment(np.full((height, width, 3), radiance, np.float32))


def texel_of(direction, width, height):
    uv = orc.env_direction_to_uv(direction)
    return int(uv[0] * width), int(uv[1] * height)


def test_direction_uv_roundtrip_on_axes():
    for d in np.eye(3).tolist() + (-np.eye(3)).tolist():
        uv = orc.env_direction_to_uv(d)
        assert np.allclose(orc.env_uv_to_direction(*uv), d, atol=1e-5), d


def test_uv_to_direction_is_unit():
    assert abs(np.linalg.norm(orc.env_uv_to_direction(0.37, 0.62)) - 1.0) < 1e-5


@pytest.mark.parametrize("w,h,uv,tol", [(128, 64, (0.25, 0.5), 5e-3), (120, 60, (0.31, 0.47), 1e-2)])
def test_uniform_environment_has_inverse_sphere_pdf(w, h, uv, tol):
    env = uniform(w, h, 1.0)
    assert abs(env.pdf(orc.env_uv_to_direction(*uv)) - 1.0 / (4.0 * PI)) < tol


def _check_samples_match_pdf(env, us, compensated=False):
    for u, v in us:
        s = env.sample(u, v, compensated)
        assert s is not None
        q = env.pdf(s["direction"], compensated)
        assert abs(s["pdf"] - q) / max(s["pdf"], 1e-6) < 1e-3, (s["pdf"], q)
        assert abs(np.linalg.norm(s["direction"]) - 1.0) < 1e-5
        assert s["pdf"] > 0.0


US = [(0.1, 0.1), (0.5, 0.5), (0.8, 0.3), (0.95, 0.85)]


def test_sample_pdf_matches_pdf_query():
    px = np.full((8, 16, 3), 0.05, np.float32)
    px[3, 9] = 10.0
    _check_samples_match_pdf(orc.Environment(px), US)


def test_zero_radiance_environment_returns_no_sample():
    env = uniform(8, 4, 0.0)
    assert env.sample(0.5, 0.5) is None
    assert env.pdf((0, 1, 0)) == 0.0


def test_uniform_environment_has_no_mis_compensated_samples():
    env = uniform(8, 4, 1.0)
    assert env.sample(0.5, 0.5, compensated=True) is None
    assert env.pdf((0, 1, 0), compensated=True) == 0.0


def test_peaked_environment_concentrates_samples_on_bright_pixel():
    px = np.full((16, 32, 3), 1e-4, np.float32)
    px[6, 10] = 1e6
    env = orc.Environment(px)
    for u, v in [(0.1, 0.1), (0.4, 0.4), (0.7, 0.7), (0.95, 0.05)]:
        assert texel_of(env.sample(u, v)["direction"], 32, 16) == (10, 6)


def test_mis_compensated_environment_keeps_only_above_mean_texels():
    px = np.ones((2, 4, 3), np.float32)
    px[1, 2] = 9.0
    env = orc.Environment(px)
    assert env.pdf(orc.env_uv_to_direction(0.125, 0.25), compensated=True) == 0.0
    assert env.pdf(orc.env_uv_to_direction(2.5 / 4, 1.5 / 2), compensated=True) > 0.0
    for u, v in [(0.1, 0.1), (0.4, 0.4), (0.7, 0.7), (0.95, 0.95)]:
        assert texel_of(env.sample(u, v, compensated=True)["direction"], 4, 2) == (2, 1)


def test_mis_compensated_mean_uses_spherical_jacobian():
    px = np.zeros((4, 1, 3), np.float32)
    px[0] = 4.0
    px[1] = 1.2
    env = orc.Environment(px)
    assert env.pdf(orc.env_uv_to_direction(0.5, 0.375), compensated=True) > 0.0


def test_mis_compensated_sample_pdf_matches_pdf_query():
    px = np.full((8, 16, 3), 0.2, np.float32)
    px[2, 4] = 8.0
    px[5, 11] = 4.0
    _check_samples_match_pdf(orc.Environment(px), US, compensated=True)


def test_integrated_pdf_over_sphere_is_one():
    env = uniform(64, 32, 1.0)
    n, acc = 4096, 0.0
    for k in range(n):
        u1 = ((k * 2654435761) & 0xFFFFFF) / float(0x1000000)
        u2 = ((k * 40503) & 0xFFFFFF) / float(0x1000000)
        z = 1.0 - 2.0 * u1
        r = math.sqrt(max(1.0 - z * z, 0.0))
        phi = 2.0 * PI * u2
        acc += env.pdf((r * math.cos(phi), z, r * math.sin(phi)))
    assert abs(acc / n * 4.0 * PI - 1.0) < 5e-2


def test_pyramid_root_holds_total_weight_and_levels_collapse_to_root():
    # environment.rs:754-777 on weights luminance(pixel) * sin(row centre): a
    # 3 x 2 map pads to 4 x 2 and collapses (4, 2) -> (2, 1) -> (1, 1)
    vals = np.arange(1, 7, dtype=np.float32).reshape(2, 3)
    env = orc.Environment(np.repeat(vals[:, :, None], 3, axis=2))
    dims, total, leaf = env.pyramid()
    assert dims == [(1, 1), (2, 1), (4, 2)]
    st = np.sin(np.float32((np.arange(2) + 0.5) / 2) * np.float32(PI)).astype(np.float32)
    lum = np.float32(0.2126) * vals + np.float32(0.7152) * vals + np.float32(0.0722) * vals
    assert np.array_equal(leaf[:, :3], (lum * st[:, None]).astype(np.float32))
    assert np.all(leaf[:, 3] == 0.0)
    assert abs(total - leaf.sum()) <= 1e-5 * total


def test_non_power_of_two_environment_sample_lands_in_valid_region():
    px = np.full((3, 5, 3), 1e-3, np.float32)
    px[1, 3] = 8.0
    env = orc.Environment(px)
    for u, v in [(0.05, 0.05), (0.5, 0.5), (0.95, 0.5), (0.5, 0.95)]:
        s = env.sample(u, v)
        i, j = texel_of(s["direction"], 5, 3)
        assert i < 5 and j < 3
        assert abs(s["pdf"] - env.pdf(s["direction"])) / max(s["pdf"], 1e-6) < 1e-3


def test_rotate_y_rotates_radiance_and_keeps_pdf_consistent():
    px = np.full((8, 16, 3), 0.05, np.float32)
    px[3, 4] = 20.0
    rot = PI / 2
    rotated, plain = orc.Environment(px, 1.0, rot), orc.Environment(px, 1.0, 0.0)
    local = orc.env_uv_to_direction(4.5 / 16, 3.5 / 8)
    c, s = math.cos(rot), math.sin(rot)
    turned = np.array([c * local[0] + s * local[2], local[1], -s * local[0] + c * local[2]], np.float32)
    assert np.linalg.norm(plain.radiance(local) - rotated.radiance(turned)) < 1e-3
    _check_samples_match_pdf(rotated, [(0.1, 0.2), (0.4, 0.6), (0.85, 0.55)])


def test_total_power_of_uniform_map():
    # total_power = total weight x scale x texel solid angle ~ 4 pi L for a uniform map
    env = orc.Environment(np.full((32, 64, 3), 0.5, np.float32), scale=2.0)
    assert abs(env.total_power() - 4.0 * PI * 1.0) < 2e-2 * 4.0 * PI


# ---- the MIS integrator with an environment ---------------------------------

def floor_scene(albedo=0.8):
    return {"meshes": [{"positions": np.array([[-50, 0, -50], [50, 0, -50], [50, 0, 50], [-50, 0, 50]], np.float32),
                        "normals": np.array([[0, 1, 0]] * 4, np.float32),
                        "indices": np.array([0, 2, 1, 0, 3, 2], np.uint32)}],
            "materials": [{"kind": tpt_scenes.LAMBERT, "rho": np.full(3, albedo, np.float32)}],
            "instances": [tpt_scenes.identity_instance(0, 0)]}


def test_camera_ray_escape_reads_environment():
    # mis.rs:490-505: a camera ray that leaves the scene returns the map's radiance
    sc = floor_scene()
    sc["environment"] = {"pixels": np.tile(np.array([0.1, 0.4, 0.9], np.float32), (8, 16, 1))}
    ref = orc.RenderScene(sc, NO_TREE)
    cam = {"eye": (0.0, 1.0, 0.0), "look_at": (0.0, 5.0, 0.1), "up": (0.0, 0.0, 1.0), "fov_y": 0.2}
    smp = ref.samples(cam, 4, 4, 2, 4, 0, 32)
    assert np.allclose(smp, [0.1, 0.4, 0.9], atol=1e-6)


def test_floor_under_uniform_environment_is_albedo_times_radiance():
    # a uniform map has no MIS-compensated samples (NEE returns zero) and an
    # escaping BSDF sample then takes MIS weight balance(pdf, 0) = 1
    # (mis.rs:461-488): every sample is albedo x L exactly
    sc = floor_scene(0.8)
    sc["environment"] = {"pixels": np.full((16, 32, 3), 2.0, np.float32)}
    ref = orc.RenderScene(sc, NO_TREE)
    cam = {"eye": (0.0, 3.0, 0.0), "look_at": (0.0, 0.0, 0.5), "up": (0.0, 1.0, 0.0), "fov_y": 0.5}
    smp = ref.samples(cam, 8, 8, 4, 5, 0, 256)
    assert np.allclose(smp, np.float32(0.8) * np.float32(2.0), rtol=1e-6)


def test_environment_nee_closed_form():
    # direct_light_mis_contribution with the environment as the only category
    # (pmf 1): Li f cos / pdf x balance(pdf, bsdf_pdf) on a Lambert floor
    px = np.full((8, 16, 3), 0.2, np.float32)
    px[2, 3] = (9.0, 6.0, 3.0)
    px[1, 12] = (4.0, 4.0, 4.0)
    sc = floor_scene(0.8)
    sc["environment"] = {"pixels": px, "scale": 1.5, "rotate_y": 0.3}
    ref = orc.RenderScene(sc, NO_TREE)
    env = orc.Environment(px, 1.5, 0.3)
    hits = 0
    for us in [(0.1, 0.2), (0.3, 0.7), (0.6, 0.4), (0.9, 0.9), (0.45, 0.15)]:
        r = ref.direct_light(0, 0, (0.2, 0.3, 0.5), (0, -1, 0), 0.0, us, 0.5)
        s = env.sample(*us, compensated=True)
        if s is None or s["direction"][1] <= 0.0:
            assert np.all(r == 0.0)
            continue
        cos = float(s["direction"][1])
        f, bsdf_pdf = 0.8 / PI, cos / PI
        mis = s["pdf"] / (s["pdf"] + bsdf_pdf)
        expected = s["radiance"] * f * cos * mis / s["pdf"]
        assert np.allclose(r, expected, rtol=1e-4), (r, expected)
        hits += 1
    assert hits >= 2


def test_area_light_and_environment_mix():
    # mis.rs:627-654
    sc = tpt_scenes.cornell_box(1, tpt_scenes.LAMBERT)
    sc["environment"] = {"pixels": np.full((8, 16, 3), 0.2, np.float32)}
    ref = orc.RenderScene(sc, tpt.build_light_tree(sc))
    for integrator in (0, 1):  # MIS, BDPT
        img = ref.render(sc["camera"], 16, 16, 4, 4, integrator=integrator)
        assert np.all(np.isfinite(img)) and np.all(img.mean(0) > 0.0)
