"""The oracle's path-replay adjoint (CPU, test infrastructure).

The reference renderer is not differentiable, so the adjoint has no reference
known answers; these tests pin the oracle's estimator with identities that hold
exactly for any set of samples:

* Base colour, one bounce: with specular_weight 0 and metalness 0 the OpenPBR
  BSDF is linear in base_color, so at max_depth 1 every sample that scatters
  once satisfies sum_c bc_c * dL/dbc_c = L_c (the central difference of a
  linear function is exact).  Summed over the image: sum_m bc[m] * grad[m] =
  image(depth 1) - image(depth 0), per channel.  With a directional light or
  an environment map the light samples at the first vertex (f at the light
  direction) and the escaping rays enter both sides.
* Masking: groups left out of the mask get exactly zero; groups are computed
  independently of each other.
* Linearity in dLoss/dimage, and zero gradients for a zero dLoss/dimage.
"""
import numpy as np
import pytest

import oracle as orc
import tpt
import tpt_scenes


SUN = {"direction": (-0.35, -0.45, -1.0), "color": (1.0, 0.95, 0.9), "intensity": 1.5}


def linear_scene(extra=None):
    sc = tpt_scenes.cornell_patches()
    for m in sc["materials"][:64]:
        m["specular_weight"] = 0.0
        m["base_metalness"] = 0.0
    if extra == "directional":  # light samples at OpenPBR vertices: f at the light direction
        sc["directional_lights"] = [SUN]
    elif extra == "environment":  # the same, plus escaping rays
        sc["environment"] = tpt_scenes.sky_environment(rotate_y=0.35)
    return sc


@pytest.fixture(scope="module", params=[None, "directional", "environment"],
                ids=["area", "area+directional", "area+environment"])
def lin(request):
    sc = linear_scene(request.param)
    return sc, orc.RenderScene(sc, tpt.build_light_tree(sc))


def test_linear_base_color_identity(lin):
    sc, R = lin
    W, spp = 24, 8
    d_image = np.ones(W * W * 3, np.float32)
    g = R.adjoint(sc["camera"], W, W, spp, 1, d_image, mask=tpt.GRAD_MASK_BASE_COLOR)
    img1 = R.render(sc["camera"], W, W, spp, 1).astype(np.float64).sum(0)
    img0 = R.render(sc["camera"], W, W, spp, 0).astype(np.float64).sum(0)
    bc = np.array([m["base_color"] for m in sc["materials"][:64]], np.float64)
    lhs = (g[:64, :3] * bc).sum(0)
    assert np.all(lhs > 0)
    np.testing.assert_allclose(lhs, img1 - img0, rtol=2e-4)
    assert np.all(g[64] == 0)  # the emitter has no parameters


@pytest.fixture(scope="module")
def patches():
    sc = tpt_scenes.cornell_patches()
    return sc, orc.RenderScene(sc, tpt.build_light_tree(sc))


def test_mask_selects_groups(patches):
    sc, R = patches
    W, spp = 24, 16
    d_image = np.random.default_rng(3).uniform(0.5, 1.5, W * W * 3).astype(np.float32)
    full = R.adjoint(sc["camera"], W, W, spp, 6, d_image, mask=tpt.GRAD_ALL)
    for bit, cols in ((tpt.GRAD_MASK_BASE_COLOR, [0, 1, 2]), (tpt.GRAD_MASK_ROUGHNESS, [3]),
                      (tpt.GRAD_MASK_METALNESS, [4]), (tpt.GRAD_MASK_COAT, [6])):
        g = R.adjoint(sc["camera"], W, W, spp, 6, d_image, mask=bit)
        others = [c for c in range(7) if c not in cols]
        assert np.all(g[:, others] == 0)
        np.testing.assert_allclose(g[:, cols], full[:, cols], rtol=1e-12)  # thread sums: any order
    assert np.any(full[:, 3] != 0) and np.any(full[:, 6] != 0)


def test_linear_in_d_image(patches):
    sc, R = patches
    W, spp = 24, 16
    rng = np.random.default_rng(4)
    d1 = rng.uniform(0.0, 1.0, W * W * 3).astype(np.float32)
    d2 = rng.uniform(-1.0, 1.0, W * W * 3).astype(np.float32)
    g1 = R.adjoint(sc["camera"], W, W, spp, 6, d1)
    g2 = R.adjoint(sc["camera"], W, W, spp, 6, d2)
    g12 = R.adjoint(sc["camera"], W, W, spp, 6, (d1 + d2).astype(np.float32))
    assert np.abs(g1).max() > 0
    np.testing.assert_allclose(g12, g1 + g2, rtol=1e-5, atol=1e-6 * np.abs(g1).max())
    assert np.all(R.adjoint(sc["camera"], W, W, spp, 6, np.zeros(W * W * 3, np.float32)) == 0)


def test_seeded_streams_are_independent_and_unbiased(patches):
    """Sample-stream seeds: seed 0 is the default image; another seed gives a
    different image of the same expectation (the two images' pixel-mean
    difference is within noise)."""
    sc, R = patches
    W, spp = 24, 16
    a = R.render(sc["camera"], W, W, spp, 4)
    assert np.array_equal(a, R.render(sc["camera"], W, W, spp, 4, seed=0))
    imgs = np.stack([R.render(sc["camera"], W, W, spp, 4, seed=s) for s in range(1, 17)])
    assert not np.array_equal(imgs[0], a)
    means = imgs.reshape(16, -1).mean(1)
    se = means.std(ddof=1) / np.sqrt(len(means))
    assert abs(float(a.mean()) - float(means.mean())) < 4.0 * se * np.sqrt(17.0)


def test_backward_with_another_seed_is_unbiased_at_the_truth(patches):
    """At the true parameters the gradient of an L2 loss against an
    independent target has zero mean when the backward pass replays paths of
    another seed than the forward image's (the default of tpt.render_function);
    replaying the forward's own paths biases it by the covariance of the image
    noise with the path derivatives."""
    sc, R = patches
    W, spp, depth, reps = 16, 8, 4, 48
    totals = {False: [], True: []}
    for k in range(reps):
        target = R.render(sc["camera"], W, W, 64, depth, seed=1000 + k).reshape(-1)
        fs = 2 * k + 1
        d = 2.0 * (R.render(sc["camera"], W, W, spp, depth, seed=fs).reshape(-1) - target)
        for same in (False, True):
            seed = fs if same else (fs + tpt.ADJOINT_SEED_STEP) & 0xFFFFFFFF
            g = R.adjoint(sc["camera"], W, W, spp, depth, d.astype(np.float32), mask=tpt.GRAD_MASK_BASE_COLOR,
                          seed=seed)
            totals[same].append(g[:64, :3].sum())
    z = {s: np.mean(t) / (np.std(t, ddof=1) / np.sqrt(reps)) for s, t in totals.items()}
    print("z of the summed gradient: other seed", z[False], "same paths", z[True])
    assert abs(z[False]) < 3.5
    assert z[True] > 5.0
