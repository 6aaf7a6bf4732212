"""The device path-replay adjoint (tpt_adjoint_device) and material updates.

* Parity: on the 64-patch Cornell box the device gradients equal the oracle's
  (the same estimator on the CPU with the same per-pixel streams, accumulated
  in double) to 1e-4 relative over the whole gradient vector.
* Exact identity: with a BSDF linear in base_color (specular_weight 0,
  metalness 0) and one bounce, sum_m bc[m] * grad[m] = image(depth 1) -
  image(depth 0).
* Unbiasedness: against central finite differences of the forward renderer
  with common random numbers (h = 1e-2) on a linear loss, each of the 12
  largest components agrees within 4 combined standard errors; both standard
  errors come from 16 interleaved pixel subsets.  (Finite differences of the
  attached renderer move sampled directions and flip lobe and Russian-roulette
  decisions with theta, so their variance is far above the adjoint's.)
* Material updates: a render after tpt_scene_set_openpbr equals a render of a
  freshly uploaded scene with the new parameters, bit for bit.
* Inverse rendering: Adam on the 64 patch materials from a perturbed start
  lowers the L2 image loss (measured at 256 spp) against a 1024-spp target.
"""
import numpy as np
import pytest

import oracle as orc
import tpt
import tpt_scenes

pytestmark = pytest.mark.gpu

PARITY_TOL = 1e-4
Z_MAX = 4.0


@pytest.fixture(scope="module")
def patches(ctx):
    sc = tpt_scenes.cornell_patches()
    scene = tpt.Scene(ctx, sc["meshes"], sc["instances"], materials=sc["materials"])
    return sc, scene


def _stream():
    import torch

    return torch.cuda.current_stream().cuda_stream


def render(scene, sc, W, spp, depth=6):
    import torch

    job = scene.job(sc["camera"], W, W, spp, depth)
    img = torch.empty(W * W * 3, device="cuda")
    scene.render_device(job, img.data_ptr(), _stream())
    torch.cuda.synchronize()
    return img.double().cpu().numpy()


def adjoint(scene, sc, W, spp, d_image, depth=6, mask=0, step=0.0, seed=0):
    import torch

    job = scene.job(sc["camera"], W, W, spp, depth, seed=seed)
    d = torch.from_numpy(np.ascontiguousarray(d_image, np.float32)).cuda()
    g = torch.zeros(scene.n_materials * tpt.GRAD_PARAMS, dtype=torch.float64, device="cuda")
    scene.adjoint_device(job, d.data_ptr(), g.data_ptr(), mask, step, _stream())
    torch.cuda.synchronize()
    return g.cpu().numpy().reshape(scene.n_materials, tpt.GRAD_PARAMS)


def set_params(scene, params):
    scene.set_openpbr(list(range(len(params))), [tpt_scenes.patch_material(p) for p in params], stream=_stream())


def test_adjoint_matches_oracle(patches):
    sc, scene = patches
    W, spp = 32, 16
    d_image = np.random.default_rng(0).uniform(0.5, 1.5, W * W * 3).astype(np.float32)
    gd = adjoint(scene, sc, W, spp, d_image)
    go = orc.RenderScene(sc, scene.light_tree()).adjoint(sc["camera"], W, W, spp, 6, d_image)
    assert np.abs(go).max() > 0
    assert np.linalg.norm(gd - go) / np.linalg.norm(go) <= PARITY_TOL
    # host-buffer entry point: the same computation
    gh = scene.adjoint(scene.job(sc["camera"], W, W, spp, 6), d_image)
    assert np.linalg.norm(gh - gd) / np.linalg.norm(gd) <= 1e-12
    # another sample-stream seed: the oracle's gradient of that seed
    seed = tpt.ADJOINT_SEED_STEP
    gs = adjoint(scene, sc, W, spp, d_image, seed=seed)
    gso = orc.RenderScene(sc, scene.light_tree()).adjoint(sc["camera"], W, W, spp, 6, d_image, seed=seed)
    assert np.linalg.norm(gs - gso) / np.linalg.norm(gso) <= PARITY_TOL
    assert np.linalg.norm(gs - gd) / np.linalg.norm(gd) > 1e-3


def test_linear_base_color_identity(ctx):
    sc = tpt_scenes.cornell_patches()
    for m in sc["materials"][:64]:
        m["specular_weight"] = 0.0
        m["base_metalness"] = 0.0
    scene = tpt.Scene(ctx, sc["meshes"], sc["instances"], materials=sc["materials"])
    W, spp = 64, 16
    g = adjoint(scene, sc, W, spp, np.ones(W * W * 3, np.float32), depth=1, mask=tpt.GRAD_MASK_BASE_COLOR)
    img1 = render(scene, sc, W, spp, 1).reshape(-1, 3).sum(0)
    img0 = render(scene, sc, W, spp, 0).reshape(-1, 3).sum(0)
    bc = np.array([m["base_color"] for m in sc["materials"][:64]], np.float64)
    lhs = (g[:64, :3] * bc).sum(0)
    np.testing.assert_allclose(lhs, img1 - img0, rtol=2e-4)
    assert np.all(g[:, 3:] == 0)
    scene.close()


def test_adjoint_agrees_with_finite_differences(patches):
    sc, scene = patches
    W, spp, h, K = 128, 256, 1e-2, 16
    rng = np.random.default_rng(1)
    w = rng.uniform(0.5, 1.5, W * W * 3).astype(np.float32)
    pix = np.arange(W * W)
    subsets = [np.repeat(pix % K == k, 3) for k in range(K)]
    g_sub = np.stack([adjoint(scene, sc, W, spp, np.where(m, w, 0.0)) for m in subsets])
    g = g_sub.sum(0)
    se_adj = np.sqrt(K) * g_sub.std(0, ddof=1)
    p0 = sc["params"].copy()
    top = np.argsort(-np.abs(g[:64, :5]).reshape(-1))[:12]
    zs = []
    try:
        for o in top:
            mi, k = divmod(int(o), 5)
            pp, pm = p0.copy(), p0.copy()
            pp[mi, k] += h
            pm[mi, k] -= h
            set_params(scene, pp)
            ip = render(scene, sc, W, spp)
            set_params(scene, pm)
            im = render(scene, sc, W, spp)
            per_pix = ((ip - im) / (2 * h) * w)
            fd_sub = np.array([per_pix[m].sum() for m in subsets])
            fd, se_fd = fd_sub.sum(), np.sqrt(K) * fd_sub.std(ddof=1)
            z = (g[mi, k] - fd) / np.hypot(se_adj[mi, k], se_fd)
            zs.append(z)
            print(f"material {mi} param {k}: adjoint {g[mi, k]:.4g} +- {se_adj[mi, k]:.2g}  fd {fd:.4g} +- {se_fd:.2g}"
                  f"  z {z:.2f}")
    finally:
        set_params(scene, p0)
    assert np.max(np.abs(zs)) <= Z_MAX


def test_set_openpbr_matches_fresh_upload(ctx, patches):
    sc, scene = patches
    p = tpt_scenes.patch_params(5, start=True)
    set_params(scene, p)
    try:
        a = render(scene, sc, 48, 8)
        sc2 = tpt_scenes.with_patch_params(sc, p)
        fresh = tpt.Scene(ctx, sc2["meshes"], sc2["instances"], materials=sc2["materials"])
        b = render(fresh, sc2, 48, 8)
        fresh.close()
        assert np.array_equal(a, b)
    finally:
        set_params(scene, sc["params"])
    with pytest.raises(tpt.TptError):
        scene.set_openpbr([64], [tpt_scenes.patch_material(p[0])])  # the emitter is not OpenPBR


def test_adjoint_rejects_bdpt_and_bad_masks(patches):
    import torch

    sc, scene = patches
    d = torch.ones(16 * 16 * 3, device="cuda")
    g = torch.zeros(scene.n_materials * 7, dtype=torch.float64, device="cuda")
    job = scene.job(sc["camera"], 16, 16, 4, 4, integrator=tpt.INTEGRATOR_BDPT)
    with pytest.raises(tpt.TptError):
        scene.adjoint_device(job, d.data_ptr(), g.data_ptr())
    job = scene.job(sc["camera"], 16, 16, 4, 4)
    with pytest.raises(tpt.TptError):
        scene.adjoint_device(job, d.data_ptr(), g.data_ptr(), mask=64)


def visible_patches(scene, sc, W, min_frac=0.01):
    """Materials (one per patch instance) seen directly by at least min_frac of
    the pixels: the parameters the image constrains."""
    out = scene.closest_hit(tpt_scenes.pixel_center_rays(sc["camera"], W, W), want_instance=True)
    inst = out["inst"][out["prim"] >= 0]
    counts = np.bincount(inst, minlength=len(sc["instances"]))[:tpt_scenes.N_PATCH_MATERIALS]
    return np.nonzero(counts >= min_frac * W * W)[0]


def test_inverse_rendering_lowers_loss(ctx):
    """200 Adam steps (lr 0.003) on the 64 patch materials from a perturbed
    start, 128x128 at 16 spp forward and adjoint, every step with fresh sample
    streams (seed = step + 1; the backward pass replays another seed's paths,
    so they are independent of the forward image's): the image loss measured
    at 256 spp against the 1024-spp target must fall below 0.6 of its start,
    and the base-colour error of the patches the camera sees (at least 1 % of
    the pixels each) must fall.  Roughness and metalness are
    printed, not checked: they trade off against each other and against base
    colour in the image."""
    import torch

    sc = tpt_scenes.cornell_patches()
    W, spp, depth = 128, 16, 6
    st = _stream()
    target_scene = tpt.Scene(ctx, sc["meshes"], sc["instances"], materials=sc["materials"])
    target = torch.from_numpy(render(target_scene, sc, W, 1024, depth)).float().cuda().view(W, W, 3)
    target_scene.close()
    start = tpt_scenes.patch_params(5, start=True)
    sc0 = tpt_scenes.with_patch_params(sc, start)
    scene = tpt.Scene(ctx, sc0["meshes"], sc0["instances"], materials=sc0["materials"])

    def clean_loss(p):
        set_params(scene, p)
        img = torch.from_numpy(render(scene, sc, W, 256, depth)).float().cuda().view(W, W, 3)
        return float(((img - target) ** 2).sum())

    loss0 = clean_loss(start)
    RenderFunction = tpt.render_function()
    params = torch.tensor(start, requires_grad=True)
    opt = torch.optim.Adam([params], lr=0.003)
    lo = torch.tensor([0.02, 0.02, 0.02, 0.05, 0.0])
    hi = torch.tensor([0.98, 0.98, 0.98, 1.0, 1.0])
    mask = tpt.GRAD_MASK_BASE_COLOR | tpt.GRAD_MASK_ROUGHNESS | tpt.GRAD_MASK_METALNESS
    for step in range(200):
        opt.zero_grad()
        job = scene.job(sc["camera"], W, W, spp, depth, seed=step + 1)
        img = RenderFunction.apply(params, scene, job, list(range(64)), tpt_scenes.patch_material, mask)
        loss = ((img - target) ** 2).sum()
        loss.backward()
        opt.step()
        with torch.no_grad():
            params.copy_(torch.maximum(torch.minimum(params, hi), lo))
    p = params.detach().numpy()
    loss1 = clean_loss(p)
    vis = visible_patches(scene, sc, W)
    bc0 = np.abs(start[vis, :3] - sc["params"][vis, :3]).mean()
    bc1 = np.abs(p[vis, :3] - sc["params"][vis, :3]).mean()
    print("256-spp image loss", loss0, "->", loss1, "; all parameters' error", np.abs(start - sc["params"]).mean(),
          "->", np.abs(p - sc["params"]).mean(), f"; base colour of the {len(vis)} visible patches", bc0, "->", bc1,
          "; roughness", np.abs(start[vis, 3] - sc["params"][vis, 3]).mean(), "->",
          np.abs(p[vis, 3] - sc["params"][vis, 3]).mean(), "; metalness",
          np.abs(start[vis, 4] - sc["params"][vis, 4]).mean(), "->", np.abs(p[vis, 4] - sc["params"][vis, 4]).mean())
    assert len(vis) >= 20
    assert loss1 < 0.6 * loss0
    assert bc1 < bc0
    scene.close()
