"""Device-side checks surface through the C ABI.

The reference's traversal stack holds 128 entries (`qbvh.rs:609`, checked by a
debug_assert at `qbvh.rs:666`), and scene queries report misuse through
`ClosestHitError` (`scene/mod.rs:100-113`).  On the device the stack-depth
check sets a per-context error word and stops the ray without writing past the
stack.  Host-buffer calls read that word before returning; `*_device` calls
leave it for `tpt_context_check`, which names the entry points whose work set it.

The scene here is a valid QBVH (every child index in range, every leaf range
inside the primitive list) that is deliberately deep: a chain of 200 interior
nodes, each with two hit children — the next chain node (near) and a small
box farther along the ray — so a closest-hit query keeps one more entry on the
stack per level and passes 128 entries at level 129.
"""
import numpy as np
import pytest

import tpt

pytestmark = pytest.mark.gpu

EMPTY = 0x80000000
LEAF_ONE = 0x80000000 | (1 << 24)  # leaf with primitive range [0, 1)
INF = np.float32(np.inf)


def deep_chain_qbvh(levels=200):
    """Nodes 2k (chain) and 2k+1 (side box) for k < levels, then the chain's end."""
    n = 2 * levels + 1
    nodes = np.zeros(n, tpt.NODE_DTYPE)
    nodes["b"][:, 0:3, :] = INF  # empty lanes: inverted boxes
    nodes["b"][:, 3:6, :] = -INF
    nodes["children"][:] = EMPTY

    def lane(i, k, lo, hi, word):
        for a in range(3):
            nodes["b"][i, a, k] = lo[a]
            nodes["b"][i, 3 + a, k] = hi[a]
        nodes["children"][i, k] = word
        nodes["valid_mask"][i] |= 1 << k

    chain_lo, chain_hi = (-2, -2, -5), (2, 2, 60)
    side_lo, side_hi = (-2, -2, 40), (2, 2, 60)
    for k in range(levels):
        i = 2 * k
        lane(i, 0, chain_lo, chain_hi, i + 2)  # entered at t = 5: popped first
        lane(i, 1, side_lo, side_hi, i + 1)  # entered at t = 50: stays on the stack
        lane(i + 1, 0, side_lo, side_hi, LEAF_ONE)
    lane(n - 1, 0, side_lo, side_hi, LEAF_ONE)
    return nodes, np.zeros(1, np.uint32)


def deep_scene(ctx):
    mesh = {
        "positions": np.array([[-1, -1, 50], [1, -1, 50], [0, 1, 50]], np.float32),
        "indices": np.array([0, 1, 2], np.uint32),
        "qbvh": deep_chain_qbvh(),
    }
    eye = np.eye(4, dtype=np.float32)
    inst = {"mesh": 0, "local_to_world": eye, "world_to_local": eye, "normal_to_world": np.eye(3, dtype=np.float32)}
    return tpt.Scene(ctx, [mesh], [inst])


def rays_down_the_chain(n=64):
    r = np.zeros((7, n), np.float32)
    r[0] = np.linspace(-0.1, 0.1, n)
    r[2] = -10.0
    r[5] = 1.0
    r[6] = np.inf
    return r


def test_deep_tree_is_valid_and_shallow_rays_still_hit(ctx):
    """The chain uploads (the validator accepts it); a ray that misses the
    chain's boxes stays shallow and reports no error."""
    scene = deep_scene(ctx)
    r = rays_down_the_chain(4)
    r[0] = 5.0  # x = 5: outside every box
    out = scene.closest_hit(r)
    assert np.all(out["prim"] == -1)
    ctx.check()
    scene.close()


def test_stack_overflow_reported_by_host_call(ctx):
    scene = deep_scene(ctx)
    with pytest.raises(tpt.TptError) as ei:
        scene.closest_hit(rays_down_the_chain())
    assert ei.value.status == 6  # TPT_ERR_DEVICE_CHECK
    assert "stack depth 128" in str(ei.value)
    ctx.check()  # the host call read and cleared the word
    scene.close()


def test_stack_overflow_reported_by_context_check_after_device_call(ctx):
    import torch

    scene = deep_scene(ctx)
    r = torch.from_numpy(rays_down_the_chain()).cuda()
    n = r.shape[1]
    prim = torch.empty(n, dtype=torch.int32, device="cuda")
    t = torch.empty(n, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    # the launch itself succeeds: its device-side check is read later
    scene.traverse_device(r.data_ptr(), n, tpt.CLOSEST_HIT, prim.data_ptr(), t.data_ptr(), stream=stream)
    with pytest.raises(tpt.TptError) as ei:
        ctx.check(stream)
    assert ei.value.status == 6
    assert "tpt_traverse_device" in str(ei.value)
    ctx.check(stream)  # cleared: a second check passes
    # any-hit queries overflow as well: every leaf sits in a side box that is
    # deferred on the stack, so no hit ends the descent first
    scene.traverse_device(r.data_ptr(), n, tpt.ANY_HIT, prim.data_ptr(), t.data_ptr(), stream=stream)
    with pytest.raises(tpt.TptError):
        ctx.check(stream)
    scene.close()


def test_check_passes_after_clean_device_work(ctx):
    import tpt_scenes
    import torch

    mesh = tpt_scenes.sphere_soup(seed=3, n_spheres=16, cube=10.0)
    scene = tpt.Scene(ctx, [mesh], [tpt_scenes.identity_instance()])
    rays = torch.from_numpy(tpt_scenes.incoherent_rays(1024, seed=2, cube=10.0)).cuda()
    prim = torch.empty(1024, dtype=torch.int32, device="cuda")
    t = torch.empty(1024, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    scene.traverse_device(rays.data_ptr(), 1024, tpt.CLOSEST_HIT, prim.data_ptr(), t.data_ptr(), stream=stream)
    ctx.check(stream)
    scene.close()
