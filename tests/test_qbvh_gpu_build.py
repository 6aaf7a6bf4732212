"""The GPU QBVH builder (tpt_qbvh_build_device) against the host builder.

The host builder produces the reference's tree (byte-identical nodes and
primitive order; tests/test_host_boundary.py).  The GPU builder must give the
same bytes for every input without -0.0 on a box face (+0.0 and -0.0 are
equal values, and the host keeps whichever it meets first): sizes around the
leaf limits and the one-thread threshold (512), random and clustered boxes,
sets with coincident centroids (forced median splits on both the thread and
the level paths), and the 1M-triangle sphere soup.  A scene uploaded with
GPU builds renders and traverses exactly like the default upload.
"""
import time

import numpy as np
import pytest

import tpt
import tpt_scenes

pytestmark = pytest.mark.gpu


def gpu_build(ctx, bounds):
    import torch

    d = torch.from_numpy(np.ascontiguousarray(bounds, np.float32)).cuda()
    out = tpt.build_qbvh_device(ctx, d.data_ptr(), bounds.shape[0], torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return out


def same(a, b):
    (na, pa), (nb, pb) = a, b
    return na.tobytes() == nb.tobytes() and np.array_equal(pa, pb)


def tri_bounds(mesh):
    tri = mesh["positions"][mesh["indices"].reshape(-1, 3)]
    return (np.concatenate([tri.min(1), tri.max(1)], 1) + np.float32(0.0)).astype(np.float32)


def random_boxes(rng, n, spread=100.0, size=1.0):
    lo = rng.uniform(0, spread, (n, 3)).astype(np.float32)
    hi = lo + rng.uniform(0, size, (n, 3)).astype(np.float32)
    return np.concatenate([lo, hi], 1) + np.float32(0.0)


@pytest.mark.parametrize("n", [1, 3, 4, 5, 16, 17, 100, 511, 512, 513, 1000, 4097, 70000])
def test_random_boxes_equal_host(ctx, n):
    rng = np.random.default_rng(n)
    b = random_boxes(rng, n)
    assert same(gpu_build(ctx, b), tpt.build_qbvh(b))


def test_clustered_and_coincident_centroids(ctx):
    rng = np.random.default_rng(3)
    # clusters of identical boxes: forced median splits, on large and small ranges
    base = random_boxes(rng, 40, spread=10.0)
    b = np.repeat(base, rng.integers(1, 3000, 40), axis=0)
    rng.shuffle(b)
    assert same(gpu_build(ctx, b), tpt.build_qbvh(b))
    # every centroid equal: no binned split anywhere
    same_box = np.tile(np.array([[1, 2, 3, 4, 5, 6]], np.float32), (5000, 1))
    assert same(gpu_build(ctx, same_box), tpt.build_qbvh(same_box))
    # coplanar centroids (zero extent on two axes) and a mix of tiny and huge boxes
    flat = random_boxes(rng, 20000)
    flat[:, [1, 4]] = np.float32(7.0)
    flat[:, [2, 5]] = np.float32(9.0)
    flat[:100, 3:] += np.float32(80.0)
    assert same(gpu_build(ctx, flat), tpt.build_qbvh(flat))


def test_sphere_soup_equals_host_and_is_faster(ctx):
    mesh = tpt_scenes.sphere_soup(seed=1)
    b = tri_bounds(mesh)
    gpu_build(ctx, b[:100000])  # warm-up
    t0 = time.perf_counter()
    g = gpu_build(ctx, b)
    t1 = time.perf_counter()
    h = tpt.build_qbvh(b)
    t2 = time.perf_counter()
    print(f"1M triangles: GPU build {1e3 * (t1 - t0):.1f} ms, host build {1e3 * (t2 - t1):.1f} ms")
    assert same(g, h)


def test_upload_with_gpu_builds(ctx):
    mesh = tpt_scenes.sphere_soup(seed=5, n_spheres=256, cube=20.0)
    mesh["positions"] = mesh["positions"] + np.float32(0.0)
    inst = [tpt_scenes.identity_instance()]
    a = tpt.Scene(ctx, [mesh], inst)
    ctx.set_gpu_build(True)
    try:
        b = tpt.Scene(ctx, [mesh], inst)
    finally:
        ctx.set_gpu_build(False)
    rays = tpt_scenes.incoherent_rays(1 << 16, seed=9, cube=20.0)
    ra, rb = a.closest_hit(rays), b.closest_hit(rays)
    assert np.array_equal(ra["prim"], rb["prim"])
    assert np.array_equal(ra["t"].view(np.uint32), rb["t"].view(np.uint32))
    a.close()
    b.close()
