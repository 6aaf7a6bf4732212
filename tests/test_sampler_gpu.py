"""The device's sample streams equal the oracle's, value for value.

The sampler (`sampler/{zsobol,pcg,path_sampler}.rs`) is integer work: the
Z-Sobol index permutation (`zsobol.rs:230-285`), the Owen-scrambled Sobol
points (`zsobol.rs:183-192`), `uint_to_float` (`zsobol.rs:35-39`) and the PCG
hash of the aux seeds (`path_sampler.rs:135-141`).  Every value the render
kernels draw for a (pixel, sample) comes from these calls, so they are compared
bit for bit through `tpt_sampler_values_device` against the oracle (itself
pinned by the reference's sampler unit tests in test_oracle_sampler.py): the
camera sample, every vertex dimension of depths 0..16 (u_category .. u_rr),
the initial aux seed (dimension 0x80000000) and each vertex's aux seed, on
power-of-two and other spp, square and 1920x1080 images.
"""
import numpy as np
import pytest

import oracle as orc

pytestmark = pytest.mark.gpu

CASES = [  # width, height, spp
    (256, 256, 64),  # the plain-MIS Cornell configuration
    (1920, 1080, 256),  # the large-scene configuration
    (1920, 1080, 48),  # spp not a power of two (odd log2 after rounding up)
    (128, 128, 16),  # the differentiable-render configuration
    (640, 480, 3),
    (1024, 768, 1),
    (7, 5, 1000),
]


def queries(w, h, spp, n, seed):
    rng = np.random.default_rng(seed)
    q = np.empty((n, 4), np.uint32)
    q[:, 0] = rng.integers(0, w, n)
    q[:, 1] = rng.integers(0, h, n)
    q[:, 2] = rng.integers(0, spp, n)
    q[:, 3] = np.arange(n) % 17  # depths 0..16
    # the image corners and the last sample of the last pixel
    q[:4, 0] = [0, w - 1, 0, w - 1]
    q[:4, 1] = [0, 0, h - 1, h - 1]
    q[:4, 2] = [0, spp - 1, spp - 1, spp - 1]
    return q


@pytest.mark.parametrize("w,h,spp", CASES)
def test_sampler_values_bit_identical(ctx, w, h, spp):
    q = queries(w, h, spp, 1 << 16, seed=w * 31 + spp)
    dv, ds = ctx.sampler_values(w, h, spp, q)
    ov, os_ = orc.sampler_values(w, h, spp, q)
    bad = np.nonzero((dv.view(np.uint32) != ov.view(np.uint32)).any(1) | (ds != os_).any(1))[0]
    assert bad.size == 0, f"{bad.size} queries differ, first {q[bad[:3]].tolist()}"
    assert np.all((dv >= 0) & (dv < 1))


def test_every_sample_of_a_pixel_block(ctx):
    """All 64 samples of every pixel of a 16x16 block, every depth 0..16."""
    w = h = 256
    spp = 64
    px, py, s, d = np.meshgrid(np.arange(100, 116), np.arange(40, 56), np.arange(spp), np.arange(17), indexing="ij")
    q = np.stack([px.ravel(), py.ravel(), s.ravel(), d.ravel()], 1).astype(np.uint32)
    dv, ds = ctx.sampler_values(w, h, spp, q)
    ov, os_ = orc.sampler_values(w, h, spp, q)
    assert np.array_equal(dv.view(np.uint32), ov.view(np.uint32))
    assert np.array_equal(ds, os_)
