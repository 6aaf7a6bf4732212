"""CPU checks of the C ABI boundary and the host-side scene preparation.

* libtpt_cuda.so loads and exports every function include/tpt.h declares;
* the library's own host QBVH builder produces exactly the oracle's tree
  (node bytes and primitive order) — the oracle restates qbvh.rs:144-516;
* error behaviour without a device (no CPU fallback).
"""
import os
import re

import numpy as np
import pytest

import oracle as orc
import tpt
import tpt_scenes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    text = open(os.path.join(ROOT, "include", "tpt.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(tpt_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = tpt.lib()
    names = header_functions()
    assert len(names) >= 10
    for n in names:
        assert hasattr(lib, n), f"{n} declared in include/tpt.h but not exported"
    assert set(names) <= set(tpt.EXPORTED_SYMBOLS) | set(names)


def test_version_string():
    assert b"sm_100a" in tpt.lib().tpt_version()


def _same_tree(a, b):
    na, pa = a
    nb, pb = b
    assert len(na) == len(nb)
    assert np.array_equal(pa, pb)
    assert na.tobytes() == nb.tobytes()


@pytest.mark.parametrize("case", ["grid", "coincident", "random", "skewed", "few"])
def test_host_builder_matches_oracle_builder(case):
    rng = np.random.default_rng(7)
    if case == "grid":
        mins = np.array([[(i * 73) % 211, (i * 37) % 191, (i * 53) % 173] for i in range(20000)], np.float32)
        b = np.concatenate([mins, mins + 0.5], 1)
    elif case == "coincident":
        b = np.tile(np.array([[0, 0, 0, 1, 1, 1]], np.float32), (300, 1))
    elif case == "random":
        lo = rng.uniform(-50, 50, (50000, 3)).astype(np.float32)
        b = np.concatenate([lo, lo + rng.uniform(0, 2, (50000, 3)).astype(np.float32)], 1)
    elif case == "skewed":
        i = np.arange(5000, dtype=np.float32)
        t = i / 5000
        lo = np.stack([t * t * 100, np.sin(i) * 0.5, np.cos(i) * 0.5], 1).astype(np.float32)
        b = np.concatenate([lo, lo + 0.2], 1)
    else:
        b = np.array([[0, 0, 0, 1, 1, 1], [2, 2, 2, 3, 3, 3], [1, 0, 0, 2, 1, 1]], np.float32)
    mine = tpt.build_qbvh(b, threads=4)
    ref = orc.BoxQbvh(b).arrays()
    _same_tree(mine, ref)


def test_host_builder_matches_oracle_on_sphere_mesh():
    m = tpt_scenes.sphere_soup(seed=5, n_spheres=256)
    pos = m["positions"]
    tri = pos[m["indices"].reshape(-1, 3)]
    b = np.concatenate([tri.min(1), tri.max(1)], 1)
    _same_tree(tpt.build_qbvh(b), orc.BoxQbvh(b).arrays())


def test_builder_rejects_empty_input():
    with pytest.raises(tpt.TptError) as e:
        tpt.build_qbvh(np.zeros((0, 6), np.float32))
    assert e.value.status == 1


def test_context_without_device_fails_loudly():
    import torch

    if torch.cuda.is_available():
        pytest.skip("device present")
    with pytest.raises(tpt.TptError) as e:
        tpt.Context(0)
    assert e.value.status == 3  # TPT_ERR_CUDA: no CPU fallback
