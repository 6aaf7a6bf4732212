"""Checks of the oracle's BDPT restatement (integrator/bdpt.rs) that need no GPU.

The reference's own BDPT tests exercise point, spot, directional and
environment lights and mirrors, none of which are in scope.  What pins the
area-light path instead: at max_depth 1 BDPT estimates exactly what MIS does
(visible emission plus one-bounce direct light: the single connection strategy
has weight 1), so the two means agree within their statistical error; at
max_depth 0 BDPT traces nothing.
"""
import numpy as np

import oracle as orc
import tpt
import tpt_scenes


def _scene(kind, seed=1):
    sc = tpt_scenes.cornell_box(seed, kind)
    return sc, orc.RenderScene(sc, tpt.build_light_tree(sc))


def test_depth_one_bdpt_estimates_the_same_as_mis():
    for kind in (tpt_scenes.LAMBERT, tpt_scenes.OPENPBR):
        sc, ref = _scene(kind)
        w = h = 32
        spp = 64
        n = w * h * spp
        m = ref.samples(sc["camera"], w, h, spp, 1, 0, n, integrator=0).astype(np.float64)
        b = ref.samples(sc["camera"], w, h, spp, 1, 0, n, integrator=1).astype(np.float64)
        mm, mb = m.mean(0), b.mean(0)
        se = np.sqrt(m.var(0) / n + b.var(0) / n)
        assert np.all(np.abs(mm - mb) <= 5 * se + 1e-7), (kind, mm, mb, se)
        assert mb.min() > 0


def test_depth_zero_bdpt_is_black():
    sc, ref = _scene(tpt_scenes.LAMBERT)
    img = ref.render(sc["camera"], 16, 16, 2, 0, integrator=1)
    assert np.count_nonzero(img) == 0


def test_bdpt_is_finite_and_deterministic():
    sc, ref = _scene(tpt_scenes.OPENPBR, seed=3)
    a = ref.render(sc["camera"], 16, 16, 4, 8, integrator=1)
    b = ref.render(sc["camera"], 16, 16, 4, 8, integrator=1, nthreads=1)
    assert np.all(np.isfinite(a)) and a.mean() > 0
    assert np.array_equal(a, b)
