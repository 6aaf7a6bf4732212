"""Pins the oracle's geometry against the reference's own known-answer tests.

Each test restates one `#[test]` of the reference crate (file:line given) and
runs it against the oracle's C++ restatement.
"""
import math

import numpy as np
import pytest

import oracle as orc

INF = float("inf")
UNIT = ((0.0, 0.0, 0.0), (1.0, 0.0, 0.0), (0.0, 1.0, 0.0))


# ---- math/ray.rs:229-321 ----------------------------------------------------
def test_intersect_triangle_returns_hit():
    t, b = orc.intersect_triangle((0.25, 0.25, 1.0), (0, 0, -1), INF, *UNIT)
    assert abs(t - 1.0) < 1e-6
    assert np.allclose(b, [0.5, 0.25, 0.25], atol=1e-6)


def test_intersect_triangle_outside_and_parallel_and_degenerate():
    assert orc.intersect_triangle((1.25, 1.25, 1.0), (0, 0, -1), INF, *UNIT) is None
    assert orc.intersect_triangle((0.25, 0.25, 1.0), (1, 0, 0), INF, *UNIT) is None
    assert orc.intersect_triangle((0.25, 0.0, 1.0), (0, 0, -1), INF, (0, 0, 0), (1, 0, 0), (2, 0, 0)) is None


def test_intersect_triangle_edge_vertex_tmax_origin_backface():
    _, b = orc.intersect_triangle((0.5, 0.0, 1.0), (0, 0, -1), INF, *UNIT)
    assert np.allclose(b, [0.5, 0.5, 0.0], atol=1e-6)
    _, b = orc.intersect_triangle((0.0, 0.0, 1.0), (0, 0, -1), INF, *UNIT)
    assert np.allclose(b, [1.0, 0.0, 0.0], atol=1e-6)
    assert orc.intersect_triangle((0.25, 0.25, 2.0), (0, 0, -1), 1.5, *UNIT) is None
    assert orc.intersect_triangle((0.25, 0.25, 2.0), (0, 0, -1), 2.5, *UNIT) is not None
    assert orc.intersect_triangle((0.25, 0.25, 0.0), (0, 0, -1), INF, *UNIT) is None
    t, _ = orc.intersect_triangle((0.25, 0.25, -1.0), (0, 0, 1), INF, *UNIT)
    assert abs(t - 1.0) < 1e-6


def test_intersect_triangle_against_fp64_on_random_rays():
    """t within 1e-5 relative of a float64 Moller-Trumbore solve on clear, non-grazing hits."""
    rng = np.random.default_rng(0)
    checked = 0
    for _ in range(2000):
        v = rng.uniform(-1, 1, (3, 3)).astype(np.float32)
        o = rng.uniform(-3, 3, 3).astype(np.float32)
        target = (v[0] * 0.3 + v[1] * 0.3 + v[2] * 0.4).astype(np.float64)
        d = (target - o.astype(np.float64))
        d /= np.linalg.norm(d)
        d = d.astype(np.float32)
        h = orc.intersect_triangle(tuple(o), tuple(d), INF, *map(tuple, v))
        e1 = v[1].astype(np.float64) - v[0]
        e2 = v[2].astype(np.float64) - v[0]
        pv = np.cross(d.astype(np.float64), e2)
        det = e1 @ pv
        nrm = np.cross(e1, e2)
        if abs(d.astype(np.float64) @ nrm) < 0.2 * np.linalg.norm(nrm):
            continue  # grazing incidence: f32 shear error grows as 1/cos
        tv = o.astype(np.float64) - v[0]
        u = (tv @ pv) / det
        qv = np.cross(tv, e1)
        w = (d.astype(np.float64) @ qv) / det
        t64 = (e2 @ qv) / det
        if u < 1e-3 or w < 1e-3 or u + w > 1 - 1e-3 or t64 < 1e-3:
            continue
        assert h is not None
        assert abs(h[0] - t64) <= 1e-5 * abs(t64)
        checked += 1
    assert checked > 500


# ---- qbvh.rs:686-1183 --------------------------------------------------------
def _boxes(mins, size):
    mins = np.asarray(mins, np.float32)
    return np.concatenate([mins, mins + np.float32(size)], 1)


def verify_invariants(nodes, prims, bounds):
    n = len(bounds)
    assert sorted(prims.tolist()) == list(range(n))
    if len(nodes) == 0:
        return

    def subtree(word, acc):
        if word & 0x80000000:
            cnt = (word >> 24) & 0x7F
            off = word & 0xFFFFFF
            for k in range(off, off + cnt):
                b = bounds[prims[k]]
                acc[0] = np.minimum(acc[0], b[:3])
                acc[1] = np.maximum(acc[1], b[3:])
        else:
            for s in range(4):
                if nodes[word]["valid_mask"] >> s & 1:
                    subtree(int(nodes[word]["children"][s]), acc)

    total = 0
    for node in nodes:
        for s in range(4):
            if not (node["valid_mask"] >> s & 1):
                continue
            w = int(node["children"][s])
            acc = [np.full(3, np.inf, np.float32), np.full(3, -np.inf, np.float32)]
            subtree(w, acc)
            lo = node["b"][0:3, s]
            hi = node["b"][3:6, s]
            assert np.all(lo <= acc[0] + 1e-4) and np.all(hi + 1e-4 >= acc[1])
            if w & 0x80000000:
                cnt = (w >> 24) & 0x7F
                assert 1 <= cnt <= 16
                total += cnt
    assert total == n


def slab_scalar(b, o, d):
    with np.errstate(divide="ignore", invalid="ignore"):
        inv = np.where(d == 0, np.inf, 1.0 / np.where(d == 0, 1, d)).astype(np.float32)
        t1 = (b[:3] - o) * inv
        t2 = (b[3:] - o) * inv
    tmin = np.fmax(np.fmax(np.fmax(np.fmin(t1, t2)[0], np.fmin(t1, t2)[1]), np.fmin(t1, t2)[2]), 0)
    tmax = np.fmin(np.fmin(np.fmax(t1, t2)[0], np.fmax(t1, t2)[1]), np.fmax(t1, t2)[2])
    return tmin if tmin <= tmax else None


def brute_closest(bounds, o, d):
    best = None
    for i, b in enumerate(bounds):
        t = slab_scalar(b, np.asarray(o, np.float32), np.asarray(d, np.float32))
        if t is not None and (best is None or t < best[1]):
            best = (i, t)
    return best


def test_empty_and_single_and_root_leaf():
    q = orc.BoxQbvh(_boxes([[0, 0, 0]], 1.0))
    nodes, prims = q.arrays()
    assert len(nodes) == 0 and prims.tolist() == [0]
    for n in range(1, 5):
        b = _boxes([[i, i, i] for i in range(n)], 0.5)
        q = orc.BoxQbvh(b)
        nodes, _ = q.arrays()
        assert len(nodes) == 0
        bf = brute_closest(b, (0.25, 0.25, -10), (0, 0, 1))
        qb = q.closest_box((0.25, 0.25, -10), (0, 0, 1))
        assert (bf and bf[0]) == (qb and qb[0])


@pytest.mark.parametrize(
    "bounds",
    [
        _boxes([[i % 4, (i // 4) % 4, i // 16] for i in range(32)], 0.5),
        _boxes([[0, 0, 0]] * 20, 1.0),
        _boxes([[0, 0, 0]] * 120, 1.0),
        _boxes([[(i * 73) % 211, (i * 37) % 191, (i * 53) % 173] for i in range(8192 * 2 + 17)], 0.5),
    ],
    ids=["clusters", "coincident", "many_coincident", "parallel_threshold"],
)
def test_build_invariants(bounds):
    q = orc.BoxQbvh(bounds)
    verify_invariants(*q.arrays(), bounds)


def test_traverse_matches_brute_force_on_grid():
    bounds = _boxes([[(i * 19) % 41, (i * 11) % 37, (i * 7) % 31] for i in range(200)], 0.4)
    q = orc.BoxQbvh(bounds)
    c = 0.5 * (bounds[:, :3].min(0) + bounds[:, 3:].max(0))
    dirs = [(0, 0, -1), (0, 0, 1), (-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0)]
    dirs += [tuple(np.asarray(v) / np.linalg.norm(v)) for v in [(1, 1, 1), (-1, 0.5, 0.3), (0.2, -0.7, 0.6)]]
    hits = 0
    for d in dirs:
        d = np.asarray(d, np.float32)
        for i in range(50):
            jit = np.array([((i * 13) % 47) * 0.5 - 12, ((i * 17) % 43) * 0.5 - 11, ((i * 7) % 41) * 0.5 - 10],
                           np.float32)
            o = (c + jit - d * 80).astype(np.float32)
            bf = brute_closest(bounds, o, d)
            qb = q.closest_box(o, d)
            assert (bf is None) == (qb is None)
            if bf:
                assert abs(bf[1] - qb[1]) <= 1e-3 * max(abs(bf[1]), 1)
                hits += 1
    assert hits > 0


def test_traverse_axis_aligned_and_inside():
    bounds = _boxes([[i % 8, (i // 8) % 4, 0] for i in range(32)], 0.5)
    q = orc.BoxQbvh(bounds)
    for o, d in [((-10, .25, .25), (1, 0, 0)), ((10, .25, .25), (-1, 0, 0)), ((.25, -10, .25), (0, 1, 0)),
                 ((.25, 10, .25), (0, -1, 0)), ((.25, .25, -10), (0, 0, 1)), ((.25, .25, 10), (0, 0, -1))]:
        bf = brute_closest(bounds, o, d)
        qb = q.closest_box(o, d)
        assert (bf and bf[0]) == (qb and qb[0])
    b = np.array([[0, 0, 0, 2, 2, 2], [5, 5, 5, 6, 6, 6], [-3, -3, -3, -2, -2, -2], [10, 10, 10, 11, 11, 11],
                  [20, 20, 20, 21, 21, 21]], np.float32)
    qb = orc.BoxQbvh(b).closest_box((1, 1, 1), (1, 0, 0))
    assert qb[0] == 0 and abs(qb[1]) < 1e-5


def test_skewed_distribution():
    n = 500
    i = np.arange(n, dtype=np.float32)
    t = i / n
    mins = np.stack([t * t * 100, np.sin(i) * 0.5, np.cos(i * np.float32(0.137)) * 0.5], 1).astype(np.float32)
    bounds = _boxes(mins, 0.2)
    q = orc.BoxQbvh(bounds)
    verify_invariants(*q.arrays(), bounds)
    hits = 0
    for d in [(1, 0, 0), (-1, 0, 0), (1, 0.2, 0), (-1, -0.1, 0.05)]:
        d = np.asarray(d, np.float32) / np.float32(np.linalg.norm(d))
        for k in range(30):
            o = np.array([-50 + k * 0.3, np.sin(k) * 0.4, 0], np.float32)
            bf = brute_closest(bounds, o, d)
            qb = q.closest_box(o, d)
            assert (bf and bf[0]) == (qb and qb[0])
            hits += bf is not None
    assert hits > 0


# ---- scene/camera.rs:104-160 ------------------------------------------------
def test_camera_center_and_normalised_and_differentials():
    p = np.array([0, 0, 5, 0, 0, 0, 0, 1, 0, math.radians(60), 1], np.float32)
    r = orc.camera_ray(p, 3, 3, 1, 1, 0.5, 0.5, 1)
    assert np.allclose(r[0:3], [0, 0, 5], atol=1e-6)
    assert np.allclose(r[3:6], [0, 0, -1], atol=1e-6)
    p[9] = math.radians(45)
    r = orc.camera_ray(p, 512, 512, 0, 0, 0.5, 0.5, 1)
    assert abs(np.linalg.norm(r[3:6]) - 1) < 1e-6
    assert np.all(r[6:9] == r[0:3]) and np.all(r[9:12] == r[0:3])
    assert np.any(r[12:15] != r[3:6]) and np.any(r[15:18] != r[3:6])
    assert r[19] > 0


def test_oracle_traversal_matches_fp64_brute_force():
    """The oracle's QBVH traversal (qbvh.rs:611-675 + math/ray.rs:107-209 in f32)
    finds the nearest triangle of an FP64 brute force over every triangle, as
    the reference's traverse_closest_matches_brute_force_on_grid
    (qbvh.rs:902-969) checks: the same triangle, or a tie within 1e-6 t."""
    import tpt_scenes

    mesh = tpt_scenes.sphere_soup(seed=5, n_spheres=64, cube=8.0)
    rays = tpt_scenes.incoherent_rays(4096, seed=9, cube=8.0)
    g = orc.Geometry()
    g.add_mesh(mesh["positions"], mesh["indices"])
    g.add_instance(0, 0, np.eye(4, dtype=np.float32), np.eye(4, dtype=np.float32), np.eye(3, dtype=np.float32))
    g.build()
    ref = g.query(rays, 0)
    bp, bt, _ = orc.brute_force_f64(mesh["positions"], mesh["indices"], rays)
    assert (bp >= 0).sum() > 1000
    assert np.array_equal(ref["prim"] >= 0, bp >= 0)
    t64, _ = orc.triangle_f64(mesh["positions"], mesh["indices"], ref["prim"], rays)
    same = ref["prim"] == bp
    with np.errstate(invalid="ignore"):  # inf - inf on rays both miss (they are `same`)
        assert np.all(same | (np.abs(t64 - bt) <= 1e-6 * bt))
    hit = bp >= 0
    assert np.all(np.abs(ref["t"][hit] - bt[hit]) <= 1e-5 * bt[hit] + 2.0 ** -20 * 8.0)
