"""Pins the oracle's sampler against the reference's known-answer tests
(crates/renderer/src/sampler/pcg.rs:27-56, zsobol.rs:289-488)."""
import numpy as np

import oracle as orc

PRIMES = [2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53, 59, 61, 67, 71]
ONE_MINUS_EPS = np.frombuffer(np.uint32(0x3F7FFFFF).tobytes(), np.float32)[0]


def L():
    return orc.lib()


def test_pcg_state_and_output():
    lib = L()
    assert lib.orc_pcg_state_transition(0) != 0
    assert lib.orc_pcg_output(0) == 0
    for p in PRIMES:
        assert lib.orc_pcg_state_transition(p) != p
        assert lib.orc_pcg_output(p) != p
        assert lib.orc_pcg_state_transition(p) != lib.orc_pcg_output(p)
        # hash(init(seed)) == rng(init(seed)): init(seed) = state_transition(0) + seed
        st = (lib.orc_pcg_state_transition(0) + p) & 0xFFFFFFFF
        assert lib.orc_pcg_hash(st) == lib.orc_pcg_output(lib.orc_pcg_state_transition(st))


def test_uint_to_float_edges():
    f = L().orc_uint_to_float
    assert f(0) == 0.0
    assert 0.0 < f(1) < f(2)
    assert np.float32(f(0xFFFFFFFF)) == ONE_MINUS_EPS
    assert np.float32(f(0xFFFFFEFF)) < ONE_MINUS_EPS
    assert np.float32(f(0xFFFFFF00)) == ONE_MINUS_EPS
    assert f(0x7FFFFFFF) < 0.5
    assert f(0x80000000) == 0.5
    assert f(0x800000FF) == 0.5
    assert f(0x80000100) > 0.5


def test_morton():
    m = L().orc_encode_morton_2
    assert [m(0, 0), m(1, 0), m(0, 1), m(1, 1), m(2, 0), m(0, 2), m(3, 3), m(4, 0)] == [0, 1, 2, 3, 4, 8, 15, 16]


def test_zsobol_indices_unique_and_pixel_aligned():
    si = L().orc_zsobol_sample_index
    rx, ry = 16, 9
    for log_s in range(0, 11, 2):
        spp = 1 << log_s
        for dim in (0, 3, 6):
            seen = set()
            for y in range(ry):
                for x in range(rx):
                    base = None
                    for i in range(spp):
                        idx = si(spp, rx, ry, x, y, i, dim)
                        assert idx not in seen
                        seen.add(idx)
                        b = idx // spp
                        base = b if base is None else base
                        assert b == base


def test_laine_karras_low_bit_preserving():
    lk = L().orc_laine_karras
    for v in [0x55553333, 0xFF00F0F0, 0xFFFF00FF, 0xFFFFFFFF, 0]:
        for p in PRIMES:
            a, b = lk(v, p), lk(v ^ 0x10000, p)
            assert a & 0xFFFF == b & 0xFFFF
            assert a & ~0xFFFF & 0xFFFFFFFF != b & ~0xFFFF & 0xFFFFFFFF


def _rev(v):
    return int(f"{v:032b}"[::-1], 2)


def test_shuffle_is_permutation():
    rs = L().orc_reverse_and_shuffle
    for p in PRIMES:
        seen = set()
        for i in range(16):
            seen.add(_rev(rs(i, p)) & 15)
        assert seen == set(range(16))


def test_sobol_02_sequence_and_shirley_property():
    out = np.zeros(2, np.uint32)
    seed = L().orc_pcg_hash(0)
    samples = []
    for idx in range(256):
        L().orc_shuffled_scrambled_sobol(idx, seed, 2, out.ctypes.data)
        samples.append(out.copy())
    samples = np.asarray(samples, np.uint64)
    for i in range(9):
        xr, yr = 1 << i, 1 << (8 - i)
        xw, yw = 0xFFFFFFFF // xr, 0xFFFFFFFF // yr
        cells = set((samples[:, 0] // xw + (samples[:, 1] // yw) * xr).tolist())
        assert len(cells) == 256
    w = 0xFFFFFFFF // 8
    first64 = samples[:64]
    for i in range(8):
        ys = [int(s[1] // w) for s in first64 if int(s[0] // w) == i]
        assert sorted(ys) == list(range(8))


def test_vertex_randoms_in_unit_interval_and_deterministic():
    a, sa = orc.vertex_randoms(3, 5, 7, 64, 256, 256, 2)
    b, sb = orc.vertex_randoms(3, 5, 7, 64, 256, 256, 2)
    assert np.array_equal(a, b) and sa == sb
    assert np.all((a >= 0) & (a < 1))
    c, _ = orc.vertex_randoms(3, 5, 8, 64, 256, 256, 2)
    assert not np.array_equal(a, c)


def test_sampler_values_layout_matches_the_per_call_queries():
    """orc_sampler_values (the layout the device query is compared in) gives the
    same values as camera_sample / vertex_randoms, which the tests above pin to
    the reference's known answers."""
    rng = np.random.default_rng(5)
    for w, h, spp in ((256, 256, 64), (1920, 1080, 48), (5, 3, 1)):
        q = np.stack([rng.integers(0, w, 200), rng.integers(0, h, 200), rng.integers(0, spp, 200),
                      rng.integers(0, 17, 200)], 1).astype(np.uint32)
        vals, seeds = orc.sampler_values(w, h, spp, q)
        for i in range(0, 200, 7):
            px, py, s, d = (int(x) for x in q[i])
            cam, seed0 = orc.camera_sample(px, py, s, spp, w, h)
            vr, seed_v = orc.vertex_randoms(px, py, s, spp, w, h, d)
            assert np.array_equal(vals[i, :2], cam) and seeds[i, 0] == seed0
            # vertex_randoms: 11 values without u_extra2/3, then u_rr
            assert np.array_equal(vals[i, 2:13], vr[:11]) and vals[i, 15] == vr[11]
            assert seeds[i, 1] == seed_v
