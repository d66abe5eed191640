"""Morton-key known-answer tests of the oracle.

Restates the reference's key tests, cpp/tests/test_morton_key.cpp:24-362
(Dim = 3, uint64 keys; the two Dim = 2 tests there, LETRequirement and
CalcRegion, are restated for the 3-D key the FMM path uses).
"""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def L(oracle_mod):
    return oracle_mod.lib()


def gen_key(L, path):
    k = 0
    for i in path:
        k = L.oracle_key_child(k, i)
    return k


def next_key(L, k, n=1):
    return L.oracle_key_next(k, n)


def children(L, k):
    return [L.oracle_key_child(k, i) for i in range(8)]


def test_parent(L):  # test_morton_key.cpp:24-32
    assert L.oracle_key_parent(gen_key(L, [0, 1, 2])) == gen_key(L, [0, 1])


def test_next(L):  # :34-46
    assert next_key(L, gen_key(L, [0, 1, 1])) == gen_key(L, [0, 1, 2])
    assert next_key(L, gen_key(L, [0, 1, 7])) == gen_key(L, [0, 2, 0])


def test_is_descendant(L):  # :48-69
    a, a2 = gen_key(L, [0, 1]), gen_key(L, [0, 2])
    d, d2 = gen_key(L, [0, 1, 3]), gen_key(L, [0, 1, 2, 3, 4, 5])
    assert L.oracle_key_is_descendant(a, d) and L.oracle_key_is_descendant(a, d2)
    assert not L.oracle_key_is_descendant(d, a) and not L.oracle_key_is_descendant(d2, a)
    assert not L.oracle_key_is_descendant(a2, d) and not L.oracle_key_is_descendant(a2, d2)


def test_owner_lookup(L):  # :71-98, restated for 3-D keys
    procs = [gen_key(L, [0, 0]), gen_key(L, [0, 7]), gen_key(L, [7, 0])]
    rm = [p >> 5 for p in procs]
    assert np.searchsorted(rm, gen_key(L, [5, 7]) >> 5, side="right") - 1 == 1
    assert np.searchsorted(rm, gen_key(L, [7, 0]) >> 5, side="right") - 1 == 2


def test_overlapped(L):  # :100-175
    R = 0
    Rn = next_key(L, R)
    ch = children(L, R)
    for c in ch:
        assert L.oracle_key_overlapped(R, Rn, c, next_key(L, c))
        assert L.oracle_key_overlapped(c, next_key(L, c), R, Rn)
    for i in range(8):
        for j in range(i + 1, 8):
            x1, y1 = ch[i], ch[j]
            assert not L.oracle_key_overlapped(x1, next_key(L, x1), y1, next_key(L, y1))
            assert not L.oracle_key_overlapped(y1, next_key(L, y1), x1, next_key(L, x1))
    assert L.oracle_key_overlapped(R, Rn, R, Rn)
    for c in ch:
        assert L.oracle_key_overlapped(c, next_key(L, c), c, next_key(L, c))
    for i in range(8):
        for j in range(8):
            if i == j:
                continue
            for nep in children(L, ch[j]):
                assert not L.oracle_key_overlapped(ch[i], next_key(L, ch[i]), nep,
                                                   next_key(L, nep))
                assert not L.oracle_key_overlapped(nep, next_key(L, nep), ch[i],
                                                   next_key(L, ch[i]))
    rng = np.random.default_rng(0)
    anc = dec = ch[0]
    for _ in range(10):
        dec = children(L, dec)[int(rng.integers(8))]
        assert L.oracle_key_overlapped(anc, next_key(L, anc), dec, next_key(L, dec))
    first = (0 << 5) | 10
    last = 0
    for _ in range(10):
        last = children(L, last)[7]
    last = next_key(L, last)
    for c in ch:
        assert L.oracle_key_overlapped(first, last, c, next_key(L, c))
        assert L.oracle_key_overlapped(c, next_key(L, c), first, last)


def test_includes(L):  # :177-216
    R = 0
    S = next_key(L, R)
    ch = children(L, R)
    for c in ch:
        assert L.oracle_key_includes_range(R, S, c)
    for i in range(8):
        for j in range(i + 1, 8):
            assert not L.oracle_key_includes_range(ch[i], ch[j], R)
    c0, c1, c2 = ch[0], ch[1], ch[2]
    assert L.oracle_key_includes_range(c0, c2, c1)
    for k0 in children(L, c0):
        for k2 in children(L, c2):
            assert L.oracle_key_includes_range(k0, k2, c1)
            for k1 in children(L, c1):
                assert L.oracle_key_includes_range(k0, k2, k1)


def test_dir_on_depth(L):  # :219-261
    k = gen_key(L, [0, 0, 0])
    for dim in range(3):
        for dep in (1, 2, 3):
            assert L.oracle_key_dir_on_depth(k, dim, dep) == 0
    k = gen_key(L, [7, 3, 2])
    assert [L.oracle_key_dir_on_depth(k, 0, d) for d in (1, 2, 3)] == [1, 1, 0]
    assert [L.oracle_key_dir_on_depth(k, 1, d) for d in (1, 2, 3)] == [1, 1, 1]
    assert [L.oracle_key_dir_on_depth(k, 2, d) for d in (1, 2, 3)] == [1, 0, 0]


def test_calc_region(L, oracle_mod):  # :277-340, restated in 3-D
    import ctypes
    rmin = np.array([-1.0, -1.0, -1.0])
    rmax = np.array([1.0, 1.0, 1.0])

    def region(path):
        k = gen_key(L, path)
        mn = np.zeros(3)
        mx = np.zeros(3)
        L.oracle_key_region(k, *[a.ctypes.data_as(ctypes.c_void_p) for a in (rmin, rmax, mn, mx)])
        return mn, mx

    mn, mx = region([])
    assert np.allclose(mn, -1) and np.allclose(mx, 1)
    mn, mx = region([7])
    assert np.allclose(mn, 0) and np.allclose(mx, 1)
    mn, mx = region([0])
    assert np.allclose(mn, -1) and np.allclose(mx, 0)
    mn, mx = region([7, 7])
    assert np.allclose(mn, 0.5) and np.allclose(mx, 1)
    mn, mx = region([0, 2])  # x low, y high within the (-1,0) octant
    assert np.allclose(mn, [-1, -0.5, -1]) and np.allclose(mx, [-0.5, 0, -0.5])


def test_msbits(L):  # :343-362
    ch = children(L, 0)
    for i in range(8):
        assert L.oracle_key_msbits(ch[i], 3) == i
    for i in range(8):
        g = children(L, ch[i])
        for j in range(8):
            assert L.oracle_key_msbits(g[j], 6) == i * 8 + j


def test_finest_key_interleave(L):
    # CalcFinestKey (sfc_morton.h:387-402): per level z, y, x bits, depth 19.
    k = L.oracle_key_finest(1 << 18, 0, 0)  # top-level x bit -> bit 54 of the key body
    assert k == ((1 << 54) << 5) | 19
    k = L.oracle_key_finest(0, 0, 1 << 18)  # top-level z bit -> bit 56
    assert k == ((1 << 56) << 5) | 19
    k = L.oracle_key_finest(1, 1, 1)
    assert k == (7 << 5) | 19
