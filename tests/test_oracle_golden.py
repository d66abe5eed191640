"""Pins the oracle (fmm_oracle.c) to golden vectors made by the reference.

The fixtures in tests/golden/ were produced by running the unmodified
reference example (tests/golden/make_golden.py).  The oracle must reproduce
them bit for bit: keys, cell ranges, leaf flags, centres, widths, the M2L and
P2P counts, the per-body results and (small cases) M and L.
"""
import pathlib

import numpy as np
import pytest

GOLDEN = sorted(p for p in (pathlib.Path(__file__).parent / "golden").glob("*.npz")
                if not p.stem.startswith(("bh_", "refsample_", "io_")))
BH_GOLDEN = sorted((pathlib.Path(__file__).parent / "golden").glob("bh_*.npz"))


@pytest.mark.parametrize("path", BH_GOLDEN, ids=[p.stem for p in BH_GOLDEN])
def test_bh_oracle_matches_reference(path, oracle_mod):
    """The Barnes-Hut restatement reproduces the reference sample bit for bit."""
    g = np.load(path)
    res, _ = oracle_mod.barnes_hut(g["x"], g["y"], g["z"], g["m"], ncrit=int(g["ncrit"]),
                                   theta=float(g["theta"]), eps2=float(g["eps2"]))
    np.testing.assert_array_equal(res, g["bh"])


@pytest.mark.parametrize("path", GOLDEN, ids=[p.stem for p in GOLDEN])
def test_oracle_matches_reference(path, oracle_mod):
    g = np.load(path)
    mutual = int(g["mutual"]) if "mutual" in g else 0
    o = oracle_mod.Oracle(g["x"], g["y"], g["z"], g["q"], P=int(g["P"]), ncrit=int(g["ncrit"]),
                          theta=float(g["theta"]), mutual=mutual)
    c = o.cells()
    order = np.argsort(c["key"], kind="stable")
    assert np.array_equal(c["key"][order], g["cell_key"])
    assert np.array_equal(c["leaf"][order], g["cell_leaf"])
    assert np.array_equal(c["nb"][order], g["cell_nb"])
    leaf = g["cell_leaf"] == 1
    assert np.array_equal(c["bid"][order][leaf], g["cell_bid"][leaf])
    assert np.array_equal(c["center"][order], g["cell_center"])
    assert np.array_equal(c["width"][order], g["cell_width"])
    assert len(o.m2l_list()[0]) == int(g["n_m2l"])
    assert o.p2p_interactions() == int(g["n_p2p_interactions"])
    orig, _, _ = o.bodies()
    assert np.array_equal(orig, g["order"])
    np.testing.assert_array_equal(o.result(), g["trg"])
    if "M" in g:
        M, L = o.expansions()
        np.testing.assert_array_equal(M[order], g["M"])
        np.testing.assert_array_equal(L[order], g["L"])


def test_oracle_accuracy_vs_direct(oracle_mod):
    """The restated FMM is as accurate as the reference says it should be
    (rel-L2 < 5e-3 is the reference's own gate, test.sh:234,271-288)."""
    g = np.load(GOLDEN[0])
    x, y, z, q = g["x"], g["y"], g["z"], g["q"]
    o = oracle_mod.Oracle(x, y, z, q, P=10, ncrit=32, theta=0.4)
    tg = np.arange(0, len(x), 7)
    d = oracle_mod.direct(x, y, z, q, tg)
    ep, ea = oracle_mod.rel_l2(o.result()[tg], d)
    assert ep < 1e-4 and ea < 1e-3


SAMPLED = sorted((pathlib.Path(__file__).parent / "golden").glob("refsample_*.npz"))


@pytest.mark.parametrize("path", SAMPLED, ids=[p.stem for p in SAMPLED])
def test_sampled_fixture_inputs_regenerate(path, tb):
    """The benchmark-sized fixtures keep only a sample of the reference's
    results; their inputs are regenerated from the seed, and the generator
    must still produce the bodies the reference ran on."""
    g = np.load(path)
    n = int(g["n"])
    x, y, z, q = tb.datasets.make(str(g["dist"]), n, int(g["seed"]))
    w = np.arange(1, n + 1, dtype=np.float64) % 1009.0 + 1.0
    # a weighted sum: its last bits depend on the host's BLAS kernel
    np.testing.assert_allclose(np.array([np.dot(w, a) for a in (x, y, z, q)]), g["checksum"],
                               rtol=1e-12, atol=0)
    np.testing.assert_array_equal(g["idx"], tb.datasets.sample_targets(n, len(g["idx"]), 1234))


def test_oracle_matches_reference_at_100k(tb, oracle_mod):
    """The restatement against the reference at the 100k-body cube (P=10,
    theta=0.4, ncrit=64): bit for bit on the sampled bodies, same counters."""
    g = np.load(pathlib.Path(__file__).parent / "golden" / "refsample_cube_n100000_p10.npz")
    x, y, z, q = tb.datasets.make(str(g["dist"]), int(g["n"]), int(g["seed"]))
    o = oracle_mod.Oracle(x, y, z, q, P=int(g["P"]), ncrit=int(g["ncrit"]),
                          theta=float(g["theta"]))
    assert len(o.m2l_list()[0]) == int(g["n_m2l"])
    assert o.p2p_interactions() == int(g["n_p2p_interactions"])
    np.testing.assert_array_equal(o.result()[g["idx"]], g["trg"])
