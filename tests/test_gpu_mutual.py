"""Mutual interaction (the reference example's -m 1) on the GPU.

The reference's mutual traversal visits every unordered cell pair once and
applies M2L and P2P both ways (ex/tapas_exafmm.cxx:209-286 with mutual,
LaplaceSphericalCPU_tapas.h:208-273, LaplaceP2PCPU_tapas.h:48-74).  Its
lists therefore differ from the mutual = 0 lists, and so do its results, at
the truncation-error level.  Bars:
* the directed lists equal the oracle's mutual pairs taken both ways (sets);
* FP64 results within 1e-11 (max relative) of the oracle's mutual restatement,
  which is itself pinned bit for bit to the reference's -m 1 output
  (tests/golden/mutual_*.npz);
* the mixed form within 2e-6 (rel-L2) of the FP64 mutual form.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FP64_RTOL = 1e-11


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _directed(keys, t, s):
    """Set of directed (target key, source key) pairs of unordered pairs."""
    out = set(zip(keys[t].tolist(), keys[s].tolist()))
    out |= set(zip(keys[s].tolist(), keys[t].tolist()))
    return out


CASES = [
    ("plummer", 20000, 3, 8, 32, 0.4),        # root of > 1000 bodies: split-order path
    ("uniform_cube", 12000, 5, 10, 64, 0.5),
    ("two_gaussians", 8000, 6, 6, 16, 0.35),
    ("uniform_cube", 600, 7, 4, 1, 0.6),      # ncrit = 1
]


@pytest.mark.parametrize("case", CASES, ids=[f"{c[0]}-n{c[1]}-ncrit{c[4]}" for c in CASES])
def test_mutual_lists_and_results(case, tb, ctx, oracle_mod):
    dist, n, seed, P, ncrit, theta = case
    x, y, z, q = tb.datasets.make(dist, n, seed)
    o = oracle_mod.Oracle(x, y, z, q, P=P, ncrit=ncrit, theta=theta, mutual=1)
    ctx.partition(x, y, z, q, ncrit=ncrit)
    ctx.upward(P, tb.FP64)
    ctx.set_reference_lists(True)
    try:
        ctx.build_lists(theta, mutual=1)
        (gmt, gms), (gpt, gps) = ctx.lists()
    finally:
        ctx.set_reference_lists(False)
    gkeys, okeys = ctx.cells()["key"], o.cells()["key"]
    omt, oms = o.m2l_list()
    opt, ops = o.p2p_list()
    assert len(gmt) == 2 * len(omt)
    assert set(zip(gkeys[gmt].tolist(), gkeys[gms].tolist())) == _directed(okeys, omt, oms)
    assert set(zip(gkeys[gpt].tolist(), gkeys[gps].tolist())) == _directed(okeys, opt, ops)
    for t, s in ((gmt, gms), (gpt, gps)):
        assert np.all(np.diff(t.astype(np.int64) * (1 << 32) + s) > 0)
    # results, default (pruned) lists
    ctx.traverse(theta, 1, tb.FP64)
    ctx.downward(tb.FP64)
    r = ctx.results(tb.ORDER_ORIGINAL)
    assert _rel(r, o.result()) < FP64_RTOL


def test_mutual_mixed_close_to_fp64_mutual(tb, ctx, oracle_mod):
    x, y, z, q = tb.datasets.make("sphere_surface", 60000, 9)
    res = {}
    for prec in (tb.FP64, tb.MIXED):
        ctx.partition(x, y, z, q, ncrit=64)
        ctx.upward(12, prec)
        ctx.traverse(0.4, 1, prec)
        ctx.downward(prec)
        res[prec] = ctx.results(tb.ORDER_ORIGINAL)
    ep, ea = oracle_mod.rel_l2(res[tb.MIXED], res[tb.FP64])
    assert ep < 2e-6 and ea < 2e-6
    # the same accuracy class as mutual = 0 against the direct sum
    tg = tb.datasets.sample_targets(len(x), 400, seed=3)
    d = ctx.direct(tg)
    r0 = ctx.evaluate(x, y, z, q, P=12, ncrit=64, theta=0.4, precision=tb.FP64)
    e0 = oracle_mod.rel_l2(r0[tg], d)
    e1 = oracle_mod.rel_l2(res[tb.FP64][tg], d)
    assert e1[0] < 3 * e0[0] + 1e-9 and e1[1] < 3 * e0[1] + 1e-9


def test_mutual_fp64_deterministic(tb, ctx):
    x, y, z, q = tb.datasets.make("plummer", 30000, 13)
    out = []
    for _ in range(2):
        ctx.partition(x, y, z, q, ncrit=32)
        ctx.upward(8, tb.FP64)
        ctx.traverse(0.4, 1, tb.FP64)
        ctx.downward(tb.FP64)
        out.append(ctx.results(tb.ORDER_ORIGINAL))
    assert np.array_equal(out[0], out[1])
