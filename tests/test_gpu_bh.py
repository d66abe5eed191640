"""GPU: the Barnes-Hut path against the reference sample and the oracle.

Bars: FP64 form bit-exact (same operations in the same order as the sample);
FP32 form within 1e-5 relative of the FP64 form; accuracy against direct sum
below the reference's own gate (force and potential error < 1e-2,
test.sh:180-228)."""
import pathlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BH_GOLDEN = sorted((pathlib.Path(__file__).parent / "golden").glob("bh_*.npz"))


@pytest.mark.parametrize("path", BH_GOLDEN, ids=[p.stem for p in BH_GOLDEN])
def test_bh_fp64_bit_exact_against_reference(path, tb, ctx):
    g = np.load(path)
    r = ctx.bh_evaluate(g["x"], g["y"], g["z"], g["m"], ncrit=int(g["ncrit"]),
                        theta=float(g["theta"]), eps2=float(g["eps2"]), precision=tb.FP64)
    np.testing.assert_array_equal(r, g["bh"])


@pytest.mark.parametrize("ncrit", [1, 8, 32])
def test_bh_fp64_matches_oracle(ncrit, tb, ctx, oracle_mod):
    x, y, z, m = tb.datasets.make("plummer", 20000, 81)
    r = ctx.bh_evaluate(x, y, z, m, ncrit=ncrit, theta=0.5, eps2=1e-6, precision=tb.FP64)
    ref, cnt = oracle_mod.barnes_hut(x, y, z, m, ncrit=ncrit, theta=0.5, eps2=1e-6)
    np.testing.assert_array_equal(r, ref)
    na, nd = ctx.bh_counts()
    assert (na, nd) == (int(cnt[0]), int(cnt[1]))


def _bh_direct(x, y, z, m, tg, eps2):
    out = np.zeros((len(tg), 4))
    for k, i in enumerate(tg):
        dx, dy, dz = x - x[i], y - y[i], z - z[i]
        r2 = dx * dx + dy * dy + dz * dz + eps2
        ir = 1.0 / np.sqrt(r2)
        ir3 = ir ** 3
        out[k] = [np.sum(dx * ir3 * m), np.sum(dy * ir3 * m), np.sum(dz * ir3 * m),
                  np.sum(ir * m)]
    return out


def test_bh_fp32_and_accuracy(tb, ctx):
    x, y, z, m = tb.datasets.make("plummer", 50000, 82)
    r64 = ctx.bh_evaluate(x, y, z, m, ncrit=32, theta=0.5, eps2=1e-6, precision=tb.FP64)
    r32 = ctx.bh_evaluate(x, y, z, m, ncrit=32, theta=0.5, eps2=1e-6, precision=tb.MIXED)
    num = np.linalg.norm(r32 - r64, axis=0)
    den = np.linalg.norm(r64, axis=0)
    assert np.all(num / den < 1e-5)
    tg = tb.datasets.sample_targets(len(x), 200, seed=3)
    d = _bh_direct(x, y, z, m, tg, 1e-6)
    ef = np.sqrt(np.sum((r64[tg, :3] - d[:, :3]) ** 2) / np.sum(d[:, :3] ** 2))
    ep = np.sqrt(np.sum((r64[tg, 3] - d[:, 3]) ** 2) / np.sum(d[:, 3] ** 2))
    assert ef < 1e-2 and ep < 1e-2
