"""Both evaluation forms against the reference's own FP64 output at the
benchmark's configurations.

Fixtures (tests/golden/, made by make_golden.py from the unmodified reference
built in oracle/_ref):
* ``refsample_*``: benchmark-sized body sets regenerated from their seeds (an
  input checksum guards the generator), with the reference's results on a
  seeded sample of bodies and its list counters:
  - the 100k uniform cube at P=10, theta=0.4, ncrit=64 (the reference's own
    CPU-runnable configuration);
  - 1M Plummer bodies at P=10, theta=0.4, ncrit=64;
  - 1M and 16M sphere-surface bodies (zero-mean charges) at P=15, theta=0.4,
    ncrit=128, and the 16M set at P=13 and P=12 with theta=0.35, ncrit=128 (the
    settings the learned chooser has picked for the 16M workload);
* the small full-output fixtures, for the mixed form.
Bars: FP64 form max relative difference <= 1e-11 of the reference's values;
mixed form rel-L2 <= 2e-6 (potential and acceleration) against them.
"""
import pathlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GDIR = pathlib.Path(__file__).parent / "golden"
SAMPLED = ["refsample_cube_n100000_p10", "refsample_plummer_n1000000_p10",
           "refsample_sphere_n1000000_p15", "refsample_sphere_n16000000_p15",
           "refsample_sphere_n16000000_p13", "refsample_sphere_n16000000_p12"]
SMALL = sorted(p for p in GDIR.glob("*.npz")
               if not p.stem.startswith(("bh_", "refsample_", "mutual_", "io_")))


def _rel_max(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def _rel_l2(a, b):
    ep = np.linalg.norm(a[:, 0] - b[:, 0]) / np.linalg.norm(b[:, 0])
    ea = np.linalg.norm(a[:, 1:] - b[:, 1:]) / np.linalg.norm(b[:, 1:])
    return float(ep), float(ea)


@pytest.mark.parametrize("name", SAMPLED)
def test_benchmark_configs_against_reference(name, tb, ctx):
    g = np.load(GDIR / f"{name}.npz")
    n, P, ncrit, theta = int(g["n"]), int(g["P"]), int(g["ncrit"]), float(g["theta"])
    x, y, z, q = tb.datasets.make(str(g["dist"]), n, int(g["seed"]))
    w = np.arange(1, n + 1, dtype=np.float64) % 1009.0 + 1.0
    # a weighted sum: its last bits depend on the host's BLAS kernel
    np.testing.assert_allclose(np.array([np.dot(w, a) for a in (x, y, z, q)]), g["checksum"],
                               rtol=1e-12, atol=0)
    idx, ref = g["idx"], g["trg"]
    # the reference's list counters, on the lists as the reference visits them
    ctx.partition(x, y, z, q, ncrit=ncrit)
    assert ctx.tree_info()["n_cells"] == int(g["ncells"])
    ctx.set_reference_lists(True)
    try:
        li = ctx.build_lists(theta)
    finally:
        ctx.set_reference_lists(False)
    assert li["n_m2l"] == int(g["n_m2l"])
    assert li["n_p2p_interactions"] == int(g["n_p2p_interactions"])
    r64 = ctx.evaluate(x, y, z, q, P=P, ncrit=ncrit, theta=theta, precision=tb.FP64)
    assert _rel_max(r64[idx], ref) < 1e-11
    rmx = ctx.evaluate(x, y, z, q, P=P, ncrit=ncrit, theta=theta, precision=tb.MIXED)
    ep, ea = _rel_l2(rmx[idx], ref)
    assert ep < 2e-6 and ea < 2e-6, (ep, ea)


@pytest.mark.parametrize("path", SMALL, ids=[p.stem for p in SMALL])
def test_mixed_against_reference_goldens(path, tb, ctx):
    """The mixed form directly against the reference's full FP64 output."""
    g = np.load(path)
    r = ctx.evaluate(g["x"], g["y"], g["z"], g["q"], P=int(g["P"]), ncrit=int(g["ncrit"]),
                     theta=float(g["theta"]), precision=tb.MIXED)
    ok = ~np.isnan(g["trg"]).any(axis=1)
    if ok.sum() < 2:
        pytest.skip("fewer than two bodies with a finite reference value")
    ep, ea = _rel_l2(r[ok], g["trg"][ok])
    assert ep < 2e-6 and ea < 2e-6, (ep, ea)
