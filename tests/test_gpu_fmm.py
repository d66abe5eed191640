"""GPU parity tests: the CUDA library through its C ABI against the oracle.

Bars (stated per check):
* tree, keys, body order, M2L/P2P list sets: bit-exact;
* FP64 expansions and results: relative error <= 1e-11 (different summation
  order and libm vs CUDA math, both FP64);
* mixed form: rel-L2 vs the FP64 form <= 2e-6, and vs direct sum the same
  accuracy class as FP64.
"""
import pathlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = sorted(p for p in (pathlib.Path(__file__).parent / "golden").glob("*.npz")
                if not p.stem.startswith(("bh_", "refsample_", "io_")))
FP64_RTOL = 1e-11


def _cells_by_key(c, key_name="key"):
    order = np.argsort(c[key_name], kind="stable")
    return order


def _rel(a, b):
    scale = max(np.max(np.abs(b)), 1e-300)
    return float(np.max(np.abs(a - b)) / scale)


def _rel_rows(a, b):
    """max over rows of |a-b| / |b| (row norms), for per-body 4-vectors."""
    num = np.linalg.norm(a - b, axis=-1)
    den = np.maximum(np.linalg.norm(b, axis=-1), 1e-300)
    return float(np.max(num / den))


CASES = [
    ("uniform_cube", 20000, 1, 10, 64, 0.4),
    ("plummer", 30000, 2, 8, 32, 0.5),
    ("sphere_surface", 25000, 5, 6, 16, 0.35),
    ("two_gaussians", 15000, 4, 12, 128, 0.3),
    ("uniform_cube", 3000, 7, 4, 1, 0.6),
]
IDS = [f"{c[0]}-n{c[1]}-p{c[3]}-ncrit{c[4]}" for c in CASES]


@pytest.fixture(scope="module", params=CASES, ids=IDS)
def run(request, tb, oracle_mod, ctx):
    dist, n, seed, P, ncrit, theta = request.param
    x, y, z, q = tb.datasets.make(dist, n, seed)
    o = oracle_mod.Oracle(x, y, z, q, P=P, ncrit=ncrit, theta=theta)
    ctx.partition(x, y, z, q, ncrit=ncrit)
    ctx.upward(P, tb.FP64)
    # lists exactly as the reference's traversal visits them ...
    ctx.set_reference_lists(True)
    ctx.build_lists(theta)
    lists = ctx.lists()
    linfo = ctx.list_info()
    # ... and the default lists without pairs of empty cells, used for the results
    ctx.set_reference_lists(False)
    ctx.build_lists(theta)
    pruned = ctx.lists()
    ctx.m2l(tb.FP64)
    ctx.p2p(tb.FP64)
    ctx.downward(tb.FP64)
    res = ctx.results(tb.ORDER_ORIGINAL)
    cells = ctx.cells()
    sorted_idx, sorted_keys = ctx.sorted_bodies()
    M, L = ctx.expansions()
    return dict(x=x, y=y, z=z, q=q, P=P, theta=theta, o=o, res=res, cells=cells, lists=lists,
                sorted_idx=sorted_idx, sorted_keys=sorted_keys, M=M, L=L,
                info=ctx.tree_info(), linfo=linfo, pruned=pruned)


def test_tree_bit_exact(run):
    o = run["o"]
    oi, ok, _ = o.bodies()
    assert np.array_equal(run["sorted_keys"], ok)
    assert np.array_equal(run["sorted_idx"], oi)
    oc = o.cells()
    gc = run["cells"]
    assert len(gc["key"]) == len(oc["key"])
    go, oo = _cells_by_key(gc), _cells_by_key(oc)
    assert np.array_equal(gc["key"][go], oc["key"][oo])
    assert np.array_equal(gc["leaf"][go], oc["leaf"][oo])
    assert np.array_equal(gc["nb"][go], oc["nb"][oo])
    assert np.array_equal(gc["bbeg"][go].astype(np.int64), oc["bid"][oo])
    assert np.array_equal(gc["center"][go], oc["center"][oo])
    assert np.array_equal(gc["width"][go], oc["width"][oo])
    lo_hi = o.bbox()
    assert run["info"]["box_lo"] == lo_hi[0] and run["info"]["box_hi"] == lo_hi[1]


def _pair_keys(keys, t, s):
    return set(zip(keys[t].tolist(), keys[s].tolist()))


def test_lists_equal_as_sets(run):
    o = run["o"]
    okeys = o.cells()["key"]
    gkeys = run["cells"]["key"]
    (gmt, gms), (gpt, gps) = run["lists"]
    omt, oms = o.m2l_list()
    opt, ops = o.p2p_list()
    assert len(gmt) == len(omt) and len(gpt) == len(opt)
    assert _pair_keys(gkeys, gmt, gms) == _pair_keys(okeys, omt, oms)
    assert _pair_keys(gkeys, gpt, gps) == _pair_keys(okeys, opt, ops)
    assert run["linfo"]["n_p2p_interactions"] == o.p2p_interactions()
    # sorted by (target, source)
    packed = gmt.astype(np.int64) * (1 << 32) + gms
    assert np.all(np.diff(packed) > 0)


def test_pruned_lists_drop_only_empty_pairs(run):
    """Default lists = reference lists minus the pairs with an empty cell."""
    gkeys, nb = run["cells"]["key"], run["cells"]["nb"]
    (rmt, rms), (rpt, rps) = run["lists"]
    (pmt, pms), (ppt, pps) = run["pruned"]
    keep = (nb[rmt] > 0) & (nb[rms] > 0)
    assert _pair_keys(gkeys, pmt, pms) == _pair_keys(gkeys, rmt[keep], rms[keep])
    assert _pair_keys(gkeys, ppt, pps) == _pair_keys(gkeys, rpt, rps)


def test_expansions_fp64(run):
    o = run["o"]
    oM, oL = o.expansions()
    oc, gc = o.cells(), run["cells"]
    go, oo = _cells_by_key(gc), _cells_by_key(oc)
    assert _rel(run["M"][go], oM[oo]) < FP64_RTOL
    # L of empty cells is never used (and not computed on the GPU).
    ne = oc["nb"][oo] > 0
    assert _rel(run["L"][go][ne], oL[oo][ne]) < FP64_RTOL


def test_results_fp64(run):
    ref = run["o"].result()
    res = run["res"]
    assert _rel(res[:, 0], ref[:, 0]) < FP64_RTOL
    assert _rel(res[:, 1:], ref[:, 1:]) < FP64_RTOL
    assert _rel_rows(res, ref) < 1e-9


@pytest.mark.parametrize("path", GOLDEN, ids=[p.stem for p in GOLDEN])
def test_against_reference_goldens(path, tb, ctx):
    """Directly against outputs of the unmodified reference (with the golden's
    mutual option: the example's -m)."""
    g = np.load(path)
    mutual = int(g["mutual"]) if "mutual" in g else 0
    ctx.set_reference_lists(True)
    try:
        ctx.partition(g["x"], g["y"], g["z"], g["q"], ncrit=int(g["ncrit"]))
        ctx.upward(int(g["P"]), tb.FP64)
        ctx.traverse(float(g["theta"]), mutual, tb.FP64)
        ctx.downward(tb.FP64)
        res = ctx.results(tb.ORDER_ORIGINAL)
    finally:
        ctx.set_reference_lists(False)
    c = ctx.cells()
    order = np.argsort(c["key"], kind="stable")
    assert np.array_equal(c["key"][order], g["cell_key"])
    assert np.array_equal(c["nb"][order], g["cell_nb"])
    assert np.array_equal(c["leaf"][order], g["cell_leaf"])
    li = ctx.list_info()
    if mutual:
        # the lists hold both directions of every unordered pair the reference
        # visited; its counters count visits (j <= i within a leaf)
        (mt, ms), (pt, ps) = ctx.lists()
        nb = c["nb"].astype(np.int64)
        up = pt < ps
        self_ = pt == ps
        visits = int(np.sum(nb[pt[up]] * nb[ps[up]]) +
                     np.sum(nb[pt[self_]] * (nb[pt[self_]] + 1) // 2))
        assert li["n_m2l"] == 2 * int(g["n_m2l"])
        assert visits == int(g["n_p2p_interactions"])
    else:
        assert li["n_m2l"] == int(g["n_m2l"])
        assert li["n_p2p_interactions"] == int(g["n_p2p_interactions"])
    assert _rel(res, g["trg"]) < FP64_RTOL
    if "M" in g:
        M, L = ctx.expansions()
        assert _rel(M[order], g["M"]) < FP64_RTOL
        ne = g["cell_nb"] > 0
        assert _rel(L[order][ne], g["L"][ne]) < FP64_RTOL


@pytest.mark.parametrize("dist,ncrit", [("plummer", 64), ("plummer", 16),
                                        ("sphere_surface", 128), ("uniform_cube", 128)])
def test_mixed_close_to_fp64(dist, ncrit, tb, ctx, oracle_mod):
    """Mixed near field and tensor-core M2L against the FP64 form: small
    leaves (4-target P2P tiles) and full leaves (3-target tiles at 16 warps)."""
    x, y, z, q = tb.datasets.make(dist, 40000, 21)
    r64 = ctx.evaluate(x, y, z, q, P=10, ncrit=ncrit, theta=0.4, precision=tb.FP64)
    rmx = ctx.evaluate(x, y, z, q, P=10, ncrit=ncrit, theta=0.4, precision=tb.MIXED)
    ep, ea = oracle_mod.rel_l2(rmx, r64)
    assert ep < 2e-6 and ea < 2e-6
    tg = tb.datasets.sample_targets(len(x), 500)
    d = ctx.direct(tg)
    e64 = oracle_mod.rel_l2(r64[tg], d)
    emx = oracle_mod.rel_l2(rmx[tg], d)
    assert emx[0] < 1.5 * e64[0] + 1e-6 and emx[1] < 1.5 * e64[1] + 1e-6


@pytest.mark.parametrize("P", [14, 16])
def test_mixed_high_order_deep_tree(P, tb, ctx, oracle_mod):
    """Mixed form at high order on a deep tree: in small cells the local
    coefficients of degree n grow like 1/R^(n+1), beyond the FP32 range, so
    the FP32 L2P must work in units of the leaf width.  The results are finite
    and within 2e-6 (rel-L2) of the FP64 form."""
    x, y, z, q = tb.datasets.make("two_gaussians", 200000, 7)
    r64 = ctx.evaluate(x, y, z, q, P=P, ncrit=32, theta=0.4, precision=tb.FP64)
    rmx = ctx.evaluate(x, y, z, q, P=P, ncrit=32, theta=0.4, precision=tb.MIXED)
    assert np.isfinite(rmx).all()
    ep, ea = oracle_mod.rel_l2(rmx, r64)
    assert ep < 2e-6 and ea < 2e-6


@pytest.mark.parametrize("P", [4, 6, 8, 10, 11, 12, 14, 16])
def test_tensorcore_m2l_matches_fp64(P, tb, ctx):
    """Split-TF32 tensor-core M2L (mixed) against the FP64 M2L: per cell,
    ||L_mixed - L_fp64|| / ||L_fp64|| <= 2e-5 (FP32 accumulation of ~100-300
    translations of ~1e-7 relative accuracy each)."""
    x, y, z, q = tb.datasets.make("plummer", 60000, 61)
    ctx.partition(x, y, z, q, ncrit=32)
    ctx.upward(P, tb.FP64)
    ctx.build_lists(0.4)
    ctx.m2l(tb.FP64)
    _, L64 = ctx.expansions()
    ctx.m2l(tb.MIXED)
    _, Lmx = ctx.expansions()
    nb = ctx.cells()["nb"]
    ne = (nb > 0) & (np.linalg.norm(L64, axis=1) > 0)
    rel = np.linalg.norm(Lmx[ne] - L64[ne], axis=1) / np.linalg.norm(L64[ne], axis=1)
    assert rel.max() < 2e-5, (rel.max(), np.median(rel))


def test_gpu_direct_matches_oracle_direct(tb, ctx, oracle_mod):
    x, y, z, q = tb.datasets.make("uniform_cube", 20000, 3)
    ctx.partition(x, y, z, q, ncrit=64)
    tg = tb.datasets.sample_targets(len(x), 64)
    d = ctx.direct(tg)
    ref = oracle_mod.direct(x, y, z, q, tg, field=True)
    assert _rel(d, ref) < 1e-12


def test_fp64_accuracy_vs_direct(tb, ctx, oracle_mod):
    # The reference's own accuracy gate is rel-L2 < 5e-3 (test.sh:234); at
    # P=10, theta=0.4 the method gives ~1e-5 on zero-mean-free data.
    x, y, z, q = tb.datasets.make("uniform_cube", 50000, 9)
    r = ctx.evaluate(x, y, z, q, P=10, ncrit=64, theta=0.4, precision=tb.FP64)
    tg = tb.datasets.sample_targets(len(x), 300)
    ep, ea = oracle_mod.rel_l2(r[tg], ctx.direct(tg))
    assert ep < 1e-4 and ea < 1e-3


def test_deterministic(tb, ctx):
    """The FP64 form is bit-reproducible (lists sorted, no atomics).  The mixed
    form adds tensor-core M2L columns into FP32 locals with atomic reductions,
    so the summation order, and the last bits, vary between runs: repeat runs
    agree to 1e-7 relative."""
    x, y, z, q = tb.datasets.make("plummer", 30000, 23)
    a = ctx.evaluate(x, y, z, q, P=8, ncrit=32, theta=0.4, precision=tb.FP64)
    b = ctx.evaluate(x, y, z, q, P=8, ncrit=32, theta=0.4, precision=tb.FP64)
    assert np.array_equal(a, b)
    a = ctx.evaluate(x, y, z, q, P=8, ncrit=32, theta=0.4, precision=tb.MIXED)
    b = ctx.evaluate(x, y, z, q, P=8, ncrit=32, theta=0.4, precision=tb.MIXED)
    assert _rel(a, b) < 1e-7


def test_class_key_ranges_reused_and_renewed(tb, ctx):
    """The M2L class keys are packed with the field ranges of the previous
    classification; a list with larger offsets (smaller theta) misses them and
    is classified again.  Either way the classes, and so the FP64 class-GEMM
    result, equal a fresh context's bit for bit."""
    x, y, z, q = tb.datasets.make("plummer", 60000, 41)
    fresh = tb.Context(0)
    try:
        ref = {th: fresh.evaluate(x, y, z, q, P=8, ncrit=32, theta=th, precision=tb.FP64)
               for th in (0.3, 0.6)}
    finally:
        fresh.close()
    for th in (0.6, 0.3, 0.3, 0.6):
        r = ctx.evaluate(x, y, z, q, P=8, ncrit=32, theta=th, precision=tb.FP64)
        assert np.array_equal(r, ref[th])


def test_mixed_traverse_lists_sorted_on_demand(tb, ctx):
    """The mixed form's traversal leaves each target's sources unsorted in both
    lists (its M2L regroups the pairs by offset class, its FP32 near field sums
    in any order); the list accessor and a later FP64 M2L and P2P see them
    sorted, as build_lists gives them, so an FP64 evaluation after a mixed
    traversal equals a plain one bit for bit."""
    x, y, z, q = tb.datasets.make("sphere_surface", 40000, 3)
    fp64 = ctx.evaluate(x, y, z, q, P=6, ncrit=32, theta=0.4, precision=tb.FP64)
    (mt0, ms0), (pt0, ps0) = ctx.lists()
    ctx.upward(P=6, precision=tb.FP64)
    ctx.traverse(0.4, 0, tb.MIXED)
    (mt, ms), (pt, ps) = ctx.lists()
    for a, b in ((mt, mt0), (ms, ms0), (pt, pt0), (ps, ps0)):
        assert np.array_equal(a, b)
    assert np.all(np.diff(mt.astype(np.int64) * (1 << 32) + ms) > 0)
    ctx.traverse(0.4, 0, tb.MIXED)
    ctx.m2l(tb.FP64)
    ctx.p2p(tb.FP64)
    ctx.downward(tb.FP64)
    assert np.array_equal(ctx.results(), fp64)


@pytest.mark.parametrize("n,ncrit", [(1, 64), (2, 1), (5, 2), (50, 64), (64, 64), (65, 64)])
def test_small_and_root_leaf(n, ncrit, tb, ctx, oracle_mod):
    """Tiny inputs, including a root that is itself a leaf (which the reference
    itself cannot run) and the bounding-cube quirk with few bodies."""
    x, y, z, q = tb.datasets.make("uniform_cube", n, 31 + n)
    o = oracle_mod.Oracle(x, y, z, q, P=6, ncrit=ncrit, theta=0.4)
    r = ctx.evaluate(x, y, z, q, P=6, ncrit=ncrit, theta=0.4, precision=tb.FP64)
    ref = o.result()
    assert np.array_equal(np.isnan(r), np.isnan(ref))
    ok = ~np.isnan(ref)
    if ok.any():
        assert _rel(r[ok], ref[ok]) < FP64_RTOL
    gi, gk = ctx.sorted_bodies()
    oi, ok2, _ = o.bodies()
    assert np.array_equal(gk, ok2) and np.array_equal(gi, oi)


def test_coincident_bodies_reach_max_depth(tb, ctx, oracle_mod):
    """More than ncrit bodies at one point: cells split to the deepest key
    level (19), where they become leaves."""
    x, y, z, q = [a.copy() for a in tb.datasets.make("uniform_cube", 400, 41)]
    x[:40] = 0.123
    y[:40] = -0.456
    z[:40] = 0.789
    o = oracle_mod.Oracle(x, y, z, q, P=4, ncrit=8, theta=0.5)
    r = ctx.evaluate(x, y, z, q, P=4, ncrit=8, theta=0.5, precision=tb.FP64)
    assert ctx.tree_info()["max_depth"] == 19
    ref = o.result()
    assert _rel(r, ref) < FP64_RTOL


def test_errors_are_status_codes(tb):
    with tb.Context(0) as c:
        with pytest.raises(tb.TapasError) as e:
            c.upward(10)
        assert e.value.code == -4  # state: no tree
        x, y, z, q = tb.datasets.make("uniform_cube", 1000, 1)
        c.partition(x, y, z, q, ncrit=16)
        with pytest.raises(tb.TapasError) as e:
            c.upward(17)
        assert e.value.code == -6
        c.upward(6)
        with pytest.raises(tb.TapasError) as e:
            c.build_lists(0.4, mutual=2)
        assert e.value.code == -1
        with pytest.raises(tb.TapasError) as e:
            c.downward()
        assert e.value.code == -4
        with pytest.raises(tb.TapasError) as e:
            c.partition(x, y, z, q, ncrit=0)
        assert e.value.code == -1


def test_device_pointers(tb, ctx):
    torch = pytest.importorskip("torch")
    x, y, z, q = tb.datasets.make("uniform_cube", 10000, 51)
    ref = ctx.evaluate(x, y, z, q, P=6, ncrit=32, theta=0.4)
    dx, dy, dz, dq = [torch.from_numpy(a).cuda() for a in (x, y, z, q)]
    out = torch.zeros((len(x), 4), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    ctx.evaluate(dx, dy, dz, dq, P=6, ncrit=32, theta=0.4, out=out)
    assert np.array_equal(out.cpu().numpy(), ref)


@pytest.mark.parametrize("ncrit,nsparse,longest", [(64, 120, 4000), (8, 16, 30000)],
                         ids=["block-sorted", "radix-sorted"])
def test_long_list_segments(tb, oracle_mod, ctx, ncrit, nsparse, longest):
    """Leaves of a sparse half-cube beside a dense half each have a P2P list of
    thousands of small leaves: longer than one warp sorts (a block sorts
    them), or longer than one block sorts (the whole list goes through the
    radix sort).  Both lists must still equal the reference traversal's as
    sets, in (target, source) order."""
    rng = np.random.default_rng(11)
    dense = rng.random((120000, 3))
    dense[:, 0] *= 0.5
    sparse = rng.random((nsparse, 3))
    sparse[:, 0] = 0.5 + 0.5 * sparse[:, 0]
    pts = np.vstack([dense, sparse])
    x, y, z = (np.ascontiguousarray(pts[:, d]) for d in range(3))
    q = rng.random(len(x)) / len(x)
    o = oracle_mod.Oracle(x, y, z, q, P=4, ncrit=ncrit, theta=0.3, run=False)
    assert oracle_mod.lib().oracle_build(o.h) == 0
    assert oracle_mod.lib().oracle_traverse(o.h) == 0
    ctx.partition(x, y, z, q, ncrit=ncrit)
    ctx.set_reference_lists(True)
    try:
        ctx.build_lists(0.3)
        (gmt, gms), (gpt, gps) = ctx.lists()
    finally:
        ctx.set_reference_lists(False)
    assert np.bincount(gpt).max() > longest  # the path is exercised
    gkeys, okeys = ctx.cells()["key"], o.cells()["key"]
    omt, oms = o.m2l_list()
    opt, ops = o.p2p_list()
    assert _pair_keys(gkeys, gmt, gms) == _pair_keys(okeys, omt, oms)
    assert _pair_keys(gkeys, gpt, gps) == _pair_keys(okeys, opt, ops)
    for t, s in ((gmt, gms), (gpt, gps)):
        assert np.all(np.diff(t.astype(np.int64) * (1 << 32) + s) > 0)


def test_long_source_lists_are_split(tb, ctx):
    """A Plummer set has leaves whose near-field lists hold far more than the
    32,768 source bodies one P2P work item takes; those lists are cut into
    pieces whose partial sums are added in piece order, so the FP64 form stays
    bit-reproducible and both forms keep their accuracy."""
    x, y, z, q = tb.datasets.make("plummer", 200000, 31)
    ctx.partition(x, y, z, q, ncrit=64)
    ctx.build_lists(0.3)
    c = ctx.cells()
    _, (pt, ps) = ctx.lists()
    per_target = np.bincount(pt, weights=c["nb"][ps].astype(np.float64), minlength=len(c["nb"]))
    assert per_target.max() > 4 * 32768  # the case is exercised
    a = ctx.evaluate(x, y, z, q, P=8, ncrit=64, theta=0.3, precision=tb.FP64)
    b = ctx.evaluate(x, y, z, q, P=8, ncrit=64, theta=0.3, precision=tb.FP64)
    assert np.array_equal(a, b)
    tg = tb.datasets.sample_targets(len(x), 400, seed=5)
    d = ctx.direct(tg)
    num = np.linalg.norm(a[tg] - d, axis=0)
    den = np.linalg.norm(d, axis=0)
    assert num[0] / den[0] < 1e-5 and np.linalg.norm(num[1:]) / np.linalg.norm(den[1:]) < 1e-4
    m = ctx.evaluate(x, y, z, q, P=8, ncrit=64, theta=0.3, precision=tb.MIXED)
    assert np.linalg.norm(m[:, 0] - a[:, 0]) / np.linalg.norm(a[:, 0]) < 2e-6


def test_tensorcore_m2l_wait_timeout_is_a_status(tb, ctx):
    """The tensor-core M2L's designed failure path: with a wait bound of 100
    clock cycles the MMA thread's first wait for a copy gives up, every role
    leaves its loop, the CTA drains its copies and MMAs and frees its tensor
    memory, and the call returns TAPAS_B200_ERR_TIMEOUT.  The same context then
    evaluates normally with the default bound."""
    x, y, z, q = tb.datasets.make("plummer", 60000, 61)
    ctx.partition(x, y, z, q, ncrit=32)
    ctx.upward(8, tb.FP64)
    ctx.build_lists(0.4)
    ctx.m2l(tb.FP64)
    _, L64 = ctx.expansions()
    try:
        ctx.set_wait_limit(100)
        with pytest.raises(tb.TapasError) as e:
            ctx.m2l(tb.MIXED)
        assert e.value.code == tb._lib.ERR_TIMEOUT
        assert "gave up" in str(e.value)
    finally:
        ctx.set_wait_limit(0)
    ctx.m2l(tb.MIXED)
    _, Lmx = ctx.expansions()
    nb = ctx.cells()["nb"]
    ne = (nb > 0) & (np.linalg.norm(L64, axis=1) > 0)
    rel = np.linalg.norm(Lmx[ne] - L64[ne], axis=1) / np.linalg.norm(L64[ne], axis=1)
    assert rel.max() < 2e-5


@pytest.mark.parametrize("P", [6, 12, 16])
def test_mixed_tree_translations_per_cell(P, tb, ctx):
    """The mixed form's tree translations (M2M: split-TF32 tensor-core GEMMs
    with level-independent operators on the deepest three parent levels below
    level 3, FP64 level GEMMs above them; L2L: FP64) on a deep tree, per cell
    against the FP64 form: multipoles within 1e-6 of
    the cell's multipoles of |q| (see below), local expansions after the
    downward pass within 5e-5 of the FP64 ones."""
    x, y, z, q = tb.datasets.make("two_gaussians", 200000, 19)
    ctx.partition(x, y, z, np.abs(q), ncrit=32)
    ctx.upward(P, tb.FP64)
    Mabs, _ = ctx.expansions()
    assert ctx.tree_info()["max_depth"] >= 8  # levels below the FP64 ones exist
    out = {}
    for prec in (tb.FP64, tb.MIXED):
        ctx.partition(x, y, z, q, ncrit=32)
        ctx.upward(P, prec)
        ctx.traverse(0.4, 0, prec)
        ctx.downward(prec)
        out[prec] = ctx.expansions()
    (M64, L64), (Mmx, Lmx) = out[tb.FP64], out[tb.MIXED]
    scale = np.linalg.norm(Mabs, axis=1)
    ok = scale > 0
    relM = np.linalg.norm(Mmx[ok] - M64[ok], axis=1) / scale[ok]
    assert relM.max() < 1e-6, relM.max()
    nrm = np.linalg.norm(L64, axis=1)
    ne = (ctx.cells()["nb"] > 0) & (nrm > 0)
    relL = np.linalg.norm(Lmx[ne] - L64[ne], axis=1) / nrm[ne]
    assert relL.max() < 5e-5, (relL.max(), np.median(relL))


@pytest.mark.parametrize("P", [4, 10, 16])
@pytest.mark.parametrize("dist", ["sphere_surface", "two_gaussians"])
def test_fp32_p2m_per_cell(P, dist, tb, ctx):
    """The mixed form's P2M (FP32 terms in units of the leaf width, FP32 warp
    reduce-scatter, FP64 sums over body chunks) followed by its M2M (FP64 at
    the top levels, split-TF32 tensor cores below), against the FP64 upward
    pass, per cell.  An FP32 term rounds to ~6e-8 of
    itself, so the error of a cell's M is bounded by its scale without
    cancellation: ||M_mixed - M_fp64|| <= 1e-6 ||M_|q|||, M_|q| the FP64
    multipoles of the charges' magnitudes.  (Where zero-mean charges cancel,
    M_fp64 itself can be far smaller than that scale.)  The sphere-surface set
    has zero-mean charges; the Gaussian clusters give a deep tree."""
    x, y, z, q = tb.datasets.make(dist, 150000, 17)
    ctx.partition(x, y, z, np.abs(q), ncrit=32)
    ctx.upward(P, tb.FP64)
    Mabs, _ = ctx.expansions()
    ctx.partition(x, y, z, q, ncrit=32)
    ctx.upward(P, tb.FP64)
    M64, _ = ctx.expansions()
    ctx.upward(P, tb.MIXED)
    Mmx, _ = ctx.expansions()
    scale = np.linalg.norm(Mabs, axis=1)
    ok = scale > 0
    rel = np.linalg.norm(Mmx[ok] - M64[ok], axis=1) / scale[ok]
    assert rel.max() < 1e-6, (rel.max(), np.median(rel))
    assert ctx.tree_info()["max_depth"] >= 6
