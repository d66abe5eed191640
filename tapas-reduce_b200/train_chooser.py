"""Data generation, training and held-out evaluation of the learned chooser.

Run on a GPU, from the repository root:
    python tapas-reduce_b200/train_chooser.py generate   # 2,320 FMM runs -> chooser_data.npz
    python tapas-reduce_b200/train_chooser.py train      # own CUDA kernels -> chooser_model.npz
    python tapas-reduce_b200/train_chooser.py evaluate   # 200 held-out systems

Training systems: 250 seeded body sets, N log-uniform in [1e4, 1e6], and 40
with N log-uniform in [1e6, 1.6e7] (theta >= 0.25, ncrit >= 32), the
distribution drawn from {uniform cube [-1,1]^3, Plummer, two Gaussian clusters
sigma 0.1 with centres 1.0 apart, unit sphere surface}, charges equal positive
or zero-mean U[-1,1] with equal odds; 8 random settings each (P in 4..16, theta in [0.2, 0.7], ncrit in
{16, 32, 64, 128}, mixed or FP64) = 2,320 runs.  Each run records the
relative-L2 potential error against an FP64 direct sum on 256 sampled targets
and the device time of the evaluation (sum of the library's CUDA-event phase
timings: tree, upward, traversal, M2L, P2P, downward).
"""
from __future__ import annotations

import importlib.util
import json
import pathlib
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
DATA_PATH = HERE / "chooser_data.npz"
# The three distributions of the chooser's specification plus the sphere
# surface of the large 16M-body run, so that run is inside the training set.
DISTS = ["uniform_cube", "plummer", "two_gaussians", "sphere_surface"]
PHASES = ("bbox_keys", "sort", "tree", "upward", "traverse", "list_sort", "m2l", "p2p",
          "downward")


def _pkg():
    if "tapas_reduce_b200" in sys.modules:
        return sys.modules["tapas_reduce_b200"]
    spec = importlib.util.spec_from_file_location(
        "tapas_reduce_b200", HERE / "__init__.py", submodule_search_locations=[str(HERE)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["tapas_reduce_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def make_system(tb, i, seed_base, log10_n=(4.0, 6.0)):
    rng = np.random.default_rng(seed_base + i)
    n = int(round(10 ** rng.uniform(*log10_n)))
    dist = DISTS[int(rng.integers(len(DISTS)))]
    x, y, z, _ = tb.datasets.make(dist, n, seed_base + i)
    if rng.random() < 0.5:  # zero-mean charges
        q = 2.0 * tb.datasets.uniform01(seed_base + i, 91, n) - 1.0
        q = q - q.mean()
    else:  # equal positive charges
        q = np.full(n, 1.0 / n)
    return dist, n, (x, y, z, q), rng


def timed_run(tb, ctx, bodies, P, theta, ncrit, prec):
    ctx.set_profiling(True)
    res = ctx.evaluate(*bodies, P=P, ncrit=ncrit, theta=theta, precision=prec)
    res = ctx.evaluate(*bodies, P=P, ncrit=ncrit, theta=theta, precision=prec)
    t = ctx.timings()
    ctx.set_profiling(False)
    return res, float(sum(t[k] for k in PHASES))


def generate(n_systems=250, per_system=8, seed_base=10_000, out=DATA_PATH, n_large=40):
    """n_systems body sets of 1e4..1e6 bodies, then n_large of 1e6..1.6e7 (the
    large runs keep theta >= 0.25 and ncrit >= 32, so every run's lists stay
    within a few GB)."""
    tb = _pkg()
    from tapas_reduce_b200 import chooser, verify
    rows = []
    sets = [(i, seed_base, (4.0, 6.0)) for i in range(n_systems)]
    sets += [(i, seed_base + 50_000, (6.0, chooser.LOG10_N_MAX)) for i in range(n_large)]
    with tb.Context(0) as ctx:
        for k, (i, base, log10_n) in enumerate(sets):
            dist, n, bodies, rng = make_system(tb, i, base, log10_n)
            large = n > 1_000_000
            feats = chooser.system_features(ctx, *bodies)
            tg = tb.datasets.sample_targets(n, 256, seed=base + i)
            d = ctx.direct(tg)
            for _ in range(per_system):
                for attempt in range(4):  # a setting too large for the device: draw again
                    P = int(rng.integers(4, 17))
                    theta = float(np.round(rng.uniform(0.25 if large else 0.2, 0.7), 2))
                    ncrit = int(rng.choice([32, 64, 128] if large else [16, 32, 64, 128]))
                    fp64 = int(rng.random() < 0.3)
                    try:
                        res, ms = timed_run(tb, ctx, bodies, P, theta, ncrit,
                                            tb.FP64 if fp64 else tb.MIXED)
                        break
                    except tb.TapasError as err:
                        print(f"system {k} n={n} {dist} P={P} theta={theta} ncrit={ncrit}: "
                              f"{err}", flush=True)
                        if attempt == 3:
                            raise
                err = verify.rel_l2(res[tg], d)[0]
                if not (np.isfinite(err) and np.isfinite(ms)):
                    raise RuntimeError(f"system {k} n={n} {dist} P={P} theta={theta} "
                                       f"ncrit={ncrit} fp64={fp64}: non-finite result")
                rows.append(np.concatenate([feats, [P, theta, ncrit, fp64,
                                                    np.log10(max(err, 1e-16)),
                                                    np.log10(ms), n, DISTS.index(dist)]]))
            if (k + 1) % 25 == 0:
                print(f"{k + 1}/{len(sets)} systems", flush=True)
    data = np.array(rows)
    np.savez_compressed(out, data=data, nfeat=len(feats))
    print(f"wrote {out}: {data.shape}")
    return data


def training_arrays(data, nfeat):
    from tapas_reduce_b200 import chooser
    feats = data[:, :nfeat]
    P, th, nc, f64 = data[:, nfeat], data[:, nfeat + 1], data[:, nfeat + 2], data[:, nfeat + 3]
    X = np.concatenate([chooser.encode(f, p, t, c, b) for f, p, t, c, b in
                        zip(feats, P, th, nc, f64)], axis=0)
    Y = data[:, nfeat + 4:nfeat + 6]
    return X, Y


def train(data_path=DATA_PATH, out=None, rounds=120, epochs_per_round=5, patience=12,
          seed=0, per_system=8):
    """Adam on the GPU (own kernels) with early stopping: 10 % of the training
    SYSTEMS (all runs of a system together) are held out for validation; the
    parameters with the lowest validation loss are kept.  The safety margin
    is the 90th percentile of how far the held-out error was under-predicted."""
    tb = _pkg()
    from tapas_reduce_b200 import chooser
    out = out or chooser.MODEL_PATH
    z = np.load(data_path)
    data, nfeat = z["data"], int(z["nfeat"])
    X, Y = training_arrays(data, nfeat)
    rng = np.random.default_rng(seed)
    nsys = len(X) // per_system
    vsys = rng.choice(nsys, max(1, nsys // 10), replace=False)
    is_val = np.isin(np.arange(len(X)) // per_system, vsys)
    val, trn = np.flatnonzero(is_val), np.flatnonzero(~is_val)
    x_mean, x_std = X[trn].mean(0), X[trn].std(0) + 1e-6
    y_mean, y_std = Y[trn].mean(0), Y[trn].std(0) + 1e-6
    Xs = ((X - x_mean) / x_std).astype(np.float32)
    Ys = ((Y - y_mean) / y_std).astype(np.float32)
    dims = [X.shape[1], 64, 64, 64, 2]
    hist, vhist = [], []
    with tb.Context(0) as ctx:
        ctx.mlp_create(dims[0], 64, 3, 2, seed=seed)
        best, best_p, since = np.inf, ctx.mlp_params(), 0
        for r in range(rounds):
            h = ctx.mlp_train(Xs[trn], Ys[trn], epochs=epochs_per_round, batch=64, lr=1e-3,
                              seed=seed + r)
            hist.extend(h.tolist())
            pv = ctx.mlp_forward(Xs[val]).astype(np.float64)
            vl = float(np.mean((pv - Ys[val]) ** 2))
            vhist.append(vl)
            if vl < best:
                best, best_p, since = vl, ctx.mlp_params(), 0
            else:
                since += 1
                if since >= patience:
                    break
        ctx.mlp_set_params(best_p)
        pv = ctx.mlp_forward(Xs[val]).astype(np.float64) * y_std + y_mean
    res = Y[val] - pv
    margin = float(np.quantile(res[:, 0], 0.90))  # under-prediction of log10 error
    np.savez_compressed(out, dims=np.array(dims), params=best_p, x_mean=x_mean, x_std=x_std,
                        y_mean=y_mean, y_std=y_std, margin=max(margin, 0.0),
                        loss=np.array(hist), val_loss=np.array(vhist))
    info = {"train_loss_first": float(hist[0]), "train_loss_last": float(hist[-1]),
            "best_val_loss": best, "rounds": len(vhist),
            "val_rmse_log10_err": float(np.sqrt(np.mean(res[:, 0] ** 2))),
            "val_rmse_log10_ms": float(np.sqrt(np.mean(res[:, 1] ** 2))),
            "margin_log10": margin, "n_train": int(len(trn)), "n_val": int(len(val))}
    print(json.dumps(info))
    return info


def evaluate(n_systems=200, seed_base=90_000, targets=256):
    """Held-out systems, random tolerance in [1e-7, 1e-3] each: the learned
    choice against the fixed setting (P=10, theta=0.4, ncrit=64) in the same
    mixed arithmetic and in FP64."""
    tb = _pkg()
    from tapas_reduce_b200 import chooser, verify
    recs = []
    with tb.Context(0) as ctx:
        lc = chooser.learned_chooser(ctx)
        for i in range(n_systems):
            dist, n, bodies, rng = make_system(tb, i, seed_base)
            tol = float(10 ** rng.uniform(-7, -3))
            feats = chooser.system_features(ctx, *bodies)
            tg = tb.datasets.sample_targets(n, targets, seed=seed_base + i)
            d = ctx.direct(tg)
            prm = lc.choose(feats, tol)
            res, ms = timed_run(tb, ctx, bodies, prm["P"], prm["theta"], prm["ncrit"],
                                tb.FP64 if prm["precision"] == "fp64" else tb.MIXED)
            e = verify.rel_l2(res[tg], d)[0]
            rf, msf = timed_run(tb, ctx, bodies, 10, 0.4, 64, tb.MIXED)
            ef = verify.rel_l2(rf[tg], d)[0]
            r64, ms64 = timed_run(tb, ctx, bodies, 10, 0.4, 64, tb.FP64)
            e64 = verify.rel_l2(r64[tg], d)[0]
            recs.append(dict(n=n, dist=dist, tol=tol, params=prm, err=e, ms=ms, err_fixed=ef,
                             ms_fixed=msf, err_fixed64=e64, ms_fixed64=ms64))
    hit = np.mean([r["err"] <= r["tol"] for r in recs])
    hit_fixed = np.mean([r["err_fixed"] <= r["tol"] for r in recs])
    hit_fixed64 = np.mean([r["err_fixed64"] <= r["tol"] for r in recs])
    def gm(rs, key):
        return float(np.exp(np.mean([np.log(r[key] / r["ms"]) for r in rs]))) if rs else None

    both = [r for r in recs if r["err"] <= r["tol"] and r["err_fixed64"] <= r["tol"]]
    summary = {"systems": n_systems, "hit_rate_learned": float(hit),
               "hit_rate_fixed_mixed": float(hit_fixed), "hit_rate_fixed_fp64": float(hit_fixed64),
               "geomean_speedup_vs_fixed_mixed": gm(recs, "ms_fixed"),
               "geomean_speedup_vs_fixed_fp64": gm(recs, "ms_fixed64"),
               "geomean_speedup_vs_fixed_fp64_where_both_meet": gm(both, "ms_fixed64"),
               "n_both_meet": len(both)}
    return summary, recs


if __name__ == "__main__":
    cmd = sys.argv[1] if len(sys.argv) > 1 else "all"
    if cmd in ("generate", "all"):
        generate()
    if cmd in ("train", "all"):
        train()
    if cmd in ("evaluate", "all"):
        s, recs = evaluate()
        print(json.dumps(s))
        out = pathlib.Path(sys.argv[2]) if len(sys.argv) > 2 else None
        if out:
            out.write_text(json.dumps({"summary": s, "records": recs}, default=str))
