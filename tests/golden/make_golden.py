"""Generates the golden fixtures in this directory from the UNMODIFIED reference.

Each case runs the reference ExaFMM/Tapas example (built from its own sources
by ``make -C oracle ref`` into oracle/_ref/, see oracle/ref_driver.cxx) on a
seeded synthetic body set and stores its inputs and outputs:

* ``x, y, z, q``            inputs (original order)
* ``trg``                   reference TRG per body, ORIGINAL order (pot, ax, ay, az)
* ``order``                 original index of each body in the reference's sorted order
* ``cell_key/leaf/nb/bid``  cells sorted by key; ``cell_center``, ``cell_width``
* ``M``, ``L``              per-cell expansions (small cases only)
* ``n_m2l``, ``n_p2p_interactions``  the reference's -DCOUNT counters

Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import importlib.util
import os
import pathlib
import sys

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "oracle"))
import oracle  # noqa: E402

spec = importlib.util.spec_from_file_location("ds", ROOT / "tapas-reduce_b200" / "datasets.py")
ds = importlib.util.module_from_spec(spec)
spec.loader.exec_module(ds)

# name: (distribution, n, seed, P, ncrit, theta, keep_expansions)
CASES = {
    "cube_n2000_p10": ("uniform_cube", 2000, 11, 10, 32, 0.4, False),
    "plummer_n3000_p8": ("plummer", 3000, 12, 8, 24, 0.5, False),
    "sphere_n2500_p6": ("sphere_surface", 2500, 13, 6, 16, 0.35, False),
    "gauss_n1500_p4": ("two_gaussians", 1500, 14, 4, 8, 0.6, False),
    "cube_n400_p6_ML": ("uniform_cube", 400, 15, 6, 16, 0.4, True),
    "cube_n300_ncrit1_p4": ("uniform_cube", 300, 16, 4, 1, 0.5, False),
    "tiny_n1": ("uniform_cube", 1, 17, 4, 64, 0.4, True),
    "tiny_n2": ("uniform_cube", 2, 18, 4, 1, 0.4, True),
    "tiny_n7": ("plummer", 7, 19, 6, 2, 0.4, True),
    "root_leaf_n50": ("uniform_cube", 50, 20, 8, 64, 0.4, True),
}
# The example's -m 1 (mutual interaction): same fields plus mutual = 1.
MUTUAL_CASES = {
    "mutual_plummer_n4000_p8": ("plummer", 4000, 23, 8, 32, 0.4, False),
    "mutual_gauss_n3000_p10": ("two_gaussians", 3000, 24, 10, 16, 0.5, False),
    "mutual_cube_n500_p6_ML": ("uniform_cube", 500, 25, 6, 16, 0.4, True),
}


def make(name, dist, n, seed, P, ncrit, theta, keep, mutual=0):
    x, y, z, q = ds.make(dist, n, seed)
    R = oracle.run_reference(x, y, z, q, P=P, ncrit=ncrit, theta=theta, mutual=mutual)
    b = R["bodies"]
    trg = np.empty((n, 4))
    trg[b["ibody"]] = b["trg"]
    c = R["cells"]
    out = dict(x=x, y=y, z=z, q=q, P=P, ncrit=ncrit, theta=theta, trg=trg,
               order=b["ibody"].astype(np.int64),
               cell_key=c["key"], cell_leaf=c["leaf"], cell_nb=c["nb"], cell_bid=c["bid"],
               cell_center=c["center"], cell_width=c["width"],
               n_m2l=R["n_m2l"], n_p2p_interactions=R["n_p2p_interactions"], mutual=mutual)
    if keep:
        out["M"] = c["M"][..., 0] + 1j * c["M"][..., 1]
        out["L"] = c["L"][..., 0] + 1j * c["L"][..., 1]
    np.savez_compressed(pathlib.Path(__file__).parent / f"{name}.npz", **out)
    print(name, n, "cells", len(c), "m2l", R["n_m2l"], "p2p", R["n_p2p_interactions"])


# Barnes-Hut sample (ncrit = 1, theta = 0.5, EPS2 = 1e-6 fixed by bh.cc):
# name: (distribution, n, seed); "unit_cube_mass" is the sample's own data
# model (positions uniform in [0,1)^3, masses U[0,1)/N, bh.cc:414-427)
# restated with this project's generator.
BH_CASES = {
    "bh_unitcube_n2000": ("unit_cube_mass", 2000, 21),
    "bh_plummer_n1500": ("plummer", 1500, 22),
}


def make_bh(name, dist, n, seed):
    if dist == "unit_cube_mass":
        x, y, z = (ds.uniform01(seed, s, n) for s in (1, 2, 3))
        m = ds.uniform01(seed, 4, n) / n
    else:
        x, y, z, m = ds.make(dist, n, seed)
    res = oracle.run_bh_reference(x, y, z, m)
    np.savez_compressed(pathlib.Path(__file__).parent / f"{name}.npz", x=x, y=y, z=z, m=m,
                        bh=res, ncrit=1, theta=0.5, eps2=1e-6)
    print(name, n)


# Benchmark-sized cases: the inputs are regenerated from the seed (datasets.py)
# and only a seeded sample of the reference's results is kept, with a checksum
# of the inputs.  name: (distribution, n, seed, P, ncrit, theta, samples)
SAMPLED_CASES = {
    "refsample_cube_n100000_p10": ("uniform_cube", 100_000, 101, 10, 64, 0.4, 2000),
    "refsample_plummer_n1000000_p10": ("plummer", 1_000_000, 102, 10, 64, 0.4, 2000),
    "refsample_sphere_n1000000_p15": ("sphere_surface", 1_000_000, 104, 15, 128, 0.4, 4000),
    "refsample_sphere_n16000000_p15": ("sphere_surface", 16_000_000, 5, 15, 128, 0.4, 4000),
    "refsample_sphere_n16000000_p13": ("sphere_surface", 16_000_000, 5, 13, 128, 0.35, 4000),
    "refsample_sphere_n16000000_p12": ("sphere_surface", 16_000_000, 5, 12, 128, 0.35, 4000),
}


def input_checksum(x, y, z, q):
    """Order-dependent checksum of a body set (detects a changed generator)."""
    w = np.arange(1, len(x) + 1, dtype=np.float64) % 1009.0 + 1.0
    return np.array([np.dot(w, a) for a in (x, y, z, q)])


def make_sampled(name, dist, n, seed, P, ncrit, theta, samples):
    x, y, z, q = ds.make(dist, n, seed)
    R = oracle.run_reference(x, y, z, q, P=P, ncrit=ncrit, theta=theta, timeout=6 * 3600)
    b = R["bodies"]
    trg = np.empty((n, 4))
    trg[b["ibody"]] = b["trg"]
    idx = ds.sample_targets(n, samples, seed=1234)
    t = R["times"]
    np.savez_compressed(pathlib.Path(__file__).parent / f"{name}.npz", dist=dist, n=n, seed=seed,
                        P=P, ncrit=ncrit, theta=theta, idx=idx, trg=trg[idx],
                        checksum=input_checksum(x, y, z, q), n_m2l=R["n_m2l"],
                        n_p2p_interactions=R["n_p2p_interactions"],
                        ncells=R["ncells"],
                        ref_seconds=t["tree"] + t["upward"] + t["traverse"] + t["downward"])
    print(name, n, "reference", t)


def make_io():
    """The reference's file formats, written and read by its own code
    (oracle/_ref/io_ref, oracle/io_ref_driver.cxx): io_source0000.dat and
    io_target0000.dat for a seeded 37-body set with values of many magnitudes,
    the values the reference's readers get back from them in two successive
    calls (18 + 19 bodies), and a main.csv row."""
    import subprocess
    import tempfile
    rng = np.random.default_rng(2024)
    n = 37
    v = rng.standard_normal((n, 8)) * 10.0 ** rng.integers(-12, 12, (n, 8))
    v[0, :] = [0.0, -0.0, 1.0, -1.0, 0.1, 1e-300, 123456789.0, 2.5e-8]
    v[1, :4] = [np.pi, -np.e, 1.0 / 3.0, 7.0]
    gdir = pathlib.Path(__file__).parent
    with tempfile.TemporaryDirectory() as d:
        fin, fout = os.path.join(d, "in.bin"), os.path.join(d, "out.bin")
        with open(fin, "wb") as f:
            f.write(np.int64(n).tobytes())
            f.write(v.tobytes())
        subprocess.run([str(oracle.REF_DIR / "io_ref"), "dat", fin, d, fout], check=True)
        back = np.fromfile(fout).reshape(n, 8)
        for stem in ("source", "target"):
            (gdir / f"io_{stem}0000.dat").write_bytes(open(os.path.join(d, f"{stem}0000.dat"),
                                                           "rb").read())
        csv_args = ["3.79", "0.143", "3.39", "0.18", "0.071", "164050000", "579992"]
        subprocess.run([str(oracle.REF_DIR / "io_ref"), "csv", str(gdir / "io_main.csv"),
                        *csv_args], check=True)
    np.savez_compressed(gdir / "io_formats.npz", values=v, readback=back,
                        csv_args=np.array(csv_args))
    print("io fixtures", n)


if __name__ == "__main__":
    import subprocess
    oracle.build_reference(quiet=False)
    if len(sys.argv) > 1 and sys.argv[1] == "io":
        make_io()
        sys.exit(0)
    if len(sys.argv) > 1:  # named sampled cases only
        for name in sys.argv[1:]:
            make_sampled(name, *SAMPLED_CASES[name])
        sys.exit(0)
    for name, args in BH_CASES.items():
        make_bh(name, *args)
    for name, args in MUTUAL_CASES.items():
        make(name, *args, mutual=1)
    for name, args in CASES.items():
        try:
            make(name, *args)
        except subprocess.CalledProcessError as e:
            # The reference aborts when the root cell is itself a leaf
            # (n <= ncrit): its Map direction probe calls subcell() on it
            # ("Cell::subcell(int) is called for a leaf cell").  No golden.
            print(name, "reference failed:", e.returncode)
