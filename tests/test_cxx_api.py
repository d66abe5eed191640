"""The C++ Tapas-API header (include/tapas_b200/tapas.hpp) over the C ABI.

tests/cxx/tapas_api_driver.cxx is written the way the reference's drivers
call Tapas (ex/tapas_exafmm.cxx:560-641, sample/barnes-hut/bh.cc:228-245).
CPU: it compiles against the header, links against libtapas_b200.so, and
reports a missing GPU as a library error (exit 3), not a crash.
GPU: its results equal the C ABI's own (bit for bit in FP64: same kernels,
deterministic order), the FMM matches the oracle within 1e-11 and the
Barnes-Hut walk matches the oracle bit for bit.
"""
import pathlib
import shutil
import struct
import subprocess

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent
SRC = ROOT / "tests" / "cxx" / "tapas_api_driver.cxx"


@pytest.fixture(scope="module")
def driver(tb, tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("no C++ compiler")
    from importlib import import_module
    lib = pathlib.Path(import_module("tapas_reduce_b200.build").build())
    exe = tmp_path_factory.mktemp("cxx") / "tapas_api_driver"
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I", str(ROOT / "include"),
           str(SRC), "-L", str(lib.parent), "-ltapas_b200", f"-Wl,-rpath,{lib.parent}",
           "-o", str(exe)]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def _run(driver, tmp, mode, x, y, z, q, P=8, ncrit=32, theta=0.4, mixed=0):
    inp, out = tmp / f"{mode}_in.bin", tmp / f"{mode}_out.bin"
    with open(inp, "wb") as f:
        f.write(struct.pack("<q", len(x)))
        for a in (x, y, z, q):
            f.write(np.ascontiguousarray(a, dtype="<f8").tobytes())
    p = subprocess.run([str(driver), mode, str(inp), str(out), str(P), str(ncrit), str(theta),
                        str(mixed)], capture_output=True, text=True, timeout=600)
    if p.returncode != 0:
        return p, None, None
    raw = out.read_bytes()
    n = struct.unpack("<q", raw[:8])[0]
    rec = np.frombuffer(raw[8:], dtype=[("i", "<i8"), ("r", "<f8", (4,))], count=n)
    return p, rec["i"].copy(), rec["r"].copy()


def _no_gpu():
    try:
        import torch
        return not torch.cuda.is_available()
    except ImportError:
        return True


def test_header_compiles_and_reports_missing_gpu(driver, tb, tmp_path):
    if not _no_gpu():
        pytest.skip("a GPU is present")
    x, y, z, q = tb.datasets.make("uniform_cube", 100, 1)
    p, _, _ = _run(driver, tmp_path, "fmm", x, y, z, q)
    assert p.returncode == 3
    assert "tapas_b200 error -2" in p.stderr


def _unsort(idx, r):
    out = np.empty_like(r)
    out[idx] = r
    return out


@pytest.mark.gpu
def test_fmm_through_cxx_api(driver, tb, ctx, oracle_mod, tmp_path):
    x, y, z, q = tb.datasets.make("plummer", 20000, 11)
    p, idx, r = _run(driver, tmp_path, "fmm", x, y, z, q, P=8, ncrit=32, theta=0.4)
    assert p.returncode == 0, p.stderr
    # bodies come back in the tree's order, each carrying its original index
    assert np.array_equal(np.sort(idx), np.arange(len(x)))
    res = _unsort(idx, r)
    capi = ctx.evaluate(x, y, z, q, P=8, ncrit=32, theta=0.4, precision=tb.FP64)
    np.testing.assert_array_equal(res, capi)
    assert np.array_equal(idx, ctx.sorted_bodies()[0])
    ref = oracle_mod.Oracle(x, y, z, q, P=8, ncrit=32, theta=0.4).result()
    for cols in (slice(0, 1), slice(1, 4)):
        assert np.max(np.abs(res[:, cols] - ref[:, cols])) <= 1e-11 * np.max(np.abs(ref[:, cols]))
    p, idx2, rm = _run(driver, tmp_path, "fmm", x, y, z, q, P=8, ncrit=32, theta=0.4, mixed=1)
    assert p.returncode == 0, p.stderr
    ep, ea = oracle_mod.rel_l2(_unsort(idx2, rm), ref)
    assert ep < 2e-6 and ea < 2e-6


@pytest.mark.gpu
def test_barnes_hut_through_cxx_api(driver, tb, oracle_mod, tmp_path):
    x, y, z, m = tb.datasets.make("plummer", 20000, 12)
    p, idx, r = _run(driver, tmp_path, "bh", x, y, z, m, ncrit=1, theta=0.5)
    assert p.returncode == 0, p.stderr
    ref, _ = oracle_mod.barnes_hut(x, y, z, m, ncrit=1, theta=0.5, eps2=1e-6)
    np.testing.assert_array_equal(_unsort(idx, r), ref)


# ---- user functors on the GPU (include/tapas_b200/device.cuh) ---------------
DEVICE_SRC = ROOT / "tests" / "cxx" / "device_api_test.cu"


@pytest.fixture(scope="module")
def device_driver(tb, tmp_path_factory):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not pathlib.Path(nvcc).exists():
        pytest.skip("no nvcc")
    from importlib import import_module
    lib = pathlib.Path(import_module("tapas_reduce_b200.build").build())
    exe = tmp_path_factory.mktemp("cu") / "device_api_test"
    cmd = [nvcc, "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-O2",
           "-Xcompiler", "-Wall", "-I", str(ROOT / "include"), str(DEVICE_SRC), "-L",
           str(lib.parent), "-ltapas_b200", "-Xlinker", "-rpath", "-Xlinker", str(lib.parent),
           "-o", str(exe)]
    p = subprocess.run(cmd, capture_output=True, text=True)
    assert p.returncode == 0, p.stderr[-3000:]
    return exe


def test_device_functor_program_builds(device_driver):
    """The device templates compile for sm_100a with a user's functors; without
    a GPU the program reports the library's error and exits 3."""
    if not _no_gpu():
        pytest.skip("a GPU is present (the GPU test runs the program)")
    p = subprocess.run([str(device_driver), "1000", "6", "32", "0.4"], capture_output=True,
                       text=True, timeout=120)
    assert p.returncode == 3, (p.returncode, p.stderr)


@pytest.mark.gpu
def test_user_functors_on_gpu(device_driver):
    """A user P2P functor written like the reference's CUDA one, run through
    FMM_DTT_With, gives the library P2P's results (1e-12: sqrt vs rsqrt);
    MapReduce sums match host sums per cell; Reduce counts the cells per level."""
    import json
    p = subprocess.run([str(device_driver), "30000", "8", "32", "0.4"], capture_output=True,
                       text=True, timeout=600)
    assert p.returncode == 0, (p.returncode, p.stdout, p.stderr)
    d = json.loads(p.stdout.strip().splitlines()[-1])
    assert d["max_rel_user_p2p"] < 1e-12 and d["max_rel_mapreduce"] < 1e-13
    assert d["reduce_levels_ok"] and d["levels"] >= 4
