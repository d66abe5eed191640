"""The sharded multi-GPU driver (tapas-reduce_b200/sharded.py) as real
processes on CPU: world sizes 2 and 3 over gloo, each rank holding its own
slice of the bodies, with the oracle standing in for each rank's GPU (the
driver's collectives, ownership split and step order are the product code;
tests/test_gpu_sharded.py runs the same steps on the GPU kernels).  Every
rank's results must equal the one-process evaluation bit for bit."""
import os
import socket
import subprocess
import sys
import pathlib

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("size", [2, 3])
def test_sharded_ranks_equal_one_process(size, tmp_path, tb, oracle_mod):
    n, P, ncrit, theta = 6000, 8, 32, 0.4
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node",
           str(size), "--master-addr", "127.0.0.1", "--master-port", str(_free_port()),
           str(ROOT / "tests" / "sharded_gloo_rank.py"), str(tmp_path), str(n), str(P),
           str(ncrit), str(theta)]
    env = dict(os.environ, OMP_NUM_THREADS="1")
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=str(ROOT), env=env)
    assert p.returncode == 0, p.stderr[-3000:]
    x, y, z, q = tb.datasets.make("plummer", n, 41)
    ref = oracle_mod.Oracle(x, y, z, q, P=P, ncrit=ncrit, theta=theta).result()
    for r in range(size):
        d = np.load(tmp_path / f"rank{r}.npz")
        np.testing.assert_array_equal(d["everything"], ref)
        np.testing.assert_array_equal(d["mine"], ref[int(d["start"]):int(d["stop"])])


def test_ownership_split(tb, oracle_mod):
    """Each non-empty leaf's bodies belong to exactly one rank, ranges are
    contiguous in Morton order, and the owner of a leaf owns the local
    expansions of the leaf and all its ancestors."""
    from tapas_reduce_b200 import sharded
    x, y, z, q = tb.datasets.make("two_gaussians", 8000, 5)
    ctx = oracle_mod.OracleContext()
    ctx.partition(x, y, z, q, ncrit=16)
    c = ctx.cells()
    leaf = (c["leaf"] != 0) & (c["nb"] > 0)
    for size in (1, 2, 5):
        masks = [sharded.ownership_mask(c, r, size) for r in range(size)]
        body_owner = np.sum([(m & 2) > 0 for m in masks], axis=0)
        assert np.all(body_owner[leaf] == 1) and np.all(body_owner[~leaf] == 0)
        for r, m in enumerate(masks):
            own = np.flatnonzero(m & 2)
            starts = np.sort(c["bbeg"][own])
            if len(starts):
                ends = np.sort(c["bbeg"][own] + c["nb"][own])
                assert np.all(starts[1:] == ends[:-1])  # contiguous bodies
            for cell in own:
                a = c["parent"][cell]
                while a >= 0:
                    assert m[a] & 1
                    a = c["parent"][a]
