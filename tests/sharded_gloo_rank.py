"""One rank of the multi-process CPU test of the sharded driver
(tests/test_sharded_gloo.py launches it with torch.distributed.run, backend
gloo).  Each rank holds its own slice of a seeded body set, runs
tapas-reduce_b200/sharded.evaluate_sharded with the oracle standing in for its
GPU, and writes its results to OUT_DIR/rank<r>.npz.

usage: sharded_gloo_rank.py OUT_DIR N P NCRIT THETA
"""
import datetime
import importlib.util
import pathlib
import sys

import numpy as np
import torch.distributed as dist

ROOT = pathlib.Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT / "oracle"))
spec = importlib.util.spec_from_file_location(
    "tapas_reduce_b200", ROOT / "tapas-reduce_b200" / "__init__.py",
    submodule_search_locations=[str(ROOT / "tapas-reduce_b200")])
tb = importlib.util.module_from_spec(spec)
sys.modules["tapas_reduce_b200"] = tb
spec.loader.exec_module(tb)

import oracle  # noqa: E402
from tapas_reduce_b200 import sharded  # noqa: E402


def main():
    out_dir, n, P, ncrit, theta = (sys.argv[1], int(sys.argv[2]), int(sys.argv[3]),
                                   int(sys.argv[4]), float(sys.argv[5]))
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
    rank, size = dist.get_rank(), dist.get_world_size()
    x, y, z, q = tb.datasets.make("plummer", n, 41)
    # uneven slices: rank r holds bodies [b_r, b_{r+1})
    cuts = np.linspace(0, n, size + 1).astype(np.int64)
    cuts[1:-1] += 17
    sl = slice(cuts[rank], cuts[rank + 1])
    comm = sharded.TorchComm(dist)
    mine, everything = sharded.evaluate_sharded(oracle.OracleContext(), comm, x[sl], y[sl], z[sl],
                                                q[sl], P=P, ncrit=ncrit, theta=theta)
    np.savez(pathlib.Path(out_dir) / f"rank{rank}.npz", mine=mine, everything=everything,
             start=cuts[rank], stop=cuts[rank + 1])
    dist.barrier()
    dist.destroy_process_group()


if __name__ == "__main__":
    main()
