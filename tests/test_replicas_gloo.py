"""Multi-process (world size 2, gloo on CPU) checks of bench.py's replica
plumbing.  The evaluation path does not shard: each GPU builds and evaluates
its own tree, and ranks exchange only scalars (the slowest step time and the
body count).  These tests run that exchange and the reference arm's
rank-0-only rule as real processes."""
import importlib.util
import json
import os
import pathlib
import socket
import subprocess
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _load_bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _rank_main(rank, world, port, out_dir):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    bench = _load_bench()
    w, r, local, pg = bench.dist_setup(None)
    assert (w, r, local) == (world, rank, rank)
    bench.barrier(pg)
    # rank r: step time 10*(r+1) ms over n = 1000*(r+1) bodies
    ms_max, n_total, value = bench.replica_throughput(pg, 10.0 * (rank + 1), 1000 * (rank + 1))
    bench.barrier(pg)
    pg.destroy_process_group()
    (pathlib.Path(out_dir) / f"rank{rank}.json").write_text(
        json.dumps({"ms_max": ms_max, "n_total": n_total, "value": value}))


def test_replica_throughput_two_ranks(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    for r in range(2):
        d = json.loads((tmp_path / f"rank{r}.json").read_text())
        assert d["ms_max"] == 20.0
        assert d["n_total"] == 3000.0
        assert d["value"] == pytest.approx(3000.0 / 0.020)


def test_single_process_needs_no_group():
    bench = _load_bench()
    assert bench.replica_throughput(None, 5.0, 100) == (5.0, 100.0, 100.0 / 0.005)


def test_reference_arm_prints_once_under_torchrun(oracle_mod):
    """``bench.py --impl reference`` launched as two ranks: rank 0 times the
    reference CPU implementation and prints one JSON line; rank 1 exits 0."""
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), str(ROOT / "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0",
           "--ref-sample", "3000"]
    env = dict(os.environ, OMP_NUM_THREADS="1")
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=str(ROOT), env=env)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, p.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2
    assert d["value"] > 0 and d["cpu_baseline"]["value"] == d["value"]
    assert d["cpu_baseline"]["kind"] in ("reference", "port")
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["gpu_launches"] == 0
