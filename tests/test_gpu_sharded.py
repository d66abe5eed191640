"""The sharded evaluation (tapas-reduce_b200/sharded.py) on the GPU kernels.

Ranks are emulated in one process on one GPU: one context per rank, the
steps run rank after rank and the two sums are done here (no kernel waits on
another rank's kernel).  FP64: every result equals the one-context evaluation
bit for bit; mixed: within 2e-6 (its tensor-core M2L adds with FP32 atomics,
so even two one-context runs differ in the last bits).  A process group of
one NCCL rank runs evaluate_sharded itself on device tensors."""
import os
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _emulate(tb, x, y, z, q, size, P, ncrit, theta, precision, mutual=0):
    from tapas_reduce_b200 import sharded
    ctxs = [tb.Context(0) for _ in range(size)]
    try:
        ranks = [sharded.ShardedRank(c, r, size) for r, c in enumerate(ctxs)]
        masks = [r.setup(x, y, z, q, ncrit) for r in ranks]
        M = np.sum([r.leaf_multipoles(P, precision) for r in ranks], axis=0)
        R = np.sum([r.finish(M, theta, precision, mutual) for r in ranks], axis=0)
        return R, masks
    finally:
        for c in ctxs:
            c.close()


@pytest.mark.parametrize("size", [2, 3])
@pytest.mark.parametrize("dist,n,P,ncrit", [("plummer", 60000, 8, 32),
                                            ("sphere_surface", 300000, 12, 64)])
def test_sharded_fp64_bit_exact(size, dist, n, P, ncrit, tb, ctx):
    x, y, z, q = tb.datasets.make(dist, n, 7)
    ref = ctx.evaluate(x, y, z, q, P=P, ncrit=ncrit, theta=0.4, precision=tb.FP64)
    R, masks = _emulate(tb, x, y, z, q, size, P, ncrit, 0.4, tb.FP64)
    assert all(((m & 2) > 0).sum() > 0 for m in masks)  # every rank has bodies
    np.testing.assert_array_equal(R, ref)


def test_sharded_mutual_fp64_bit_exact(tb, ctx):
    x, y, z, q = tb.datasets.make("two_gaussians", 50000, 8)
    ctx.partition(x, y, z, q, ncrit=32)
    ctx.upward(10, tb.FP64)
    ctx.traverse(0.4, 1, tb.FP64)
    ctx.downward(tb.FP64)
    ref = ctx.results(tb.ORDER_ORIGINAL)
    R, _ = _emulate(tb, x, y, z, q, 2, 10, 32, 0.4, tb.FP64, mutual=1)
    np.testing.assert_array_equal(R, ref)


def test_sharded_mixed(tb, ctx, oracle_mod):
    x, y, z, q = tb.datasets.make("sphere_surface", 200000, 9)
    ref = ctx.evaluate(x, y, z, q, P=12, ncrit=64, theta=0.4, precision=tb.MIXED)
    R, _ = _emulate(tb, x, y, z, q, 3, 12, 64, 0.4, tb.MIXED)
    ep, ea = oracle_mod.rel_l2(R, ref)
    assert ep < 2e-6 and ea < 2e-6


def test_evaluate_sharded_nccl_device_tensors(tb, ctx):
    """evaluate_sharded with a one-rank NCCL group on device tensors (the
    all-gather and all-reduce calls of the multi-GPU run)."""
    torch = pytest.importorskip("torch")
    import torch.distributed as dist
    from tapas_reduce_b200 import sharded
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("nccl", rank=0, world_size=1)
    try:
        x, y, z, q = tb.datasets.make("plummer", 40000, 10)
        ref = ctx.evaluate(x, y, z, q, P=8, ncrit=32, theta=0.4, precision=tb.FP64)
        dev = [torch.from_numpy(a).cuda() for a in (x, y, z, q)]
        with tb.Context(0) as c2:
            mine, allr = sharded.evaluate_sharded(c2, sharded.TorchComm(dist), *dev, P=8,
                                                  ncrit=32, theta=0.4, precision=tb.FP64)
            torch.cuda.synchronize()
        np.testing.assert_array_equal(mine.cpu().numpy(), ref)
        np.testing.assert_array_equal(allr.cpu().numpy(), ref)
    finally:
        dist.destroy_process_group()
