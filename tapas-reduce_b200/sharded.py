"""FMM evaluation sharded over several GPUs, one process per GPU.

The reference spreads one evaluation over MPI ranks: it samples the bodies,
cuts the Morton curve into per-rank key ranges, moves the bodies there
(cpp/include/tapas/hot/buildtree.h:162-324,461-483) and builds a locally
essential tree per rank by running the user's traversal on proxy cells
(hot/exact_let.h:675-1247).  Between GPUs of one node the bodies are cheap to
replicate, so here every rank builds the same tree and evaluates only the
targets it owns:

1. all-gather the ranks' bodies in rank order: every rank has the same input;
2. partition: the tree is a deterministic function of the input, so it is the
   same on every rank;
3. ownership (``ownership_mask``): the non-empty leaves, in Morton order, are
   cut into ``size`` contiguous ranges of about equal body count; a rank owns
   the bodies of its leaves and the local expansions of those leaves and of all
   their ancestors (a parent's local expansion is needed by each rank below it);
4. P2M of the owned leaves, one all-reduce (sum) of the multipoles, M2M
   everywhere.  Every leaf's multipole is non-zero on exactly one rank, so the
   sum is that value exactly and the tree's multipoles are the one-GPU ones;
5. traversal everywhere; M2L and P2P for owned targets only, L2L, L2P of the
   owned leaves;
6. one all-reduce (sum) of the results: rows of bodies another rank owns are
   exactly zero there.
In the FP64 form every result equals the one-GPU evaluation bit for bit.

``evaluate_sharded`` runs the steps for one rank with a communicator
(``TorchComm``: torch.distributed, NCCL for device tensors or gloo for host
arrays).  ``ShardedRank`` exposes the steps so that several ranks can also be
driven in one process (tests do that on one GPU).  The context only needs the
methods of ``Context`` used below.
"""
from __future__ import annotations

import numpy as np


def ownership_mask(cells: dict, rank: int, size: int) -> np.ndarray:
    """Per-cell ownership bytes of `rank` among `size`: bit 0 = computes the
    cell's local expansion, bit 1 = evaluates the cell's bodies."""
    nb = cells["nb"].astype(np.int64)
    leaf = (cells["leaf"] != 0) & (nb > 0)
    bbeg = cells["bbeg"].astype(np.int64)
    n = int(nb[0]) if len(nb) else 0  # the root holds every body
    mask = np.zeros(len(nb), np.uint8)
    if n == 0 or size < 1:
        return mask
    lo, hi = (rank * n) // size, ((rank + 1) * n) // size
    own_leaf = leaf & (bbeg >= lo) & (bbeg < hi)  # a leaf goes with its first body
    mask[own_leaf] = 3
    parent = cells["parent"].astype(np.int64)
    cur = np.unique(parent[own_leaf])
    cur = cur[cur >= 0]
    while len(cur):
        mask[cur] |= 1
        cur = np.unique(parent[cur])
        cur = cur[cur >= 0]
    return mask


class ShardedRank:
    """The steps of one rank's sharded evaluation on `ctx`."""

    def __init__(self, ctx, rank: int, size: int):
        self.ctx, self.rank, self.size = ctx, rank, size

    def setup(self, x, y, z, q, ncrit: int):
        """Partition the full (gathered) body set and take this rank's share."""
        self.ctx.partition(x, y, z, q, ncrit=ncrit)
        self.mask = ownership_mask(self.ctx.cells(), self.rank, self.size)
        self.ctx.set_owned_cells(self.mask)
        return self.mask

    def leaf_multipoles(self, P: int, precision: int, out=None):
        """P2M of the owned leaves; the multipoles (2 x ncells x NT floats) to
        be summed over the ranks."""
        self.ctx.p2m(P, precision)
        if out is None:
            C = self.ctx.tree_info()["n_cells"]
            out = np.zeros(2 * C * (P * (P + 1) // 2))
        return self.ctx.multipoles(out=out)

    def finish(self, M, theta: float, precision: int, mutual: int = 0, out=None):
        """M2M from the summed leaf multipoles, M2L / P2P of the owned targets,
        downward pass; results in the caller's order (zero rows for bodies
        another rank owns), to be summed over the ranks."""
        self.ctx.set_multipoles(M)
        self.ctx.m2m()
        self.ctx.traverse(theta, mutual, precision)
        self.ctx.downward(precision)
        return self.ctx.results(out=out)


class TorchComm:
    """Collectives of torch.distributed (process group already initialised):
    NCCL on device tensors, gloo on CPU tensors."""

    def __init__(self, dist, device=None):
        self.dist = dist
        self.rank = dist.get_rank()
        self.size = dist.get_world_size()
        if device is None and dist.get_backend() == "nccl":  # NCCL takes device tensors only
            import torch
            device = torch.device("cuda", torch.cuda.current_device())
        self.device = device

    def _tensor(self, a):
        import torch
        t = a if isinstance(a, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(a))
        return t.to(self.device) if self.device is not None else t

    def allgather_concat(self, a):
        """Concatenation of every rank's array, in rank order."""
        import torch
        t = self._tensor(a)
        n = torch.tensor([t.shape[0]], dtype=torch.int64, device=t.device)
        sizes = [torch.zeros_like(n) for _ in range(self.size)]
        self.dist.all_gather(sizes, n)
        mx = int(max(int(s.item()) for s in sizes))
        buf = torch.zeros((mx,) + tuple(t.shape[1:]), dtype=t.dtype, device=t.device)
        buf[: t.shape[0]] = t
        parts = [torch.zeros_like(buf) for _ in range(self.size)]
        self.dist.all_gather(parts, buf)
        out = torch.cat([p[: int(s.item())] for p, s in zip(parts, sizes)])
        return out if isinstance(a, torch.Tensor) else out.cpu().numpy()

    def allreduce_sum_(self, a):
        """In-place sum over the ranks (a numpy array or a tensor)."""
        import torch
        if isinstance(a, torch.Tensor):
            self.dist.all_reduce(a, op=self.dist.ReduceOp.SUM)
            return a
        t = self._tensor(a)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        if t.device.type != "cpu":
            a[...] = t.cpu().numpy()
        return a


def evaluate_sharded(ctx, comm, x, y, z, q, P=10, ncrit=64, theta=0.4, precision=0, mutual=0):
    """This rank's share of one sharded evaluation.  x, y, z, q: this rank's
    bodies (host arrays, or device tensors with an NCCL communicator).
    Returns (results of this rank's bodies [n_local, 4], results of all
    bodies in gathered order [n, 4])."""
    n_local = len(x)
    X, Y, Z, Q = (comm.allgather_concat(a) for a in (x, y, z, q))
    offs = comm.allgather_concat(np.array([n_local], np.int64))
    start = int(np.sum(offs[: comm.rank]))
    r = ShardedRank(ctx, comm.rank, comm.size)
    r.setup(X, Y, Z, Q, ncrit)
    dev = hasattr(X, "is_cuda") and X.is_cuda
    C = ctx.tree_info()["n_cells"]
    nt = P * (P + 1) // 2
    if dev:
        import torch
        mbuf = torch.zeros(2 * C * nt, dtype=torch.float64, device=X.device)
        rbuf = torch.zeros((len(X), 4), dtype=torch.float64, device=X.device)
    else:
        mbuf, rbuf = np.zeros(2 * C * nt), np.zeros((len(X), 4))
    r.leaf_multipoles(P, precision, out=mbuf)
    comm.allreduce_sum_(mbuf)
    r.finish(mbuf, theta, precision, mutual, out=rbuf)
    comm.allreduce_sum_(rbuf)
    return rbuf[start:start + n_local], rbuf
