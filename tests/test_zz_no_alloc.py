"""The allocation-free direct-sum entry point (tapas_b200_direct_noalloc).

It serves callers that must not allocate device memory where they check
accuracy (a solver loop that reserved its memory up front, or code sharing
the GPU with other streams, where cudaMalloc/cudaFree would synchronise the
device).  Checked through the C ABI against the allocating entry point
tapas_b200_direct on the same bodies and targets, on two calls in a row
(the second with a different target set, so stale scratch contents would
show), to 1e-12 relative.

This file is collected last so that a run stopping at the first failure has
run every other test; it also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(L, dev, targets, k, out, stream=None):
    fn = L.tapas_b200_direct_noalloc
    fn.argtypes = [ctypes.c_void_p] * 4 + [ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64,
                                           ctypes.c_void_p, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    x, y, z, q = dev
    return fn(x.data_ptr(), y.data_ptr(), z.data_ptr(), q.data_ptr(), x.numel(),
              targets.data_ptr(), k, out.data_ptr(), stream)


def test_direct_noalloc_matches_direct(tb):
    torch = pytest.importorskip("torch")
    L = tb.lib()
    L.tapas_b200_last_error.restype = ctypes.c_char_p
    x, y, z, q = tb.datasets.make("plummer", 200_000, 71)
    dev = [torch.from_numpy(a).cuda() for a in (x, y, z, q)]
    with tb.Context(0) as ctx:
        ctx.partition(x, y, z, q, ncrit=64)
        for call, seed in enumerate((5, 6)):
            tg = tb.datasets.sample_targets(len(x), 1000 + 500 * call, seed=seed)
            ref = ctx.direct(tg)  # allocating entry point
            tg_d = torch.from_numpy(tg).cuda()
            out = torch.full((len(tg), 4), 7.0, dtype=torch.float64, device="cuda")
            torch.cuda.synchronize()
            rc = _noalloc(L, dev, tg_d, len(tg), out)
            assert rc == 0, L.tapas_b200_last_error(None)
            torch.cuda.synchronize()
            got = out.cpu().numpy()
            scale = np.max(np.abs(ref), axis=0)
            assert np.all(np.abs(got - ref) <= 1e-12 * scale), call


def test_direct_noalloc_bad_index_and_stream(tb):
    """A target index outside [0, n) gives an all-NaN row (the other rows are
    unaffected), and the work runs on the caller's stream: results read after
    synchronising only that stream match the allocating entry point."""
    torch = pytest.importorskip("torch")
    L = tb.lib()
    L.tapas_b200_last_error.restype = ctypes.c_char_p
    x, y, z, q = tb.datasets.make("uniform_cube", 50_000, 73)
    dev = [torch.from_numpy(a).cuda() for a in (x, y, z, q)]
    n = len(x)
    tg = np.array([3, -1, 17, n, 4999], dtype=np.int64)
    good = np.array([0, 2, 4])
    with tb.Context(0) as ctx:
        ctx.partition(x, y, z, q, ncrit=64)
        ref = ctx.direct(tg[good])
    stream = torch.cuda.Stream()
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        tg_d = torch.from_numpy(tg).to("cuda", non_blocking=False)
        out = torch.zeros((len(tg), 4), dtype=torch.float64, device="cuda")
    stream.synchronize()
    rc = _noalloc(L, dev, tg_d, len(tg), out, stream=stream.cuda_stream)
    assert rc == 0, L.tapas_b200_last_error(None)
    stream.synchronize()
    got = out.cpu().numpy()
    assert np.isnan(got[1]).all() and np.isnan(got[3]).all()
    scale = np.max(np.abs(ref), axis=0)
    assert np.all(np.abs(got[good] - ref) <= 1e-12 * scale)


def test_direct_noalloc_rejects_too_many_targets(tb):
    torch = pytest.importorskip("torch")
    L = tb.lib()
    L.tapas_b200_last_error.restype = ctypes.c_char_p
    x, y, z, q = tb.datasets.make("uniform_cube", 1000, 72)
    dev = [torch.from_numpy(a).cuda() for a in (x, y, z, q)]
    k = 4097
    tg = torch.zeros(k, dtype=torch.int64, device="cuda")
    out = torch.zeros((k, 4), dtype=torch.float64, device="cuda")
    rc = _noalloc(L, dev, tg, k, out)
    assert rc == -5
    assert b"4096" in L.tapas_b200_last_error(None)
