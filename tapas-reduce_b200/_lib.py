"""ctypes binding of libtapas_b200.so (C ABI in include/tapas_b200.h).

Loading fails loudly when the library is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import pathlib

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
LIB_PATH = HERE / "libtapas_b200.so"

OK = 0
ERR_ARG, ERR_CUDA, ERR_NOMEM, ERR_STATE, ERR_CAPACITY, ERR_UNSUPPORTED, ERR_TIMEOUT = (
    -1, -2, -3, -4, -5, -6, -7)
HOST, DEVICE = 0, 1
FP64, MIXED = 0, 1
ORDER_SORTED, ORDER_ORIGINAL = 0, 1

# Every symbol include/tapas_b200.h declares (checked by tests/test_abi.py).
EXPORTS = (
    "tapas_b200_ctx_create", "tapas_b200_ctx_destroy", "tapas_b200_set_stream",
    "tapas_b200_set_profiling", "tapas_b200_set_reference_lists", "tapas_b200_get_timings",
    "tapas_b200_set_wait_limit",
    "tapas_b200_last_error",
    "tapas_b200_kernel_launches", "tapas_b200_partition", "tapas_b200_tree_info",
    "tapas_b200_get_cells", "tapas_b200_get_sorted", "tapas_b200_upward",
    "tapas_b200_traverse", "tapas_b200_build_lists", "tapas_b200_list_info",
    "tapas_b200_get_lists", "tapas_b200_m2l", "tapas_b200_p2p", "tapas_b200_downward",
    "tapas_b200_get_expansions", "tapas_b200_get_results", "tapas_b200_evaluate",
    "tapas_b200_direct", "tapas_b200_direct_noalloc", "tapas_b200_leaf_depth_histogram",
    "tapas_b200_mlp_create", "tapas_b200_mlp_num_params", "tapas_b200_mlp_set_params",
    "tapas_b200_mlp_get_params", "tapas_b200_mlp_forward", "tapas_b200_mlp_gradients",
    "tapas_b200_mlp_train", "tapas_b200_bh_upward", "tapas_b200_bh_interact",
    "tapas_b200_bh_counts", "tapas_b200_bh_evaluate",
    "tapas_b200_write_sources", "tapas_b200_write_targets", "tapas_b200_read_sources",
    "tapas_b200_read_targets", "tapas_b200_write_main_csv", "tapas_b200_write_report",
    "tapas_b200_set_owned_cells", "tapas_b200_p2m", "tapas_b200_m2m",
    "tapas_b200_get_multipoles", "tapas_b200_set_multipoles",
)


class TreeStats(ctypes.Structure):
    _fields_ = [("n_bodies", ctypes.c_int64), ("n_cells", ctypes.c_int64),
                ("n_leaves", ctypes.c_int64), ("max_depth", ctypes.c_int32),
                ("ncrit", ctypes.c_int32), ("box_lo", ctypes.c_double),
                ("box_hi", ctypes.c_double)]


class ListStats(ctypes.Structure):
    _fields_ = [("n_m2l", ctypes.c_int64), ("n_p2p", ctypes.c_int64),
                ("n_p2p_interactions", ctypes.c_uint64),
                ("traverse_iterations", ctypes.c_int32), ("n_m2l_tc", ctypes.c_int64),
                ("tc_classes", ctypes.c_int64), ("tc_tiles", ctypes.c_int64),
                ("pairs_visited", ctypes.c_int64)]


_TIMING_FIELDS = ("upload", "bbox_keys", "sort", "tree", "upward", "p2m", "m2m", "traverse",
                  "list_sort", "m2l", "p2p", "downward", "l2l", "l2p", "download", "m2l_fp64",
                  "m2l_tc", "m2l_setup")


class Timings(ctypes.Structure):
    _fields_ = [(f, ctypes.c_double) for f in _TIMING_FIELDS]


class TapasError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[{code}] {msg}")
        self.code = code


_lib = None
_vp = ctypes.c_void_p
_i64 = ctypes.c_int64
_int = ctypes.c_int
_dbl = ctypes.c_double


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is not built; run __graft_entry__.build() "
                          "or python tapas-reduce_b200/build.py")
    L = ctypes.CDLL(str(LIB_PATH))
    sig = {
        "tapas_b200_ctx_create": [_int, ctypes.POINTER(_vp)],
        "tapas_b200_ctx_destroy": [_vp],
        "tapas_b200_set_stream": [_vp, _vp],
        "tapas_b200_set_profiling": [_vp, _int],
        "tapas_b200_set_reference_lists": [_vp, _int],
        "tapas_b200_set_wait_limit": [_vp, _i64],
        "tapas_b200_get_timings": [_vp, ctypes.POINTER(Timings)],
        "tapas_b200_partition": [_vp, _vp, _vp, _vp, _vp, _i64, _int, _int],
        "tapas_b200_tree_info": [_vp, ctypes.POINTER(TreeStats)],
        "tapas_b200_get_cells": [_vp] + [_vp] * 8,
        "tapas_b200_get_sorted": [_vp, _vp, _vp],
        "tapas_b200_upward": [_vp, _int, _int],
        "tapas_b200_traverse": [_vp, _dbl, _int, _int],
        "tapas_b200_build_lists": [_vp, _dbl, _int],
        "tapas_b200_list_info": [_vp, ctypes.POINTER(ListStats)],
        "tapas_b200_get_lists": [_vp, _vp, _vp, _vp, _vp],
        "tapas_b200_m2l": [_vp, _int],
        "tapas_b200_p2p": [_vp, _int],
        "tapas_b200_downward": [_vp, _int],
        "tapas_b200_get_expansions": [_vp, _vp, _vp],
        "tapas_b200_get_results": [_vp, _vp, _int, _int],
        "tapas_b200_evaluate": [_vp, _vp, _vp, _vp, _vp, _i64, _int, _int, _dbl, _int, _vp,
                                _int, _int],
        "tapas_b200_direct": [_vp, _vp, _i64, _vp, _int],
    }
    for name, args in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = _int
    sig2 = {
        "tapas_b200_leaf_depth_histogram": [_vp, _int, _vp],
        "tapas_b200_mlp_create": [_vp, _int, _int, _int, _int, ctypes.c_uint64],
        "tapas_b200_mlp_set_params": [_vp, _vp],
        "tapas_b200_mlp_get_params": [_vp, _vp],
        "tapas_b200_mlp_forward": [_vp, _vp, _i64, _vp],
        "tapas_b200_mlp_gradients": [_vp, _vp, _vp, _i64, _vp, _vp],
        "tapas_b200_mlp_train": [_vp, _vp, _vp, _i64, _int, _int, ctypes.c_float,
                                 ctypes.c_uint64, _vp],
        "tapas_b200_direct_noalloc": [_vp] * 4 + [_i64, _vp, _i64, _vp, _vp],
        "tapas_b200_bh_upward": [_vp],
        "tapas_b200_bh_interact": [_vp, _dbl, _dbl, _int],
        "tapas_b200_bh_counts": [_vp, _vp, _vp],
        "tapas_b200_bh_evaluate": [_vp, _vp, _vp, _vp, _vp, _i64, _int, _dbl, _dbl, _int, _vp,
                                   _int, _int],
    }
    _cp = ctypes.c_char_p
    sig2.update({
        "tapas_b200_write_sources": [_cp, _int, _i64, _vp, _vp, _vp, _vp, _int],
        "tapas_b200_write_targets": [_cp, _int, _i64, _vp, _int],
        "tapas_b200_read_sources": [_cp, _int, _i64, _vp, _vp, _vp, _vp, _vp],
        "tapas_b200_read_targets": [_cp, _int, _i64, _vp, _vp],
        "tapas_b200_write_main_csv": [_cp, _int, _dbl, _dbl, _dbl, _dbl, _dbl,
                                      ctypes.c_uint64, ctypes.c_uint64],
        "tapas_b200_write_report": [_vp, _cp, _cp],
        "tapas_b200_set_owned_cells": [_vp, _vp, _int],
        "tapas_b200_p2m": [_vp, _int, _int],
        "tapas_b200_m2m": [_vp],
        "tapas_b200_get_multipoles": [_vp, _vp, _int],
        "tapas_b200_set_multipoles": [_vp, _vp, _int],
    })
    for name, args in sig2.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = _int
    L.tapas_b200_mlp_num_params.argtypes = [_vp]
    L.tapas_b200_mlp_num_params.restype = _i64
    L.tapas_b200_last_error.argtypes = [_vp]
    L.tapas_b200_last_error.restype = ctypes.c_char_p
    L.tapas_b200_kernel_launches.argtypes = [_vp, _int]
    L.tapas_b200_kernel_launches.restype = _i64
    _lib = L
    return L


def _ptr(a):
    """Host numpy array or torch tensor -> (void*, mem kind)."""
    if isinstance(a, np.ndarray):
        return a.ctypes.data_as(_vp), HOST
    # torch tensors (plumbing only): device pointers pass through as DEVICE.
    if hasattr(a, "data_ptr"):
        return _vp(a.data_ptr()), (DEVICE if a.is_cuda else HOST)
    raise TypeError(f"unsupported array type {type(a)}")


def _check_free(rc):
    """Status of a call that takes no context (message from the thread's last error)."""
    if rc != OK:
        msg = lib().tapas_b200_last_error(None)
        raise TapasError(rc, msg.decode() if msg else "")


def _cstr(s):
    return None if s is None else str(s).encode()


# ---- the reference's file formats (host code, no GPU) ------------------------
def write_sources(directory, rank, x, y, z, q, digits=0):
    """<directory>/source%04d.dat as the reference's Dataset::writeSources
    writes it (digits <= 0: its 6-significant-digit default)."""
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z, q)]
    _check_free(lib().tapas_b200_write_sources(_cstr(directory), rank, len(arrs[0]),
                                               *[a.ctypes.data_as(_vp) for a in arrs], digits))


def write_targets(directory, rank, trg4, digits=0):
    t = np.ascontiguousarray(trg4, dtype=np.float64).reshape(-1, 4)
    _check_free(lib().tapas_b200_write_targets(_cstr(directory), rank, len(t),
                                               t.ctypes.data_as(_vp), digits))


def read_sources(directory, rank, n, position=0):
    """n bodies from <directory>/source%04d.dat starting at byte `position`:
    (x, y, z, q, next position)."""
    arrs = [np.zeros(n) for _ in range(4)]
    pos = ctypes.c_int64(position)
    _check_free(lib().tapas_b200_read_sources(_cstr(directory), rank, n,
                                              *[a.ctypes.data_as(_vp) for a in arrs],
                                              ctypes.byref(pos)))
    return (*arrs, int(pos.value))


def read_targets(directory, rank, n, position=0):
    """n bodies' (pot, ax, ay, az) from <directory>/target%04d.dat: (trg[n, 4], next position)."""
    t = np.zeros((n, 4))
    pos = ctypes.c_int64(position)
    _check_free(lib().tapas_b200_read_targets(_cstr(directory), rank, n, t.ctypes.data_as(_vp),
                                              ctypes.byref(pos)))
    return t, int(pos.value)


def write_main_csv(path, total, upward, traverse, downward, tree, num_p2p, num_m2l, rank=0):
    """The example's main.csv row (ex/tapas_exafmm.cxx:651-677) in the reference's layout."""
    _check_free(lib().tapas_b200_write_main_csv(_cstr(path), rank, total, upward, traverse,
                                                downward, tree, num_p2p, num_m2l))


class Context:
    """One GPU context of the library (C ABI: tapas_b200_ctx)."""

    def __init__(self, device: int = 0):
        self._L = lib()
        h = _vp()
        self._check(self._L.tapas_b200_ctx_create(device, ctypes.byref(h)), None)
        self.h = h
        self.n = 0
        self.P = None

    def close(self):
        if getattr(self, "h", None):
            self._L.tapas_b200_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc, h="self"):
        if rc != OK:
            hh = self.h if h == "self" else h
            msg = self._L.tapas_b200_last_error(hh)
            raise TapasError(rc, msg.decode() if msg else "")
        return rc

    def last_error(self) -> str:
        return self._L.tapas_b200_last_error(self.h).decode()

    # ---- configuration -------------------------------------------------
    def set_stream(self, stream_handle: int | None):
        self._check(self._L.tapas_b200_set_stream(self.h, _vp(stream_handle or 0)))

    def set_profiling(self, on: bool):
        self._check(self._L.tapas_b200_set_profiling(self.h, int(on)))

    def set_reference_lists(self, on: bool):
        """Keep the traversal's pairs with empty cells, as the reference does."""
        self._check(self._L.tapas_b200_set_reference_lists(self.h, int(on)))

    def set_wait_limit(self, cycles: int = 0):
        """Bound (GPU clock cycles) on each wait inside the tensor-core M2L
        kernel; 0 restores the default (about 2 s)."""
        self._check(self._L.tapas_b200_set_wait_limit(self.h, int(cycles)))

    def timings(self) -> dict:
        t = Timings()
        self._check(self._L.tapas_b200_get_timings(self.h, ctypes.byref(t)))
        return {f: getattr(t, f) for f in _TIMING_FIELDS}

    def write_report(self, prefix=None, suffix=None):
        """The reference's report files of the last evaluation (main.csv and
        hot/report.h's set); None: TAPAS_REPORT_PREFIX / _SUFFIX."""
        self._check(self._L.tapas_b200_write_report(self.h, _cstr(prefix), _cstr(suffix)))

    def kernel_launches(self, reset=False) -> int:
        return int(self._L.tapas_b200_kernel_launches(self.h, int(reset)))

    # ---- tree ------------------------------------------------------------
    def partition(self, x, y, z, q, ncrit: int = 64):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) if isinstance(a, np.ndarray) else a
                for a in (x, y, z, q)]
        ptrs = [_ptr(a) for a in arrs]
        mem = ptrs[0][1]
        n = len(arrs[0]) if isinstance(arrs[0], np.ndarray) else arrs[0].numel()
        self._keep = arrs
        self._check(self._L.tapas_b200_partition(self.h, *[p for p, _ in ptrs], n, ncrit, mem))
        self.n = n
        return self.tree_info()

    def tree_info(self) -> dict:
        t = TreeStats()
        self._check(self._L.tapas_b200_tree_info(self.h, ctypes.byref(t)))
        return {f: getattr(t, f) for f, _ in TreeStats._fields_}

    def cells(self) -> dict:
        C = self.tree_info()["n_cells"]
        d = dict(key=np.zeros(C, np.uint64), leaf=np.zeros(C, np.int32), nb=np.zeros(C, np.int32),
                 bbeg=np.zeros(C, np.int32), parent=np.zeros(C, np.int32),
                 child0=np.zeros(C, np.int32), center=np.zeros((C, 3)), width=np.zeros((C, 3)))
        self._check(self._L.tapas_b200_get_cells(
            self.h, *[d[k].ctypes.data_as(_vp) for k in
                      ("key", "leaf", "nb", "bbeg", "parent", "child0", "center", "width")]))
        return d

    def sorted_bodies(self):
        o = np.zeros(self.n, np.int64)
        k = np.zeros(self.n, np.uint64)
        self._check(self._L.tapas_b200_get_sorted(self.h, o.ctypes.data_as(_vp),
                                                  k.ctypes.data_as(_vp)))
        return o, k

    # ---- evaluation ------------------------------------------------------
    def upward(self, P: int = 10, precision: int = FP64):
        self.P = P
        self._check(self._L.tapas_b200_upward(self.h, P, precision))

    # ---- sharded evaluation (tapas-reduce_b200/sharded.py) ---------------
    def set_owned_cells(self, mask):
        """Per-cell ownership bytes (bit 0: local expansion, bit 1: bodies) of
        the current tree; None clears."""
        if mask is None:
            self._check(self._L.tapas_b200_set_owned_cells(self.h, None, HOST))
            return
        if isinstance(mask, np.ndarray):
            mask = np.ascontiguousarray(mask, dtype=np.uint8)
        p, mem = _ptr(mask)
        self._keep_mask = mask
        self._check(self._L.tapas_b200_set_owned_cells(self.h, p, mem))

    def p2m(self, P: int = 10, precision: int = FP64):
        self.P = P
        self._check(self._L.tapas_b200_p2m(self.h, P, precision))

    def m2m(self):
        self._check(self._L.tapas_b200_m2m(self.h))

    def multipoles(self, out=None):
        """M as (ncells, NT) complex (host) or into `out`, a float64 buffer of
        2 * ncells * NT values (host array or device tensor)."""
        C = self.tree_info()["n_cells"]
        nt = self.P * (self.P + 1) // 2
        ret = out is None
        if out is None:
            out = np.zeros((C, nt, 2))
        p, mem = _ptr(out)
        self._check(self._L.tapas_b200_get_multipoles(self.h, p, mem))
        return out[..., 0] + 1j * out[..., 1] if ret else out

    def set_multipoles(self, M):
        """M: a float64 buffer of 2 * ncells * NT values (host array or device tensor)."""
        if isinstance(M, np.ndarray):
            M = np.ascontiguousarray(M, dtype=np.float64)
        p, mem = _ptr(M)
        self._check(self._L.tapas_b200_set_multipoles(self.h, p, mem))

    def build_lists(self, theta: float = 0.4, mutual: int = 0):
        self._check(self._L.tapas_b200_build_lists(self.h, float(theta), mutual))
        return self.list_info()

    def list_info(self) -> dict:
        t = ListStats()
        self._check(self._L.tapas_b200_list_info(self.h, ctypes.byref(t)))
        return {f: getattr(t, f) for f, _ in ListStats._fields_}

    def lists(self):
        li = self.list_info()
        mt = np.zeros(li["n_m2l"], np.int32)
        ms = np.zeros(li["n_m2l"], np.int32)
        pt = np.zeros(li["n_p2p"], np.int32)
        ps = np.zeros(li["n_p2p"], np.int32)
        self._check(self._L.tapas_b200_get_lists(self.h, *[a.ctypes.data_as(_vp)
                                                          for a in (mt, ms, pt, ps)]))
        return (mt, ms), (pt, ps)

    def m2l(self, precision: int = FP64):
        self._check(self._L.tapas_b200_m2l(self.h, precision))

    def p2p(self, precision: int = FP64):
        self._check(self._L.tapas_b200_p2p(self.h, precision))

    def traverse(self, theta: float = 0.4, mutual: int = 0, precision: int = FP64):
        self._check(self._L.tapas_b200_traverse(self.h, float(theta), mutual, precision))

    def downward(self, precision: int = FP64):
        self._check(self._L.tapas_b200_downward(self.h, precision))

    def expansions(self):
        C = self.tree_info()["n_cells"]
        nt = self.P * (self.P + 1) // 2
        M = np.zeros((C, nt, 2))
        L = np.zeros((C, nt, 2))
        self._check(self._L.tapas_b200_get_expansions(self.h, M.ctypes.data_as(_vp),
                                                      L.ctypes.data_as(_vp)))
        return M[..., 0] + 1j * M[..., 1], L[..., 0] + 1j * L[..., 1]

    def results(self, order: int = ORDER_ORIGINAL, out=None):
        if out is None:
            out = np.zeros((self.n, 4))
        p, mem = _ptr(out)
        self._check(self._L.tapas_b200_get_results(self.h, p, order, mem))
        return out

    def evaluate(self, x, y, z, q, P=10, ncrit=64, theta=0.4, precision=FP64,
                 order=ORDER_ORIGINAL, out=None):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) if isinstance(a, np.ndarray) else a
                for a in (x, y, z, q)]
        ptrs = [_ptr(a) for a in arrs]
        mem = ptrs[0][1]
        n = len(arrs[0]) if isinstance(arrs[0], np.ndarray) else arrs[0].numel()
        if out is None:
            out = np.zeros((n, 4))
        op, omem = _ptr(out)
        if omem != mem:
            raise ValueError("inputs and output must live in the same memory kind")
        self._keep = arrs
        self.P = P
        self._check(self._L.tapas_b200_evaluate(self.h, *[p for p, _ in ptrs], n, P, ncrit,
                                                float(theta), precision, op, order, mem))
        self.n = n
        return out

    # ---- Barnes-Hut sample path ------------------------------------------
    def bh_evaluate(self, x, y, z, m, ncrit=1, theta=0.5, eps2=1e-6, precision=FP64,
                    order=ORDER_ORIGINAL, out=None):
        """(ax, ay, az, phi) per body, the sample's calc() (bh.cc:228-245)."""
        arrs = [np.ascontiguousarray(a, dtype=np.float64) if isinstance(a, np.ndarray) else a
                for a in (x, y, z, m)]
        ptrs = [_ptr(a) for a in arrs]
        mem = ptrs[0][1]
        n = len(arrs[0]) if isinstance(arrs[0], np.ndarray) else arrs[0].numel()
        if out is None:
            out = np.zeros((n, 4))
        op, _ = _ptr(out)
        self._keep = arrs
        self._check(self._L.tapas_b200_bh_evaluate(self.h, *[p for p, _ in ptrs], n, ncrit,
                                                   float(theta), float(eps2), precision, op,
                                                   order, mem))
        self.n = n
        return out

    def bh_counts(self):
        a, d = ctypes.c_uint64(), ctypes.c_uint64()
        self._check(self._L.tapas_b200_bh_counts(self.h, ctypes.byref(a), ctypes.byref(d)))
        return int(a.value), int(d.value)

    def leaf_depth_histogram(self, nbins: int = 16) -> np.ndarray:
        h = np.zeros(nbins, np.int64)
        self._check(self._L.tapas_b200_leaf_depth_histogram(self.h, nbins,
                                                            h.ctypes.data_as(_vp)))
        return h

    # ---- learned-chooser network (own CUDA kernels) -----------------------
    def mlp_create(self, n_in, n_hidden=64, n_layers=3, n_out=2, seed=0):
        self._check(self._L.tapas_b200_mlp_create(self.h, n_in, n_hidden, n_layers, n_out,
                                                  seed))
        return int(self._L.tapas_b200_mlp_num_params(self.h))

    def mlp_params(self) -> np.ndarray:
        p = np.zeros(int(self._L.tapas_b200_mlp_num_params(self.h)), np.float32)
        self._check(self._L.tapas_b200_mlp_get_params(self.h, p.ctypes.data_as(_vp)))
        return p

    def mlp_set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        self._check(self._L.tapas_b200_mlp_set_params(self.h, p.ctypes.data_as(_vp)))

    def mlp_forward(self, X, n_out=2) -> np.ndarray:
        X = np.ascontiguousarray(X, np.float32)
        Y = np.zeros((len(X), n_out), np.float32)
        self._check(self._L.tapas_b200_mlp_forward(self.h, X.ctypes.data_as(_vp), len(X),
                                                   Y.ctypes.data_as(_vp)))
        return Y

    def mlp_gradients(self, X, Y):
        X = np.ascontiguousarray(X, np.float32)
        Y = np.ascontiguousarray(Y, np.float32)
        g = np.zeros(int(self._L.tapas_b200_mlp_num_params(self.h)), np.float32)
        loss = ctypes.c_float()
        self._check(self._L.tapas_b200_mlp_gradients(self.h, X.ctypes.data_as(_vp),
                                                     Y.ctypes.data_as(_vp), len(X),
                                                     g.ctypes.data_as(_vp), ctypes.byref(loss)))
        return g, float(loss.value)

    def mlp_train(self, X, Y, epochs=200, batch=128, lr=1e-3, seed=0) -> np.ndarray:
        X = np.ascontiguousarray(X, np.float32)
        Y = np.ascontiguousarray(Y, np.float32)
        hist = np.zeros(epochs, np.float32)
        self._check(self._L.tapas_b200_mlp_train(self.h, X.ctypes.data_as(_vp),
                                                 Y.ctypes.data_as(_vp), len(X), epochs, batch,
                                                 ctypes.c_float(lr), seed,
                                                 hist.ctypes.data_as(_vp)))
        return hist

    def direct(self, targets) -> np.ndarray:
        tg = np.ascontiguousarray(targets, dtype=np.int64)
        out = np.zeros((len(tg), 4))
        self._check(self._L.tapas_b200_direct(self.h, tg.ctypes.data_as(_vp), len(tg),
                                              out.ctypes.data_as(_vp), HOST))
        return out
