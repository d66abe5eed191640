"""Python access to the test oracle (CPU restatement + reference build).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py as the checker.  The product never imports it.

* ``Oracle``         - ctypes wrapper of liboracle.so (fmm_oracle.c), the
                       restatement of the reference algorithm.
* ``run_reference``  - runs the unmodified reference example built into
                       oracle/_ref/ by ``make -C oracle ref`` and parses its
                       binary dump (format: oracle/ref_driver.cxx).
"""
from __future__ import annotations

import ctypes
import os
import pathlib
import subprocess
import tempfile

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"
REF_DIR = HERE / "_ref"

_c_i64 = ctypes.c_int64
_c_dp = ctypes.POINTER(ctypes.c_double)
_vp = ctypes.c_void_p

_lib = None


def build(quiet: bool = True) -> None:
    """Compile liboracle.so (and, when the reference tree is present, oracle/_ref)."""
    out = subprocess.DEVNULL if quiet else None
    subprocess.run(["make", "-C", str(HERE), "liboracle.so"], check=True, stdout=out)


def build_reference(quiet: bool = True) -> bool:
    # the reference checkout: TAPAS_REFERENCE_ROOT, else a sibling of this repository
    ref = os.environ.get("TAPAS_REFERENCE_ROOT", str(HERE.parent.parent / "reference"))
    if not pathlib.Path(ref, "cpp", "include", "tapas.h").exists():
        return False
    out = subprocess.DEVNULL if quiet else None
    subprocess.run(["make", "-C", str(HERE), "ref", f"REF={ref}"], check=True, stdout=out)
    return True


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = ctypes.CDLL(str(LIB_PATH))
        L.oracle_create.restype = _vp
        L.oracle_create.argtypes = [_c_i64, _vp, _vp, _vp, _vp, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_double]
        for f in ("oracle_build", "oracle_upward", "oracle_traverse", "oracle_downward",
                  "oracle_run_all", "oracle_max_depth"):
            getattr(L, f).argtypes = [_vp]
            getattr(L, f).restype = ctypes.c_int
        L.oracle_destroy.argtypes = [_vp]
        L.oracle_set_mutual.argtypes = [_vp, ctypes.c_int]
        L.oracle_set_mutual.restype = None
        L.oracle_set_owned.argtypes = [_vp, _vp]
        L.oracle_set_owned.restype = None
        for f in ("oracle_p2m_only", "oracle_m2m_only"):
            getattr(L, f).argtypes = [_vp]
            getattr(L, f).restype = ctypes.c_int
        L.oracle_set_multipoles.argtypes = [_vp, _vp]
        L.oracle_set_multipoles.restype = None
        L.oracle_set_theta.argtypes = [_vp, ctypes.c_double]
        L.oracle_set_theta.restype = None
        for f in ("oracle_ncells", "oracle_n_m2l", "oracle_n_p2p"):
            getattr(L, f).argtypes = [_vp]
            getattr(L, f).restype = _c_i64
        L.oracle_n_p2p_interactions.argtypes = [_vp]
        L.oracle_n_p2p_interactions.restype = ctypes.c_uint64
        L.oracle_bbox.argtypes = [_vp, _vp]
        L.oracle_get_cells.argtypes = [_vp] + [_vp] * 8
        L.oracle_get_expansions.argtypes = [_vp, _vp, _vp]
        L.oracle_get_m2l.argtypes = [_vp, _vp, _vp]
        L.oracle_get_p2p.argtypes = [_vp, _vp, _vp]
        L.oracle_get_bodies.argtypes = [_vp, _vp, _vp, _vp]
        L.oracle_bh.argtypes = [_vp, ctypes.c_double, ctypes.c_double, _vp, _vp]
        L.oracle_bh.restype = ctypes.c_int
        for f in ("oracle_direct", "oracle_direct_field"):
            getattr(L, f).argtypes = [_c_i64, _vp, _vp, _vp, _vp, _c_i64, _vp, _vp, ctypes.c_int]
        L.oracle_key_child.restype = ctypes.c_uint64
        L.oracle_key_child.argtypes = [ctypes.c_uint64, ctypes.c_int]
        L.oracle_key_parent.restype = ctypes.c_uint64
        L.oracle_key_parent.argtypes = [ctypes.c_uint64]
        L.oracle_key_next.restype = ctypes.c_uint64
        L.oracle_key_next.argtypes = [ctypes.c_uint64, ctypes.c_int]
        L.oracle_key_is_descendant.argtypes = [ctypes.c_uint64, ctypes.c_uint64]
        L.oracle_key_includes_range.argtypes = [ctypes.c_uint64] * 3
        L.oracle_key_overlapped.argtypes = [ctypes.c_uint64] * 4
        L.oracle_key_dir_on_depth.argtypes = [ctypes.c_uint64, ctypes.c_int, ctypes.c_int]
        L.oracle_key_msbits.restype = ctypes.c_uint64
        L.oracle_key_msbits.argtypes = [ctypes.c_uint64, ctypes.c_int]
        L.oracle_key_finest.restype = ctypes.c_uint64
        L.oracle_key_finest.argtypes = [ctypes.c_int] * 3
        L.oracle_key_region.argtypes = [ctypes.c_uint64, _vp, _vp, _vp, _vp]
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(_vp)


class Oracle:
    """One FMM evaluation by the CPU restatement (fmm_oracle.c)."""

    def __init__(self, x, y, z, q, P=10, ncrit=64, theta=0.4, run=True, mutual=0):
        L = lib()
        self._keep = [np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z, q)]
        self.n = len(self._keep[0])
        self.P, self.ncrit, self.theta, self.mutual = P, ncrit, theta, int(mutual)
        self.h = L.oracle_create(self.n, *[_p(a) for a in self._keep], P, ncrit, float(theta))
        if not self.h:
            raise ValueError("oracle_create rejected its arguments")
        L.oracle_set_mutual(self.h, int(mutual))
        if run:
            rc = L.oracle_run_all(self.h)
            if rc != 0:
                raise RuntimeError(f"oracle_run_all failed: {rc}")

    def __del__(self):
        if getattr(self, "h", None):
            lib().oracle_destroy(self.h)
            self.h = None

    @property
    def nterm(self):
        return self.P * (self.P + 1) // 2

    def bbox(self):
        out = np.zeros(2)
        lib().oracle_bbox(self.h, _p(out))
        return out

    def cells(self):
        L = lib()
        c = L.oracle_ncells(self.h)
        d = dict(key=np.zeros(c, np.uint64), leaf=np.zeros(c, np.int32), nb=np.zeros(c, np.int32),
                 bid=np.zeros(c, np.int64), parent=np.zeros(c, np.int32),
                 child0=np.zeros(c, np.int32), center=np.zeros((c, 3)), width=np.zeros((c, 3)))
        L.oracle_get_cells(self.h, *[_p(d[k]) for k in ("key", "leaf", "nb", "bid", "parent",
                                                           "child0", "center", "width")])
        return d

    def expansions(self):
        c = lib().oracle_ncells(self.h)
        M = np.zeros((c, self.nterm, 2))
        Lx = np.zeros((c, self.nterm, 2))
        lib().oracle_get_expansions(self.h, _p(M), _p(Lx))
        return M[..., 0] + 1j * M[..., 1], Lx[..., 0] + 1j * Lx[..., 1]

    def m2l_list(self):
        k = lib().oracle_n_m2l(self.h)
        t = np.zeros(k, np.int32)
        s = np.zeros(k, np.int32)
        lib().oracle_get_m2l(self.h, _p(t), _p(s))
        return t, s

    def p2p_list(self):
        k = lib().oracle_n_p2p(self.h)
        t = np.zeros(k, np.int32)
        s = np.zeros(k, np.int32)
        lib().oracle_get_p2p(self.h, _p(t), _p(s))
        return t, s

    def p2p_interactions(self) -> int:
        return int(lib().oracle_n_p2p_interactions(self.h))

    def bodies(self):
        """(orig_index, key, trg[n,4]) in sorted order."""
        o = np.zeros(self.n, np.int64)
        k = np.zeros(self.n, np.uint64)
        t = np.zeros((self.n, 4))
        lib().oracle_get_bodies(self.h, _p(o), _p(k), _p(t))
        return o, k, t

    def result(self):
        """Target values (pot, ax, ay, az) per body in ORIGINAL order."""
        o, _, t = self.bodies()
        out = np.empty_like(t)
        out[o] = t
        return out


class OracleContext:
    """The methods of the library's Context that the sharded driver
    (tapas-reduce_b200/sharded.py) calls, carried out by the oracle: the CPU
    stand-in for one GPU in the multi-process (gloo) test of that driver.
    FP64 form, mutual = 0."""

    def __init__(self):
        self.o = None
        self._mask = None

    def partition(self, x, y, z, q, ncrit=64):
        self._bodies = [np.ascontiguousarray(np.asarray(a), dtype=np.float64) for a in (x, y, z, q)]
        self.ncrit = ncrit
        self._new(P=2)

    def _new(self, P):
        self.o = Oracle(*self._bodies, P=P, ncrit=self.ncrit, theta=0.4, run=False)
        if lib().oracle_build(self.o.h):
            raise RuntimeError("oracle_build failed")
        if self._mask is not None:
            lib().oracle_set_owned(self.o.h, _p(self._mask))

    def tree_info(self):
        return {"n_cells": int(lib().oracle_ncells(self.o.h))}

    def cells(self):
        d = self.o.cells()
        d["bbeg"] = d["bid"]
        return d

    def set_owned_cells(self, mask):
        self._mask = None if mask is None else np.ascontiguousarray(mask, dtype=np.uint8)
        lib().oracle_set_owned(self.o.h, None if mask is None else _p(self._mask))

    def p2m(self, P=10, precision=0):
        self._new(P)
        lib().oracle_p2m_only(self.o.h)

    def multipoles(self, out=None):
        M, _ = self.o.expansions()
        flat = np.stack([M.real, M.imag], axis=-1).reshape(-1)
        if out is None:
            return M
        out.reshape(-1)[:] = flat
        return out

    def set_multipoles(self, M):
        lib().oracle_set_multipoles(self.o.h, _p(np.ascontiguousarray(M, dtype=np.float64)))

    def m2m(self):
        lib().oracle_m2m_only(self.o.h)

    def traverse(self, theta=0.4, mutual=0, precision=0):
        if mutual:
            raise ValueError("the oracle's sharded restatement covers mutual = 0")
        lib().oracle_set_theta(self.o.h, float(theta))
        lib().oracle_traverse(self.o.h)

    def downward(self, precision=0):
        lib().oracle_downward(self.o.h)

    def results(self, order=1, out=None):
        r = self.o.result()
        if out is None:
            return r
        out[...] = r
        return out


def barnes_hut(x, y, z, m, ncrit=1, theta=0.5, eps2=1e-6):
    """Barnes-Hut sample restated (fmm_oracle.c oracle_bh): (ax, ay, az, phi)
    per body in ORIGINAL order, and (approximations, direct interactions)."""
    o = Oracle(x, y, z, m, P=2, ncrit=ncrit, theta=0.5, run=False)
    if lib().oracle_build(o.h):
        raise RuntimeError("oracle_build failed")
    out = np.zeros((o.n, 4))
    cnt = np.zeros(2, np.uint64)
    lib().oracle_bh(o.h, float(theta), float(eps2), _p(out), _p(cnt))
    orig, _, _ = o.bodies()
    res = np.empty_like(out)
    res[orig] = out
    return res, cnt


def bh_reference_available() -> bool:
    return (REF_DIR / "bh_ref").exists()


def run_bh_reference(x, y, z, m, timeout=3600):
    """The unmodified reference BH sample (ncrit = 1, theta = 0.5, EPS2 = 1e-6):
    (ax, ay, az, phi) per body in ORIGINAL order (bodies matched by position)."""
    exe = REF_DIR / "bh_ref"
    n = len(x)
    with tempfile.TemporaryDirectory() as d:
        fi, fo = os.path.join(d, "in.bin"), os.path.join(d, "out.bin")
        with open(fi, "wb") as f:
            f.write(np.int64(n).tobytes())
            f.write(np.stack([x, y, z, m], axis=1).astype(np.float64).tobytes())
        subprocess.run([str(exe), fi, fo], check=True, timeout=timeout, cwd=d,
                       stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        raw = np.fromfile(fo, dtype=np.float64, offset=8).reshape(n, 8)
    pos = np.stack([x, y, z], axis=1)
    order = np.lexsort(pos.T[::-1])
    rorder = np.lexsort(raw[:, :3].T[::-1])
    res = np.empty((n, 4))
    res[order] = raw[rorder, 4:]
    return res


def direct(x, y, z, q, targets, nthreads=0, field=False):
    """FP64 direct sum at the given target indices -> [k, 4]."""
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z, q)]
    tg = np.ascontiguousarray(targets, dtype=np.int64)
    out = np.zeros((len(tg), 4))
    f = lib().oracle_direct_field if field else lib().oracle_direct
    f(len(arrs[0]), *[_p(a) for a in arrs], len(tg), _p(tg), _p(out), int(nthreads))
    return out


def rel_l2(approx: np.ndarray, ref: np.ndarray):
    """(pot, acc) relative L2 errors as in the reference's Verify (verify.h:18-90)."""
    dp = np.sum((approx[:, 0] - ref[:, 0]) ** 2)
    npot = np.sum(ref[:, 0] ** 2)
    da = np.sum((approx[:, 1:] - ref[:, 1:]) ** 2)
    na = np.sum(ref[:, 1:] ** 2)
    return float(np.sqrt(dp / npot)), float(np.sqrt(da / na))


# ---------------------------------------------------------------------------
# The unmodified reference, built by `make -C oracle ref`.
# ---------------------------------------------------------------------------

def reference_binary(P: int) -> pathlib.Path:
    return REF_DIR / f"tapas_exafmm_ref_p{P}"


def reference_available(P: int = 10) -> bool:
    return reference_binary(P).exists()


def write_input(path, x, y, z, q, ncrit, theta):
    n = len(x)
    with open(path, "wb") as f:
        f.write(np.int64(n).tobytes())
        f.write(np.int32(ncrit).tobytes())
        f.write(np.float64(theta).tobytes())
        f.write(np.stack([x, y, z, q], axis=1).astype(np.float64).tobytes())


def read_reference_output(path):
    raw = open(path, "rb").read()
    off = 0

    def take(dtype, count):
        nonlocal off
        a = np.frombuffer(raw, dtype=dtype, count=count, offset=off)
        off += a.nbytes
        return a

    n, ncells = take(np.int64, 2)
    nterm, P = take(np.int32, 2)
    np2p, nm2l = take(np.uint64, 2)
    times = take(np.float64, 5)
    brec = np.dtype([("ibody", "<i8"), ("x", "<f8", 3), ("q", "<f8"), ("trg", "<f8", 4)])
    bodies = take(brec, int(n))
    crec = np.dtype([("key", "<u8"), ("leaf", "<i4"), ("nb", "<i4"), ("bid", "<i8"),
                     ("center", "<f8", 3), ("width", "<f8", 3),
                     ("M", "<f8", (int(nterm), 2)), ("L", "<f8", (int(nterm), 2))])
    cells = take(crec, int(ncells))
    return dict(n=int(n), ncells=int(ncells), P=int(P), nterm=int(nterm),
                n_p2p_interactions=int(np2p), n_m2l=int(nm2l),
                times=dict(zip(("tree", "upward", "traverse", "downward", "total"), times)),
                bodies=bodies, cells=cells)


def run_reference(x, y, z, q, P=10, ncrit=64, theta=0.4, repeat=1, timeout=3600, mutual=0):
    exe = reference_binary(P)
    if not exe.exists():
        raise FileNotFoundError(f"{exe} not built (make -C oracle ref)")
    with tempfile.TemporaryDirectory() as d:
        fi = os.path.join(d, "in.bin")
        fo = os.path.join(d, "out.bin")
        write_input(fi, x, y, z, q, ncrit, theta)
        subprocess.run([str(exe), fi, fo, str(repeat), str(int(mutual))], check=True,
                       timeout=timeout, stdout=subprocess.DEVNULL)
        return read_reference_output(fo)
