"""ctypes binding of the CPU oracle (oracle/liboracle.so) and of the
reference shim (oracle/_ref/libvdf_ref.so).  Test infrastructure: used only by
tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg, never by the
product library."""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
ORACLE_DIR = ROOT / "oracle"
ORACLE_LIB = ORACLE_DIR / "liboracle.so"
REF_LIB = ORACLE_DIR / "_ref" / "libvdf_ref.so"

DT = {np.dtype(np.int32): 0, np.dtype(np.int64): 1, np.dtype(np.uint32): 2, np.dtype(np.uint64): 3,
      np.dtype(np.float64): 4, np.dtype(np.float32): 5}
ASC, DESC_STABLE, DESC_REVERSE = 0, 1, 2


def _vp(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def _load_oracle() -> C.CDLL:
    if not ORACLE_LIB.exists() or ORACLE_LIB.stat().st_mtime < (ORACLE_DIR / "vdf_oracle.c").stat().st_mtime:
        subprocess.run(["make", "-s", "-C", str(ORACLE_DIR), "all"], check=True)
    lib = C.CDLL(str(ORACLE_LIB))
    lib.orc_argsort.restype = C.c_int
    lib.orc_argsort.argtypes = [C.POINTER(C.c_void_p), C.POINTER(C.c_int), C.c_int, C.c_size_t, C.c_int, C.c_void_p]
    lib.orc_groupby.restype = C.c_int64
    lib.orc_groupby.argtypes = [C.POINTER(C.c_void_p), C.POINTER(C.c_int), C.c_int, C.POINTER(C.c_void_p),
                                C.POINTER(C.c_int), C.c_int, C.c_size_t, C.c_int, C.POINTER(C.c_void_p), C.c_void_p,
                                C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                                C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.c_void_p]
    lib.orc_radix_u32.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t]
    lib.orc_radix_u64.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t]
    lib.orc_order_key.restype = C.c_uint64
    lib.orc_order_key.argtypes = [C.c_void_p, C.c_int, C.c_size_t]
    lib.orc_unique.restype = C.c_int64
    lib.orc_unique.argtypes = [C.c_void_p, C.c_int, C.c_size_t, C.c_int, C.c_void_p]
    lib.orc_left_join.restype = C.c_int64
    lib.orc_left_join.argtypes = [C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t, C.c_int, C.c_int, C.c_void_p]
    return lib


_oracle = None


def oracle() -> C.CDLL:
    global _oracle
    if _oracle is None:
        _oracle = _load_oracle()
    return _oracle


def ref_available() -> bool:
    return REF_LIB.exists()


_ref = None


def ref() -> C.CDLL:
    global _ref
    if _ref is None:
        lib = C.CDLL(str(REF_LIB))
        lib.ref_sort_frame.restype = C.c_int
        lib.ref_sort_frame.argtypes = [C.POINTER(C.c_void_p), C.POINTER(C.c_int), C.c_int, C.c_size_t, C.c_int,
                                       C.c_int, C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_int), C.c_int,
                                       C.POINTER(C.c_void_p)]
        lib.ref_groupby.restype = C.c_int64
        lib.ref_groupby.argtypes = [C.POINTER(C.c_void_p), C.POINTER(C.c_int), C.c_int, C.POINTER(C.c_void_p),
                                    C.POINTER(C.c_int), C.c_int, C.c_size_t, C.c_int, C.c_void_p]
        lib.ref_radix_u32.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int, C.c_int]
        lib.ref_radix_u64.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int, C.c_int]
        _ref = lib
    return _ref


def _arr(ptrs):
    return (C.c_void_p * max(1, len(ptrs)))(*ptrs)


def _ints(xs):
    return (C.c_int * max(1, len(xs)))(*xs)


def argsort(keys, order=ASC) -> np.ndarray:
    """Oracle stable argsort over key columns (keys[0] most significant)."""
    keys = [np.ascontiguousarray(k) for k in keys]
    n = keys[0].size
    perm = np.zeros(n, np.uint32)
    rc = oracle().orc_argsort(_arr([_vp(k) for k in keys]), _ints([DT[k.dtype] for k in keys]), len(keys), n, order,
                              _vp(perm))
    assert rc == 0
    return perm


def ref_sort(keys, order=ASC, cores=1, payload=()) -> tuple:
    """The reference's own radix kernels (through the shim)."""
    keys = [np.ascontiguousarray(k) for k in keys]
    n = keys[0].size
    perm = np.zeros(n, np.uint32)
    pay_out = [np.empty_like(p) for p in payload]
    rc = ref().ref_sort_frame(_arr([_vp(k) for k in keys]), _ints([DT[k.dtype] for k in keys]), len(keys), n, order,
                              cores, _vp(perm), _arr([_vp(p) for p in payload]),
                              _ints([p.dtype.itemsize for p in payload]), len(payload),
                              _arr([_vp(p) for p in pay_out]))
    assert rc == 0
    return perm, pay_out


def ref_groupby(keys, vals, cores=1):
    keys = [np.ascontiguousarray(k) for k in keys]
    vals = [np.ascontiguousarray(v) for v in vals]
    chk = np.zeros(1 + len(vals), np.float64)
    g = ref().ref_groupby(_arr([_vp(k) for k in keys]), _ints([DT[k.dtype] for k in keys]), len(keys),
                          _arr([_vp(v) for v in vals]), _ints([DT[v.dtype] for v in vals]), len(vals),
                          keys[0].size, cores, _vp(chk))
    return int(g), chk


class OracleGroups:
    def __init__(self, n_groups, keys, count, sums, sum_hi, mins, maxs, means, abss, first):
        self.n_groups, self.keys, self.count = n_groups, keys, count
        self.sum, self.sum_hi, self.min, self.max, self.mean, self.abs, self.first = (
            sums, sum_hi, mins, maxs, means, abss, first)


def groupby(keys, vals, sorted_groups=True) -> OracleGroups:
    """Oracle hash group-by (count/sum/min/max/mean, exact sums)."""
    keys = [np.ascontiguousarray(k) for k in keys]
    vals = [np.ascontiguousarray(v) for v in vals]
    n = keys[0].size
    ok = [np.empty(n, k.dtype) for k in keys]
    cnt = np.empty(n, np.int64)
    is_f = [v.dtype.kind == "f" for v in vals]
    sums = [np.empty(n, np.float64 if f else np.int64) for f in is_f]
    his = [np.zeros(n, np.int64) for _ in vals]
    mins = [np.empty(n, v.dtype) for v in vals]
    maxs = [np.empty(n, v.dtype) for v in vals]
    means = [np.empty(n, np.float64) for _ in vals]
    abss = [np.empty(n, np.float64) for _ in vals]
    first = np.empty(n, np.int64)
    g = oracle().orc_groupby(_arr([_vp(k) for k in keys]), _ints([DT[k.dtype] for k in keys]), len(keys),
                             _arr([_vp(v) for v in vals]), _ints([DT[v.dtype] for v in vals]), len(vals), n,
                             1 if sorted_groups else 0, _arr([_vp(a) for a in ok]), _vp(cnt),
                             _arr([_vp(a) for a in sums]), _arr([_vp(a) for a in his]),
                             _arr([_vp(a) for a in mins]), _arr([_vp(a) for a in maxs]),
                             _arr([_vp(a) for a in means]), _arr([_vp(a) for a in abss]), _vp(first))
    assert g >= 0
    g = int(g)
    return OracleGroups(g, [a[:g] for a in ok], cnt[:g], [a[:g] for a in sums], [a[:g] for a in his],
                        [a[:g] for a in mins], [a[:g] for a in maxs], [a[:g] for a in means],
                        [a[:g] for a in abss], first[:g])


def unique(key, keep_last=False):
    """Oracle de-duplication: (keep mask uint8, number of distinct keys)."""
    key = np.ascontiguousarray(key)
    keep = np.zeros(key.size, np.uint8)
    d = oracle().orc_unique(_vp(key), DT[key.dtype], key.size, 1 if keep_last else 0, _vp(keep))
    assert d >= 0
    return keep, int(d)


def left_join(left, right, method=0):
    """Oracle left-join matching, method 0 First / 1 Last / 2 Aligned:
    (match uint32, UINT32_MAX where absent; matched rows)."""
    left = np.ascontiguousarray(left)
    right = np.ascontiguousarray(right)
    assert left.dtype == right.dtype
    match = np.empty(left.size, np.uint32)
    m = oracle().orc_left_join(_vp(left), left.size, _vp(right), right.size, DT[left.dtype],
                               int(method), _vp(match))
    assert m >= 0
    return match, int(m)
