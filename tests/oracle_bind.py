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
    srcs = [ORACLE_DIR / "vdf_oracle.c", ORACLE_DIR / "vdf_oracle_csv.c", ORACLE_DIR / "vdf_oracle_pivot.c"]
    if not ORACLE_LIB.exists() or any(ORACLE_LIB.stat().st_mtime < p.stat().st_mtime for p in srcs):
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
    lib.orc_csv_read.restype = C.c_void_p
    lib.orc_csv_read.argtypes = [C.c_char_p, C.c_size_t, C.c_char, C.c_int, C.c_char, C.POINTER(C.c_size_t)]
    lib.orc_csv_free.argtypes = [C.c_void_p]
    lib.orc_parse_double.restype = C.c_double
    lib.orc_parse_double.argtypes = [C.c_char_p, C.c_size_t]
    lib.orc_parse_u32.restype = C.c_uint32
    lib.orc_parse_u32.argtypes = [C.c_char_p, C.c_size_t]
    lib.orc_parse_i32.restype = C.c_int32
    lib.orc_parse_i32.argtypes = [C.c_char_p, C.c_size_t]
    lib.orc_pivot.restype = C.c_int
    lib.orc_pivot.argtypes = [C.c_size_t, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                              C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.c_void_p, C.c_void_p, C.c_void_p,
                              C.c_size_t]
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


class CsvResult:
    """A parsed CSV table in the oracle's blob layout: nrow, names, types,
    bad_row (-1 when every record has the first line's field count) and
    columns (numpy arrays, or lists of bytes for strings)."""

    NP = {"d": np.float64, "u": np.uint32, "b": np.uint8}

    def __init__(self, blob: bytes):
        nrow, ncol, _pad, bad = np.frombuffer(blob[:24], dtype=np.dtype([("a", "<u8"), ("b", "<u4"), ("c", "<u4"),
                                                                          ("d", "<i8")]))[0]
        self.nrow, self.ncol, self.bad_row = int(nrow), int(ncol), int(bad)
        p = 24
        self.types, self.names = [], []
        for _ in range(self.ncol):
            self.types.append(chr(blob[p]))
            nl = int(np.frombuffer(blob[p + 1:p + 5], dtype="<u4")[0])
            self.names.append(blob[p + 5:p + 5 + nl].decode("latin-1"))
            p += 5 + nl
        self.columns = []
        if self.nrow == 0 or self.bad_row >= 0:
            self.columns = [np.zeros(0, self.NP.get(t, np.uint8)) if t in self.NP else [] for t in self.types]
            return
        for t in self.types:
            if t in self.NP:
                w = np.dtype(self.NP[t]).itemsize
                self.columns.append(np.frombuffer(blob[p:p + w * self.nrow], dtype=self.NP[t]).copy())
                p += w * self.nrow
            else:
                off = np.frombuffer(blob[p:p + 8 * (self.nrow + 1)], dtype="<u8")
                p += 8 * (self.nrow + 1)
                data = blob[p:p + int(off[-1])]
                p += int(off[-1])
                self.columns.append([data[int(off[i]):int(off[i + 1])] for i in range(self.nrow)])


def csv_read(data: bytes, delim=",", header=True, quote="'") -> CsvResult:
    """Oracle read_csv of `data` (the C restatement)."""
    size = C.c_size_t(0)
    blob = oracle().orc_csv_read(data, len(data), delim.encode("latin-1"), 1 if header else 0,
                                 quote.encode("latin-1"), C.byref(size))
    assert blob
    try:
        return CsvResult(C.string_at(blob, size.value))
    finally:
        oracle().orc_csv_free(blob)


def parse_double(s: bytes) -> float:
    return oracle().orc_parse_double(s, len(s))


def parse_u32(s: bytes) -> int:
    return int(oracle().orc_parse_u32(s, len(s)))


def parse_i32(s: bytes) -> int:
    return int(oracle().orc_parse_i32(s, len(s)))


def ref_csv_read(data: bytes, delim=",", header=True, quote="'", cores=1) -> CsvResult:
    """The reference's own parser (oracle/_ref shim) on `data`: the same blob layout."""
    lib = ref()
    lib.ref_csv_read.restype = C.c_void_p
    lib.ref_csv_read.argtypes = [C.c_char_p, C.c_size_t, C.c_char, C.c_int, C.c_char, C.c_int,
                                 C.POINTER(C.c_size_t), C.POINTER(C.c_double)]
    lib.ref_csv_free.argtypes = [C.c_void_p]
    size = C.c_size_t(0)
    blob = lib.ref_csv_read(data, len(data), delim.encode("latin-1"), 1 if header else 0, quote.encode("latin-1"),
                            int(cores), C.byref(size), None)
    assert blob
    try:
        return CsvResult(C.string_at(blob, size.value))
    finally:
        lib.ref_csv_free(blob)


def ref_csv_seconds(data: bytes, delim=",", header=True, quote="'", cores=1, reps=1) -> float:
    """Best-of-`reps` seconds of the reference's parse + inference + conversions."""
    lib = ref()
    lib.ref_csv_time.restype = C.c_double
    lib.ref_csv_time.argtypes = [C.c_char_p, C.c_size_t, C.c_char, C.c_int, C.c_char, C.c_int, C.c_int]
    return float(lib.ref_csv_time(data, len(data), delim.encode("latin-1"), 1 if header else 0,
                                  quote.encode("latin-1"), int(cores), int(reps)))


def string_column(strings) -> tuple:
    """(bytes uint8, offsets uint64 of len + 1) of a list of str / bytes."""
    enc = [x.encode() if isinstance(x, str) else bytes(x) for x in strings]
    offs = np.zeros(len(enc) + 1, np.uint64)
    offs[1:] = np.cumsum([len(x) for x in enc], dtype=np.uint64)
    data = np.frombuffer(b"".join(enc) or b"\0", np.uint8).copy()
    return data, offs


class OraclePivot:
    def __init__(self, colkey_row, rowkey_row, matrix):
        self.colkey_row = colkey_row  # first row of each col key, in first-appearance order
        self.rowkey_row = rowkey_row
        self.matrix = matrix          # [n_colkeys, n_rowkeys]


def pivot(col_strings, row_strings, values) -> OraclePivot:
    """Oracle pivot (V/pivots/pivot.hpp:5-128): sum of values per (col key,
    row key), col and row keys in first-appearance order."""
    n = len(values)
    cb, co = string_column(col_strings)
    rb, ro = string_column(row_strings)
    values = np.ascontiguousarray(values)
    code = {np.dtype(np.int32): 0, np.dtype(np.int64): 1, np.dtype(np.uint32): 2, np.dtype(np.uint64): 3,
            np.dtype(np.float64): 4}[values.dtype]
    ckr = np.zeros(max(1, n), np.uint32)
    rkr = np.zeros(max(1, n), np.uint32)
    nc, nr = C.c_uint32(), C.c_uint32()
    lib = oracle()
    assert lib.orc_pivot(n, _vp(cb), _vp(co), _vp(rb), _vp(ro), _vp(values), code, C.byref(nc), C.byref(nr),
                         _vp(ckr), _vp(rkr), None, 0) in (0, -1)
    m = np.zeros(max(1, nc.value * nr.value), values.dtype)
    assert lib.orc_pivot(n, _vp(cb), _vp(co), _vp(rb), _vp(ro), _vp(values), code, C.byref(nc), C.byref(nr),
                         _vp(ckr), _vp(rkr), _vp(m), m.size) == 0
    return OraclePivot(ckr[:nc.value].copy(), rkr[:nr.value].copy(),
                       m[:nc.value * nr.value].reshape(nc.value, nr.value))
