"""ctypes binding of include/vdf_capi.h (libvdf_b200.so).

Columns are contiguous CUDA torch tensors; torch only provides device memory
and streams here.  Every operation runs in the CUDA library; if the library
is missing the import fails loudly -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import weakref
from dataclasses import dataclass, field
from pathlib import Path
from typing import Optional, Sequence

import numpy as np
import torch

LIB_PATH = Path(__file__).resolve().parent / "libvdf_b200.so"
HEADER_PATH = Path(__file__).resolve().parent.parent / "include" / "vdf_capi.h"

# vdf_status
OK, ERR_INVALID_ARG, ERR_OOM, ERR_TIMEOUT, ERR_DEVICE, ERR_UNSUPPORTED, ERR_WORKSPACE = range(7)
# vdf_dtype
I32, I64, U32, U64, F64, F32 = range(6)
# vdf_order
ORDER_ASC, ORDER_DESC_STABLE, ORDER_DESC_REVERSE = range(3)

KERNEL_CLASSES = ["hist", "scan", "onesweep32", "onesweep64", "gather", "segreduce", "broadcast", "pack",
                  "segscan", "segemit", "ties", "batch", "csv", "localsort", "fallback", "dict"]
# vdf_multikey_mode
MULTIKEY_LSD, MULTIKEY_PRIMARY_FIRST = 0, 1
# vdf_sort_strategy
SORT_AUTO, SORT_LSD, SORT_MSD = 0, 1, 2

TORCH_TO_VDF = {
    torch.int32: I32, torch.int64: I64, torch.uint32: U32, torch.uint64: U64,
    torch.float64: F64, torch.float32: F32,
}
VDF_TO_TORCH = {v: k for k, v in TORCH_TO_VDF.items()}
WIDTH = {I32: 4, I64: 8, U32: 4, U64: 8, F64: 8, F32: 4}


class VdfError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"vdf status {status}: {message}")
        self.status = status


class vdf_col(C.Structure):
    _fields_ = [("data", C.c_void_p), ("dtype", C.c_int32)]


class vdf_strcol(C.Structure):
    _fields_ = [("bytes", C.c_void_p), ("offsets", C.c_void_p)]


class vdf_agg_out(C.Structure):
    _fields_ = [("sum", C.c_void_p), ("sum_hi", C.c_void_p), ("min", C.c_void_p), ("max", C.c_void_p),
                ("mean", C.c_void_p)]


class vdf_sort_tuning(C.Structure):
    _fields_ = [("pass_variant32", C.c_int32), ("pass_variant64", C.c_int32)]


class vdf_sort_groupby_args(C.Structure):
    _fields_ = [
        ("n", C.c_uint64), ("keys", C.POINTER(vdf_col)), ("nkeys", C.c_int32), ("order", C.c_int32),
        ("payload", C.POINTER(vdf_col)), ("npayload", C.c_int32),
        ("perm_out", C.c_void_p), ("sorted_keys_out", C.POINTER(C.c_void_p)), ("payload_out", C.POINTER(C.c_void_p)),
        ("groupby", C.c_int32), ("agg_cols", C.POINTER(C.c_int32)), ("nagg", C.c_int32),
        ("group_keys_out", C.POINTER(C.c_void_p)), ("group_count_out", C.c_void_p),
        ("aggs", C.POINTER(vdf_agg_out)), ("group_start_out", C.c_void_p), ("row_group_out", C.c_void_p),
        ("n_groups_dev", C.c_void_p), ("n_groups_host", C.POINTER(C.c_uint64)),
        ("perm_in", C.c_void_p),
    ]


BATCH_MAX_VALS = 4


class vdf_batch_query(C.Structure):
    _fields_ = [("n", C.c_uint64), ("key", vdf_col), ("vals", C.c_void_p * BATCH_MAX_VALS)]


class vdf_batch_tuning(C.Structure):
    _fields_ = [("small_rows", C.c_uint32), ("small_bits", C.c_int32), ("seg_variant", C.c_int32)]


class vdf_batch_args(C.Structure):
    _fields_ = [
        ("nqueries", C.c_uint32), ("queries", C.POINTER(vdf_batch_query)), ("nvals", C.c_int32),
        ("val_dtypes", C.c_int32 * BATCH_MAX_VALS), ("perm_out", C.c_void_p), ("group_keys_out", C.c_void_p),
        ("group_count_out", C.c_void_p), ("aggs", vdf_agg_out * BATCH_MAX_VALS), ("row_offset_out", C.c_void_p),
        ("group_offset_out", C.c_void_p), ("n_groups_out", C.c_void_p),
    ]


def _load() -> C.CDLL:
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is not built; run `python -m visondf_b200.build` (no CPU fallback exists)")
    lib = C.CDLL(str(LIB_PATH))
    vp, u64, i32, sz = C.c_void_p, C.c_uint64, C.c_int, C.c_size_t
    st = C.c_int
    sig = {
        "vdf_abi_version": (C.c_uint32, []),
        "vdf_status_string": (C.c_char_p, [st]),
        "vdf_max_rows": (u64, []),
        "vdf_ctx_create": (st, [i32, C.POINTER(vp)]),
        "vdf_ctx_destroy": (st, [vp]),
        "vdf_ctx_last_error": (C.c_char_p, [vp]),
        "vdf_ctx_reserve": (st, [vp, sz]),
        "vdf_ctx_check": (st, [vp, vp]),
        "vdf_ctx_kernel_launches": (u64, [vp]),
        "vdf_ctx_profile": (st, [vp, i32]),
        "vdf_ctx_profile_read": (st, [vp, i32, C.POINTER(C.c_double), C.POINTER(C.c_uint64)]),
        "vdf_ctx_profile_reset": (st, [vp]),
        "vdf_sort_workspace_bytes": (sz, [u64, C.POINTER(C.c_int32), i32]),
        "vdf_sort_variant_count": (i32, []),
        "vdf_sort_variant_info": (st, [i32] + [C.POINTER(C.c_int32)] * 5),
        "vdf_sort_variant_flags": (C.c_uint32, [i32]),
        "vdf_ctx_set_group_tuning": (st, [vp, C.c_uint32]),
        "vdf_ctx_get_group_tuning": (C.c_uint32, [vp]),
        "vdf_ctx_set_sort_tuning": (st, [vp, C.POINTER(vdf_sort_tuning)]),
        "vdf_ctx_get_sort_tuning": (st, [vp, C.POINTER(vdf_sort_tuning)]),
        "vdf_groupby_workspace_bytes": (sz, [u64, i32]),
        "vdf_sort_argsort": (st, [vp, u64, C.POINTER(vdf_col), i32, i32, vp, C.POINTER(vp), vp]),
        "vdf_sort_argsort_ws": (st, [vp, u64, C.POINTER(vdf_col), i32, i32, vp, C.POINTER(vp), vp, sz, vp]),
        "vdf_sort_argsort_noalloc": (st, [u64, C.POINTER(vdf_col), i32, i32, vp, C.POINTER(vp), vp]),
        "vdf_sort_noalloc_error": (st, [C.POINTER(C.c_uint32), vp]),
        "vdf_gather": (st, [vp, u64, vp, C.POINTER(vdf_col), i32, C.POINTER(vp), vp]),
        "vdf_groupby_sorted": (st, [vp, u64, C.POINTER(vdf_col), i32, C.POINTER(vdf_col), i32, C.POINTER(vp), vp,
                                    C.POINTER(vdf_agg_out), vp, vp, vp, C.POINTER(C.c_uint64), vp]),
        "vdf_sort_groupby": (st, [vp, C.POINTER(vdf_sort_groupby_args), vp]),
        "vdf_sort_groupby_host": (st, [vp, C.POINTER(vdf_sort_groupby_args), vp]),
        "vdf_broadcast": (st, [vp, u64, vp, vp, u64, i32, vp, vp, vp]),
        "vdf_unique": (st, [vp, u64, vdf_col, i32, vp, vp, C.POINTER(C.c_uint64), vp]),
        "vdf_pivot_host": (st, [vp, u64, vdf_strcol, vdf_strcol, vdf_col, C.POINTER(C.c_uint32),
                                C.POINTER(C.c_uint32), vp, vp, vp, u64]),
        "vdf_left_join_index": (st, [vp, u64, vdf_col, u64, vdf_col, i32, vp, vp, C.POINTER(C.c_uint64), vp]),
        "vdf_gather_host": (st, [vp, u64, vp, C.POINTER(vdf_col), i32, C.POINTER(vp), vp]),
        "vdf_transform_groupby_host": (st, [vp, u64, C.POINTER(vdf_col), i32, vdf_col, C.c_int32, vp, vp,
                                            C.POINTER(C.c_uint64), vp]),
        "vdf_ctx_set_multikey_mode": (st, [vp, i32]),
        "vdf_ctx_get_multikey_mode": (i32, [vp]),
        "vdf_ctx_set_sort_strategy": (st, [vp, i32, u64]),
        "vdf_ctx_sort_stats": (st, [vp, vp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
        "vdf_ctx_dict_stats": (st, [vp, vp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
        "vdf_sort_plan_tries_dict": (i32, [u64, C.POINTER(C.c_int32), i32, i32, u64]),
        "vdf_ctx_set_local_sort_variant": (st, [vp, i32]),
        "vdf_ctx_set_test_hooks": (st, [vp, C.c_uint32, C.c_uint32, C.c_uint32]),
        "vdf_ctx_get_local_sort_variant": (i32, [vp]),
        "vdf_ctx_get_sort_strategy": (st, [vp, C.POINTER(C.c_int32), C.POINTER(C.c_uint64)]),
        "vdf_sort_plan_info": (st, [u64, C.POINTER(C.c_int32), i32, i32, u64, C.POINTER(C.c_int32),
                                    C.POINTER(C.c_uint32)]),
        "vdf_batch_variant_count": (i32, []),
        "vdf_batch_variant_info": (st, [i32, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
        "vdf_batch_default_tuning": (st, [C.POINTER(vdf_batch_tuning)]),
        "vdf_batch_create": (st, [vp, C.POINTER(vdf_batch_args), C.POINTER(vdf_batch_tuning), C.POINTER(vp)]),
        "vdf_batch_rows": (u64, [vp]),
        "vdf_batch_info": (st, [vp, C.POINTER(C.c_uint32), C.POINTER(C.c_uint64), C.POINTER(C.c_uint32),
                                C.POINTER(C.c_uint64)]),
        "vdf_batch_sort_info": (st, [vp, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
        "vdf_batch_launch": (st, [vp, vp]),
        "vdf_batch_launch_graph": (st, [vp, vp]),
        "vdf_batch_destroy": (None, [vp]),
        "vdf_csv_read": (st, [vp, vp, u64, C.c_char, i32, C.c_char, C.POINTER(vp), vp]),
        "vdf_csv_read_host": (st, [vp, vp, u64, C.c_char, i32, C.c_char, C.POINTER(vp), vp]),
        "vdf_csv_nrow": (u64, [vp]),
        "vdf_csv_ncol": (C.c_uint32, [vp]),
        "vdf_csv_name": (C.c_char_p, [vp, C.c_uint32]),
        "vdf_csv_type": (C.c_char, [vp, C.c_uint32]),
        "vdf_csv_values": (vp, [vp, C.c_uint32]),
        "vdf_csv_offsets": (vp, [vp, C.c_uint32]),
        "vdf_csv_string_bytes": (u64, [vp, C.c_uint32]),
        "vdf_csv_copy_column": (st, [vp, vp, C.c_uint32, vp, vp, vp]),
        "vdf_csv_free": (None, [vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


lib = _load()


def _ptr(t: Optional[torch.Tensor]) -> Optional[int]:
    return None if t is None else t.data_ptr()


def _col(t: torch.Tensor) -> vdf_col:
    if not t.is_cuda or not t.is_contiguous():
        raise ValueError("columns must be contiguous CUDA tensors")
    if t.dtype not in TORCH_TO_VDF:
        raise TypeError(f"unsupported column dtype {t.dtype}")
    return vdf_col(t.data_ptr(), TORCH_TO_VDF[t.dtype])


def _cols(ts: Sequence[torch.Tensor]):
    arr = (vdf_col * max(1, len(ts)))()
    for i, t in enumerate(ts):
        arr[i] = _col(t)
    return arr


def _ptrs(ts: Sequence[Optional[torch.Tensor]]):
    arr = (C.c_void_p * max(1, len(ts)))()
    for i, t in enumerate(ts):
        arr[i] = _ptr(t)
    return arr


def _stream(stream) -> Optional[int]:
    if stream is None:
        stream = torch.cuda.current_stream()
    return stream.cuda_stream


@dataclass
class AggResult:
    sum: torch.Tensor
    sum_hi: Optional[torch.Tensor]
    min: torch.Tensor
    max: torch.Tensor
    mean: torch.Tensor


@dataclass
class GroupResult:
    n_groups: int
    keys: list
    count: torch.Tensor
    aggs: list
    group_start: Optional[torch.Tensor] = None
    row_group: Optional[torch.Tensor] = None
    perm: Optional[torch.Tensor] = None
    sorted_keys: list = field(default_factory=list)
    payload: list = field(default_factory=list)

    def trimmed(self) -> "GroupResult":
        g = self.n_groups
        aggs = [AggResult(a.sum[:g], None if a.sum_hi is None else a.sum_hi[:g], a.min[:g], a.max[:g], a.mean[:g])
                for a in self.aggs]
        return GroupResult(g, [k[:g] for k in self.keys], self.count[:g], aggs,
                           None if self.group_start is None else self.group_start[:g], self.row_group, self.perm,
                           self.sorted_keys, self.payload)


def _alloc_aggs(vals: Sequence[torch.Tensor], n: int, device):
    outs, structs = [], (vdf_agg_out * max(1, len(vals)))()
    for i, v in enumerate(vals):
        is_float = v.dtype in (torch.float64, torch.float32)
        s = torch.empty(n, dtype=torch.float64 if is_float else torch.int64, device=device)
        hi = None if is_float else torch.empty(n, dtype=torch.int64, device=device)
        mn = torch.empty(n, dtype=v.dtype, device=device)
        mx = torch.empty(n, dtype=v.dtype, device=device)
        mean = torch.empty(n, dtype=torch.float64, device=device)
        outs.append(AggResult(s, hi, mn, mx, mean))
        structs[i] = vdf_agg_out(_ptr(s), _ptr(hi), _ptr(mn), _ptr(mx), _ptr(mean))
    return outs, structs


class Context:
    """One vdf_ctx: a device, a grow-only workspace and an error word."""

    def __init__(self, device: int = 0):
        self.device = device
        h = C.c_void_p()
        self._check(lib.vdf_ctx_create(device, C.byref(h)), "vdf_ctx_create", ctx=None)
        self.handle = h

    def close(self):
        if getattr(self, "handle", None):
            lib.vdf_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, status: int, what: str, ctx="self"):
        if status != OK:
            msg = lib.vdf_status_string(status).decode()
            if ctx == "self" and getattr(self, "handle", None):
                detail = lib.vdf_ctx_last_error(self.handle).decode()
                if detail:
                    msg += f" ({detail})"
            raise VdfError(status, f"{what}: {msg}")

    @property
    def kernel_launches(self) -> int:
        return int(lib.vdf_ctx_kernel_launches(self.handle))

    def check(self, stream=None):
        self._check(lib.vdf_ctx_check(self.handle, _stream(stream)), "vdf_ctx_check")

    def profile(self, enable: bool = True):
        self._check(lib.vdf_ctx_profile(self.handle, 1 if enable else 0), "vdf_ctx_profile")

    def profile_reset(self):
        self._check(lib.vdf_ctx_profile_reset(self.handle), "vdf_ctx_profile_reset")

    def profile_read(self) -> dict:
        """{kernel class name: (total device ms, launches)}"""
        out = {}
        for cls, name in enumerate(KERNEL_CLASSES):
            ms, cnt = C.c_double(0), C.c_uint64(0)
            self._check(lib.vdf_ctx_profile_read(self.handle, cls, C.byref(ms), C.byref(cnt)), "profile_read")
            out[name] = (ms.value, int(cnt.value))
        return out

    def set_sort_tuning(self, variant32: int, variant64: int):
        t = vdf_sort_tuning(variant32, variant64)
        self._check(lib.vdf_ctx_set_sort_tuning(self.handle, C.byref(t)), "vdf_ctx_set_sort_tuning")

    def set_multikey_mode(self, mode: int):
        self._check(lib.vdf_ctx_set_multikey_mode(self.handle, mode), "vdf_ctx_set_multikey_mode")

    def get_multikey_mode(self) -> int:
        return lib.vdf_ctx_get_multikey_mode(self.handle)

    def set_sort_strategy(self, strategy: int, msd_min_rows: int = 1 << 20):
        """SORT_AUTO: MSD-first sorts (one or two keys, >= msd_min_rows rows,
        8-byte key 0) with the LSD passes as the on-device fallback;
        SORT_LSD: LSD only; SORT_MSD: MSD-first for every key width."""
        self._check(lib.vdf_ctx_set_sort_strategy(self.handle, strategy, msd_min_rows), "vdf_ctx_set_sort_strategy")

    def sort_stats(self, stream=None) -> dict:
        """{"msd_sorts": sorts planned MSD-first, "msd_fallbacks": of those, LSD fallbacks on the device,
        "dict_sorts": sorts that tried the dictionary plan, "dict_taken": of those, the ones it sorted}"""
        a, b, c, d = C.c_uint64(), C.c_uint64(), C.c_uint64(), C.c_uint64()
        self._check(lib.vdf_ctx_sort_stats(self.handle, _stream(stream), C.byref(a), C.byref(b)), "sort_stats")
        self._check(lib.vdf_ctx_dict_stats(self.handle, _stream(stream), C.byref(c), C.byref(d)), "sort_stats")
        return {"msd_sorts": int(a.value), "msd_fallbacks": int(b.value), "dict_sorts": int(c.value),
                "dict_taken": int(d.value)}

    def set_group_tuning(self, striped_min_heads: int = 0):
        """Group starts per 512-row tile from which the emit takes its striped path (0: the default)."""
        self._check(lib.vdf_ctx_set_group_tuning(self.handle, striped_min_heads), "vdf_ctx_set_group_tuning")

    def get_group_tuning(self) -> int:
        return int(lib.vdf_ctx_get_group_tuning(self.handle))

    def set_test_hooks(self, spin_limit: int = 0, stall_tile: int = 0xFFFFFFFF, fail_allocs: int = 0):
        """Failure injection for tests (see vdf_ctx_set_test_hooks)."""
        self._check(lib.vdf_ctx_set_test_hooks(self.handle, spin_limit, stall_tile, fail_allocs), "set_test_hooks")

    def set_local_sort_variant(self, variant: int):
        self._check(lib.vdf_ctx_set_local_sort_variant(self.handle, variant), "vdf_ctx_set_local_sort_variant")

    def get_local_sort_variant(self) -> int:
        return lib.vdf_ctx_get_local_sort_variant(self.handle)

    def get_sort_strategy(self) -> tuple:
        st, mn = C.c_int32(), C.c_uint64()
        self._check(lib.vdf_ctx_get_sort_strategy(self.handle, C.byref(st), C.byref(mn)), "get_sort_strategy")
        return st.value, int(mn.value)

    def get_sort_tuning(self) -> tuple:
        t = vdf_sort_tuning()
        self._check(lib.vdf_ctx_get_sort_tuning(self.handle, C.byref(t)), "vdf_ctx_get_sort_tuning")
        return t.pass_variant32, t.pass_variant64

    def reserve(self, nbytes: int):
        self._check(lib.vdf_ctx_reserve(self.handle, nbytes), "vdf_ctx_reserve")

    # ---- sort ----------------------------------------------------------------
    def argsort(self, keys: Sequence[torch.Tensor], order: int = ORDER_ASC, perm_out=None,
                sorted_keys_out: Optional[Sequence[Optional[torch.Tensor]]] = None, stream=None,
                workspace: Optional[torch.Tensor] = None) -> torch.Tensor:
        n = keys[0].numel() if keys else 0
        dev = keys[0].device if keys else torch.device("cuda", self.device)
        if perm_out is None:
            perm_out = torch.empty(n, dtype=torch.int32, device=dev)
        sko = _ptrs(sorted_keys_out) if sorted_keys_out is not None else None
        if workspace is None:
            st = lib.vdf_sort_argsort(self.handle, n, _cols(keys), len(keys), order, _ptr(perm_out), sko,
                                      _stream(stream))
        else:
            st = lib.vdf_sort_argsort_ws(self.handle, n, _cols(keys), len(keys), order, _ptr(perm_out), sko,
                                         _ptr(workspace), workspace.numel() * workspace.element_size(),
                                         _stream(stream))
        self._check(st, "vdf_sort_argsort")
        return perm_out

    def gather(self, perm: torch.Tensor, cols: Sequence[torch.Tensor], out=None, stream=None):
        n = perm.numel()
        if out is None:
            out = [torch.empty(n, dtype=c.dtype, device=c.device) for c in cols]
        self._check(lib.vdf_gather(self.handle, n, _ptr(perm), _cols(cols), len(cols), _ptrs(out), _stream(stream)),
                    "vdf_gather")
        return out

    # ---- group-by ------------------------------------------------------------
    def groupby_sorted(self, keys: Sequence[torch.Tensor], vals: Sequence[torch.Tensor], want_row_group=False,
                       want_group_start=False, stream=None) -> GroupResult:
        n = keys[0].numel()
        dev = keys[0].device
        gk = [torch.empty(n, dtype=k.dtype, device=dev) for k in keys]
        cnt = torch.empty(n, dtype=torch.int64, device=dev)
        aggs, structs = _alloc_aggs(vals, n, dev)
        gs = torch.empty(n, dtype=torch.int32, device=dev) if want_group_start else None
        rg = torch.empty(n, dtype=torch.int32, device=dev) if want_row_group else None
        ng = C.c_uint64(0)
        st = lib.vdf_groupby_sorted(self.handle, n, _cols(keys), len(keys), _cols(vals), len(vals), _ptrs(gk),
                                    _ptr(cnt), structs, _ptr(gs), _ptr(rg), None, C.byref(ng), _stream(stream))
        self._check(st, "vdf_groupby_sorted")
        return GroupResult(int(ng.value), gk, cnt, aggs, gs, rg).trimmed()

    def sort_groupby(self, keys: Sequence[torch.Tensor], payload: Sequence[torch.Tensor] = (),
                     agg_cols: Sequence[int] = (), order: int = ORDER_ASC, groupby: bool = True,
                     want_perm=True, want_sorted_keys=True, want_payload=True, want_row_group=False,
                     want_group_start=False, stream=None, outputs: Optional[dict] = None) -> GroupResult:
        """Sort + payload gather + group-by in one call.  `outputs` may carry
        preallocated tensors (keys as in the returned GroupResult fields) so a
        benchmark loop allocates nothing."""
        n = keys[0].numel()
        dev = keys[0].device
        o = outputs if outputs is not None else self.alloc_sort_groupby_outputs(
            keys, payload, agg_cols, groupby, want_perm, want_sorted_keys, want_payload, want_row_group,
            want_group_start)
        args = self.pack_sort_groupby(keys, payload, agg_cols, order, groupby, o)
        self._check(lib.vdf_sort_groupby(self.handle, C.byref(args), _stream(stream)), "vdf_sort_groupby")
        g = int(o["_ng"].value) if groupby else 0
        res = GroupResult(g, o["gkeys"], o["count"], o["aggs"], o["gstart"], o["rgroup"], o["perm"],
                          o["skeys"], o["pay"])
        return res.trimmed() if groupby else res

    def alloc_sort_groupby_outputs(self, keys, payload, agg_cols, groupby=True, want_perm=True,
                                   want_sorted_keys=True, want_payload=True, want_row_group=False,
                                   want_group_start=False) -> dict:
        n = keys[0].numel()
        dev = keys[0].device
        o = {
            "perm": torch.empty(n, dtype=torch.int32, device=dev) if want_perm else None,
            "skeys": [torch.empty(n, dtype=k.dtype, device=dev) for k in keys] if want_sorted_keys else [],
            "pay": [torch.empty(n, dtype=p.dtype, device=dev) for p in payload] if want_payload else [],
            "gkeys": [], "count": None, "aggs": [], "gstart": None, "rgroup": None,
        }
        if groupby:
            o["gkeys"] = [torch.empty(n, dtype=k.dtype, device=dev) for k in keys]
            o["count"] = torch.empty(n, dtype=torch.int64, device=dev)
            o["aggs"], o["_structs"] = _alloc_aggs([payload[i] for i in agg_cols], n, dev)
            o["gstart"] = torch.empty(n, dtype=torch.int32, device=dev) if want_group_start else None
            o["rgroup"] = torch.empty(n, dtype=torch.int32, device=dev) if want_row_group else None
        return o

    def pack_sort_groupby(self, keys, payload, agg_cols, order, groupby, o, host_count=True):
        n = keys[0].numel()
        a = vdf_sort_groupby_args()
        kc, pc = _cols(keys), _cols(payload)
        o["_keep"] = [kc, pc]
        a.n = n
        a.keys, a.nkeys, a.order = kc, len(keys), order
        a.payload, a.npayload = pc, len(payload)
        a.perm_out = _ptr(o["perm"])
        if o["skeys"]:
            sk = _ptrs(o["skeys"]); o["_keep"].append(sk); a.sorted_keys_out = sk
        if o["pay"]:
            pp = _ptrs(o["pay"]); o["_keep"].append(pp); a.payload_out = pp
        a.groupby = 1 if groupby else 0
        if groupby:
            ac = (C.c_int32 * max(1, len(agg_cols)))(*agg_cols)
            gk = _ptrs(o["gkeys"])
            o["_keep"] += [ac, gk]
            a.agg_cols, a.nagg = ac, len(agg_cols)
            a.group_keys_out = gk
            a.group_count_out = _ptr(o["count"])
            a.aggs = o["_structs"]
            a.group_start_out = _ptr(o["gstart"])
            a.row_group_out = _ptr(o["rgroup"])
            o["_ng"] = C.c_uint64(0)
            if host_count:
                a.n_groups_host = C.pointer(o["_ng"])
            else:
                o["ngroups_dev"] = torch.zeros(1, dtype=torch.int64, device=keys[0].device)
                a.n_groups_dev = o["ngroups_dev"].data_ptr()
        return a

    def sort_groupby_packed(self, args, stream=None):
        self._check(lib.vdf_sort_groupby(self.handle, C.byref(args), _stream(stream)), "vdf_sort_groupby")

    def broadcast(self, row_group: torch.Tensor, group_vals: torch.Tensor, perm=None, out=None, stream=None):
        n = row_group.numel()
        if out is None:
            out = torch.empty(n, dtype=group_vals.dtype, device=group_vals.device)
        self._check(lib.vdf_broadcast(self.handle, n, _ptr(row_group), _ptr(group_vals), group_vals.numel(),
                                      group_vals.element_size(), _ptr(perm), _ptr(out), _stream(stream)),
                    "vdf_broadcast")
        return out


    def unique(self, key: torch.Tensor, keep_last: bool = False, stream=None):
        """(keep, n_unique): keep[i] = 1 (uint8) where row i is the first
        (or, with keep_last, the last) occurrence of its key."""
        n = key.numel()
        keep = torch.empty(n, dtype=torch.uint8, device=key.device)
        cnt = C.c_uint64(0)
        self._check(lib.vdf_unique(self.handle, n, _col(key), 1 if keep_last else 0, _ptr(keep), None,
                                   C.byref(cnt), _stream(stream)), "vdf_unique")
        return keep, int(cnt.value)

    def pivot_host(self, col_key, row_key, values) -> dict:
        """Pivot (the reference's pivot, pivots/pivot.hpp:5-128) of host
        columns: col_key / row_key are string columns given as (bytes uint8,
        offsets uint64 of n + 1) numpy arrays, values a numpy int32 / uint32 /
        int64 / uint64 / float64 column.  Returns {"colkey_row": first row of
        each col key, "rowkey_row": likewise, "matrix": [n_colkeys,
        n_rowkeys] sums}, keys in first-appearance order."""
        import numpy as np
        values = np.ascontiguousarray(values)
        code = {np.dtype(np.int32): I32, np.dtype(np.uint32): U32, np.dtype(np.int64): I64,
                np.dtype(np.uint64): U64, np.dtype(np.float64): F64, np.dtype(np.float32): F32}[values.dtype]
        n = values.size
        cols = []
        for b, o in (col_key, row_key):
            b = np.ascontiguousarray(b, np.uint8)
            o = np.ascontiguousarray(o, np.uint64)
            assert o.size == n + 1
            cols.append((b, o, vdf_strcol(b.ctypes.data if b.size else None, o.ctypes.data)))
        ckr = np.zeros(max(1, n), np.uint32)
        rkr = np.zeros(max(1, n), np.uint32)
        nc, nr = C.c_uint32(), C.c_uint32()
        vc = vdf_col(values.ctypes.data if n else None, code)
        st = lib.vdf_pivot_host(self.handle, n, cols[0][2], cols[1][2], vc, C.byref(nc), C.byref(nr),
                                ckr.ctypes.data, rkr.ctypes.data, None, 0)
        if st not in (OK, ERR_WORKSPACE):
            self._check(st, "vdf_pivot_host")
        m = np.zeros(max(1, nc.value * nr.value), values.dtype)
        st = lib.vdf_pivot_host(self.handle, n, cols[0][2], cols[1][2], vc, C.byref(nc), C.byref(nr),
                                ckr.ctypes.data, rkr.ctypes.data, m.ctypes.data, m.size)
        self._check(st, "vdf_pivot_host")
        return {"colkey_row": ckr[:nc.value].copy(), "rowkey_row": rkr[:nr.value].copy(),
                "matrix": m[:nc.value * nr.value].reshape(nc.value, nr.value)}

    def read_csv(self, data, delim: str = ",", header: bool = True, quote: str = "'", stream=None) -> "CsvTable":
        """Parses a CSV file's bytes (`bytes` / numpy uint8 in host memory, or
        a contiguous CUDA uint8 tensor) into device columns (read_csv, with the
        reference's defaults delim ',', header on, quote \\')."""
        h = C.c_void_p()
        d, q = delim.encode("latin-1"), quote.encode("latin-1")
        if isinstance(data, torch.Tensor):
            if not data.is_cuda or data.dtype != torch.uint8 or not data.is_contiguous():
                raise ValueError("device input must be a contiguous CUDA uint8 tensor")
            self._check(lib.vdf_csv_read(self.handle, data.data_ptr(), data.numel(), d, 1 if header else 0, q,
                                         C.byref(h), _stream(stream)), "vdf_csv_read")
        else:
            buf = np.frombuffer(data, dtype=np.uint8) if isinstance(data, (bytes, bytearray)) else \
                np.ascontiguousarray(data, dtype=np.uint8)
            self._check(lib.vdf_csv_read_host(self.handle, buf.ctypes.data if buf.size else None, buf.size, d,
                                              1 if header else 0, q, C.byref(h), _stream(stream)),
                        "vdf_csv_read_host")
        return CsvTable(self, h.value)

    def left_join_index(self, left: torch.Tensor, right: torch.Tensor, method: int = 0, stream=None):
        """(match, n_matched): match[i] = the row of `right` that left row i
        takes -- method 0: the first row holding its key, 1: the last, 2
        (aligned): the k-th one for the key's k-th left occurrence -- or
        UINT32_MAX (int32 view: -1) where there is none."""
        n = left.numel()
        match = torch.empty(n, dtype=torch.int32, device=left.device)
        cnt = C.c_uint64(0)
        self._check(lib.vdf_left_join_index(self.handle, n, _col(left), right.numel(), _col(right), int(method),
                                            _ptr(match), None, C.byref(cnt), _stream(stream)), "vdf_left_join_index")
        return match, int(cnt.value)


class CsvTable:
    """A parsed CSV file: device-resident columns owned by the table
    (vdf_csv_read).  `types[k]` is 'd' (float64), 'u' (uint32), 'b' (uint8
    0/1), 's' or 'c' (strings: offsets + bytes)."""

    _NP = {"d": np.float64, "u": np.uint32, "b": np.uint8}

    def __init__(self, ctx: "Context", handle: int):
        self._ctx = ctx
        self.handle = handle
        self._live_views = 0    # view() tensors still alive
        self._closing = False   # close() called: free once the last view is gone
        self.nrow = int(lib.vdf_csv_nrow(handle))
        self.ncol = int(lib.vdf_csv_ncol(handle))
        self.names = [lib.vdf_csv_name(handle, k).decode("latin-1") for k in range(self.ncol)]
        self.types = [lib.vdf_csv_type(handle, k).decode("latin-1") for k in range(self.ncol)]

    def device_column(self, k: int) -> dict:
        """{'values': device pointer, 'offsets': device pointer or None, 'bytes': string bytes}."""
        return dict(values=lib.vdf_csv_values(self.handle, k), offsets=lib.vdf_csv_offsets(self.handle, k),
                    bytes=int(lib.vdf_csv_string_bytes(self.handle, k)))

    _TORCH = {"d": torch.float64, "u": torch.uint32, "b": torch.uint8}

    _TYPESTR = {"d": "<f8", "u": "<u4", "b": "|u1"}

    def view(self, k: int) -> torch.Tensor:
        """Numeric column k as a CUDA tensor over the table's own memory (no
        copy): parsed columns go straight into the sort and group-by; writes
        through it change the table.  The tensor keeps the table alive, and
        close() while views are alive frees the table's memory only when the
        last of them is gone.  uint32 columns come back as torch.uint32."""
        ty = self.types[k]
        if ty not in self._TYPESTR:
            raise ValueError("string columns have no tensor view")
        if not self.handle or self._closing:
            raise ValueError("the table is closed")
        table = self

        class _Col:
            __cuda_array_interface__ = {"shape": (self.nrow,), "typestr": self._TYPESTR[ty],
                                        "data": (int(lib.vdf_csv_values(self.handle, k) or 0), False),
                                        "version": 3, "strides": None}
            owner = table

        holder = _Col()
        t = torch.as_tensor(holder, device=f"cuda:{self._ctx.device}")
        t._vdf_owner = holder  # the table outlives the view
        self._live_views += 1
        weakref.finalize(holder, CsvTable._view_gone, self)
        return t

    @staticmethod
    def _view_gone(table: "CsvTable"):
        table._live_views -= 1
        if table._closing and table._live_views == 0:
            table._free()

    def copy_column(self, k: int, values: int, offsets: Optional[int] = None, stream=None):
        """Copies column k into caller memory (host or device addresses):
        the values (or string bytes) and, for strings, nrow + 1 offsets."""
        self._ctx._check(lib.vdf_csv_copy_column(self._ctx.handle, self.handle, k, values, offsets,
                                                 _stream(stream)), "vdf_csv_copy_column")

    def tensor(self, k: int, stream=None) -> torch.Tensor:
        """Numeric column k copied into a new CUDA tensor (uint32 columns as
        torch.uint32, as view() gives them, so both sort the same way)."""
        ty = self.types[k]
        if ty not in self._TORCH:
            raise ValueError("string columns have no tensor form")
        out = torch.empty(self.nrow, dtype=self._TORCH[ty], device=f"cuda:{self._ctx.device}")
        self._ctx._check(lib.vdf_csv_copy_column(self._ctx.handle, self.handle, k, out.data_ptr(), None,
                                                 _stream(stream)), "vdf_csv_copy_column")
        return out

    def column(self, k: int, stream=None):
        """Column k on the host: a numpy array, or a list of bytes for strings."""
        ty = self.types[k]
        if ty in self._NP:
            out = np.empty(self.nrow, dtype=self._NP[ty])
            self._ctx._check(lib.vdf_csv_copy_column(self._ctx.handle, self.handle, k, out.ctypes.data, None,
                                                        _stream(stream)), "vdf_csv_copy_column")
            return out
        nb = int(lib.vdf_csv_string_bytes(self.handle, k))
        data = np.empty(max(nb, 1), dtype=np.uint8)
        off = np.empty(self.nrow + 1, dtype=np.uint64)
        self._ctx._check(lib.vdf_csv_copy_column(self._ctx.handle, self.handle, k, data.ctypes.data,
                                                    off.ctypes.data, _stream(stream)), "vdf_csv_copy_column")
        raw = data.tobytes()
        return [raw[int(off[i]):int(off[i + 1])] for i in range(self.nrow)]

    def close(self):
        """Frees the table's device memory, or, while view() tensors are
        alive, as soon as the last of them is gone (their memory must not go
        back to the pool under them)."""
        self._closing = True
        if self._live_views == 0:
            self._free()

    def _free(self):
        if self.handle:
            lib.vdf_csv_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self._free()
        except Exception:
            pass


def sort_variants() -> list:
    """[{index, key_width, threads, items, digit_bits, match, tma}] of the compiled radix-pass variants
    (tma: tiles staged by bulk copies on a persistent grid)."""
    out = []
    for i in range(lib.vdf_sort_variant_count()):
        vals = [C.c_int32() for _ in range(5)]
        if lib.vdf_sort_variant_info(i, *[C.byref(v) for v in vals]) == OK:
            out.append(dict(index=i, key_width=vals[0].value, threads=vals[1].value, items=vals[2].value,
                            digit_bits=vals[3].value, match=vals[4].value,
                            tma=bool(lib.vdf_sort_variant_flags(i) & 1)))
    return out


def sort_plan_info(n: int, dtypes: Sequence[int], strategy: int = SORT_AUTO, msd_min_rows: int = 1 << 20) -> dict:
    """The plan of a sort: {"msd_passes": global MSD passes (0 = LSD), "chunks": shared-memory chunks,
    "dict": whether the dictionary plan is tried first}."""
    dts = (C.c_int32 * len(dtypes))(*dtypes)
    p, c = C.c_int32(), C.c_uint32()
    tries = lib.vdf_sort_plan_tries_dict(n, dts, len(dtypes), strategy, msd_min_rows)
    st = lib.vdf_sort_plan_info(n, dts, len(dtypes), strategy, msd_min_rows, C.byref(p), C.byref(c))
    if st != OK:
        raise VdfError(st, "vdf_sort_plan_info")
    return {"msd_passes": p.value, "chunks": c.value, "dict": tries == 1}


def header_functions() -> list[str]:
    """Names of the functions include/vdf_capi.h declares."""
    import re
    text = HEADER_PATH.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(vdf_[a-z0-9_]+)\s*\(", text)))


def batch_variants() -> list:
    """[{index, digit_bits, tile_rows}] of the segmented radix-pass variants."""
    out = []
    for i in range(lib.vdf_batch_variant_count()):
        b, t = C.c_int32(), C.c_int32()
        if lib.vdf_batch_variant_info(i, C.byref(b), C.byref(t)) == OK:
            out.append(dict(index=i, digit_bits=b.value, tile_rows=t.value))
    return out


def default_batch_tuning() -> dict:
    t = vdf_batch_tuning()
    lib.vdf_batch_default_tuning(C.byref(t))
    return dict(small_rows=t.small_rows, small_bits=t.small_bits, seg_variant=t.seg_variant)


@dataclass
class QueryResult:
    """One query's results (device tensor views into the batch arenas)."""
    perm: torch.Tensor
    n_groups: int
    keys: torch.Tensor
    count: torch.Tensor
    aggs: list


class Batch:
    """Many independent sort + group-by queries planned once (vdf_batch_*).

    `queries` is a list of (key tensor, [value tensors]); every query has
    the same value dtypes.  Outputs live in arenas owned by this object;
    `result(q)` returns views of query q's part after a launch."""

    @staticmethod
    def alloc_outputs(capacity: int, val_dtypes, device) -> dict:
        """Output arenas for batches of up to `capacity` rows, reusable by
        successive batches (pass as `outputs=`)."""
        N = max(1, int(capacity))
        aggs = []
        for dt in val_dtypes:
            fl = dt in (torch.float64, torch.float32)
            aggs.append(AggResult(torch.empty(N, dtype=torch.float64 if fl else torch.int64, device=device),
                                  None if fl else torch.empty(N, dtype=torch.int64, device=device),
                                  torch.empty(N, dtype=dt, device=device), torch.empty(N, dtype=dt, device=device),
                                  torch.empty(N, dtype=torch.float64, device=device)))
        return {"capacity": N, "perm": torch.empty(N, dtype=torch.int32, device=device),
                "gkeys": torch.empty(N, dtype=torch.int64, device=device),
                "count": torch.empty(N, dtype=torch.int64, device=device), "aggs": aggs,
                "val_dtypes": list(val_dtypes)}

    def __init__(self, ctx: "Context", queries, tuning: Optional[dict] = None, outputs: Optional[dict] = None):
        self.ctx = ctx
        self.queries = [(k, list(vs)) for k, vs in queries]
        nq = len(self.queries)
        nvals = len(self.queries[0][1]) if nq else 0
        if nvals > BATCH_MAX_VALS:
            raise ValueError(f"at most {BATCH_MAX_VALS} value columns")
        self.val_dtypes = [v.dtype for v in self.queries[0][1]] if nq else []
        for k, vs in self.queries:
            if [v.dtype for v in vs] != self.val_dtypes:
                raise ValueError("every query must have the same value dtypes")
        dev = torch.device("cuda", ctx.device)
        self.n_total = sum(int(k.numel()) for k, _ in self.queries)
        if outputs is None:
            outputs = Batch.alloc_outputs(self.n_total, self.val_dtypes, dev)
        elif outputs["capacity"] < self.n_total or outputs["val_dtypes"] != self.val_dtypes:
            raise ValueError("output arenas too small or of other value dtypes")
        self.perm, self.gkeys, self.count, self.aggs = outputs["perm"], outputs["gkeys"], outputs["count"], outputs["aggs"]
        structs = (vdf_agg_out * BATCH_MAX_VALS)()
        for j, a in enumerate(self.aggs):
            structs[j] = vdf_agg_out(_ptr(a.sum), _ptr(a.sum_hi), _ptr(a.min), _ptr(a.max), _ptr(a.mean))
        self.row_offset = torch.zeros(max(1, nq), dtype=torch.int64, device=dev)
        self.group_offset = torch.zeros(max(1, nq), dtype=torch.int64, device=dev)
        self.n_groups = torch.zeros(max(1, nq), dtype=torch.int64, device=dev)
        qs = (vdf_batch_query * max(1, nq))()
        for i, (k, vs) in enumerate(self.queries):
            qs[i].n = k.numel()
            qs[i].key = _col(k)
            for j, v in enumerate(vs):
                if not v.is_cuda or not v.is_contiguous() or v.numel() != k.numel():
                    raise ValueError("value columns must be contiguous CUDA tensors of the key's length")
                qs[i].vals[j] = v.data_ptr()
        a = vdf_batch_args()
        a.nqueries = nq
        a.queries = qs
        a.nvals = nvals
        for j, dt in enumerate(self.val_dtypes):
            a.val_dtypes[j] = TORCH_TO_VDF[dt]
        a.perm_out = _ptr(self.perm)
        a.group_keys_out = _ptr(self.gkeys)
        a.group_count_out = _ptr(self.count)
        a.aggs = structs
        a.row_offset_out = _ptr(self.row_offset)
        a.group_offset_out = _ptr(self.group_offset)
        a.n_groups_out = _ptr(self.n_groups)
        self._args = a
        t = None
        if tuning is not None:
            t = vdf_batch_tuning(int(tuning["small_rows"]), int(tuning["small_bits"]), int(tuning["seg_variant"]))
        h = C.c_void_p()
        st = lib.vdf_batch_create(ctx.handle, C.byref(a), None if t is None else C.byref(t), C.byref(h))
        ctx._check(st, "vdf_batch_create")
        self.handle = h
        self._host = None

    def info(self) -> dict:
        sq, lq = C.c_uint32(), C.c_uint32()
        sr, lr = C.c_uint64(), C.c_uint64()
        lib.vdf_batch_info(self.handle, C.byref(sq), C.byref(sr), C.byref(lq), C.byref(lr))
        return dict(small_queries=sq.value, small_rows=sr.value, large_queries=lq.value, large_rows=lr.value,
                    rows=lib.vdf_batch_rows(self.handle))

    def sort_info(self, fallbacks: bool = False) -> dict:
        """Queries on the MSD-first sort and on the LSD passes; with
        fallbacks=True also (after waiting for the device) the MSD queries of
        the last launch that fell back to the LSD passes."""
        mq, lq, fb = C.c_uint32(), C.c_uint32(), C.c_uint32()
        st = lib.vdf_batch_sort_info(self.handle, C.byref(mq), C.byref(lq), C.byref(fb) if fallbacks else None)
        self.ctx._check(st, "vdf_batch_sort_info")
        out = dict(msd_queries=mq.value, lsd_queries=lq.value)
        if fallbacks:
            out["fallbacks"] = fb.value
        return out

    def launch(self, stream=None):
        self._host = None
        self.ctx._check(lib.vdf_batch_launch(self.handle, _stream(stream)), "vdf_batch_launch")

    def launch_graph(self, stream=None):
        self._host = None
        self.ctx._check(lib.vdf_batch_launch_graph(self.handle, _stream(stream)), "vdf_batch_launch_graph")

    def _offsets(self):
        if self._host is None:
            self._host = (self.row_offset.cpu().tolist(), self.group_offset.cpu().tolist(),
                          self.n_groups.cpu().tolist())
        return self._host

    def result(self, q: int) -> QueryResult:
        ro, go, ng = self._offsets()
        k = self.queries[q][0]
        n = k.numel()
        G = int(ng[q])
        r0, g0 = int(ro[q]), int(go[q])
        kb = self.gkeys.view(torch.uint8)[8 * g0: 8 * g0 + k.element_size() * G]
        keys = kb.view(k.dtype) if G else torch.empty(0, dtype=k.dtype, device=k.device)
        aggs = [AggResult(a.sum[g0:g0 + G], None if a.sum_hi is None else a.sum_hi[g0:g0 + G], a.min[g0:g0 + G],
                          a.max[g0:g0 + G], a.mean[g0:g0 + G]) for a in self.aggs]
        return QueryResult(self.perm[r0:r0 + n], G, keys, self.count[g0:g0 + G], aggs)

    def close(self):
        if getattr(self, "handle", None):
            lib.vdf_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
