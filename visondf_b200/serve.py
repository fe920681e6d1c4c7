"""Request loop for sort + group-by queries over device-resident columns.

Requests (a key column and value columns, each a slice of tables that stay
resident in HBM) arrive over time.  The loop admits them first-come first-
served while the device memory they need fits the HBM budget, and runs them
with continuous batching: every request that has arrived and been admitted
when an execution slot frees up joins the next batch (vdf_batch_*: one
planned set of launches for all of them), and up to `slots` batches are in
flight at once on separate streams, so a batch formed while another runs
overlaps it on the device.  A request's latency runs from its arrival to the
completion of the batch holding it.

The reference has no serving layer; its per-query work is one sort_by_mt
call plus one transform_group_by_onecol_mt call.  `PerCallExecutor` runs the
same requests one library call each (vdf_sort_groupby), one at a time, as the
baseline the batched loop is measured against.

The scheduler only talks to an executor through `start(requests) -> handle`,
`done(handle)` and `finish(handle)`, so its admission and batching logic is
tested on the CPU with a simulated executor.
"""
from __future__ import annotations

import collections
import statistics
import time
from dataclasses import dataclass, field
from typing import Callable, Optional, Sequence

# Device bytes per row a request holds while its batch is in flight: the
# output arenas (u32 permutation, 8-byte group key slot, int64 count) plus
# per value column sum/min/max/mean (+ the high sum word for integers).
OUT_BYTES_PER_ROW_BASE = 4 + 8 + 8


def out_bytes_per_row(val_is_float: Sequence[bool]) -> int:
    return OUT_BYTES_PER_ROW_BASE + sum(32 if f else 40 for f in val_is_float)


# Upper bound of the batch workspace per row (arena keys, segment ids, value
# copies in both orders, sorted keys, group scratch, and the largest of the
# radix, gather and reduction scratch); each slot reserves it once for its
# largest batch.
WS_BYTES_PER_ROW = 136


@dataclass
class Request:
    rid: int
    arrival: float          # seconds from the start of the trace
    rows: int
    key: object = None      # device column (resident slice)
    vals: list = field(default_factory=list)
    need_bytes: int = 0     # device memory held while in flight
    # filled in by the loop
    admitted: Optional[float] = None
    started: Optional[float] = None
    completed: Optional[float] = None
    result: object = None

    @property
    def latency(self) -> Optional[float]:
        return None if self.completed is None else self.completed - self.arrival


@dataclass
class TraceStats:
    requests: int
    rows: int
    seconds: float          # first arrival to last completion
    rows_per_s: float
    p50_ms: float
    p99_ms: float
    mean_ms: float
    batches: int
    max_in_flight_bytes: int

    def as_dict(self) -> dict:
        return dict(requests=self.requests, rows=self.rows, seconds=self.seconds, rows_per_s=self.rows_per_s,
                    p50_ms=self.p50_ms, p99_ms=self.p99_ms, mean_ms=self.mean_ms, batches=self.batches,
                    max_in_flight_bytes=self.max_in_flight_bytes)


def percentile(xs: Sequence[float], q: float) -> float:
    """Nearest-rank percentile (q in [0, 100])."""
    s = sorted(xs)
    if not s:
        return float("nan")
    k = max(0, min(len(s) - 1, int(-(-q * len(s) // 100)) - 1))
    return s[k]


class Loop:
    """Admission by HBM budget + continuous batching over an executor.

    budget_bytes: device memory the loop may use in total, including
        `fixed_bytes` (resident columns, reserved workspaces) held throughout.
    max_batch_rows / max_batch_queries: limits of one batch.
    """

    def __init__(self, executor, budget_bytes: int, fixed_bytes: int = 0, max_batch_rows: int = 1 << 27,
                 max_batch_queries: int = 4096, clock: Callable[[], float] = time.perf_counter,
                 idle_sleep: Callable[[float], None] = time.sleep):
        self.ex = executor
        self.budget = int(budget_bytes)
        self.fixed = int(fixed_bytes)
        self.max_rows = int(max_batch_rows)
        self.max_queries = int(max_batch_queries)
        self.clock = clock
        self.sleep = idle_sleep
        if self.fixed > self.budget:
            raise ValueError("resident columns and workspaces exceed the HBM budget")

    def run(self, requests: Sequence[Request]) -> TraceStats:
        reqs = sorted(requests, key=lambda r: (r.arrival, r.rid))
        for r in reqs:
            if self.fixed + r.need_bytes > self.budget:
                raise ValueError(f"request {r.rid} alone needs more than the HBM budget")
            if r.rows > self.max_rows:
                raise ValueError(f"request {r.rid} has more rows than a batch may hold")
        waiting: collections.deque = collections.deque()
        inflight = []  # (handle, [requests], bytes)
        in_use = self.fixed
        peak = in_use
        nxt = 0
        batches = 0
        t0 = self.clock()
        done = 0
        while done < len(reqs):
            now = self.clock() - t0
            while nxt < len(reqs) and reqs[nxt].arrival <= now:
                waiting.append(reqs[nxt])
                nxt += 1
            # completions free their slot and memory
            still = []
            for h, rs, nbytes in inflight:
                if self.ex.done(h):
                    results = self.ex.finish(h)
                    t = self.clock() - t0
                    for r, res in zip(rs, results):
                        r.completed = t
                        r.result = res
                    in_use -= nbytes
                    done += len(rs)
                else:
                    still.append((h, rs, nbytes))
            inflight = still
            # admit first-come first-served into one batch while memory, the
            # batch limits and a free slot allow
            if waiting and self.ex.free_slots(len(inflight)):
                batch, rows, nbytes = [], 0, 0
                while waiting:
                    r = waiting[0]
                    if (len(batch) >= self.max_queries or rows + r.rows > self.max_rows or
                            in_use + nbytes + r.need_bytes > self.budget):
                        break
                    waiting.popleft()
                    r.admitted = now
                    batch.append(r)
                    rows += r.rows
                    nbytes += r.need_bytes
                if batch:
                    t = self.clock() - t0
                    for r in batch:
                        r.started = t
                    inflight.append((self.ex.start(batch), batch, nbytes))
                    in_use += nbytes
                    peak = max(peak, in_use)
                    batches += 1
                    continue
            if not inflight and not waiting and nxt < len(reqs):
                self.sleep(max(0.0, min(reqs[nxt].arrival - (self.clock() - t0), 0.001)))
            else:
                self.sleep(0)
        lat = [r.latency for r in reqs]
        rows = sum(r.rows for r in reqs)
        span = max(r.completed for r in reqs) - min(r.arrival for r in reqs)
        return TraceStats(len(reqs), rows, span, rows / span if span > 0 else float("inf"),
                          percentile(lat, 50) * 1e3, percentile(lat, 99) * 1e3, statistics.fmean(lat) * 1e3,
                          batches, peak)


class BatchExecutor:
    """Runs a batch of requests with vdf_batch_* on one of `slots` contexts,
    each with its own stream and a workspace reserved up front (so creating a
    batch never reallocates it)."""

    def __init__(self, device: int = 0, slots: int = 2, max_batch_rows: int = 1 << 27, tuning: Optional[dict] = None,
                 use_graph: bool = False, val_dtypes=None):
        """val_dtypes: with it, each slot keeps output arenas for
        max_batch_rows rows that every batch on the slot reuses (no
        allocation per batch; a request's result is then valid until its
        slot runs another batch).  Without it each batch allocates its own
        outputs, which stay valid as long as the result is held."""
        import torch

        from . import _lib
        self.torch = torch
        self._lib = _lib
        self.slots = [_lib.Context(device) for _ in range(slots)]
        self.streams = [torch.cuda.Stream(device=device) for _ in range(slots)]
        for c in self.slots:
            c.reserve(WS_BYTES_PER_ROW * max_batch_rows)
        self.free = list(range(slots))
        self.tuning = tuning
        self.use_graph = use_graph
        self.reserved_bytes = WS_BYTES_PER_ROW * max_batch_rows * slots
        self.outputs = None
        if val_dtypes is not None:
            dev = torch.device("cuda", device)
            self.outputs = [_lib.Batch.alloc_outputs(max_batch_rows, val_dtypes, dev) for _ in range(slots)]
            is_float = [dt in (torch.float64, torch.float32) for dt in val_dtypes]
            self.reserved_bytes += slots * max_batch_rows * out_bytes_per_row(is_float)

    def free_slots(self, inflight: int) -> bool:
        return bool(self.free)

    def start(self, requests):
        slot = self.free.pop(0)
        b = self._lib.Batch(self.slots[slot], [(r.key, r.vals) for r in requests], self.tuning,
                            None if self.outputs is None else self.outputs[slot])
        s = self.streams[slot]
        if self.use_graph:
            b.launch_graph(s)
        else:
            b.launch(s)
        ev = self.torch.cuda.Event()
        ev.record(s)
        return (slot, b, ev, len(requests))

    def done(self, h) -> bool:
        return h[2].query()

    def finish(self, h):
        slot, b, ev, nq = h
        ev.synchronize()
        self.slots[slot].check(self.streams[slot])
        self.free.append(slot)
        return [(b, q) for q in range(nq)]


class PerCallExecutor:
    """One request per library call (vdf_sort_groupby), one call at a time.

    With `reuse_outputs=(max_rows, key_dtype, val_dtypes)` every call writes
    into the same preallocated outputs (a result is then valid until the
    next call)."""

    def __init__(self, device: int = 0, reuse_outputs=None):
        import torch

        from . import _lib
        self.torch = torch
        self.ctx = _lib.Context(device)
        self.stream = torch.cuda.Stream(device=device)
        self.reserved_bytes = 0
        self.outputs = None
        if reuse_outputs is not None:
            rows, kdt, vdts = reuse_outputs
            dev = torch.device("cuda", device)
            k = torch.empty(rows, dtype=kdt, device=dev)
            vs = [torch.empty(rows, dtype=dt, device=dev) for dt in vdts]
            self.outputs = self.ctx.alloc_sort_groupby_outputs([k], vs, list(range(len(vs))))
            del k, vs
            is_float = [dt in (torch.float64, torch.float32) for dt in vdts]
            self.reserved_bytes = rows * (out_bytes_per_row(is_float) + 4 + 4 + 16)

    def free_slots(self, inflight: int) -> bool:
        return inflight == 0

    def start(self, requests):
        out = []
        for r in requests:
            g = self.ctx.sort_groupby([r.key], r.vals, agg_cols=list(range(len(r.vals))), stream=self.stream,
                                      outputs=self.outputs)
            out.append(g)
        return out

    def done(self, h) -> bool:
        return True

    def finish(self, h):
        return h


def request_bytes(rows: int, val_is_float: Sequence[bool]) -> int:
    return rows * out_bytes_per_row(val_is_float)


# ---------------------------------------------------------------------------
# The library's own request loop (vdf_server_*): the scheduler thread runs in
# C++; this is its Python view and a trace client for it.
# ---------------------------------------------------------------------------
def _server_lib():
    import ctypes as C

    from . import _lib

    lib = _lib.lib
    if getattr(lib, "_server_bound", False):
        return lib, _lib

    class Config(C.Structure):
        _fields_ = [("device", C.c_int32), ("hbm_budget_bytes", C.c_uint64), ("resident_bytes", C.c_uint64),
                    ("slots", C.c_uint32), ("max_batch_rows", C.c_uint64), ("max_batch_queries", C.c_uint32),
                    ("nvals", C.c_int32), ("val_dtypes", C.c_int32 * _lib.BATCH_MAX_VALS),
                    ("use_default_tuning", C.c_int32), ("small_rows", C.c_uint32), ("small_bits", C.c_int32),
                    ("seg_variant", C.c_int32), ("use_graph", C.c_int32)]

    class Result(C.Structure):
        _fields_ = [("n", C.c_uint64), ("n_groups", C.c_uint64), ("perm", C.c_void_p), ("group_keys", C.c_void_p),
                    ("group_count", C.c_void_p), ("aggs", _lib.vdf_agg_out * _lib.BATCH_MAX_VALS),
                    ("t_submit", C.c_double), ("t_start", C.c_double), ("t_done", C.c_double)]

    class Stats(C.Structure):
        _fields_ = [("batches", C.c_uint64), ("completed", C.c_uint64), ("queued", C.c_uint64),
                    ("in_use_bytes", C.c_uint64), ("max_in_use_bytes", C.c_uint64), ("fixed_bytes", C.c_uint64),
                    ("host_start_seconds", C.c_double), ("host_finish_seconds", C.c_double)]

    vp, st = C.c_void_p, C.c_int
    for name, res, args in [
        ("vdf_server_default_config", st, [C.POINTER(Config)]),
        ("vdf_server_create", st, [C.POINTER(Config), C.POINTER(vp)]),
        ("vdf_server_submit", st, [vp, C.POINTER(_lib.vdf_batch_query), C.POINTER(C.c_uint64)]),
        ("vdf_server_poll", st, [vp, C.c_uint64, C.POINTER(C.c_int32), C.POINTER(Result)]),
        ("vdf_server_wait", st, [vp, C.c_uint64, C.c_double, C.POINTER(Result)]),
        ("vdf_server_release", st, [vp, C.c_uint64]),
        ("vdf_server_read_stats", st, [vp, C.POINTER(Stats)]),
        ("vdf_server_inject_failure", st, [vp, C.c_int, C.c_uint32, C.c_int]),
        ("vdf_server_last_error", C.c_char_p, [vp]),
        ("vdf_server_destroy", None, [vp]),
    ]:
        f = getattr(lib, name)
        f.restype, f.argtypes = res, args
    lib._server_types = (Config, Result, Stats)
    lib._server_bound = True
    return lib, _lib


class _DevArray:
    """A device buffer seen through __cuda_array_interface__ (so torch can wrap it)."""

    def __init__(self, ptr, n, typestr):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": typestr, "data": (int(ptr or 0), False),
                                         "version": 3, "strides": None}


def _tensor(ptr, n, dtype):
    import numpy as np
    import torch
    typestr = np.dtype(str(dtype).replace("torch.", "")).str
    if n == 0 or not ptr:
        return torch.empty(0, dtype=dtype, device="cuda")
    return torch.as_tensor(_DevArray(ptr, n, typestr), device="cuda")


@dataclass
class ServedResult:
    perm: object
    n_groups: int
    keys: object
    count: object
    aggs: list
    t_submit: float
    t_start: float
    t_done: float


class Server:
    """vdf_server_*: the library's request loop (admission by HBM budget,
    continuous batching over `slots` in-flight batches)."""

    def __init__(self, device: int = 0, budget_bytes: float = 150e9, resident_bytes: int = 0, slots: int = 2,
                 max_batch_rows: int = 1 << 27, max_batch_queries: int = 4096, val_dtypes=(),
                 tuning: Optional[dict] = None, use_graph: bool = False):
        import ctypes as C

        import torch
        lib, _lib = _server_lib()
        Config, _, _ = lib._server_types
        self.lib, self._lib, self.C = lib, _lib, C
        c = Config()
        lib.vdf_server_default_config(C.byref(c))
        c.device = device
        c.hbm_budget_bytes = int(budget_bytes)
        c.resident_bytes = int(resident_bytes)
        c.slots = slots
        c.max_batch_rows = int(max_batch_rows)
        c.max_batch_queries = int(max_batch_queries)
        self.val_dtypes = list(val_dtypes)
        c.nvals = len(self.val_dtypes)
        for j, dt in enumerate(self.val_dtypes):
            c.val_dtypes[j] = _lib.TORCH_TO_VDF[dt]
        if tuning is not None:
            c.use_default_tuning = 0
            c.small_rows, c.small_bits, c.seg_variant = tuning["small_rows"], tuning["small_bits"], tuning["seg_variant"]
        c.use_graph = 1 if use_graph else 0
        h = C.c_void_p()
        stt = lib.vdf_server_create(C.byref(c), C.byref(h))
        if stt != _lib.OK:
            raise _lib.VdfError(stt, "vdf_server_create failed")
        self.handle = h
        self.torch = torch
        self._keys = {}

    def submit(self, key, vals) -> int:
        q = self._lib.vdf_batch_query()
        q.n = key.numel()
        q.key = self._lib._col(key)
        for j, v in enumerate(vals):
            q.vals[j] = v.data_ptr()
        rid = self.C.c_uint64()
        st = self.lib.vdf_server_submit(self.handle, self.C.byref(q), self.C.byref(rid))
        if st != self._lib.OK:
            raise self._lib.VdfError(st, "vdf_server_submit")
        self._keys[rid.value] = key.dtype
        return rid.value

    def _result(self, rid, r) -> ServedResult:
        kdt = self._keys[rid]
        aggs = []
        for j, dt in enumerate(self.val_dtypes):
            a = r.aggs[j]
            fl = dt in (self.torch.float64, self.torch.float32)
            g = r.n_groups
            aggs.append(self._lib.AggResult(_tensor(a.sum, g, self.torch.float64 if fl else self.torch.int64),
                                            None if fl else _tensor(a.sum_hi, g, self.torch.int64),
                                            _tensor(a.min, g, dt), _tensor(a.max, g, dt),
                                            _tensor(a.mean, g, self.torch.float64)))
        return ServedResult(_tensor(r.perm, r.n, self.torch.int32), int(r.n_groups), _tensor(r.group_keys, r.n_groups, kdt),
                            _tensor(r.group_count, r.n_groups, self.torch.int64), aggs, r.t_submit, r.t_start,
                            r.t_done)

    def poll(self, rid: int, want_result: bool = True):
        """(state, result): state 0 queued, 1 running, 2 done; the result
        (device tensors) once done, or just its timestamps with
        want_result=False."""
        _, Result, _ = self.lib._server_types
        state = self.C.c_int32()
        r = Result()
        st = self.lib.vdf_server_poll(self.handle, rid, self.C.byref(state), self.C.byref(r))
        if st != self._lib.OK:
            raise self._lib.VdfError(st, self.lib.vdf_server_last_error(self.handle).decode())
        if state.value != 2:
            return state.value, None
        if not want_result:
            return state.value, ServedResult(None, int(r.n_groups), None, None, [], r.t_submit, r.t_start, r.t_done)
        return state.value, self._result(rid, r)

    def wait(self, rid: int, timeout: float = 120.0) -> ServedResult:
        _, Result, _ = self.lib._server_types
        r = Result()
        st = self.lib.vdf_server_wait(self.handle, rid, timeout, self.C.byref(r))
        if st != self._lib.OK:
            raise self._lib.VdfError(st, self.lib.vdf_server_last_error(self.handle).decode())
        return self._result(rid, r)

    def release(self, rid: int):
        self._keys.pop(rid, None)
        st = self.lib.vdf_server_release(self.handle, rid)
        if st != self._lib.OK:
            raise self._lib.VdfError(st, "vdf_server_release")

    def inject_failure(self, where: str, count: int = 1, status: int = 4):
        """Test hook: the next `count` batches fail with `status` when they
        start ("start") or when their results are read back ("finish")."""
        st = self.lib.vdf_server_inject_failure(self.handle, {"start": 0, "finish": 1}[where], count, status)
        if st != self._lib.OK:
            raise self._lib.VdfError(st, "vdf_server_inject_failure")

    def stats(self) -> dict:
        _, _, Stats = self.lib._server_types
        s = Stats()
        self.lib.vdf_server_read_stats(self.handle, self.C.byref(s))
        return {k: getattr(s, k) for k, _ in Stats._fields_}

    def close(self):
        if getattr(self, "handle", None):
            self.lib.vdf_server_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def serve_trace(server: Server, requests: Sequence[Request], keep_results: bool = False,
                clock: Callable[[], float] = time.perf_counter) -> TraceStats:
    """Submits each request at its arrival time (seconds from the start),
    releases results as they complete (keep_results: after copying them to
    r.result), and returns the trace statistics with latencies on the
    server's clock."""
    reqs = sorted(requests, key=lambda r: (r.arrival, r.rid))
    ids = {}
    outstanding = []
    batches0 = int(server.stats()["batches"])
    t0 = clock()
    nxt = 0
    done = 0
    while done < len(reqs):
        now = clock() - t0
        while nxt < len(reqs) and reqs[nxt].arrival <= now:
            r = reqs[nxt]
            ids[r.rid] = server.submit(r.key, r.vals)
            outstanding.append(r)
            nxt += 1
        still = []
        for r in outstanding:
            state, res = server.poll(ids[r.rid], want_result=keep_results)
            if state == 2:
                r.started, r.completed = res.t_start, res.t_done
                r.admitted = res.t_submit
                if keep_results:  # copies: a slot's arenas are reused once released
                    r.result = ServedResult(res.perm.clone(), res.n_groups, res.keys.clone(), res.count.clone(),
                                            [server._lib.AggResult(*(None if x is None else x.clone()
                                                                     for x in (a.sum, a.sum_hi, a.min, a.max, a.mean)))
                                             for a in res.aggs], res.t_submit, res.t_start, res.t_done)
                server.release(ids[r.rid])
                done += 1
            else:
                still.append(r)
        outstanding = still
        if nxt < len(reqs) and not outstanding:
            time.sleep(max(0.0, min(reqs[nxt].arrival - (clock() - t0), 0.0005)))
    lat = [r.completed - r.admitted for r in reqs]
    rows = sum(r.rows for r in reqs)
    span = max(r.completed for r in reqs) - min(r.admitted for r in reqs)
    st = server.stats()
    return TraceStats(len(reqs), rows, span, rows / span if span > 0 else float("inf"),
                      percentile(lat, 50) * 1e3, percentile(lat, 99) * 1e3, statistics.fmean(lat) * 1e3,
                      int(st["batches"]) - batches0, int(st["max_in_use_bytes"]))
