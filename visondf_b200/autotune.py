"""Autotuner for the radix sort's kernel variants.

The library compiles the radix pass in several variants (key width, threads
per CTA, keys per thread, digit bits, warp digit-match method; see
vdf_sort_variant_info).  A context uses one variant per key width.  This
module times every variant on the caller's own workload shape and picks the
fastest per key width, keyed by a size class (power-of-two bucket of the row
count), so a serving loop can keep one choice per class.

Timing uses the library's per-launch CUDA-event profiler (vdf_ctx_profile),
so the 4-byte-key and 8-byte-key passes of one run are measured separately
and each width is tuned independently.  Variants differ in digit width (8 or
11 bits: 4 or 3 passes over a 4-byte key, 8 or 6 over an 8-byte key), so the
figure compared is the time of all of a width's passes in one run.
"""
from __future__ import annotations

import json
import math
from dataclasses import dataclass, field
from pathlib import Path
from typing import Callable, Optional

from . import _lib


def size_class(n: int) -> int:
    """Power-of-two bucket of a row count (0 for n <= 1)."""
    return 0 if n <= 1 else int(math.ceil(math.log2(n)))


@dataclass
class TuningTable:
    """Best (variant32, variant64) per size class."""

    entries: dict = field(default_factory=dict)  # size class -> [v32, v64, ms32, ms64]

    def lookup(self, n: int) -> Optional[tuple]:
        e = self.entries.get(size_class(n))
        return None if e is None else (e[0], e[1])

    def save(self, path: Path):
        Path(path).write_text(json.dumps({str(k): v for k, v in self.entries.items()}, indent=1) + "\n")

    @classmethod
    def load(cls, path: Path) -> "TuningTable":
        d = json.loads(Path(path).read_text())
        return cls({int(k): v for k, v in d.items()})


def tune(ctx: "_lib.Context", run: Callable[[], None], reps: int = 2) -> dict:
    """Times `run` (one sort or sort + group-by on the context) under every
    variant assignment and returns {"variant32": i, "variant64": j,
    "ms32": {i: ms per run}, "ms64": {j: ms per run}, "local": k,
    "ms_local": {k: ms per run}} (time of all radix passes over keys of that
    width in one run, and of the MSD-first sort's shared-memory finish);
    leaves the best tuning set on the context."""
    variants = _lib.sort_variants()
    v32 = [v["index"] for v in variants if v["key_width"] == 4]
    v64 = [v["index"] for v in variants if v["key_width"] == 8]
    ms32, ms64 = {}, {}
    saved = ctx.get_sort_tuning()
    # every key's passes run in the LSD mode and strategy, so both widths get
    # timed (the primary-key-first mode and the MSD-first plan skip passes)
    mode = ctx.get_multikey_mode()
    strategy = ctx.get_sort_strategy()
    ctx.set_multikey_mode(_lib.MULTIKEY_LSD)
    ctx.set_sort_strategy(_lib.SORT_LSD, strategy[1])
    try:
        run()  # warm the workspace and the kernels
        for i in range(max(len(v32), len(v64))):
            a, b = v32[i % len(v32)], v64[i % len(v64)]
            ctx.set_sort_tuning(a, b)
            run()
            ctx.profile(True)
            ctx.profile_reset()
            for _ in range(reps):
                run()
            prof = ctx.profile_read()
            ctx.profile(False)
            t32, c32 = prof["onesweep32"]
            t64, c64 = prof["onesweep64"]
            if c32:
                ms32[a] = min(ms32.get(a, math.inf), t32 / reps)
            if c64:
                ms64[b] = min(ms64.get(b, math.inf), t64 / reps)
    finally:
        ctx.set_multikey_mode(mode)
        ctx.set_sort_strategy(*strategy)
    best32 = min(ms32, key=ms32.get) if ms32 else saved[0]  # a width not timed keeps its choice
    best64 = min(ms64, key=ms64.get) if ms64 else saved[1]
    ctx.set_sort_tuning(best32, best64)
    # the shared-memory finish of the MSD-first plan (where the plan applies)
    ms_local = {}
    for k in (0, 1):
        ctx.set_local_sort_variant(k)
        run()
        ctx.profile(True)
        ctx.profile_reset()
        for _ in range(reps):
            run()
        t, c = ctx.profile_read()["localsort"]
        ctx.profile(False)
        if c:
            ms_local[k] = t / reps
    best_local = min(ms_local, key=ms_local.get) if ms_local else 0
    ctx.set_local_sort_variant(best_local)
    return {"variant32": best32, "variant64": best64, "ms32": ms32, "ms64": ms64, "local": best_local,
            "ms_local": ms_local}


def batch_candidates() -> list:
    """Tunings of the batched executor: the size-class boundary (largest
    query run by one CTA in shared memory: none, 2048, 4096 or 8192 rows),
    that kernel's digit width (4 or 8 bits) and the segmented radix-pass
    variant (digit width 8 or 11, 2048-4096-row tiles) for the larger
    queries."""
    segs = [v["index"] for v in _lib.batch_variants()]
    out = []
    for seg in segs:
        out.append({"small_rows": 0, "small_bits": 8, "seg_variant": seg})
        for small in (2048, 4096, 8192):
            for bits in (4, 8):
                out.append({"small_rows": small, "small_bits": bits, "seg_variant": seg})
    return out


def tune_batch(ctx: "_lib.Context", queries, reps: int = 2, candidates: Optional[list] = None) -> dict:
    """Times one batch of `queries` under every candidate tuning (graph
    launches, CUDA events) and returns {"best": tuning, "best_ms": ms,
    "table": [(tuning, ms), ...]}."""
    import torch

    stream = torch.cuda.current_stream()
    table = []
    for t in candidates or batch_candidates():
        b = _lib.Batch(ctx, queries, t)
        b.launch_graph(stream)  # capture + warm
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            b.launch_graph(stream)
        e1.record(stream)
        e1.synchronize()
        ctx.check(stream)
        table.append((dict(t), e0.elapsed_time(e1) / reps))
        b.close()
        del b
    best, best_ms = min(table, key=lambda x: x[1])
    return {"best": best, "best_ms": best_ms, "table": table}
