#!/usr/bin/env python
"""Benchmark of the B200 sort + group-by path.

Workload (one "step"): the 100,000,000-row two-key frame -- key1 int64 over
the full 64-bit range, key2 int32 Zipf(s=1.1) over 1,000,000 distinct values,
payload f64 N(0,1), int32 uniform and a uint64 row id -- is stably sorted by
(key1, key2), every payload column is gathered into sorted order, and the
frame is grouped by (key1, key2) with count/sum/min/max/mean of the f64 and
int32 payloads.  One vdf_sort_groupby call per step through the C-ABI.

  value  rows/s with the inputs resident in HBM (device-timed, CUDA events).
  e2e    the same call fed from pinned HOST buffers: every step copies the five
         input columns host->device, runs the call, and copies the result
         (permutation + the group table) device->host; issued from two host
         threads with a context and stream each, so one step's uploads overlap
         the other's downloads (e2e.single_stream: one call at a time).
  roofline   the dominant kernel's algorithmic bytes per launch / its average
             launch time (CUDA events around each launch, inside the timed
             region), against the measured HBM copy bandwidth.
  cpu_baseline   the reference's own radix kernels (+ the hash group-by restated
                 on the reference's map and hash) on the host cores, on a
                 10,000,000-row sample of the same workload.

  configs    the other configurations, timed like the headline with parity
             checks and the reference CPU path beside each: c1_ties (key1 from
             a 50M pool), c0 (1M rows, int32 key over 10,000 values), c2a
             (200M rows, 50M distinct int64 keys), c2b (200M rows, 16 int32
             keys: the dictionary plan).
  batched    4,096 independent sort + group-by queries (rows log-uniform
             1e3..1e7 scaled to a 2 GiB batch, int32/int64 keys, f64 + int64
             values) as one CUDA graph launch per batch (vdf_batch_*), autotuned,
             against one vdf_sort_groupby call per query.
  served     a Poisson request stream (rows lognormal, median 1e6) over a
             resident 100M-row table through the library's request loop
             (vdf_server_*: HBM-budget admission, continuous batching): capacity
             and p50/p99 latency at 50/70/90 % of batched capacity, against one
             vdf_sort_groupby call per request on the same traces; more_slots:
             the same server with three slots (capacity, 90 % load).
  unique_join  vdf_unique over 100M int64 keys and vdf_left_join_index of 100M
             left rows against 10M right keys, with the oracle's hash walks
             on a 10M-row sample as the CPU baseline.
  csv        read_csv of a ~1 GiB synthetic airline delay-cause table (the
             reference's read benchmark shape) from HBM and end to end from
             pinned host memory, against the reference's own parser.
  (all single-GPU, after the headline measurement; --sections selects them)

--gpus N (launched by torchrun for N > 1) runs N independent replicas, one per
GPU ("replicas only": the single-GPU path has no exchange step); value is all
rows processed / the slowest rank's time.

--impl reference times the reference CPU path alone (rank 0), each step a
bounded sample of the workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "rows/s & %HBM peak, 100M-row sort+group-by; served p99 and rows/s vs per-call"
UNIT = "rows/s"
WORKLOAD = ("two-key stable radix sort (key1 int64 full range, key2 int32 Zipf s=1.1 over 1M values) "
            "+ gather of 3 payload columns (f64, int32, uint64 row id) + group-by (key1, key2) "
            "count/sum/min/max/mean of the f64 and int32 payloads")
# Canonical algorithmic bytes per row (8-bit digits over the full key widths,
# u32 row ids, each pass reading and writing key + row id once): sort 344
# (key2 68, key1 220, key2 emit 12, payload gather 44) + group-by with G ~= N
# 108 (sorted keys 12 + values 12 read, 84 written per group).
SORT_BYTES_PER_ROW = 344
GROUPBY_BYTES_PER_ROW_G_EQ_N = 108


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def measured_peaks() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        rows = []
        try:
            for line in Path(self.path).read_text().splitlines():
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        finally:
            os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def cpu_info() -> str:
    try:
        out = subprocess.run(["lscpu"], capture_output=True, text=True).stdout
        for line in out.splitlines():
            if line.startswith("Model name:"):
                return line.split(":", 1)[1].strip()
    except FileNotFoundError:
        pass
    return "unknown"


def cpu_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def run_reference_sample(n_sample: int, cores: int):
    """One step of the reference CPU path on an n_sample-row frame; returns
    (seconds, kind, cores_used)."""
    sys.path.insert(0, str(ROOT / "tests"))
    import oracle_bind as ob
    from visondf_b200 import datagen

    f = datagen.frame_w1(n_sample)
    keys = [f["key1"], f["key2"]]
    pay = [f["f64"], f["i32"], f["rowid"]]
    if ob.ref_available():
        cores = max(1, min(cores, 32))  # the reference's tables hold MAX_THREADS = 32
        t0 = time.perf_counter()
        perm, pay_out = ob.ref_sort(keys, ob.ASC, cores=cores, payload=pay)
        ob.ref_groupby(keys, [f["f64"], f["i32"]], cores=cores)
        return time.perf_counter() - t0, "reference", cores
    t0 = time.perf_counter()
    perm = ob.argsort(keys)
    for p in pay:
        p[perm]
    ob.groupby(keys, [f["f64"], f["i32"]], sorted_groups=False)
    return time.perf_counter() - t0, "port", 1


def reference_arm(args, rank: int, world: int):
    if rank != 0:
        return
    cores = cpu_threads()
    times = []
    kind, used = "reference", cores
    for step in range(args.warmup + args.steps):
        dt, kind, used = run_reference_sample(args.ref_sample, cores)
        if step >= args.warmup:
            times.append(dt)
    sec = statistics.median(times)
    value = args.ref_sample / sec
    sample = (f"{args.ref_sample:,} rows of the same two-key workload per step (same generators), "
              f"sort + payload gather + group-by; host CPU: {cpu_info()}")
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "rows": args.ref_sample, "parallelism": f"{used} host threads"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": used, "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def c0_canonical_bytes(n: int, key_width: int, n_groups: int) -> int:
    """Canonical bytes of one one-key query (8-bit digits over the key, u32 row
    ids, f64 + int64 values): sort w + w*2(w+4) + payload gather 4 + 2*16;
    group-by reads keys + values once and writes per group key + count 8 +
    f64 32 + int 40."""
    w = key_width
    return n * (w + w * 2 * (w + 4) + 4 + 32 + w + 16) + n_groups * (w + 8 + 32 + 40)


def kernel_bytes(cls: str, n: int, key_w, gather_w, val_w, n_groups: int, val_float):
    """Algorithmic bytes of ONE launch of a kernel class (the canonical model's
    per-kernel terms): a radix pass reads and writes (key, u32 row id); the
    shared-memory finish reads key images + row ids and writes raw keys + the
    permutation; the payload gather reads the permutation once and each
    gathered column once and writes it once; the group-by emit reads the sorted
    keys and values and writes each group's record (keys, count 8, per float
    column sum/min/max/mean 32, per integer column sum128 16 + min/max 2w +
    mean 8); the reduce pass reads the sorted keys and values.  None: no
    model (histograms, scans, the pack)."""
    out = sum(key_w) + 8 + sum(32 if f else 16 + 2 * w + 8 for w, f in zip(val_w, val_float))
    return {"onesweep64": 2 * (8 + 4) * n, "onesweep32": 2 * (4 + 4) * n,
            "localsort": 2 * (key_w[0] + 4) * n,
            "gather": (4 + 2 * sum(gather_w)) * n if gather_w else None,
            "segemit": (sum(key_w) + sum(val_w)) * n + n_groups * out,
            "segreduce": (sum(key_w) + sum(val_w)) * n}.get(cls)


def roofline_from_profile(prof: dict, steps: int, n: int, key_w, gather_w, val_w, n_groups: int, val_float,
                          peak: float, peak_kind: str) -> dict:
    """The dominant kernel (most device time among the classes with a byte
    model): its algorithmic bytes per launch / average launch time (library
    CUDA events inside the timed region) against the HBM peak."""
    best = None
    for cls, (ms, cnt) in prof.items():
        b = kernel_bytes(cls, n, key_w, gather_w, val_w, n_groups, val_float)
        if b is None or not cnt or ms <= 0:
            continue
        if best is None or ms > best[1]:
            best = (cls, ms, cnt, b)
    if best is None:
        return None
    cls, ms, cnt, b = best
    avg = ms / cnt
    achieved = b / (avg / 1e3) / 1e9
    roof = {"bound": "hbm", "kernel": cls, "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_kind": peak_kind, "algorithmic_bytes_per_launch": b,
            "avg_launch_ms": avg, "launches_per_step": cnt / steps}
    if cls == "localsort":
        roof["note"] = ("the shared-memory finish moves only about its algorithmic bytes and is issue- and "
                        "latency-bound (ncu: about 49 % issue active, two CTAs per SM by shared memory and "
                        "registers), so HBM bandwidth is not what limits it")
    return roof


def group_parity_sample(gr, keys_h, vals_h, n_sample: int, seed: int) -> dict:
    """Exact per-group check of a random sample of groups of a device result
    (size-independent: any row count): the group's rows come from the group
    starts and the permutation; keys, counts and integer sum/min/max must be
    bit-exact, float sums within 1e-12 of the exact value (math.fsum), and the
    groups that pass only the condition-aware bound 1e-12 * sum|x| (cancelling
    sums) are counted apart."""
    import math

    import torch
    G = int(gr.n_groups)
    rng = np.random.default_rng(seed)
    gi = np.unique(rng.integers(0, G, size=n_sample)) if G > n_sample else np.arange(G)
    dgi = torch.from_numpy(gi).to(gr.count.device)
    pick = lambda t: t[dgi].cpu().numpy()  # noqa: E731
    starts = pick(gr.group_start).view(np.uint32).astype(np.int64)
    counts = pick(gr.count)
    idx = np.concatenate([np.arange(s0, s0 + c) for s0, c in zip(starts, counts)])
    rows = gr.perm[torch.from_numpy(idx).to(gr.perm.device)].cpu().numpy().view(np.uint32)
    gkeys = [pick(k) for k in gr.keys]
    aggs = []
    for v, vh in enumerate(vals_h):
        a = gr.aggs[v]
        if vh.dtype.kind == "f":
            aggs.append((pick(a.sum), None, pick(a.min), pick(a.max)))
        else:
            aggs.append((pick(a.sum), pick(a.sum_hi), pick(a.min), pick(a.max)))
    bad = {"keys": 0, "counts": int((counts <= 0).sum()), "int": 0, "float_min_max": 0, "float_cond": 0}
    plain_fail, worst = 0, 0.0
    o = 0
    for j in range(gi.size):
        r = rows[o:o + counts[j]]
        o += counts[j]
        for kh, gk in zip(keys_h, gkeys):
            if not (kh[r] == gk[j]).all():
                bad["keys"] += 1
        for vh, (sm, hi, mn, mx) in zip(vals_h, aggs):
            x = vh[r]
            if vh.dtype.kind == "f":
                exact = math.fsum(x.tolist())
                absum = math.fsum(np.abs(x).tolist())
                err = abs(float(sm[j]) - exact)
                if err > 1e-12 * max(absum, abs(exact)) + 1e-300:
                    bad["float_cond"] += 1
                if err > 1e-12 * abs(exact):
                    plain_fail += 1
                if exact:
                    worst = max(worst, err / abs(exact))
                if mn[j] != x.min() or mx[j] != x.max():
                    bad["float_min_max"] += 1
            else:
                exact = int(sum(int(t) for t in x))
                got = ((int(hi[j]) << 64) | (int(sm[j]) & ((1 << 64) - 1)))
                if got >= 1 << 127:
                    got -= 1 << 128
                if got != exact or int(mn[j]) != int(x.min()) or int(mx[j]) != int(x.max()):
                    bad["int"] += 1
    return {"groups_checked": int(gi.size), "rows_checked": int(idx.size), "bit_exact_failures": bad,
            "f64_plain_relative_failures": plain_fail, "f64_worst_relative_error": worst,
            "rule": "keys, counts, integer sum/min/max and f64 min/max bit-exact; f64 sums within 1e-12 of "
                    "math.fsum, groups passing only 1e-12 * sum|x| counted as plain-relative failures"}


def config_section(args, local_rank: int, name: str) -> dict:
    """One more configuration of the sort + gather + group-by pipeline, device-
    resident and timed like the headline (CUDA events around args.steps calls,
    library events per kernel class), with its canonical %HBM, the dominant
    kernel's roofline, a parity summary and the reference CPU path on the
    first rows of the same seeded inputs:
      c1_ties  the two-key frame with key1 drawn from 50M values (about two
               rows per key1 value, so key2 orders them)
      c0       1M rows, int32 key over 10,000 values, f64 + int64 values
      c2a      200M rows, int64 key over 50M values, lognormal f64 + int64 values
      c2b      200M rows, int32 key over 16 values, 90/10 skew, same values
    (--c2-rows sets the c2a / c2b row count, e.g. for a profiler capture of a
    smaller case)"""
    import torch

    import visondf_b200 as vdf
    from visondf_b200 import datagen

    sys.path.insert(0, str(ROOT / "tests"))
    import oracle_bind as ob

    dev = torch.device("cuda", local_rank)
    t0 = time.time()
    if name == "c1_ties":
        n = args.rows
        f = datagen.frame_w1(n, key1_pool=n // 2)
        knames, pnames, agg = ["key1", "key2"], ["f64", "i32", "rowid"], [0, 1]
        workload = (f"{n:,} rows: the two-key frame with key1 drawn from {n // 2:,} distinct full-range int64 "
                    f"values (about two rows per value, ordered by key2), same payload and group-by")
    elif name == "c0":
        n = 1_000_000
        f = datagen.frame_w0(n)
        knames, pnames, agg = ["key"], ["v1", "v2"], [0, 1]
        workload = ("1,000,000 rows, int32 key over 10,000 distinct values, f64 N(0,1) + int64 U[-1e9, 1e9]; "
                    "sort by key, group-by count/sum/min/max/mean of both")
    elif name == "c2a":
        n = args.c2_rows
        f = datagen.frame_w2a(n)
        knames, pnames, agg = ["key"], ["v1", "v2"], [0, 1]
        workload = (f"{n:,} rows, int64 key over 50,000,000 distinct values, f64 lognormal(0,1) + int64 "
                    "U[0, 2^40); sort, gather, group-by count/sum/min/max/mean")
    elif name == "c2b":
        n = args.c2_rows
        f = datagen.frame_w2b(n)
        knames, pnames, agg = ["key"], ["v1", "v2"], [0, 1]
        workload = (f"{n:,} rows, int32 key over 16 distinct values (two take 45 % each, 14 share 10 %), "
                    "f64 lognormal(0,1) + int64 U[0, 2^40); sort, gather, group-by")
    else:
        raise ValueError(name)
    log(f"[{name}] generated {n:,} rows in {time.time() - t0:.1f}s")
    keys = [torch.from_numpy(f[k]).to(dev) for k in knames]
    payload = [torch.from_numpy(f[k]).to(dev) for k in pnames]
    ctx = vdf.Context(local_rank)
    if args.section_tuning:
        ctx.set_sort_tuning(*args.section_tuning[:2])
        ctx.set_local_sort_variant(args.section_tuning[2])
    stream = torch.cuda.current_stream()
    outs = ctx.alloc_sort_groupby_outputs(keys, payload, agg, want_group_start=True)
    packed = ctx.pack_sort_groupby(keys, payload, agg, vdf.ORDER_ASC, True, outs, host_count=False)
    steps = args.steps * (10 if n <= 1_000_000 else 1)
    for _ in range(args.warmup):
        ctx.sort_groupby_packed(packed, stream)
    ctx.check(stream)
    st0 = ctx.sort_stats(stream)
    ctx.profile(True)
    ctx.profile_reset()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = ctx.kernel_launches
    e0.record(stream)
    for _ in range(steps):
        ctx.sort_groupby_packed(packed, stream)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    launches = (ctx.kernel_launches - l0) / steps
    prof = ctx.profile_read()
    ctx.profile(False)
    ctx.check(stream)
    st1 = ctx.sort_stats(stream)
    G = int(outs["ngroups_dev"].item())
    peak, peak_kind = measured_peaks()
    key_w = [k.element_size() for k in keys]
    gather_w = key_w[1:] + [p.element_size() for p in payload]
    val_w = [payload[i].element_size() for i in agg]
    val_float = [payload[i].dtype.is_floating_point for i in agg]
    if name == "c1_ties":
        canonical = (SORT_BYTES_PER_ROW + 24) * n + G * 84
    else:
        canonical = c0_canonical_bytes(n, key_w[0], G)
    roof = roofline_from_profile(prof, steps, n, key_w, gather_w, val_w, G, val_float, peak, peak_kind)
    res = {"workload": workload, "rows": n, "n_groups": G, "unit": UNIT, "steps": steps,
           "ms_per_step": ms, "value": n / (ms / 1e3), "hbm_frac_canonical": canonical / (ms / 1e3) / 1e9 / peak,
           "canonical_bytes": canonical, "gpu_launches_per_step": launches,
           "sort_plan": {**vdf._lib.sort_plan_info(n, [vdf._lib.TORCH_TO_VDF[k.dtype] for k in keys]),
                         "msd_sorts": st1["msd_sorts"] - st0["msd_sorts"],
                         "msd_fallbacks": st1["msd_fallbacks"] - st0["msd_fallbacks"]},
           "kernels": {k: {"ms_per_step": v[0] / steps, "launches_per_step": v[1] / steps}
                       for k, v in prof.items() if v[1]},
           "roofline": roof}
    if name == "c2b":
        res["hbm_frac_sort_free_20B"] = 20 * n / (ms / 1e3) / 1e9 / peak
    # parity: the whole group table against the oracle where that is quick
    # (c0: 1M rows; c2b: 16 groups), an exact check of sampled groups otherwise
    gr = vdf.GroupResult(G, outs["gkeys"], outs["count"], outs["aggs"], outs["gstart"], None, outs["perm"],
                         outs["skeys"], outs["pay"]).trimmed()
    keys_h = [f[k] for k in knames]
    vals_h = [f[pnames[i]] for i in agg]
    if name in ("c0", "c2b"):
        og = ob.groupby(keys_h, vals_h)
        ok = {"n_groups": og.n_groups == G,
              "keys": all((k.cpu().numpy() == o).all() for k, o in zip(gr.keys, og.keys)),
              "counts": bool((gr.count.cpu().numpy() == og.count).all())}
        plain = 0
        for v in range(len(vals_h)):
            a = gr.aggs[v]
            if vals_h[v].dtype.kind == "f":
                got = a.sum.cpu().numpy()
                err = np.abs(got - og.sum[v])
                ok[f"v{v}_sum_cond"] = bool((err <= 1e-12 * np.maximum(og.abs[v], np.abs(og.sum[v])) + 1e-300).all())
                plain += int(np.count_nonzero(err > 1e-12 * np.abs(og.sum[v])))
                ok[f"v{v}_min_max"] = bool((a.min.cpu().numpy() == og.min[v]).all() and
                                           (a.max.cpu().numpy() == og.max[v]).all())
            else:
                ok[f"v{v}_sum"] = bool((a.sum.cpu().numpy() == og.sum[v]).all() and
                                       (a.sum_hi.cpu().numpy() == og.sum_hi[v]).all())
                ok[f"v{v}_min_max"] = bool((a.min.cpu().numpy() == og.min[v]).all() and
                                           (a.max.cpu().numpy() == og.max[v]).all())
        res["parity"] = {"against": "oracle group-by of every row (exact 128-bit integer sums, long double "
                                    "Neumaier float sums)", "checks": ok, "all_ok": all(ok.values()),
                         "f64_plain_relative_failures": plain}
    else:
        res["parity"] = {"against": "exact sums of sampled groups", **group_parity_sample(
            gr, keys_h, vals_h, 2000, seed=17)}
    ctx.close()
    del keys, payload, outs, packed, gr
    torch.cuda.empty_cache()
    # the reference CPU path on the first rows of the same inputs
    if not args.no_cpu_baseline:
        m = min(n, args.ref_sample)
        ks = [np.ascontiguousarray(f[k][:m]) for k in knames]
        ps = [np.ascontiguousarray(f[k][:m]) for k in pnames]
        cores = cpu_threads()
        if ob.ref_available():
            cores = max(1, min(cores, 32))
            c0 = time.perf_counter()
            ob.ref_sort(ks, ob.ASC, cores=cores, payload=ps)
            ob.ref_groupby(ks, [ps[i] for i in agg], cores=cores)
            sec, kind = time.perf_counter() - c0, "reference"
        else:
            c0 = time.perf_counter()
            perm = ob.argsort(ks)
            for q in ps:
                q[perm]
            ob.groupby(ks, [ps[i] for i in agg], sorted_groups=False)
            sec, kind, cores = time.perf_counter() - c0, "port", 1
        res["cpu_baseline"] = {"value": m / sec, "unit": UNIT, "cores": cores, "kind": kind,
                               "sample": f"first {m:,} rows of the same inputs; host CPU: {cpu_info()}"}
    del f
    return res


def batched_section(args, local_rank: int) -> dict:
    """Many independent queries as one graph-launched batch, against the same
    queries run one library call each."""
    import numpy as np
    import torch

    import visondf_b200 as vdf
    from visondf_b200 import autotune, datagen

    dev = torch.device("cuda", local_rank)
    t0 = time.time()
    specs = datagen.batch_specs(nq=args.batch_queries, budget_bytes=args.batch_bytes)
    parts = [datagen.batch_query(s) for s in specs]
    # one resident buffer per column kind; each query's columns are slices of it
    cols = {}
    for name, pick in (("k32", lambda p: p[0] if p[0].dtype == np.int32 else None),
                       ("k64", lambda p: p[0] if p[0].dtype == np.int64 else None),
                       ("v1", lambda p: p[1]), ("v2", lambda p: p[2])):
        arrs = [a for a in (pick(p) for p in parts) if a is not None]
        cols[name] = torch.from_numpy(np.concatenate(arrs)).to(dev)
    off = {"k32": 0, "k64": 0, "v": 0}
    queries = []
    for key, v1, v2 in parts:
        n = key.size
        kk = "k32" if key.dtype == np.int32 else "k64"
        k = cols[kk][off[kk]:off[kk] + n]
        off[kk] += n
        queries.append((k, [cols["v1"][off["v"]:off["v"] + n], cols["v2"][off["v"]:off["v"] + n]]))
        off["v"] += n
    del parts
    rows = sum(int(k.numel()) for k, _ in queries)
    log(f"[batched] {len(queries)} queries, {rows:,} rows, generated in {time.time() - t0:.1f}s")
    ctx = vdf.Context(local_rank)
    stream = torch.cuda.current_stream()
    if args.no_batch_autotune:
        tuned = {"best": vdf._lib.default_batch_tuning(), "best_ms": float("nan"), "table": []}
    else:
        tuned = autotune.tune_batch(ctx, queries, reps=2)
    log(f"[batched] tuning: {tuned['best']} ({tuned['best_ms']:.2f} ms)")
    b = vdf.Batch(ctx, queries, tuned["best"])
    for _ in range(args.warmup):
        b.launch_graph(stream)
    ctx.check(stream)
    torch.cuda.synchronize()
    l0 = ctx.kernel_launches
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        b.launch_graph(stream)
    e1.record(stream)
    torch.cuda.synchronize()
    ctx.check(stream)
    ms = e0.elapsed_time(e1) / args.steps
    launches = (ctx.kernel_launches - l0) / args.steps
    ng = b.n_groups.cpu().tolist()
    canonical = sum(c0_canonical_bytes(int(k.numel()), k.element_size(), int(g)) for (k, _), g in zip(queries, ng))
    peak, _ = measured_peaks()
    info = b.info()
    # per-kernel-class split of one batch (plain launches with the library's
    # event profiler; the one-CTA-per-query kernel runs on a side stream and
    # is not in it), after the timed region
    ctx.profile(True)
    ctx.profile_reset()
    prof_reps = 3
    for _ in range(prof_reps):
        b.launch(stream)
    torch.cuda.synchronize()
    split = {k: round(v[0] / prof_reps, 4) for k, v in ctx.profile_read().items() if v[1]}
    ctx.profile(False)
    b.close()

    # one library call per query (vdf_sort_groupby, group count read back), one at a time
    per_call_q = queries if args.per_call_queries <= 0 else queries[:args.per_call_queries]
    for k, vs in per_call_q[:8]:
        ctx.sort_groupby([k], vs, agg_cols=[0, 1])
    torch.cuda.synchronize()
    c0 = time.perf_counter()
    for k, vs in per_call_q:
        ctx.sort_groupby([k], vs, agg_cols=[0, 1])
    torch.cuda.synchronize()
    pc_sec = time.perf_counter() - c0
    pc_rows = sum(int(k.numel()) for k, _ in per_call_q)
    ctx.close()
    del queries, cols
    torch.cuda.empty_cache()
    value = rows / (ms / 1e3)
    per_call = pc_rows / pc_sec
    return {
        "workload": f"{len(specs)} independent sort + group-by queries, rows log-uniform 1e3..1e7 scaled to a "
                    f"2 GiB batch (floor 1,000), int32/int64 keys 50/50, key cardinality log-uniform in "
                    f"[2, rows/2], f64 + int64 values",
        "queries": len(specs), "rows": rows, "value": value, "unit": UNIT, "ms_per_batch": ms,
        "launch": "one CUDA graph per batch (captured once, replayed)", "gpu_launches_per_batch": launches,
        "hbm_frac_canonical": canonical / (ms / 1e3) / 1e9 / peak, "canonical_bytes": canonical,
        "split": info, "kernel_ms": split, "tuning": tuned["best"], "tuning_ms": tuned["table"],
        "per_call": {"value": per_call, "unit": UNIT, "queries": len(per_call_q), "seconds": pc_sec,
                     "call": "vdf_sort_groupby per query, group count read back (host sync) after each"},
        "speedup_vs_per_call": value / per_call,
    }


def unique_join_section(args, local_rank: int) -> dict:
    """De-duplication (vdf_unique) of a 100M-row int64 column and left-join
    row matching (vdf_left_join_index) of 100M left rows against 10M right
    rows, device-resident, CUDA events around each call (count read back);
    the oracle's hash walks on a 10M / 1M-row sample as the CPU baseline (the
    reference's own de-duplication and join cannot run: the first calls a
    filter the reference does not define, the second does not compile)."""
    import numpy as np
    import torch

    import visondf_b200 as vdf

    dev = torch.device("cuda", local_rank)
    rng = np.random.default_rng(0xB200 + 16 * 5)
    n, n_right = args.rows, args.rows // 10
    ukey = torch.from_numpy(rng.integers(0, n // 2, size=n, dtype=np.int64)).to(dev)  # ~86 % distinct
    right = rng.integers(-(1 << 61), 1 << 61, size=n_right, dtype=np.int64) * 2  # even keys
    left = right[rng.integers(0, n_right, size=n)]
    left[rng.random(n) < 0.25] += 1  # odd: absent from the right side
    left_d, right_d = torch.from_numpy(left).to(dev), torch.from_numpy(right).to(dev)
    ctx = vdf.Context(local_rank)
    stream = torch.cuda.current_stream()

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            out = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / args.steps, out

    u_ms, (_, distinct) = timed(lambda: ctx.unique(ukey))
    j_ms, (_, matched) = timed(lambda: ctx.left_join_index(left_d, right_d))
    ctx.close()
    cpu = None
    if not args.no_cpu_baseline:
        sys.path.insert(0, str(ROOT / "tests"))
        import oracle_bind as ob
        s_n = min(n, 10_000_000)
        k_host = ukey[:s_n].cpu().numpy()
        t0 = time.perf_counter()
        ob.unique(k_host)
        u_cpu = s_n / (time.perf_counter() - t0)
        s_r = max(1, s_n // 10)
        t0 = time.perf_counter()
        ob.left_join(left[:s_n], right[:s_r])
        j_cpu = s_n / (time.perf_counter() - t0)
        cpu = {"unique_rows_per_s": u_cpu, "left_join_rows_per_s": j_cpu, "cores": 1, "kind": "port",
               "sample": f"{s_n:,} rows (left join: {s_n:,} x {s_r:,}); host CPU: {cpu_info()}"}
    del ukey, left_d, right_d
    torch.cuda.empty_cache()
    return {
        "workload": f"unique: {n:,} int64 keys drawn from [0, {n // 2:,}); left join: {n:,} left rows x "
                    f"{n_right:,} distinct right int64 keys (75 % of left rows present), first match",
        "unique": {"ms": u_ms, "rows_per_s": n / (u_ms / 1e3), "distinct": distinct},
        "left_join": {"ms": j_ms, "rows_per_s": n / (j_ms / 1e3), "matched": matched},
        "cpu_baseline": cpu,
    }


def csv_section(args, local_rank: int) -> dict:
    """CSV ingest (vdf_csv_read) of a ~1 GiB synthetic file shaped like the
    reference's read benchmark input (benchmarks/readf.cpp:9-21: readf of an
    airline delay-cause table, delimiter ',', quote '"', header on; its
    metric is MB/s of file bytes).  `device`: file bytes resident in HBM,
    CUDA events around each call (outputs allocated inside the call);
    `e2e`: file bytes in pinned host memory -> vdf_csv_read_host -> every
    column copied back to pinned host memory; CPU baseline: the reference's
    own record parser and fast_float (oracle/_ref) on a bounded sample, its
    per-column conversions on 4 threads as readf<0, 0, 4> asks (its
    multi-core record parser computes every chunk's end from the first
    chunk's, standard_parser_mt.inl:30-37, so only the single-core one runs)."""
    import numpy as np
    import torch

    import visondf_b200 as vdf
    from visondf_b200 import datagen

    dev = torch.device("cuda", local_rank)
    data = datagen.airline_csv(args.csv_bytes)
    nbytes = len(data)
    host = torch.from_numpy(np.frombuffer(data, dtype=np.uint8).copy()).pin_memory()
    dbuf = host.to(dev)
    ctx = vdf.Context(local_rank)
    stream = torch.cuda.current_stream()
    t = ctx.read_csv(dbuf, quote='"')
    nrow, types = t.nrow, "".join(t.types)
    out_bytes = sum((8 * nrow if ty == "d" else 4 * nrow if ty == "u" else nrow if ty == "b" else
                     8 * (nrow + 1) + t.device_column(k)["bytes"]) for k, ty in enumerate(t.types))
    t.close()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(args.warmup):
        ctx.read_csv(dbuf, quote='"').close()
    launches0 = ctx.kernel_launches
    dev_ms = []
    for _ in range(args.steps):
        torch.cuda.synchronize()
        e0.record(stream)
        tt = ctx.read_csv(dbuf, quote='"')
        e1.record(stream)
        torch.cuda.synchronize()
        dev_ms.append(e0.elapsed_time(e1))
        tt.close()
    launches = (ctx.kernel_launches - launches0) / max(1, args.steps)
    # end to end: pinned host bytes in, every column back in pinned host memory
    sink = torch.empty(out_bytes + 4096 * (t.ncol + 1), dtype=torch.uint8).pin_memory()

    def e2e_once():
        tt = ctx.read_csv(host.numpy(), quote='"')
        o = sink.data_ptr()
        for k, ty in enumerate(tt.types):
            dc = tt.device_column(k)
            if ty in "dub":
                w = {"d": 8, "u": 4, "b": 1}[ty]
                tt.copy_column(k, o)
                o += (w * nrow + 255) // 256 * 256
            else:
                tt.copy_column(k, o, o + (dc["bytes"] + 255) // 256 * 256)
                o += (dc["bytes"] + 255) // 256 * 256 + (8 * (nrow + 1) + 255) // 256 * 256
        tt.close()

    for _ in range(args.warmup):
        e2e_once()
    e2e_ms = []
    for _ in range(args.steps):
        torch.cuda.synchronize()
        e0.record(stream)
        e2e_once()
        e1.record(stream)
        torch.cuda.synchronize()
        e2e_ms.append(e0.elapsed_time(e1))
    ctx.close()
    del dbuf
    torch.cuda.empty_cache()
    cpu = None
    if not args.no_cpu_baseline:
        sys.path.insert(0, str(ROOT / "tests"))
        import oracle_bind as ob
        sample = data[: min(nbytes, 64 << 20)]
        sample = sample[: sample.rfind(b"\n") + 1]
        if ob.ref_available():
            sec = ob.ref_csv_seconds(sample, quote='"', cores=4, reps=2)
            kind = "reference"
        else:
            t0 = time.perf_counter()
            ob.csv_read(sample, quote='"')
            sec, kind = time.perf_counter() - t0, "port"
        cpu = {"value": len(sample) / sec / 1e9, "unit": "GB/s", "cores": 4 if kind == "reference" else 1,
               "kind": kind, "sample": f"first {len(sample) / 1e6:.1f} MB of the same file; host CPU: {cpu_info()}"}
    d_best, e_best = min(dev_ms), min(e2e_ms)
    algo = nbytes + out_bytes
    peak, peak_kind = measured_peaks()
    return {
        "workload": f"read_csv of a {nbytes / 1e6:.0f} MB synthetic airline delay-cause table "
                    f"({nrow:,} rows, 21 columns: 2 unsigned, 4 strings, 15 two-decimal numbers), ',' / '\"' / header",
        "bytes": nbytes, "rows": nrow, "types": types, "unit": "GB/s",
        "device": {"ms": d_best, "ms_median": float(np.median(dev_ms)), "value": nbytes / (d_best / 1e3) / 1e9,
                   "gpu_launches": launches},
        "e2e": {"ms": e_best, "value": nbytes / (e_best / 1e3) / 1e9, "h2d_bytes_per_step": nbytes,
                "d2h_bytes_per_step": out_bytes},
        "roofline": {"bound": "hbm", "algorithmic_bytes": algo, "achieved": algo / (d_best / 1e3) / 1e9,
                     "peak": peak, "peak_kind": peak_kind, "frac": algo / (d_best / 1e3) / 1e9 / peak,
                     "note": "file read once + columns written once; the parse is instruction-bound"},
        "cpu_baseline": cpu,
        "speedup_vs_cpu": (nbytes / (d_best / 1e3) / 1e9) / cpu["value"] if cpu else None,
        "e2e_speedup_vs_cpu": (nbytes / (e_best / 1e3) / 1e9) / cpu["value"] if cpu else None,
    }


def served_section(args, local_rank: int) -> dict:
    """Poisson request stream over resident columns: continuous batching with
    HBM-budget admission, against one library call per request."""
    import numpy as np
    import torch

    from visondf_b200 import datagen, serve

    dev = torch.device("cuda", local_rank)
    table_rows = args.served_table_rows
    f = datagen.frame_w0(n=table_rows, distinct=10_000)
    key = torch.from_numpy(f["key"]).to(dev)
    v1 = torch.from_numpy(f["v1"]).to(dev)
    v2 = torch.from_numpy(f["v2"]).to(dev)
    del f
    resident = table_rows * (4 + 8 + 8)
    budget = int(args.hbm_budget_gb * 1e9)
    max_rows = 1 << 27
    per_row_out = serve.out_bytes_per_row([True, False])
    rng = np.random.default_rng(datagen.seed(4, 9))

    def make_trace(rate, nreq, seed_col):
        specs = datagen.stream_specs(nreq, rate, seed_col=seed_col)
        reqs = []
        for i, s in enumerate(specs):
            n = min(s["n"], table_rows)
            o = int(rng.integers(0, table_rows - n + 1))
            reqs.append(serve.Request(rid=i, arrival=s["t"], rows=n, key=key[o:o + n],
                                      vals=[v1[o:o + n], v2[o:o + n]], need_bytes=n * per_row_out))
        return reqs

    # batched: the library's request loop (C++ scheduler thread, two batches
    # in flight); per call: one vdf_sort_groupby per request, one at a time,
    # into preallocated outputs
    vdts = [torch.float64, torch.int64]
    server = serve.Server(local_rank, budget_bytes=budget, resident_bytes=resident, slots=2,
                          max_batch_rows=max_rows, val_dtypes=vdts)
    per_call_ex = serve.PerCallExecutor(local_rank, reuse_outputs=(table_rows, torch.int32, vdts))
    per_call_ex.ctx.reserve(serve.WS_BYTES_PER_ROW * table_rows)

    def run(which, reqs):
        if which == "batched":
            st = serve.serve_trace(server, reqs)
        else:
            loop = serve.Loop(per_call_ex, budget, resident + per_call_ex.reserved_bytes, max_batch_rows=max_rows,
                              max_batch_queries=1)
            st = loop.run(reqs)
        for r in reqs:
            r.result = None
        return st

    nreq = args.served_requests
    # warm both paths (kernels, workspaces, allocator pools)
    run("batched", make_trace(1e9, 64, 7))
    run("per_call", make_trace(1e9, 16, 7))
    torch.cuda.synchronize()
    # capacity: every request waiting at t = 0
    cap_b = run("batched", make_trace(1e12, nreq, 0))
    cap_p = run("per_call", make_trace(1e12, nreq, 0))
    mean_rows = cap_b.rows / cap_b.requests
    rates = []
    for frac in args.served_fractions:
        rate = frac * cap_b.rows_per_s / mean_rows
        sb = run("batched", make_trace(rate, nreq, 1))
        sp = run("per_call", make_trace(rate, nreq, 1))
        rates.append({"fraction_of_batched_capacity": frac, "requests_per_s": rate,
                      "offered_rows_per_s": rate * mean_rows, "batched": sb.as_dict(), "per_call": sp.as_dict()})
    server_stats = server.stats()
    server.close()
    # the same server with three slots (three batches in flight): capacity
    # and the 90 % load point
    slots_more = None
    if args.served_slots_more > 2:
        more = serve.Server(local_rank, budget_bytes=budget, resident_bytes=resident, slots=args.served_slots_more,
                            max_batch_rows=max_rows, val_dtypes=vdts)
        server = more
        run("batched", make_trace(1e9, 64, 7))
        cap_m = run("batched", make_trace(1e12, nreq, 0))
        rate = 0.9 * cap_b.rows_per_s / mean_rows
        sm = run("batched", make_trace(rate, nreq, 1))
        slots_more = {"slots": args.served_slots_more, "capacity_rows_per_s": cap_m.rows_per_s,
                      "speedup": cap_m.rows_per_s / cap_p.rows_per_s, "at_0.9_of_two_slot_capacity": sm.as_dict(),
                      "fixed_bytes": more.stats()["fixed_bytes"]}
        more.close()
    del key, v1, v2
    torch.cuda.empty_cache()
    return {
        "workload": f"Poisson arrivals, {nreq} requests per trace, rows lognormal (median 1e6, sigma 1.0, cap 1e8), "
                    f"int32 key over min(10,000, rows) values + f64 + int64 values, slices of a resident "
                    f"{table_rows:,}-row table; sort + group-by count/sum/min/max/mean per request",
        "hbm_budget_bytes": budget, "resident_bytes": resident, "slots": 2,
        "batched_impl": "vdf_server_* (C++ scheduler thread: admission by HBM budget, continuous batching, "
                        "2 batches in flight)",
        "per_call_impl": "one vdf_sort_groupby call per request, one at a time, group count read back",
        "server_stats": server_stats,
        "capacity": {"batched_rows_per_s": cap_b.rows_per_s, "per_call_rows_per_s": cap_p.rows_per_s,
                     "speedup": cap_b.rows_per_s / cap_p.rows_per_s,
                     "batched": cap_b.as_dict(), "per_call": cap_p.as_dict()},
        "rates": rates,
        "more_slots": slots_more,
    }


def our_arm(args, rank: int, world: int, local_rank: int):
    import torch
    import torch.distributed as dist

    import visondf_b200 as vdf
    from visondf_b200 import datagen, replicas

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    n = args.rows
    t0 = time.time()
    f = datagen.frame_w1(n)
    log(f"[rank {rank}] generated {n:,} rows in {time.time() - t0:.1f}s")
    names = ["key1", "key2", "f64", "i32", "rowid"]
    host = {k: torch.from_numpy(f[k]).pin_memory() for k in names}
    del f
    d = {k: host[k].to(dev, non_blocking=True) for k in names}
    torch.cuda.synchronize()
    keys = [d["key1"], d["key2"]]
    payload = [d["f64"], d["i32"], d["rowid"]]
    agg_cols = [0, 1]
    ctx = vdf.Context(local_rank)
    stream = torch.cuda.current_stream()
    outs = ctx.alloc_sort_groupby_outputs(keys, payload, agg_cols)
    packed = ctx.pack_sort_groupby(keys, payload, agg_cols, vdf.ORDER_ASC, True, outs, host_count=False)

    def barrier():
        if world > 1:
            dist.barrier()

    # ---- autotune the radix-pass variants on this shape (untimed) ------------------
    from visondf_b200 import autotune
    if args.no_autotune:
        if args.variants:
            ctx.set_sort_tuning(*args.variants)
        v32, v64 = ctx.get_sort_tuning()
        tuned = {"variant32": v32, "variant64": v64, "ms32": {}, "ms64": {}}
    else:
        tuned = autotune.tune(ctx, lambda: ctx.sort_groupby_packed(packed, stream), reps=2)
    log(f"[rank {rank}] autotune: {tuned}")

    # ---- device-resident timing ------------------------------------------------
    for _ in range(args.warmup):
        ctx.sort_groupby_packed(packed, stream)
    ctx.check(stream)
    sstats0 = ctx.sort_stats(stream)
    ctx.profile(True)
    ctx.profile_reset()
    barrier()
    torch.cuda.synchronize()
    launches0 = ctx.kernel_launches
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clocks:
        ev0.record(stream)
        for _ in range(args.steps):
            ctx.sort_groupby_packed(packed, stream)
        ev1.record(stream)
        torch.cuda.synchronize()
    barrier()
    ms = ev0.elapsed_time(ev1) / args.steps
    launches = ctx.kernel_launches - launches0
    prof = ctx.profile_read()
    ctx.profile(False)
    ctx.check(stream)
    sstats = ctx.sort_stats(stream)
    n_groups = int(outs["ngroups_dev"].item())
    clk = clocks.summary()
    ms = replicas.max_over_ranks(ms, world, dev)
    value = replicas.whole_job_rate(n, world, ms)

    # ---- roofline of the dominant kernel ------------------------------------------
    peak, peak_kind = measured_peaks()
    roofline = roofline_from_profile(prof, args.steps, n, [8, 4], [4, 8, 4, 8], [8, 4], n_groups, [True, False],
                                     peak, peak_kind)
    tfile = ROOT / "profiles" / "traffic.json"
    roofline["traffic"] = None
    if tfile.exists():
        tj = json.loads(tfile.read_text())
        ent = tj.get(roofline["kernel"])
        if ent and ent.get("rows"):
            roofline["traffic"] = ent["bytes_per_launch"] * n / ent["rows"]
            roofline["traffic_source"] = (f"scaled from profiles/traffic.json: ncu dram__bytes_read.sum + "
                                          f"dram__bytes_write.sum of one {ent['rows']:,}-row launch")
    kernels = {k: {"ms_per_step": v[0] / args.steps, "launches_per_step": v[1] / args.steps}
               for k, v in prof.items() if v[1]}
    canonical = (SORT_BYTES_PER_ROW + GROUPBY_BYTES_PER_ROW_G_EQ_N) * n
    step_frac = canonical / (ms / 1e3) / 1e9 / peak

    # ---- end to end from host buffers -------------------------------------------
    # One vdf_sort_groupby_host call per step: the five input columns are copied
    # from pinned host memory to the device, the path runs, and the permutation
    # plus the group table come back to pinned host memory.
    e2e = None
    if not args.no_e2e:
        import ctypes as C
        from visondf_b200 import _lib
        h2d = sum(host[k].numel() * host[k].element_size() for k in names)
        pin = lambda dtype: torch.empty(n, dtype=dtype).pin_memory()  # noqa: E731

        def host_call(c, strm):
            """One vdf_sort_groupby_host call's argument block with its own
            pinned output buffers, on context c and stream strm."""
            hp = {"perm": pin(torch.int32), "gk1": pin(torch.int64), "gk2": pin(torch.int32), "cnt": pin(torch.int64),
                  "f_sum": pin(torch.float64), "f_min": pin(torch.float64), "f_max": pin(torch.float64),
                  "f_mean": pin(torch.float64), "i_sum": pin(torch.int64), "i_hi": pin(torch.int64),
                  "i_min": pin(torch.int32), "i_max": pin(torch.int32), "i_mean": pin(torch.float64)}
            hk = (_lib.vdf_col * 2)(_lib.vdf_col(host["key1"].data_ptr(), vdf.I64),
                                    _lib.vdf_col(host["key2"].data_ptr(), vdf.I32))
            hpay = (_lib.vdf_col * 3)(_lib.vdf_col(host["f64"].data_ptr(), vdf.F64),
                                      _lib.vdf_col(host["i32"].data_ptr(), vdf.I32),
                                      _lib.vdf_col(host["rowid"].data_ptr(), vdf.U64))
            hagg = (_lib.vdf_agg_out * 2)(
                _lib.vdf_agg_out(hp["f_sum"].data_ptr(), None, hp["f_min"].data_ptr(), hp["f_max"].data_ptr(),
                                 hp["f_mean"].data_ptr()),
                _lib.vdf_agg_out(hp["i_sum"].data_ptr(), hp["i_hi"].data_ptr(), hp["i_min"].data_ptr(),
                                 hp["i_max"].data_ptr(), hp["i_mean"].data_ptr()))
            hgk = (C.c_void_p * 2)(hp["gk1"].data_ptr(), hp["gk2"].data_ptr())
            hac = (C.c_int32 * 2)(0, 1)
            ng = C.c_uint64(0)
            ha = _lib.vdf_sort_groupby_args()
            ha.n, ha.keys, ha.nkeys, ha.order = n, hk, 2, vdf.ORDER_ASC
            ha.payload, ha.npayload = hpay, 3
            ha.perm_out = hp["perm"].data_ptr()
            ha.groupby, ha.agg_cols, ha.nagg, ha.aggs = 1, hac, 2, hagg
            ha.group_keys_out, ha.group_count_out = hgk, hp["cnt"].data_ptr()
            ha.n_groups_host = C.pointer(ng)
            keep = (hp, hk, hpay, hagg, hgk, hac)  # the structs point into these

            def step():
                c._check(vdf.lib.vdf_sort_groupby_host(c.handle, C.byref(ha), strm.cuda_stream),
                         "vdf_sort_groupby_host")
            return step, ng, keep

        # (1) one stream: each call's copies and kernels in turn
        step_a, ng, keep_a = host_call(ctx, stream)
        for _ in range(max(1, args.warmup)):
            step_a()
        torch.cuda.synchronize()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            step_a()
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        ems_single = replicas.max_over_ranks(e0.elapsed_time(e1) / args.steps, world, dev)
        g = int(ng.value)
        d2h = 4 * n + g * (8 + 4 + 8 + 4 * 8 + (8 + 8 + 4 + 4 + 8))

        # (2) two host threads, each with its own context and stream (the
        # library's rule for concurrent use), so one step's uploads run while
        # the other's results come back over the full-duplex link; the events
        # span both streams
        import threading
        ctx_b = vdf.Context(local_rank)
        stream_b = torch.cuda.Stream(device=dev)
        step_b, _, keep_b = host_call(ctx_b, stream_b)
        for _ in range(max(1, args.warmup)):
            step_b()
        torch.cuda.synchronize()
        barrier()
        k_a = (args.steps + 1) // 2
        k_b = args.steps - k_a
        e0, e1, eb = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record(stream)
        stream_b.wait_event(e0)
        worker = threading.Thread(target=lambda: [step_b() for _ in range(k_b)])
        worker.start()
        for _ in range(k_a):
            step_a()
        worker.join()
        eb.record(stream_b)
        stream.wait_event(eb)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        ems = replicas.max_over_ranks(e0.elapsed_time(e1) / args.steps, world, dev)
        ctx_b.close()
        del keep_a, keep_b
        e2e = {"value": replicas.whole_job_rate(n, world, ems), "unit": UNIT, "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "ms_per_step": ems,
               "call": "vdf_sort_groupby_host (pinned host buffers) from two host threads, one context and stream "
                       "each, consecutive steps overlapping",
               "single_stream": {"value": replicas.whole_job_rate(n, world, ems_single), "ms_per_step": ems_single,
                                 "call": "vdf_sort_groupby_host, one call at a time"}}

    # ---- CPU baseline (rank 0, one GPU only) -------------------------------------
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        sec, kind, used = run_reference_sample(args.ref_sample, cpu_threads())
        cpu = {"value": args.ref_sample / sec, "unit": UNIT, "cores": used, "kind": kind,
               "sample": f"{args.ref_sample:,} rows of the same workload (same generators), one step of "
                         f"sort + payload gather + group-by; host CPU: {cpu_info()}"}

    ctx.close()
    del d, outs, packed, keys, payload
    torch.cuda.empty_cache()
    args.section_tuning = (tuned["variant32"], tuned["variant64"], tuned.get("local", 0))
    sections = set(args.sections.split(","))
    batched = served = unique_join = csv_res = None
    configs = {}
    for name in ("c1_ties", "c0", "c2a", "c2b"):
        if world == 1 and name in sections:
            configs[name] = config_section(args, local_rank, name)
    if world == 1 and "batched" in sections:
        batched = batched_section(args, local_rank)
    if world == 1 and "served" in sections:
        served = served_section(args, local_rank)
    if world == 1 and "unique_join" in sections:
        unique_join = unique_join_section(args, local_rank)
    if world == 1 and "csv" in sections:
        csv_res = csv_section(args, local_rank)
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "rows": n, "n_groups": n_groups, "key_dtypes": ["int64", "int32"],
                       "payload_dtypes": ["float64", "int32", "uint64"], "parallelism": f"replicas x{world}",
                       "l2": "inputs (3.2 GB) larger than L2 (126 MB); no flush between steps"},
            "roofline": roofline,
            "hbm_frac_canonical": step_frac,
            "canonical_bytes_per_row": SORT_BYTES_PER_ROW + GROUPBY_BYTES_PER_ROW_G_EQ_N,
            "kernels": kernels,
            "sort_plan": {**__import__("visondf_b200._lib", fromlist=["x"]).sort_plan_info(n, [1, 0]),
                          "msd_sorts": sstats["msd_sorts"] - sstats0["msd_sorts"],
                          "msd_fallbacks": sstats["msd_fallbacks"] - sstats0["msd_fallbacks"]},
            "tuning": {"variant32": tuned["variant32"], "variant64": tuned["variant64"],
                       "local_sort_variant": tuned.get("local"), "ms_local": tuned.get("ms_local"),
                       "variants": __import__("visondf_b200._lib", fromlist=["x"]).sort_variants()},
            "gpu_launches": launches,
            "clocks": clk,
            "e2e": e2e,
            "cpu_baseline": cpu,
            "configs": configs,
            "batched": batched,
            "served": served,
            "unique_join": unique_join,
            "csv": csv_res,
        }
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--rows", type=int, default=100_000_000)
    ap.add_argument("--ref-sample", type=int, default=10_000_000)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true", help="keep the library's default kernel variants")
    ap.add_argument("--variants", type=int, nargs=2, metavar=("V32", "V64"),
                    help="with --no-autotune: radix-pass variant indices for 4- and 8-byte keys")
    ap.add_argument("--csv-bytes", type=int, default=1 << 30, help="size of the synthetic CSV file (csv section)")
    ap.set_defaults(section_tuning=None)
    ap.add_argument("--c2-rows", type=int, default=200_000_000,
                    help="rows of the c2a / c2b sections (200M: the configurations as stated)")
    ap.add_argument("--sections", default="c1_ties,c0,c2a,c2b,batched,served,unique_join,csv",
                    help="extra single-GPU measurements after the headline one: batched, served, unique_join "
                         "(comma list, 'none' for none)")
    ap.add_argument("--batch-queries", type=int, default=4096)
    ap.add_argument("--no-batch-autotune", action="store_true", help="batched section: the default tuning")
    ap.add_argument("--batch-bytes", type=int, default=2 << 30, help="batched section: key + value bytes of the batch")
    ap.add_argument("--per-call-queries", type=int, default=0, help="queries of the per-call baseline (0 = all)")
    ap.add_argument("--served-requests", type=int, default=400)
    ap.add_argument("--served-table-rows", type=int, default=100_000_000)
    ap.add_argument("--served-fractions", type=float, nargs="+", default=[0.5, 0.7, 0.9])
    ap.add_argument("--served-slots-more", type=int, default=3,
                    help="served section: also measure a server with this many slots (<= 2: skip)")
    ap.add_argument("--hbm-budget-gb", type=float, default=150.0)
    args = ap.parse_args()
    if args.warmup < 3:
        log("note: fewer than 3 warm-up steps; the timing rules ask for at least 3")
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        reference_arm(args, rank, world)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local_rank))
    try:
        our_arm(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
