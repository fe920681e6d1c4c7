"""Seeded synthetic frames for the sort + group-by workloads.

There is no public dataset for this path; every input is synthetic.  The
seed of column c of workload w is 0xB200 + 16*w + c.  All generators return
numpy arrays on the host (the benchmark pins and uploads them; tests compare
GPU results with the CPU oracle on the same arrays).

  w0  small frame: N=1,000,000; int32 key uniform over 10,000 distinct random
      int32 (negatives included); f64 value N(0,1); int64 value U[-1e9, 1e9].
  w1  two-key frame: N=100,000,000; key1 int64 = 64 random bits; key2 int32
      Zipf(s=1.1) over 1,000,000 ranks (inverse-CDF table), rank r mapped to a
      fixed random distinct int32; payload f64 N(0,1), int32 uniform, uint64
      row id (= original row index).
  w2a group-by frame: N=200,000,000; int64 key uniform over a pool of
      50,000,000 distinct random int64; f64 lognormal(0,1); int64 U[0, 2^40).
  w2b same values; int32 key from 16 distinct random int32 with a 90/10 skew:
      2 hot keys take 45% of the rows each, the other 14 share 10%.
  w3  batch of independent queries (the w0 schema): row counts log-uniform in
      [1e3, 1e7], then all scaled by one factor so the batch holds a byte
      budget (2 GiB of key + value bytes), floored at 1,000 rows; key int32 or
      int64 (50/50); key cardinality log-uniform in [2, rows/2], drawn from a
      per-query pool of distinct random values.
  w4  served stream: Poisson arrivals; rows lognormal (median 1e6, sigma 1.0)
      capped at 1e8; the w0 schema (int32 key over min(10,000, rows) distinct
      values, f64 N(0,1) and int64 U[-1e9, 1e9] values).
"""
from __future__ import annotations

import numpy as np

SEED_BASE = 0xB200


def seed(workload: int, column: int) -> int:
    return SEED_BASE + 16 * workload + column


def distinct_pool(rng: np.random.Generator, size: int, dtype) -> np.ndarray:
    """`size` distinct random values of an integer dtype (full range)."""
    info = np.iinfo(dtype)
    out = np.empty(0, dtype=dtype)
    while out.size < size:
        extra = rng.integers(info.min, info.max, size=int((size - out.size) * 1.1) + 16, dtype=dtype,
                             endpoint=True)
        out = np.unique(np.concatenate([out, extra]))
    rng.shuffle(out)
    return out[:size]


def zipf_ranks(rng: np.random.Generator, n: int, ranks: int, s: float) -> np.ndarray:
    """n draws of a Zipf(s) rank in [0, ranks) by inverse-CDF table lookup."""
    w = np.arange(1, ranks + 1, dtype=np.float64) ** (-s)
    cdf = np.cumsum(w)
    cdf /= cdf[-1]
    u = rng.random(n)
    r = np.searchsorted(cdf, u, side="right")
    return np.minimum(r, ranks - 1).astype(np.int64)


def frame_w0(n: int = 1_000_000, distinct: int = 10_000):
    rng = np.random.default_rng(seed(0, 0))
    pool = distinct_pool(rng, distinct, np.int32)
    key = pool[rng.integers(0, distinct, size=n)]
    v1 = np.random.default_rng(seed(0, 1)).standard_normal(n)
    v2 = np.random.default_rng(seed(0, 2)).integers(-10**9, 10**9, size=n, dtype=np.int64, endpoint=True)
    return {"key": key, "v1": v1, "v2": v2}


def frame_w1(n: int = 100_000_000, ranks: int = 1_000_000, s: float = 1.1, key1_pool: int = 0):
    """The two-key frame; key1_pool > 0 draws key1 from that many distinct
    full-range values instead (the tie-heavy variant: key2 then decides the
    order of rows sharing key1)."""
    if key1_pool:
        r1 = np.random.default_rng(seed(1, 5))
        k1 = distinct_pool(r1, key1_pool, np.int64)[r1.integers(0, key1_pool, size=n)]
    else:
        k1 = np.random.default_rng(seed(1, 0)).integers(np.iinfo(np.int64).min, np.iinfo(np.int64).max, size=n,
                                                        dtype=np.int64, endpoint=True)
    rng2 = np.random.default_rng(seed(1, 1))
    pool = distinct_pool(rng2, ranks, np.int32)
    k2 = pool[zipf_ranks(rng2, n, ranks, s)]
    f = np.random.default_rng(seed(1, 2)).standard_normal(n)
    i = np.random.default_rng(seed(1, 3)).integers(np.iinfo(np.int32).min, np.iinfo(np.int32).max, size=n,
                                                   dtype=np.int32, endpoint=True)
    rowid = np.arange(n, dtype=np.uint64)
    return {"key1": k1, "key2": k2, "f64": f, "i32": i, "rowid": rowid}


def values_w2(n: int):
    v1 = np.exp(np.random.default_rng(seed(2, 1)).standard_normal(n))
    v2 = np.random.default_rng(seed(2, 2)).integers(0, 1 << 40, size=n, dtype=np.int64)
    return v1, v2


def frame_w2a(n: int = 200_000_000, distinct: int = 50_000_000):
    rng = np.random.default_rng(seed(2, 0))
    pool = distinct_pool(rng, distinct, np.int64)
    key = pool[rng.integers(0, distinct, size=n)]
    v1, v2 = values_w2(n)
    return {"key": key, "v1": v1, "v2": v2}


def frame_w2b(n: int = 200_000_000):
    rng = np.random.default_rng(seed(2, 3))
    pool = distinct_pool(rng, 16, np.int32)
    p = np.full(16, 0.10 / 14)
    p[:2] = 0.45
    key = pool[rng.choice(16, size=n, p=p)]
    v1, v2 = values_w2(n)
    return {"key": key, "v1": v1, "v2": v2}


def keys_for(dist: str, dtype, n: int, rng: np.random.Generator) -> np.ndarray:
    """Key columns for parity tests: uniform, few, equal, sorted, reversed, zipf, small."""
    if np.dtype(dtype).kind == "f":
        base = rng.standard_normal(n).astype(dtype)
        if dist == "few":
            base = np.array([-0.0, 0.0, -1.5, 2.25, np.inf, -np.inf], dtype=dtype)[rng.integers(0, 6, size=n)]
        elif dist == "equal":
            base = np.full(n, 3.5, dtype=dtype)
    else:
        info = np.iinfo(dtype)
        if dist in ("uniform", "sorted", "reversed"):
            base = rng.integers(info.min, info.max, size=n, dtype=dtype, endpoint=True)
        elif dist == "few":
            base = distinct_pool(rng, 7, dtype)[rng.integers(0, 7, size=n)]
        elif dist == "equal":
            base = np.full(n, info.max // 3, dtype=dtype)
        elif dist == "zipf":
            base = distinct_pool(rng, 1000, dtype)[zipf_ranks(rng, n, 1000, 1.1)]
        elif dist == "small":
            base = rng.integers(0, 300, size=n).astype(dtype)
        else:
            raise ValueError(dist)
    if dist == "sorted":
        base = np.sort(base, kind="stable")
    elif dist == "reversed":
        base = np.sort(base, kind="stable")[::-1].copy()
    return base


def batch_specs(nq: int = 4096, rows_lo: float = 1e3, rows_hi: float = 1e7, budget_bytes: int = 2 << 30,
                min_rows: int = 1000, seed_col: int = 0):
    """Query shapes of a w3 batch: list of dicts {n, dtype, card, seed}."""
    rng = np.random.default_rng(seed(3, seed_col))
    n = np.floor(10 ** rng.uniform(np.log10(rows_lo), np.log10(rows_hi), size=nq)).astype(np.int64)
    wide = rng.random(nq) < 0.5
    nbytes = n * (np.where(wide, 8, 4) + 16)
    s = min(1.0, budget_bytes / float(nbytes.sum()))
    n = np.maximum(min_rows, np.floor(n * s)).astype(np.int64)
    out = []
    for i in range(nq):
        hi = max(2.0, n[i] / 2)
        card = int(np.floor(10 ** rng.uniform(np.log10(2.0), np.log10(hi)))) if hi > 2 else 2
        out.append(dict(n=int(n[i]), dtype=np.int64 if wide[i] else np.int32, card=max(1, min(card, int(n[i]))),
                        seed=int(rng.integers(0, 2**62))))
    return out


def batch_query(spec: dict):
    """(key, v1 f64 N(0,1), v2 int64 U[-1e9, 1e9]) of one query shape."""
    rng = np.random.default_rng(spec["seed"])
    n, card = spec["n"], spec["card"]
    pool = distinct_pool(rng, card, spec["dtype"])
    key = pool[rng.integers(0, card, size=n)] if n else np.empty(0, spec["dtype"])
    v1 = rng.standard_normal(n)
    v2 = rng.integers(-10**9, 10**9, size=n, dtype=np.int64, endpoint=True)
    return key, v1, v2


def stream_specs(n_requests: int, rate_per_s: float, median_rows: float = 1e6, sigma: float = 1.0,
                 cap_rows: int = 100_000_000, seed_col: int = 0):
    """Request shapes of a w4 stream: list of dicts {t (arrival, s), n, dtype, card, seed}."""
    rng = np.random.default_rng(seed(4, seed_col))
    gaps = rng.exponential(1.0 / rate_per_s, size=n_requests)
    t = np.cumsum(gaps) - gaps[0]
    n = np.minimum(cap_rows, np.maximum(1, np.floor(rng.lognormal(np.log(median_rows), sigma, size=n_requests))))
    return [dict(t=float(t[i]), n=int(n[i]), dtype=np.int32, card=int(min(10_000, n[i])),
                 seed=int(rng.integers(0, 2**62))) for i in range(n_requests)]


def airline_csv(target_bytes: int = 1 << 30, seed_: int = 1, block_rows: int = 200_000) -> bytes:
    """A CSV file shaped like the reference's read benchmark input
    (benchmarks/readf.cpp:9, an airline delay-cause table: 21 columns -- year
    and month, a carrier code and name, an airport code and name, 15 counts
    and delay minutes with two decimals), synthetic and seeded: names with a
    comma come quoted with '"'.  One block of `block_rows` rows is generated
    and repeated up to about `target_bytes`; the header comes first."""
    rng = np.random.default_rng(seed_)
    n = block_rows
    carriers = np.array(["AA", "DL", "UA", "WN", "B6", "AS", "NK", "F9"])
    cnames = np.array(["Alpha Air Inc.", "Beta Air Lines Inc.", '"Gamma Air, Inc."', "Delta Wings Co."])
    airports = np.array(["AAA", "BBB", "CCC", "DDD", "EEE", "FFF", "GGG", "HHH"])
    anames = np.array(['"Aton, GA: Aton Municipal"', '"Bexley, IL: Bexley International"',
                       '"Corin, TX: Corin Regional"', '"Dover, CO: Dover Field"'])
    cols = [rng.integers(2003, 2025, n).astype(str), rng.integers(1, 13, n).astype(str),
            carriers[rng.integers(0, 8, n)], cnames[rng.integers(0, 4, n)],
            airports[rng.integers(0, 8, n)], anames[rng.integers(0, 4, n)]]
    for k in range(15):
        cols.append(np.char.mod("%.2f", np.round(rng.exponential(50.0 * (k + 1), n), 2)))
    rows = cols[0]
    for c in cols[1:]:
        rows = np.char.add(np.char.add(rows, ","), c)
    block = ("\n".join(rows.tolist()) + "\n").encode()
    header = ("year,month,carrier,carrier_name,airport,airport_name,"
              + ",".join(f"delay_{k}" for k in range(15)) + "\n").encode()
    return header + block * max(1, target_bytes // len(block))
