"""The pivot (vdf_pivot_host, the reference's pivots/pivot.hpp:5-128) on the
GPU against the CPU oracle's restatement: the same key orders (first
appearance) bit for bit, integer cells bit-exact (sums wrap in the value
type), f64 cells within 1e-12 of the cell's sum |x| (the oracle adds in row
order, the GPU sum is compensated)."""
import numpy as np
import pytest

import oracle_bind as ob
import visondf_b200 as vdf

pytestmark = pytest.mark.gpu


def run(ctx, cols, rows, vals):
    got = ctx.pivot_host(ob.string_column(cols), ob.string_column(rows), vals)
    exp = ob.pivot(cols, rows, vals)
    assert (got["colkey_row"] == exp.colkey_row).all()
    assert (got["rowkey_row"] == exp.rowkey_row).all()
    assert got["matrix"].shape == exp.matrix.shape
    if vals.dtype.kind == "f":
        absum = ob.pivot(cols, rows, np.abs(vals)).matrix
        err = np.abs(got["matrix"] - exp.matrix)
        assert (err <= 1e-12 * absum + 1e-300).all()
        plain = int(np.count_nonzero(err > 1e-12 * np.abs(exp.matrix)))
        print(f"f64 cells: plain-relative failures: {plain}")
    else:
        assert (got["matrix"] == exp.matrix).all()
    return got


def test_documented_example(ctx):
    cols = list("AAABBABBBAABBBB")
    rows = list("DDCCCDCDDCDCDCD")
    vals = np.array([3, 8, 0, 8, 3, 8, 3, 3, 8, 0, 8, 8, 0, 8, 3], np.float64)
    got = run(ctx, cols, rows, vals)
    assert got["matrix"].tolist() == [[27.0, 0.0], [14.0, 30.0]]


def random_keys(rng, n, pool, maxlen):
    words = []
    for i in range(pool):
        ln = int(rng.integers(0, maxlen + 1))
        words.append(bytes(rng.integers(97, 100, ln).astype(np.uint8)) + str(i % 7).encode() * (i % 3))
    words = list(dict.fromkeys(words))  # distinct
    return [words[j] for j in rng.integers(0, len(words), n)]


@pytest.mark.parametrize("dt", [np.int32, np.uint32, np.int64, np.uint64, np.float64])
@pytest.mark.parametrize("n,cpool,rpool", [(1, 1, 1), (1000, 3, 5), (50_000, 200, 40), (300_001, 40, 900)])
def test_random_frames(ctx, dt, n, cpool, rpool):
    rng = np.random.default_rng(n + cpool)
    cols = random_keys(rng, n, cpool, 12)
    rows = random_keys(rng, n, rpool, 70)  # some strings longer than 64 bytes
    if np.dtype(dt).kind == "f":
        vals = rng.standard_normal(n)
    else:
        info = np.iinfo(dt)
        vals = rng.integers(info.min // 2, info.max // 2, n, dtype=dt)  # cells wrap
    run(ctx, cols, rows, vals)


def test_keys_that_differ_in_their_last_byte_or_length(ctx):
    base = "x" * 40
    cols = [base, base + "a", base + "b", base[:-1], "", base + "a", ""] * 300
    rows = ["", "r", "r\0", "r", "", "s", "r\0"] * 300
    vals = np.arange(len(cols), dtype=np.int64)
    got = run(ctx, cols, rows, vals)
    assert got["matrix"].shape == (5, 4)


def test_bad_value_type_and_empty(ctx):
    with pytest.raises(vdf.VdfError):
        ctx.pivot_host(ob.string_column(["a"]), ob.string_column(["b"]), np.ones(1, np.float32))
    got = ctx.pivot_host(ob.string_column([]), ob.string_column([]), np.zeros(0, np.int32))
    assert got["matrix"].size == 0
