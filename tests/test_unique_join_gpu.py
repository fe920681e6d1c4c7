"""De-duplication (vdf_unique) and left-join row matching
(vdf_left_join_index) on the GPU against the oracle: bit-exact keep masks,
match indices and counts, over every key dtype, first and last
occurrence, and the edge cases (empty sides, one row, all-equal and
all-distinct keys, absent keys, -0.0 / +0.0 and NaN bit patterns)."""
import numpy as np
import pytest
import torch

import oracle_bind as ob
from gpu_util import dev, host

pytestmark = pytest.mark.gpu

DTYPES = [np.int32, np.int64, np.uint32, np.uint64, np.float64, np.float32]


def keys(dt, n, card, rng):
    if np.dtype(dt).kind == "f":
        pool = rng.standard_normal(max(1, card)).astype(dt)
        pool[: min(card, 4)] = np.array([-0.0, 0.0, np.nan, -np.inf], dtype=dt)[: min(card, 4)]
    else:
        info = np.iinfo(dt)
        pool = rng.integers(info.min, info.max, size=max(1, card), dtype=dt, endpoint=True)
    return pool[rng.integers(0, max(1, card), size=n)]


@pytest.mark.parametrize("dt", DTYPES)
@pytest.mark.parametrize("keep_last", [False, True])
@pytest.mark.parametrize("n,card", [(1, 1), (1000, 1), (4099, 37), (100_000, 100_000), (300_001, 20_000)])
def test_unique_matches_the_oracle(ctx, dt, keep_last, n, card):
    key = keys(dt, n, card, np.random.default_rng(n ^ card))
    keep, d = ctx.unique(dev(key), keep_last)
    ok, od = ob.unique(key, keep_last)
    assert d == od
    assert (host(keep) == ok).all()


def test_unique_empty_and_large(ctx):
    keep, d = ctx.unique(torch.empty(0, dtype=torch.int64, device="cuda"))
    assert d == 0 and keep.numel() == 0
    rng = np.random.default_rng(5)
    key = rng.integers(0, 3_000_000, size=8_000_000, dtype=np.int64)
    keep, d = ctx.unique(dev(key))
    ok, od = ob.unique(key)
    assert d == od and (host(keep) == ok).all()


@pytest.mark.parametrize("dt", DTYPES)
@pytest.mark.parametrize("method", [0, 1, 2])
@pytest.mark.parametrize("nl,nr,card", [(1, 1, 1), (5000, 1, 1), (20_000, 30_000, 7000), (100_000, 3, 3),
                                        (250_000, 400_000, 300_000), (60_000, 90_000, 500)])
def test_left_join_matches_the_oracle(ctx, dt, method, nl, nr, card):
    rng = np.random.default_rng(nl + 3 * nr + card)
    pool = keys(dt, card, card, rng)
    # about one left row in eight carries a key drawn outside the right side's pool
    left = pool[rng.integers(0, card, size=nl)]
    miss = rng.random(nl) < 0.125
    left[miss] = keys(dt, int(miss.sum()), 11, np.random.default_rng(nl))
    right = pool[rng.integers(0, card, size=nr)]
    match, m = ctx.left_join_index(dev(left), dev(right), method)
    om, omm = ob.left_join(left, right, method)
    assert m == omm
    assert (host(match).view(np.uint32) == om).all()


@pytest.mark.parametrize("method", [0, 1, 2])
def test_left_join_empty_sides(ctx, method):
    a = dev(np.array([3, 1, 3], np.int64))
    match, m = ctx.left_join_index(a, torch.empty(0, dtype=torch.int64, device="cuda"), method)
    assert m == 0 and (host(match).view(np.uint32) == 0xFFFFFFFF).all()
    match, m = ctx.left_join_index(torch.empty(0, dtype=torch.int64, device="cuda"), a, method)
    assert m == 0 and match.numel() == 0


def test_bad_join_method_is_rejected(ctx):
    import visondf_b200 as vdf
    with pytest.raises(vdf.VdfError):
        ctx.left_join_index(dev(np.arange(4, dtype=np.int64)), dev(np.arange(4, dtype=np.int64)), 3)


def test_signed_zero_and_nan_bits(ctx):
    key = np.array([0.0, -0.0, np.nan, 0.0, -0.0, np.nan, 2.5], dtype=np.float64)
    keep, d = ctx.unique(dev(key))
    assert d == 4 and host(keep).tolist() == [1, 1, 1, 0, 0, 0, 1]
    keep, d = ctx.unique(dev(key), keep_last=True)
    assert d == 4 and host(keep).tolist() == [0, 0, 0, 1, 1, 1, 1]
    match, m = ctx.left_join_index(dev(np.array([-0.0, 1.0, np.nan], np.float64)), dev(key), method=1)
    assert m == 2 and host(match).view(np.uint32).tolist() == [4, 0xFFFFFFFF, 5]
    left = np.array([-0.0, np.nan, -0.0, -0.0, 0.0], np.float64)
    match, m = ctx.left_join_index(dev(left), dev(key), method=2)  # k-th occurrence takes the k-th right row
    assert m == 4 and host(match).view(np.uint32).tolist() == [1, 2, 4, 0xFFFFFFFF, 0]


def test_mismatched_dtypes_are_rejected(ctx):
    import visondf_b200 as vdf
    with pytest.raises(vdf.VdfError):
        ctx.left_join_index(dev(np.arange(4, dtype=np.int64)), dev(np.arange(4, dtype=np.int32)))
