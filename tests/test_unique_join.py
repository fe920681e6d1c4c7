"""CPU: the oracle's de-duplication and left-join matching against a plain
Python restatement of the reference's set / map walks
(V/transform/transform_unique/transform_unique_mt.hpp:105-140,
V/transform/transform_left_join/transform_left_join_mt.hpp:172-205), keyed
by each element's raw bytes as the reference's string_view keys are."""
import numpy as np
import pytest

import oracle_bind as ob

DTYPES = [np.int32, np.int64, np.uint32, np.uint64, np.float64, np.float32]


def raw(a):
    return a.view(np.uint32 if a.dtype.itemsize == 4 else np.uint64).tolist()


def py_unique(key, keep_last):
    keep = np.zeros(key.size, np.uint8)
    seen = set()
    order = range(key.size - 1, -1, -1) if keep_last else range(key.size)
    for i, k in zip(order, (raw(key)[i] for i in order)):
        if k not in seen:
            seen.add(k)
            keep[i] = 1
    return keep, len(seen)


def py_left_join(left, right, method):
    if method == 2:  # Aligned: the k-th left occurrence takes the k-th right one
        rows, nxt = {}, {}
        for j, k in enumerate(raw(right)):
            rows.setdefault(k, []).append(j)
        out = []
        for k in raw(left):
            c = nxt.get(k, 0)
            if k in rows and c < len(rows[k]):
                out.append(rows[k][c])
                nxt[k] = c + 1
            else:
                out.append(0xFFFFFFFF)
        match = np.array(out, dtype=np.uint32)
        return match, int((match != 0xFFFFFFFF).sum())
    m = {}
    for j, k in enumerate(raw(right)):
        if method == 1 or k not in m:
            m[k] = j
    match = np.array([m.get(k, 0xFFFFFFFF) for k in raw(left)], dtype=np.uint32)
    return match, int((match != 0xFFFFFFFF).sum())


def keys(dt, n, card, rng):
    if np.dtype(dt).kind == "f":
        pool = rng.standard_normal(card).astype(dt)
        pool[: min(card, 4)] = np.array([-0.0, 0.0, np.nan, np.inf], dtype=dt)[: min(card, 4)]
    else:
        info = np.iinfo(dt)
        pool = rng.integers(info.min, info.max, size=card, dtype=dt, endpoint=True)
    return pool[rng.integers(0, card, size=n)]


@pytest.mark.parametrize("dt", DTYPES)
@pytest.mark.parametrize("keep_last", [False, True])
@pytest.mark.parametrize("n,card", [(0, 1), (1, 1), (257, 3), (5000, 4000), (3000, 1)])
def test_oracle_unique_matches_the_set_walk(dt, keep_last, n, card):
    key = keys(dt, n, card, np.random.default_rng(n + card))
    keep, d = ob.unique(key, keep_last)
    pk, pd = py_unique(key, keep_last)
    assert d == pd and (keep == pk).all()


@pytest.mark.parametrize("dt", DTYPES)
@pytest.mark.parametrize("method", [0, 1, 2])
@pytest.mark.parametrize("nl,nr,card", [(0, 5, 3), (7, 0, 3), (2000, 1500, 900), (100, 3000, 50)])
def test_oracle_left_join_matches_the_map_walk(dt, method, nl, nr, card):
    rng = np.random.default_rng(nl * 7 + nr)
    pool = keys(dt, card, card, rng)
    left = np.concatenate([pool[rng.integers(0, card, size=nl)], keys(dt, 3, 3, rng)])[:nl]
    right = pool[rng.integers(0, card, size=nr)]
    match, m = ob.left_join(left, right, method)
    pm, pmm = py_left_join(left, right, method)
    assert m == pmm and (match == pm).all()


def test_negative_zero_and_nan_bits_are_distinct_keys():
    key = np.array([0.0, -0.0, np.nan, 0.0, -0.0, np.nan], dtype=np.float64)
    keep, d = ob.unique(key)
    assert d == 3 and keep.tolist() == [1, 1, 1, 0, 0, 0]
    match, m = ob.left_join(np.array([-0.0, 1.0], np.float64), key)
    assert m == 1 and match.tolist() == [1, 0xFFFFFFFF]
