"""GPU stable radix argsort through the C-ABI, bit-exact against the CPU
oracle (and, through the golden fixtures, the reference's own kernels)."""
import json
from pathlib import Path

import numpy as np
import pytest
import torch

import oracle_bind as ob
import visondf_b200 as vdf
from gpu_util import bits_equal, dev, host
from visondf_b200 import datagen

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"

# tile sizes are 4096 rows (4-byte keys) and 3072 rows (8-byte keys)
SIZES = [0, 1, 2, 31, 32, 33, 255, 256, 257, 3071, 3072, 3073, 4095, 4096, 4097, 100_003]
DTYPES = [np.int32, np.int64, np.uint32, np.uint64, np.float64, np.float32]
ORDERS = [vdf.ORDER_ASC, vdf.ORDER_DESC_STABLE, vdf.ORDER_DESC_REVERSE]


def check_sort(ctx, keys, order=vdf.ORDER_ASC):
    n = keys[0].size
    dk = [dev(k) for k in keys]
    skeys = [torch.empty_like(k) for k in dk]
    perm = ctx.argsort(dk, order=order, sorted_keys_out=skeys)
    ctx.check()
    exp = ob.argsort(keys, order)
    got = host(perm).view(np.uint32)
    assert got.shape == (n,)
    assert (got == exp).all(), f"first mismatch at {np.argmax(got != exp)}"
    for k, s in zip(keys, skeys):
        assert bits_equal(host(s), k[exp])


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("dt", DTYPES)
def test_single_key_sizes(ctx, n, dt):
    rng = np.random.default_rng(n * 7 + 1)
    check_sort(ctx, [datagen.keys_for("uniform", dt, n, rng)])


@pytest.mark.parametrize("dist", ["uniform", "few", "equal", "sorted", "reversed", "zipf", "small"])
@pytest.mark.parametrize("dt", [np.int32, np.int64, np.uint64, np.float64])
@pytest.mark.parametrize("order", ORDERS)
def test_single_key_distributions(ctx, dist, dt, order):
    if dist in ("zipf", "small") and np.dtype(dt).kind == "f":
        pytest.skip("integer-only distribution")
    rng = np.random.default_rng(hash((dist, np.dtype(dt).name, order)) & 0xFFFF)
    check_sort(ctx, [datagen.keys_for(dist, dt, 250_001, rng)], order)


@pytest.mark.parametrize("order", ORDERS)
@pytest.mark.parametrize("dts", [(np.int64, np.int32), (np.int32, np.int64, np.uint32), (np.float64, np.uint64),
                                 (np.uint32, np.uint32, np.uint32, np.int64)])
def test_multi_key(ctx, dts, order):
    rng = np.random.default_rng(len(dts) * 100 + order)
    n = 200_003
    dists = ["few", "zipf", "small", "uniform"]
    keys = [datagen.keys_for(dists[i] if np.dtype(t).kind != "f" else "few", t, n, rng) for i, t in enumerate(dts)]
    check_sort(ctx, keys, order)


def test_golden_reference_radix_fixtures(ctx):
    z = np.load(GOLDEN / "ref_sort_cases.npz")
    for c in range(int(z["n_cases"][0])):
        keys, i = [], 0
        while f"c{c}_k{i}" in z:
            keys.append(z[f"c{c}_k{i}"])
            i += 1
        for order, name in [(vdf.ORDER_ASC, "asc"), (vdf.ORDER_DESC_REVERSE, "rev")]:
            perm = ctx.argsort([dev(k) for k in keys], order=order)
            assert (host(perm).view(np.uint32) == z[f"c{c}_{name}"]).all(), (c, name)


def test_golden_internals_doc_example(ctx):
    d = json.loads((GOLDEN / "internals_sort_by.json").read_text())
    col = list(d["columns"])[d["sort_col_index"]]
    key = np.array(d["columns"][col], dtype=np.uint32)
    ids = np.array(d["columns"]["col1"])
    perm = host(ctx.argsort([dev(key)], order=vdf.ORDER_ASC)).view(np.uint32)
    assert list(ids[perm]) == d["asc_col1"]
    perm = host(ctx.argsort([dev(key)], order=vdf.ORDER_DESC_STABLE)).view(np.uint32)
    assert list(ids[perm]) == d["desc_col1"]


def test_workspace_variant_and_too_small(ctx):
    rng = np.random.default_rng(9)
    k = datagen.keys_for("uniform", np.int64, 50_000, rng)
    import ctypes as C
    need = vdf.lib.vdf_sort_workspace_bytes(k.size, (C.c_int32 * 1)(vdf.I64), 1)
    ws = torch.empty(need, dtype=torch.uint8, device="cuda")
    perm = ctx.argsort([dev(k)], workspace=ws)
    assert (host(perm).view(np.uint32) == ob.argsort([k])).all()
    with pytest.raises(vdf.VdfError) as ei:
        ctx.argsort([dev(k)], workspace=ws[: need // 2])
    assert ei.value.status == vdf._lib.ERR_WORKSPACE


def test_invalid_arguments(ctx):
    k = dev(np.arange(10, dtype=np.int32))
    with pytest.raises(vdf.VdfError):
        ctx.argsort([k], order=7)
    with pytest.raises(vdf.VdfError) as ei:
        ctx.argsort([k] * 5)
    assert ei.value.status == vdf._lib.ERR_INVALID_ARG


def test_gather_widths_and_alignment(ctx):
    rng = np.random.default_rng(4)
    for n in (1, 3, 4, 5, 1001, 65_537):
        perm = rng.permutation(n).astype(np.uint32)
        cols = [rng.integers(-9, 9, n).astype(np.int32), rng.standard_normal(n),
                rng.integers(0, 2**63, n, dtype=np.uint64), rng.standard_normal(n).astype(np.float32)]
        out = ctx.gather(dev(perm).view(torch.int32), [dev(c) for c in cols])
        for c, o in zip(cols, out):
            assert bits_equal(host(o), c[perm])
    # unaligned output views take the scalar path
    n = 1003
    perm = rng.permutation(n).astype(np.uint32)
    src = rng.standard_normal(n)
    big = torch.empty(n + 1, dtype=torch.float64, device="cuda")
    ctx.gather(dev(perm).view(torch.int32), [dev(src)], out=[big[1:]])
    assert bits_equal(host(big[1:]), src[perm])


def test_repeated_calls_reuse_workspace(ctx):
    rng = np.random.default_rng(21)
    for n in (10_000, 1_000_000, 5_000, 2_000_000):
        k = datagen.keys_for("zipf", np.int64, n, rng)
        perm = ctx.argsort([dev(k)])
        assert (host(perm).view(np.uint32) == ob.argsort([k])).all()


def test_every_kernel_variant_gives_identical_results(ctx):
    variants = vdf._lib.sort_variants()
    v32 = [v["index"] for v in variants if v["key_width"] == 4]
    v64 = [v["index"] for v in variants if v["key_width"] == 8]
    rng = np.random.default_rng(17)
    n = 300_007
    keys = [datagen.keys_for("zipf", np.int64, n, rng), datagen.keys_for("few", np.int32, n, rng),
            datagen.keys_for("uniform", np.uint32, n, rng)]
    exp = ob.argsort(keys)
    saved = ctx.get_sort_tuning()
    try:
        for a in v32:
            for b in v64:
                ctx.set_sort_tuning(a, b)
                assert ctx.get_sort_tuning() == (a, b)
                perm = ctx.argsort([dev(k) for k in keys])
                assert (host(perm).view(np.uint32) == exp).all(), (a, b)
        with pytest.raises(vdf.VdfError):
            ctx.set_sort_tuning(v64[0], v32[0])  # widths swapped
    finally:
        ctx.set_sort_tuning(*saved)


def test_autotune_picks_valid_variants(ctx):
    from visondf_b200 import autotune
    rng = np.random.default_rng(3)
    k = [dev(datagen.keys_for("uniform", np.int64, 200_000, rng)), dev(datagen.keys_for("uniform", np.int32, 200_000, rng))]
    saved = ctx.get_sort_tuning()
    try:
        res = autotune.tune(ctx, lambda: ctx.argsort(k), reps=1)
        assert ctx.get_sort_tuning() == (res["variant32"], res["variant64"])
        assert res["ms32"] and res["ms64"]
    finally:
        ctx.set_sort_tuning(*saved)


@pytest.mark.parametrize("order", [ob.ASC, ob.DESC_STABLE, ob.DESC_REVERSE])
def test_eleven_bit_digits_with_every_key_type(ctx, order):
    """Plans whose passes use 11-bit digits for one or both key widths
    (3 passes per 4-byte key, 6 per 8-byte key) against the oracle, over
    signed, unsigned and floating keys."""
    variants = vdf._lib.sort_variants()
    wide32 = [v["index"] for v in variants if v["key_width"] == 4 and v["digit_bits"] == 11]
    wide64 = [v["index"] for v in variants if v["key_width"] == 8 and v["digit_bits"] == 11]
    narrow32 = [v["index"] for v in variants if v["key_width"] == 4 and v["digit_bits"] == 8]
    narrow64 = [v["index"] for v in variants if v["key_width"] == 8 and v["digit_bits"] == 8]
    assert wide32 and wide64
    rng = np.random.default_rng(1100 + order)
    n = 2_000_003
    keys = [datagen.keys_for("few", np.float64, n, rng), datagen.keys_for("zipf", np.int32, n, rng),
            datagen.keys_for("uniform", np.uint64, n, rng), datagen.keys_for("uniform", np.float32, n, rng)]
    exp = ob.argsort(keys, order)
    saved = ctx.get_sort_tuning()
    try:
        for a, b in [(wide32[0], wide64[0]), (wide32[-1], wide64[-1]), (wide32[0], narrow64[0]),
                     (narrow32[0], wide64[-1])]:
            ctx.set_sort_tuning(a, b)
            perm = ctx.argsort([dev(k) for k in keys], order=order)
            assert (host(perm).view(np.uint32) == exp).all(), (a, b)
    finally:
        ctx.set_sort_tuning(*saved)


def _primary_keys(case, n, rng):
    if case == "distinct":
        k0 = rng.integers(np.iinfo(np.int64).min, np.iinfo(np.int64).max, size=n, dtype=np.int64, endpoint=True)
        assert np.unique(k0).size == n
    elif case == "ties":
        k0 = rng.integers(0, 1000, size=n).astype(np.int64)
    elif case == "one_pair":  # distinct except the last row repeats the first
        k0 = rng.permutation(n).astype(np.int64) * 3 - n
        k0[-1] = k0[0]
    else:  # all equal
        k0 = np.full(n, -7, dtype=np.int64)
    return k0


@pytest.mark.parametrize("case", ["distinct", "ties", "one_pair", "all_equal"])
@pytest.mark.parametrize("order", [ob.ASC, ob.DESC_STABLE, ob.DESC_REVERSE])
def test_multikey_modes_give_the_oracle_order(ctx, case, order):
    rng = np.random.default_rng(77 + order)
    n = 400_003
    k0 = _primary_keys(case, n, rng)
    k1 = rng.integers(-5, 5, size=n).astype(np.int32)
    v = rng.standard_normal(n)
    exp = ob.argsort([k0, k1], order)
    keys = [dev(k0), dev(k1)]
    try:
        for mode in (vdf._lib.MULTIKEY_LSD, vdf._lib.MULTIKEY_PRIMARY_FIRST):
            ctx.set_multikey_mode(mode)
            assert ctx.get_multikey_mode() == mode
            perm = ctx.argsort(keys, order=order)
            assert (host(perm).view(np.uint32) == exp).all(), (case, mode)
            s0, s1 = torch.empty_like(keys[0]), torch.empty_like(keys[1])
            perm = ctx.argsort(keys, order=order, sorted_keys_out=[s0, s1])
            assert (host(perm).view(np.uint32) == exp).all()
            assert bits_equal(host(s0), k0[exp]) and bits_equal(host(s1), k1[exp])
            if order == ob.ASC:
                gr = ctx.sort_groupby(keys, [dev(v)], agg_cols=[0])
                assert (host(gr.perm).view(np.uint32) == exp).all()
                og = ob.groupby([k0, k1], [v])
                assert gr.n_groups == og.n_groups and (host(gr.count) == og.count).all()
    finally:
        ctx.set_multikey_mode(vdf._lib.MULTIKEY_PRIMARY_FIRST)


def test_multikey_sort_under_graph_capture(ctx):
    """Inside stream capture the primary-key check (a host read-back) is
    skipped and the LSD sort over all keys is captured instead."""
    rng = np.random.default_rng(5)
    n = 300_000
    k0 = rng.integers(0, 50, size=n).astype(np.int64)
    k1 = rng.integers(0, 1 << 31, size=n).astype(np.int32)
    keys = [dev(k0), dev(k1)]
    exp = ob.argsort([k0, k1])
    perm = torch.empty(n, dtype=torch.int32, device="cuda")
    ctx.reserve(1 << 28)
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        ctx.argsort(keys, perm_out=perm, stream=s)  # warm
    torch.cuda.current_stream().wait_stream(s)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        ctx.argsort(keys, perm_out=perm)
    perm.fill_(-1)
    g.replay()
    torch.cuda.synchronize()
    ctx.check()
    assert (host(perm).view(np.uint32) == exp).all()
    del g


def _bulk_variants(width):
    return [v["index"] for v in vdf._lib.sort_variants() if v["tma"] and v["key_width"] == width]


@pytest.mark.parametrize("order", ORDERS)
def test_bulk_load_variants_match_the_oracle(ctx, order):
    """Variants whose tiles are staged by bulk copies (persistent grid, the
    next tile's copy overlapping the current one): full and partial last
    tiles, every pass input (raw column, buffers, keys read through the
    permutation) and a column that starts off the 16-byte grid, where the
    tiles load without bulk copies."""
    from visondf_b200 import _lib
    t32, t64 = _bulk_variants(4), _bulk_variants(8)
    assert t32 and t64
    rng = np.random.default_rng(300 + order)
    saved = ctx.get_sort_tuning()
    strategy = ctx.get_sort_strategy()
    try:
        ctx.set_sort_strategy(_lib.SORT_LSD, 0)
        for n in (1, 3071, 3072, 3073, 4096 * 3, 1_000_003):
            keys = [datagen.keys_for("uniform", np.uint64, n, rng), datagen.keys_for("zipf", np.int32, n, rng)]
            exp = ob.argsort(keys, order)
            for a, b in [(t32[0], t64[0]), (t32[-1], t64[-1]), (t32[0], 2), (1, t64[-1])]:
                ctx.set_sort_tuning(a, b)
                perm = ctx.argsort([dev(k) for k in keys], order=order)
                ctx.check()
                assert (host(perm).view(np.uint32) == exp).all(), (n, a, b)
        # a column viewed one element in: its tiles are not 16-byte aligned
        n = 500_001
        base = datagen.keys_for("uniform", np.int64, n + 1, rng)
        k = dev(base)[1:]
        assert k.data_ptr() % 16 != 0
        ctx.set_sort_tuning(t32[0], t64[0])
        perm = ctx.argsort([k], order=order)
        ctx.check()
        assert (host(perm).view(np.uint32) == ob.argsort([base[1:]], order)).all()
    finally:
        ctx.set_sort_tuning(*saved)
        ctx.set_sort_strategy(*strategy)


def test_bulk_load_variants_through_a_row_view_and_the_msd_plan(ctx):
    import ctypes as C

    from test_groupby_gpu import _host_args
    from visondf_b200 import _lib
    t32, t64 = _bulk_variants(4), _bulk_variants(8)
    rng = np.random.default_rng(31)
    n = 700_001
    saved = ctx.get_sort_tuning()
    strategy = ctx.get_sort_strategy()
    try:
        for st in (_lib.SORT_LSD, _lib.SORT_AUTO):
            ctx.set_sort_strategy(st, 0)
            for b in t64:
                ctx.set_sort_tuning(t32[0], b)
                k = datagen.keys_for("uniform", np.int64, n, rng)
                view = rng.permutation(n).astype(np.uint32)
                a, out = _host_args([k], [], [], n, perm_in=view)
                a.groupby = 0
                assert vdf.lib.vdf_sort_groupby_host(ctx.handle, C.byref(a), None) == 0
                assert (out["perm"] == view[np.argsort(k[view], kind="stable")]).all(), (st, b)
    finally:
        ctx.set_sort_tuning(*saved)
        ctx.set_sort_strategy(*strategy)
