"""CSV ingest on the GPU (vdf_csv_read / vdf_csv_read_host) against the
reference's own parser output (committed fixtures) and the oracle: column
types, names, row counts, bit-exact values and string bytes, over quoting,
CR / LF / CR LF line ends, empty fields, files without a final line end,
records and quoted fields that cross the 64-byte and 16 KB split boundaries,
decimal strings that need the exact decision, and the field-count errors."""
import json

import numpy as np
import pytest
import torch

import csv_gen
import oracle_bind as ob
import visondf_b200 as vdf
from test_csv import golden_cases, hard_strings, random_strings

pytestmark = pytest.mark.gpu


def read(ctx, data: bytes, device: bool, **kw):
    if device:
        t = torch.from_numpy(np.frombuffer(data, dtype=np.uint8).copy()).cuda() if data else \
            torch.empty(0, dtype=torch.uint8, device="cuda")
        return ctx.read_csv(t, **kw)
    return ctx.read_csv(data, **kw)


def assert_same(t, r: ob.CsvResult):
    assert r.bad_row < 0
    assert t.nrow == r.nrow
    assert t.types == r.types
    assert t.names == r.names
    for k in range(t.ncol):
        got = t.column(k)
        exp = r.columns[k]
        if isinstance(exp, list):
            assert got == exp, k
        else:
            assert got.tobytes() == exp.tobytes(), k


@pytest.mark.parametrize("device", [False, True])
def test_reference_fixtures(ctx, device):
    for data, m, ref in golden_cases():
        kw = dict(delim=m["delim"], header=m["header"], quote=m["quote"])
        if ref.bad_row >= 0:
            with pytest.raises(vdf.VdfError, match=f"column number problem at row {ref.bad_row}"):
                read(ctx, data, device, **kw)
            continue
        t = read(ctx, data, device, **kw)
        assert_same(t, ref)
        t.close()


@pytest.mark.parametrize("seed", range(8))
@pytest.mark.parametrize("crlf", [False, True])
def test_generated_files_match_the_oracle(ctx, seed, crlf):
    for header in (True, False):
        for tn in (True, False):
            q = "'" if seed % 2 else '"'
            data = csv_gen.make_csv(seed, [1, 9, 500, 20_000][seed % 4] + seed, crlf=crlf, empty_frac=0.05,
                                    header=header, trailing_newline=tn, quote=q)
            t = read(ctx, data, device=bool(seed % 2), header=header, quote=q)
            assert_same(t, ob.csv_read(data, header=header, quote=q))
            t.close()


def test_large_file_matches_the_oracle(ctx):
    data = csv_gen.make_csv(77, 400_000, kinds=["u", "d", "s", "d", "b", "c", "d", "u"], empty_frac=0.01,
                            quote='"')
    assert len(data) > 16 * 1024 * 64   # many split tiles
    t = read(ctx, data, True, quote='"')
    assert_same(t, ob.csv_read(data, quote='"'))


def test_quoted_line_ends_across_tiles(ctx):
    rng = np.random.default_rng(5)
    rows = ["id,text,v"]
    for i in range(3000):
        k = int(rng.integers(0, 400))
        body = "".join(rng.choice(list("ab,\n\r xy"), k))
        rows.append(f"{i},'{body}',{i}.5")
    data = ("\n".join(rows) + "\n").encode()
    t = read(ctx, data, True)
    r = ob.csv_read(data)
    assert r.nrow == 3000
    assert_same(t, r)


def test_decimals_that_need_the_exact_decision(ctx):
    strings = [s for s in random_strings(21, 30000) + hard_strings(22, 3000)
               if s and not any(c in s for c in ",'\n\r")]
    data = ("v\n0.5\n" + "\n".join(strings) + "\n").encode()
    t = read(ctx, data, True)
    r = ob.csv_read(data)
    assert t.types == ["d"]
    assert t.column(0).tobytes() == r.columns[0].tobytes()


def test_empty_and_header_only(ctx):
    for data, header, nrow in [(b"", True, 0), (b"a,b", True, 0), (b"a,b\n", True, 0), (b"a,b\r\n", True, 0),
                               (b"1,2", False, 1), (b"1,2\n", False, 1)]:
        t = read(ctx, data, True, header=header)
        assert t.nrow == nrow, data
        t.close()


def test_field_count_errors(ctx):
    with pytest.raises(vdf.VdfError, match="column number problem at row 1"):
        read(ctx, b"a,b\n1,2\n3\n", True)
    with pytest.raises(vdf.VdfError, match="column number problem at row 0"):
        read(ctx, b"a,b\n1,2,3\n", True)
    # past the first ten records (found by the parse kernel)
    body = "".join(f"{i},{i}\n" for i in range(5000)) + "1\n" + "".join(f"{i},{i}\n" for i in range(5000))
    with pytest.raises(vdf.VdfError, match="column number problem at row 5000"):
        read(ctx, ("a,b\n" + body).encode(), True)
    # the context stays usable
    t = read(ctx, b"a,b\n1,2.5\n", True)
    assert t.column(1).tolist() == [2.5]


def test_bad_arguments(ctx):
    with pytest.raises(vdf.VdfError):
        ctx.read_csv(b"a,b\n", delim=",", quote=",")
    with pytest.raises(vdf.VdfError):
        ctx.read_csv(b"a,b\n", delim="\n")
    buf = torch.zeros(64, dtype=torch.uint8, device="cuda")
    with pytest.raises(vdf.VdfError, match="16-byte aligned"):
        ctx.read_csv(buf[1:])


def test_columns_feed_the_sort(ctx):
    """Parsed columns stay in HBM and go straight into the sort + group-by."""
    data = csv_gen.make_csv(3, 50_000, kinds=["u", "d"], quote='"')
    t = read(ctx, data, True, quote='"')
    r = ob.csv_read(data, quote='"')
    key = t.tensor(0)
    assert key.dtype == torch.uint32
    perm = ctx.argsort([key])
    exp = np.argsort(r.columns[0], kind="stable")
    assert (perm.cpu().numpy().astype(np.int64) == exp).all()
    assert t.tensor(1).cpu().numpy().tobytes() == r.columns[1].tobytes()


def test_zero_copy_views_feed_the_group_by(ctx):
    """read_csv -> sort + group-by on the parsed columns in place (no copies)."""
    data = csv_gen.make_csv(11, 30_000, kinds=["u", "d", "d"], quote='"')
    t = read(ctx, data, True, quote='"')
    r = ob.csv_read(data, quote='"')
    key, val = t.view(0), t.view(1)
    assert key.dtype == torch.uint32 and val.dtype == torch.float64
    assert key.data_ptr() == t.device_column(0)["values"]
    gr = ctx.sort_groupby([key], [val], agg_cols=[0])
    og = ob.groupby([r.columns[0]], [r.columns[1]])
    assert gr.n_groups == og.n_groups
    assert (gr.keys[0].cpu().numpy() == og.keys[0]).all()
    assert (gr.count.cpu().numpy() == og.count).all()
    del t   # the views keep the table's memory alive
    assert (key.cpu().numpy() == r.columns[0]).all()


@pytest.mark.parametrize("device", [False, True])
def test_quoting_soup_matches_the_oracle(ctx, device):
    for seed in range(40):
        q = "'" if seed % 2 else '"'
        short = 5 + seed if seed % 8 == 3 else -1
        data = csv_gen.soup_csv(100 + seed, 200 + 37 * seed, 2 + seed % 6, quote=q, short_row=short)
        r = ob.csv_read(data, quote=q)
        if r.bad_row >= 0:
            with pytest.raises(vdf.VdfError, match=f"column number problem at row {r.bad_row} "):
                read(ctx, data, device, quote=q)
            continue
        t = read(ctx, data, device, quote=q)
        assert_same(t, r)
        t.close()


def test_close_waits_for_live_views(ctx):
    """close() while a view is alive must not hand the view's memory to the
    next table: the free waits for the last view."""
    data = csv_gen.make_csv(21, 40_000, kinds=["u", "d"], quote='"')
    t = read(ctx, data, True, quote='"')
    r = ob.csv_read(data, quote='"')
    v = t.view(1)
    t.close()
    with pytest.raises(ValueError, match="closed"):
        t.view(0)
    others = [read(ctx, csv_gen.make_csv(22 + i, 40_000, kinds=["d", "d"], quote='"'), True, quote='"')
              for i in range(3)]
    assert v.cpu().numpy().tobytes() == r.columns[1].tobytes()
    assert t.handle  # still held for the view
    del v
    import gc
    gc.collect()
    assert not t.handle  # the last view went: the table is freed
    for o in others:
        o.close()


def test_unsigned_columns_sort_alike_through_view_and_tensor(ctx):
    """uint32 values at and above 2^31 order the same whichever accessor
    feeds the sort (both give torch.uint32)."""
    rng = np.random.default_rng(9)
    vals = rng.integers(0, 1 << 32, 5_000, dtype=np.uint64)
    vals[:4] = [0, (1 << 31) - 1, 1 << 31, (1 << 32) - 1]
    data = ("k\n" + "\n".join(str(int(x)) for x in vals) + "\n").encode()
    t = read(ctx, data, True, quote='"')
    assert t.types == ["u"]
    a, b = t.view(0), t.tensor(0)
    assert a.dtype == b.dtype == torch.uint32
    exp = np.argsort(vals.astype(np.uint32), kind="stable").astype(np.uint32)
    for col in (a, b):
        assert (ctx.argsort([col]).cpu().numpy().view(np.uint32) == exp).all()
    del a
    t.close()
