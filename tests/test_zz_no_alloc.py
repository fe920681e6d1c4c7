"""The allocation-free argsort entry point (vdf_sort_argsort_noalloc).

It exists for callers that cannot allocate device memory at the moment they
sort; it keeps its scratch in a fixed device array inside the library.  Here
it is called through the C-ABI and compared, bit for bit, with the
context-based vdf_sort_argsort on two calls in a row (the second call runs on
the scratch the first one left behind).  This file is collected last so that
a run stopping at the first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import visondf_b200 as vdf
from gpu_util import bits_equal, dev, host
from visondf_b200 import _lib, datagen

pytestmark = pytest.mark.gpu

MAX_ROWS = 1 << 20  # VDF_NOALLOC_MAX_ROWS


def noalloc_sort(keys, order):
    n = keys[0].numel()
    perm = torch.empty(n, dtype=torch.int32, device="cuda")
    skeys = [torch.empty_like(k) for k in keys]
    stream = torch.cuda.current_stream().cuda_stream
    st = vdf.lib.vdf_sort_argsort_noalloc(n, _lib._cols(keys), len(keys), order, perm.data_ptr(),
                                          _lib._ptrs(skeys), stream)
    assert st == _lib.OK, vdf.lib.vdf_status_string(st)
    # a normal call leaves no device error bits
    err = C.c_uint32(0xFFFFFFFF)
    assert vdf.lib.vdf_sort_noalloc_error(C.byref(err), stream) == _lib.OK
    assert err.value == 0
    torch.cuda.synchronize()
    return perm, skeys


def test_noalloc_matches_context_sort_on_two_calls(ctx):
    rng = np.random.default_rng(2024)
    cases = [
        ([datagen.keys_for("zipf", np.int64, MAX_ROWS, rng), datagen.keys_for("few", np.int32, MAX_ROWS, rng)],
         vdf.ORDER_ASC),
        ([datagen.keys_for("uniform", np.float64, 300_001, rng)], vdf.ORDER_DESC_STABLE),
    ]
    for keys_h, order in cases:
        keys = [dev(k) for k in keys_h]
        perm, skeys = noalloc_sort(keys, order)
        ref_skeys = [torch.empty_like(k) for k in keys]
        ref_perm = ctx.argsort(keys, order=order, sorted_keys_out=ref_skeys)
        torch.cuda.synchronize()
        assert (host(perm) == host(ref_perm)).all()
        for a, b in zip(skeys, ref_skeys):
            assert bits_equal(host(a), host(b))


def test_noalloc_error_query_rejects_null():
    assert vdf.lib.vdf_sort_noalloc_error(None, None) == _lib.ERR_INVALID_ARG


def test_noalloc_rejects_more_rows_than_its_scratch_holds():
    k = torch.empty(1, dtype=torch.int64, device="cuda")
    cols = (_lib.vdf_col * 1)(_lib.vdf_col(k.data_ptr(), vdf.I64))
    st = vdf.lib.vdf_sort_argsort_noalloc(MAX_ROWS + 1, cols, 1, vdf.ORDER_ASC, k.data_ptr(), None, None)
    assert st == _lib.ERR_UNSUPPORTED
