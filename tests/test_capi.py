"""The C-ABI library, without a GPU: it loads, exports every function
include/vdf_capi.h declares, and its pure host functions (sizing, limits,
status strings) behave.  No compute call is made here."""
import ctypes as C
import subprocess

import numpy as np
import pytest

import visondf_b200 as vdf
from visondf_b200 import _lib


def test_library_exports_every_declared_symbol():
    declared = _lib.header_functions()
    assert len(declared) >= 15
    out = subprocess.run(["nm", "-D", "--defined-only", str(vdf.LIB_PATH)], capture_output=True, text=True,
                         check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    missing = [f for f in declared if f not in exported]
    assert not missing, missing
    for f in declared:
        assert hasattr(vdf.lib, f)


def test_abi_version_and_limits():
    assert vdf.lib.vdf_abi_version() == 1
    assert vdf.lib.vdf_max_rows() == (1 << 30) - 1


def test_status_strings():
    for s in range(7):
        assert vdf.lib.vdf_status_string(s)
    assert vdf.lib.vdf_status_string(99) == b"unknown status"


def test_sort_workspace_sizing():
    dts = (C.c_int32 * 2)(vdf.I64, vdf.I32)
    small = vdf.lib.vdf_sort_workspace_bytes(1000, dts, 2)
    big = vdf.lib.vdf_sort_workspace_bytes(100_000_000, dts, 2)
    assert 0 < small < big
    # the largest need over all kernel variants: ping-pong keys (8 B) + row
    # ids (4 B) = 24 B/row, plus two look-back status buffers of one word per
    # bin per tile (11-bit digits over 2048-row tiles: 8 B/row each)
    assert 24 * 100_000_000 <= big <= 41 * 100_000_000
    bad = (C.c_int32 * 1)(42)
    assert vdf.lib.vdf_sort_workspace_bytes(10, bad, 1) == 0
    assert vdf.lib.vdf_sort_workspace_bytes(10, dts, 0) == 0
    assert vdf.lib.vdf_sort_workspace_bytes(10, dts, 5) == 0


def test_groupby_workspace_sizing():
    assert vdf.lib.vdf_groupby_workspace_bytes(0, 2) == 256
    a = vdf.lib.vdf_groupby_workspace_bytes(1 << 20, 2)
    b = vdf.lib.vdf_groupby_workspace_bytes(1 << 20, 4)
    assert 256 < a <= b
    assert vdf.lib.vdf_groupby_workspace_bytes(10, 5) == 0


def test_null_context_is_rejected():
    assert vdf.lib.vdf_sort_argsort(None, 0, None, 1, 0, None, None, None) == _lib.ERR_INVALID_ARG
    assert vdf.lib.vdf_ctx_destroy(None) == _lib.ERR_INVALID_ARG
    assert vdf.lib.vdf_ctx_kernel_launches(None) == 0


def test_ctx_create_without_gpu_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = C.c_void_p()
    assert vdf.lib.vdf_ctx_create(0, C.byref(h)) == _lib.ERR_DEVICE
    assert not h.value


def test_dtype_maps_are_consistent():
    import torch
    for t, code in _lib.TORCH_TO_VDF.items():
        assert _lib.WIDTH[code] == torch.empty(0, dtype=t).element_size()


def test_variant_table_is_consistent():
    vs = _lib.sort_variants()
    assert vs and {v["key_width"] for v in vs} == {4, 8}
    for v in vs:
        assert v["threads"] % 32 == 0 and v["items"] > 0 and v["digit_bits"] in (8, 11) and v["match"] in (0, 1, 2, 3)
    assert vdf.lib.vdf_sort_variant_info(len(vs), None, None, None, None, None) == _lib.ERR_INVALID_ARG


def test_autotune_size_classes():
    from visondf_b200 import autotune
    assert autotune.size_class(1) == 0
    assert autotune.size_class(1024) == 10
    assert autotune.size_class(1025) == 11
    t = autotune.TuningTable({20: [1, 2, 0.1, 0.2]})
    assert t.lookup(1 << 20) == (1, 2)
    assert t.lookup(5) is None


def test_sort_plan_choice():
    info = _lib.sort_plan_info
    # 100M rows, int64 + int32 keys: two top-digit passes, 2048-row chunks
    assert info(100_000_000, [vdf.I64, vdf.I32]) == {"msd_passes": 2, "chunks": (100_000_000 + 2047) // 2048,
                                                       "dict": False}
    # wide chunks (8,192 rows) save the third top digit up to 201M rows
    assert info(200_000_000, [vdf.I64]) == {"msd_passes": 2, "chunks": (200_000_000 + 4095) // 4096, "dict": True}
    assert info(100_000_000, [vdf.I64])["chunks"] == (100_000_000 + 2047) // 2048
    assert info(300_000_000, [vdf.I64])["msd_passes"] == 3
    # 4-byte key 0: the LSD passes unless the MSD strategy is forced
    assert info(393_216, [vdf.I32], msd_min_rows=0)["msd_passes"] == 0
    assert info(10_000_000, [vdf.U32, vdf.I64])["msd_passes"] == 0
    assert info(393_216, [vdf.I32], strategy=_lib.SORT_MSD, msd_min_rows=0)["msd_passes"] == 1
    assert info(393_217, [vdf.I32], strategy=_lib.SORT_MSD, msd_min_rows=0)["msd_passes"] == 2
    # below the row threshold, with three keys, or with the LSD strategy: LSD
    assert info(1000, [vdf.I64])["msd_passes"] == 0
    assert info(1000, [vdf.I64], msd_min_rows=0)["msd_passes"] == 1
    assert info(10_000_000, [vdf.I64, vdf.I32, vdf.I32])["msd_passes"] == 0
    assert info(10_000_000, [vdf.I64], strategy=_lib.SORT_LSD)["msd_passes"] == 0
    assert info(1, [vdf.I64], msd_min_rows=0)["msd_passes"] == 0


def test_dictionary_plan_choice():
    info = _lib.sort_plan_info
    # one key, at least the row threshold, the automatic strategy: tried first
    # from four times the row threshold (4 x 2^20 by default)
    assert info(200_000_000, [vdf.I32])["dict"] and info(4_194_304, [vdf.F64])["dict"]
    assert not info(4_194_303, [vdf.F64])["dict"]
    assert info(200_000_000, [vdf.I64])["msd_passes"] == 2  # its fallback when the values are many
    assert not info(1000, [vdf.I32])["dict"]
    assert info(1000, [vdf.I32], msd_min_rows=0)["dict"]
    assert not info(2_000_000, [vdf.I32, vdf.I32])["dict"]
    assert not info(2_000_000, [vdf.I32], strategy=_lib.SORT_LSD)["dict"]
    assert not info(2_000_000, [vdf.I32], strategy=_lib.SORT_MSD)["dict"]
    assert vdf.lib.vdf_sort_plan_tries_dict(10, None, 1, 0, 0) == -1


def test_group_tuning_bounds_without_a_context():
    assert vdf.lib.vdf_ctx_set_group_tuning(None, 10) == _lib.ERR_INVALID_ARG
    assert vdf.lib.vdf_ctx_get_group_tuning(None) == 0
