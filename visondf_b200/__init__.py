"""visondf_b200 -- VisonDF's sort + group-by hot path on NVIDIA B200 (sm_100a).

The product is libvdf_b200.so (C-ABI in include/vdf_capi.h) and the
header-only C++ dataframe layer in include/vison_b200/vison.hpp.  This
package is the Python view of the same library: a ctypes binding (`_lib`:
Context, Batch, CsvTable), the request loop (`serve`), the autotuner
(`autotune`), replica plumbing (`replicas`) and the seeded workload
generators (`datagen`) used by the tests and the benchmark.

The library is loaded on first use of any binding name (so `build` and
`datagen` import without it); a missing library raises ImportError there --
there is no CPU fallback.
"""
_EXPORTS = {"Context", "GroupResult", "VdfError", "lib", "LIB_PATH", "I32", "I64", "U32", "U64", "F64", "F32",
            "ORDER_ASC", "ORDER_DESC_STABLE", "ORDER_DESC_REVERSE", "KERNEL_CLASSES", "Batch", "QueryResult",
            "CsvTable"}

__all__ = sorted(_EXPORTS)


def __getattr__(name):
    if name in _EXPORTS:
        from . import _lib
        return getattr(_lib, name)
    raise AttributeError(f"module 'visondf_b200' has no attribute {name!r}")
