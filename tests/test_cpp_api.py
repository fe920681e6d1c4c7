"""The header-only C++ dataframe layer (include/vison_b200/vison.hpp): it
compiles standalone (CPU), and a C++ program using it runs on the GPU
against CPU-computed expectations (tests/cpp/test_vison_b200.cpp)."""
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
SRC = ROOT / "tests" / "cpp" / "test_vison_b200.cpp"
LIBDIR = ROOT / "visondf_b200"


def test_header_compiles_standalone(tmp_path):
    r = subprocess.run(["g++", "-std=c++20", "-fsyntax-only", "-Wall", "-Wextra", "-I", str(ROOT / "include"), str(SRC)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_header_compiles_as_vison_dropin(tmp_path):
    src = tmp_path / "dropin.cpp"
    src.write_text('#define VISON_B200_AS_VISON\n#include "vison_b200/vison.hpp"\n'
                   "int main(){ vison::Dataframe<> df; unsigned n = 0; df.add_col(std::vector<int>{3,1,2});\n"
                   " df.sort_by_mt<1, 8, void, true, true, vison::SortType::Radix>(n); df.materialize_mt<8>();\n"
                   " df.transform_group_by_mt<void, void, 4, vison::GroupFunction::Sum>({0}, 0, \"s\");\n"
                   " vison::Dataframe<> r = df; df.transform_unique_mt<void, 8>(0);\n"
                   " df.transform_left_join_mt<void, 8, true, vison::LeftJoinMethods::Last>(r, 0, 0, ' '); return 0; }\n")
    r = subprocess.run(["g++", "-std=c++20", "-fsyntax-only", "-I", str(ROOT / "include"), str(src)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


@pytest.mark.gpu
def test_cpp_layer_on_gpu(tmp_path):
    exe = tmp_path / "test_vison_b200"
    r = subprocess.run(["g++", "-std=c++20", "-O2", "-I", str(ROOT / "include"), str(SRC), "-o", str(exe),
                        "-L", str(LIBDIR), "-lvdf_b200", f"-Wl,-rpath,{LIBDIR}"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "all checks passed" in r.stdout
