"""CSV ingest, CPU side: the oracle restatement against the reference's own
record parser and fast_float (oracle/_ref shim) and against the committed
fixtures they produced, and the GPU path's decimal conversion code
(vdf_decimal.cuh, built for the host) against the oracle on adversarial
strings.  No GPU needed."""
from __future__ import annotations

import json
import math
import random
import shutil
import struct
import subprocess
from fractions import Fraction
from pathlib import Path

import numpy as np
import pytest

import csv_gen
import oracle_bind as ob

ROOT = Path(__file__).resolve().parent.parent
GOLDEN = ROOT / "tests" / "golden" / "ref_csv_cases.npz"


def same_table(a: ob.CsvResult, b: ob.CsvResult) -> bool:
    if a.bad_row >= 0 or b.bad_row >= 0:
        return a.bad_row == b.bad_row
    if (a.nrow, a.types, a.names) != (b.nrow, b.types, b.names):
        return False
    for x, y in zip(a.columns, b.columns):
        if isinstance(x, list):
            if x != y:
                return False
        elif x.tobytes() != y.tobytes():
            return False
    return True


def golden_cases():
    z = np.load(GOLDEN)
    meta = json.loads(z["meta"].tobytes())
    return [(z[f"csv{i}"].tobytes(), m, ob.CsvResult(z[f"blob{i}"].tobytes())) for i, m in enumerate(meta)]


def test_oracle_matches_reference_fixtures():
    cases = golden_cases()
    assert len(cases) >= 20
    for data, m, ref in cases:
        got = ob.csv_read(data, delim=m["delim"], header=m["header"], quote=m["quote"])
        assert same_table(got, ref), (data[:80], m)


@pytest.mark.skipif(not ob.ref_available(), reason="reference shim not built")
@pytest.mark.parametrize("crlf", [False, True])
@pytest.mark.parametrize("header", [True, False])
def test_oracle_matches_reference_parser(crlf, header):
    for seed in range(12):
        for tn in (True, False):
            d = csv_gen.make_csv(seed, 30 + 11 * seed, crlf=crlf, empty_frac=0.1, header=header, trailing_newline=tn,
                                 quote="'" if seed % 2 else '"')
            if d.endswith(b","):
                continue   # the reference leaves the last column short there (documented deviation)
            q = "'" if seed % 2 else '"'
            assert same_table(ob.csv_read(d, header=header, quote=q), ob.ref_csv_read(d, header=header, quote=q))


def test_final_record_ending_in_delimiter_reads_na():
    r = ob.csv_read(b"a,b\n1,x\n2,")
    assert r.nrow == 2 and r.columns[1] == [b"x", b"NA"]


def test_field_count_errors():
    assert ob.csv_read(b"a,b\n1,2\n3\n").bad_row == 1
    assert ob.csv_read(b"a,b\n1,2,3\n").bad_row == 0
    assert ob.csv_read(b"1,2\n3\n", header=False).bad_row == 1
    assert ob.csv_read(b"a,b\n1,2\n").bad_row == -1


def test_first_line_quirks():
    # no header, CR LF: the first row's last field keeps the CR (read_csv.hpp:67-69,129)
    r = ob.csv_read(b"1,2\r\n3,4\r\n", header=False)
    assert r.types == ["u", "s"] and r.columns[1] == [b"2\r", b"4"]
    # header names: empty -> "NA", quotes kept
    r = ob.csv_read(b",'b'\n1,2\n")
    assert r.names == ["NA", "'b'"]


def hard_strings(seed: int, count: int) -> list[str]:
    rnd = random.Random(seed)

    def exact(fr):
        k = fr.denominator.bit_length() - 1
        digits = str(fr.numerator * 5 ** k)
        if k == 0:
            return digits
        if len(digits) <= k:
            digits = "0" * (k - len(digits) + 1) + digits
        return digits[:-k] + "." + digits[-k:]

    out = []
    while len(out) < count:
        b = rnd.getrandbits(63) if rnd.random() < 0.8 else rnd.getrandbits(52)
        x = struct.unpack("<d", struct.pack("<Q", b))[0]
        y = math.nextafter(x, math.inf)
        if not (x > 0 and math.isfinite(y)):
            continue
        h = (Fraction(x) + Fraction(y)) / 2
        s = exact(h)
        out += [s, "-" + s, s + "0000000000000000000001", exact(h - Fraction(1, 1 << 1100))]
    return out


def random_strings(seed: int, count: int) -> list[str]:
    rng = random.Random(seed)
    alpha = "0123456789.-+eEnaifNAIF x"
    out = []
    for _ in range(count):
        k = rng.randrange(7)
        if k == 6:   # short decimals, the CSV-typical shape, with odd tails
            s = "".join(rng.choice("0123456789") for _ in range(rng.randrange(0, 10)))
            if rng.random() < 0.7:
                s += "." + "".join(rng.choice("0123456789") for _ in range(rng.randrange(0, 10)))
            s += rng.choice(["", "", "", "x", "e5", "E-2", ".", "-", " "])
            out.append(("-" if rng.random() < 0.2 else "") + s)
            continue
        if k == 0:
            s = "".join(rng.choice("0123456789") for _ in range(rng.randrange(1, 25)))
            if rng.random() < 0.5:
                s += "." + "".join(rng.choice("0123456789") for _ in range(rng.randrange(0, 25)))
        elif k == 1:
            s = f"{rng.randrange(1, 10**rng.randrange(1, 20))}e{rng.randrange(-350, 350)}"
        elif k == 2:
            s = "".join(rng.choice(alpha) for _ in range(rng.randrange(0, 12)))
        elif k == 3:
            s = repr(struct.unpack("<d", struct.pack("<Q", rng.getrandbits(63)))[0])
        elif k == 4:
            s = str(rng.randrange(0, 2 ** 34)) if rng.random() < 0.7 else str(-rng.randrange(0, 2 ** 32))
        else:
            s = "0." + "0" * rng.randrange(0, 30) + "".join(rng.choice("0123456789") for _ in range(rng.randrange(1, 40)))
        if rng.random() < 0.2:
            s = "-" + s
        out.append(s)
    return out


@pytest.fixture(scope="module")
def decimal_check(tmp_path_factory):
    gxx = shutil.which("g++")
    if not gxx:
        pytest.skip("g++ not available")
    exe = tmp_path_factory.mktemp("dec") / "decimal_check"
    subprocess.run([gxx, "-O2", "-std=c++17", "-I", str(ROOT / "visondf_b200" / "csrc"), "-o", str(exe),
                    str(ROOT / "tests" / "cpp" / "decimal_check.cpp")], check=True)
    return exe


def run_check(exe, strings):
    out = subprocess.run([str(exe)], input="\n".join(strings) + "\n", capture_output=True, text=True,
                         check=True).stdout.split("\n")
    rows = [line.split() for line in out if line]
    assert len(rows) == len(strings)
    return rows


def oracle_bits(s: str) -> str:
    return f"{struct.unpack('<Q', struct.pack('<d', ob.parse_double(s.encode())))[0]:016x}"


@pytest.mark.parametrize("kind", ["random", "halfway"])
def test_device_decimal_code_matches_oracle(decimal_check, kind):
    strings = random_strings(3, 20000) if kind == "random" else hard_strings(5, 2000)
    rows = run_check(decimal_check, strings)
    slow = fast = 0
    for s, (bits, u, i, path, scan) in zip(strings, rows):
        assert path != "2", s
        assert scan != "2", s   # the eight-byte scan gives the general scan's result
        slow += path == "1"
        fast += scan == "1"
        assert bits == oracle_bits(s), s
        assert int(u) == ob.parse_u32(s.encode()), s
        assert int(i) == ob.parse_i32(s.encode()), s
    if kind == "halfway":
        assert slow > len(strings) // 2   # the exact decision is exercised
    else:
        assert fast > len(strings) // 10  # the eight-byte scan is exercised


@pytest.mark.skipif(not ob.ref_available(), reason="reference shim not built")
def test_oracle_doubles_match_reference_fast_float():
    strings = [s for s in random_strings(9, 5000) + hard_strings(10, 400)
               if s and not any(c in s for c in ",'\n\r")]
    data = ("v\n0.5\n" + "\n".join(strings) + "\n").encode()
    ref = ob.ref_csv_read(data)
    assert ref.types == ["d"]
    got = np.array([ob.parse_double(s.encode()) for s in strings])
    assert got.tobytes() == ref.columns[0][1:].tobytes()


@pytest.mark.skipif(not ob.ref_available(), reason="reference shim not built")
def test_oracle_matches_reference_parser_on_quoting_soup():
    """Quotes mid-field, quoted delimiters and line ends, mixed line ends:
    the oracle's split equals the reference parser's (and a short record
    is the same error row)."""
    checked = 0
    for seed in range(60):
        q = "'" if seed % 2 else '"'
        short = 7 if seed % 10 == 3 else -1
        data = csv_gen.soup_csv(seed, 40 + seed, 2 + seed % 5, quote=q, short_row=short)
        o = ob.csv_read(data, quote=q)
        r = ob.ref_csv_read(data, quote=q)
        assert same_table(o, r), seed
        if short >= 0:
            assert o.bad_row == short
        checked += 1
    assert checked == 60
