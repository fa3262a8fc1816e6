"""Reference dataset files through the C ABI (host code, no GPU): the text
format the reference's generator writes and its harness reads with
sscanf("%lld") (open-harmonia/script/generate-data/util.py:37-42,
open-harmonia/src/main.cpp:50-67, open-harmonia/src/range.cu:349-355)."""
import re

import numpy as np
import pytest

from harmonia_b200 import HarmoniaError, datagen as dg
from harmonia_b200.files import read_keys, read_ranges, write_keys

LLD = re.compile(r"[ \t\r\v\f]*([+-]?\d+)")


def sscanf_lld(line):
    """What sscanf("%lld") reads from a line that holds a number."""
    return int(LLD.match(line).group(1))


def test_round_trip_matches_the_generator_format(tmp_path):
    keys = np.concatenate([dg.gen_keys(100_000, 3), np.array([0, -1, -(2**63), 2**63 - 1, 42], np.int64)])
    p = tmp_path / "insert64_0m.txt"
    write_keys(str(p), keys)
    # byte-identical to the reference generator's output_as_file: str(key) + "\n" per key
    assert p.read_text() == "".join(f"{int(k)}\n" for k in keys)
    assert (read_keys(str(p)) == keys).all()


def test_lines_are_read_as_sscanf_lld_reads_them(tmp_path):
    lines = ["  17", "\t-5 trailing text", "+9", "123abc", "7\r", "", "   ", "8"]
    p = tmp_path / "search.txt"
    p.write_text("\n".join(lines))  # no newline after the last line
    got = read_keys(str(p))
    exp = [sscanf_lld(l) for l in lines if l.strip()]
    assert got.tolist() == exp


@pytest.mark.parametrize("bad", ["abc", "-", "99999999999999999999", "-9223372036854775809", "x12"])
def test_malformed_lines_are_errors(tmp_path, bad):
    p = tmp_path / "bad.txt"
    p.write_text(f"1\n{bad}\n3\n")
    with pytest.raises(HarmoniaError) as e:
        read_keys(str(p))
    assert e.value.code == -12


def test_missing_file_and_capacity(tmp_path):
    with pytest.raises(HarmoniaError) as e:
        read_keys(str(tmp_path / "nope.txt"))
    assert e.value.code == -12
    import ctypes
    from harmonia_b200.native import lib
    p = tmp_path / "k.txt"
    write_keys(str(p), np.arange(10, dtype=np.int64))
    n = ctypes.c_size_t()
    buf = np.empty(4, np.int64)
    assert lib().hm_read_keys(str(p).encode(), buf.ctypes.data, 4, ctypes.byref(n)) == -6  # HM_ECAPACITY
    assert n.value == 10 and buf.tolist() == [0, 1, 2, 3]


def test_lines_across_read_chunks(tmp_path):
    # about 12 MB: lines straddle the reader's 4 MiB chunks
    keys = dg.gen_keys(600_000, 9)
    p = tmp_path / "big.txt"
    p.write_text("".join(f"{int(k)}\n" for k in keys))
    assert (read_keys(str(p)) == keys).all()


def test_range_pairs(tmp_path):
    lo = dg.gen_keys(1000, 4)
    hi = lo + 5247
    p = tmp_path / "range64_uniform_0m.txt"
    p.write_text("".join(f"{int(a)}\n{int(b)}\n" for a, b in zip(lo, hi)))
    s, e = read_ranges(str(p))
    assert (s == lo).all() and (e == hi).all()
    p.write_text("1\n2\n3\n")  # a start without its end
    with pytest.raises(HarmoniaError) as err:
        read_ranges(str(p))
    assert err.value.code == -12
