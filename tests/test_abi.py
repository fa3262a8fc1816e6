"""CPU tests of the C ABI: the library loads and exports every symbol the
public header declares.  No compute call is made (there is no GPU here)."""
import os
import re
import subprocess

import pytest

from harmonia_b200 import native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "harmonia.h")


def declared_symbols():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(hm_[a-z_0-9]+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(native.LIB_PATH):
        import __graft_entry__
        __graft_entry__.build()
    return native.lib()


def test_every_declared_symbol_is_exported(lib):
    syms = declared_symbols()
    assert len(syms) >= 10
    out = subprocess.run(["nm", "-D", "--defined-only", native.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (hm_\w+)", out))
    missing = [s for s in syms if s not in exported]
    assert not missing, missing
    for s in syms:
        getattr(lib, s)


def test_binding_covers_the_header():
    assert sorted(native.EXPORTS) == [s for s in declared_symbols() if s in native.EXPORTS]
    assert set(native.EXPORTS) == set(declared_symbols())


def test_strerror_and_defaults_without_gpu(lib):
    for code in list(native.ERRORS) + [0, 123]:
        assert isinstance(lib.hm_strerror(code), bytes)
    import ctypes
    c = native.Config()
    assert lib.hm_config_default(ctypes.byref(c)) == 0
    assert (c.fanout, c.leaf_cap, c.inner_fill, c.leaf_fill) == (64, 16, 64, 16)
    assert c.group_width in (1, 2, 4, 8, 16, 32) and c.sort_bits == -1 and c.cache_hints == 1


def test_library_has_no_host_fallback_symbols():
    # The product library must not link the oracle.
    out = subprocess.run(["nm", "-D", native.LIB_PATH], capture_output=True, text=True).stdout
    assert "hmo_" not in out and "hmref_" not in out
