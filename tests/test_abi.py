"""The C-ABI library loads and exports every entry point include/ofb200.h declares
(no GPU needed: nothing is called)."""
import ctypes
import os
import re

import pytest

from conftest import REPO

HEADER = os.path.join(REPO, "include", "ofb200.h")
LIB = os.path.join(REPO, "opticalflow-ri_b200", "ofb200", "libofb200.so")


def declared():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:int|size_t|unsigned long long)\s+(of_\w+)\s*\(", src, flags=re.M)))


def test_header_parses():
    names = declared()
    assert "of_ls_solve" in names and "of_lk_dense" in names and len(names) >= 20


def test_library_exports_every_declared_symbol():
    if not os.path.exists(LIB):
        pytest.skip("libofb200.so not built")
    L = ctypes.CDLL(LIB)
    missing = [n for n in declared() if not hasattr(L, n)]
    assert not missing, missing


def test_binding_covers_header():
    from ofb200 import _lib
    assert set(declared()) <= set(_lib.exported_symbols()) | {"of_version", "of_last_error"}


def test_version_and_error_string_without_gpu():
    if not os.path.exists(LIB):
        pytest.skip("libofb200.so not built")
    L = ctypes.CDLL(LIB)
    L.of_version.restype = ctypes.c_int
    assert L.of_version() >= 100
    # argument validation runs on the host and reports through of_last_error
    L.of_prefilter_f32.restype = ctypes.c_int
    rc = L.of_prefilter_f32(None, 0, None, 0, 0, 0, None, 3, None)
    assert rc == -1
    buf = ctypes.create_string_buffer(256)
    L.of_last_error(buf, 256)
    assert b"of_prefilter_f32" in buf.value
