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


def test_host_copy_without_gpu():
    """of_host_copy (the staging copy of host-buffer calls) is host code: byte-exact for
    sizes below and above the 1 MiB pool threshold, including lengths that do not split
    into whole pages, and it rejects overlapping buffers."""
    if not os.path.exists(LIB):
        pytest.skip("libofb200.so not built")
    import numpy as np
    from ofb200 import _lib, par_copyto
    L = _lib.lib()
    rng = np.random.default_rng(3)
    for n in (0, 1, 4095, 1 << 20, (1 << 20) + 13, 4 * 1024 * 1024 + 4097, 9 * 1024 * 1024 + 1):
        src = rng.integers(0, 256, n, dtype=np.uint8)
        dst = np.zeros(n, dtype=np.uint8)
        assert L.of_host_copy(dst.ctypes.data, src.ctypes.data, n) == 0
        assert np.array_equal(dst, src)
    buf = np.zeros(1 << 21, dtype=np.uint8)
    assert L.of_host_copy(buf.ctypes.data + 16, buf.ctypes.data, 1 << 20) == -1
    # the Python helper: same-dtype planes natively, casts through numpy
    a = rng.random((1024, 1024), dtype=np.float32)
    b = np.empty_like(a)
    par_copyto(b, a)
    assert np.array_equal(a, b)
    u8 = rng.integers(0, 256, (1024, 1024), dtype=np.uint8)
    f = np.empty((1024, 1024), dtype=np.float32)
    par_copyto(f, u8)
    assert np.array_equal(f, u8.astype(np.float32))


def test_spline_pair_argument_checks_without_gpu():
    """of_spline_upsample_pair validates its arguments on the host before any CUDA call:
    aliased outputs and a workspace under two single-plane workspaces are rejected with
    the entry point named in the error message."""
    if not os.path.exists(LIB):
        pytest.skip("libofb200.so not built")
    from ofb200 import _lib
    L = _lib.lib()
    fake = ctypes.c_void_p(4096)  # never dereferenced: the checks fail first
    rc = L.of_spline_upsample_pair(fake, fake, 8, 8, 8, fake, fake, 16, 16, 16, 1.0, 1.0, fake, 1 << 20, None)
    assert rc == -1 and "alias" in _lib.last_error()
    other = ctypes.c_void_p(8192)
    need = 2 * L.of_spline_workspace_size(8, 8, 16, 16)
    rc = L.of_spline_upsample_pair(fake, fake, 8, 8, 8, fake, other, 16, 16, 16, 1.0, 1.0, fake, need - 8, None)
    assert rc == -3 and "workspace" in _lib.last_error()


def test_resize_table_sizes_without_gpu():
    """The drop-in's estimate of Pillow's taps per output (which decides when a resize uses
    kept weight tables) is the library's kernel width: of_resize_table_size holds 2 ints and
    that many doubles per output sample.  The tabled resize rejects a missing table and a
    small workspace on the host."""
    if not os.path.exists(LIB):
        pytest.skip("libofb200.so not built")
    from ofb200 import _lib, ops
    L = _lib.lib()

    def up256(x):
        return (x + 255) // 256 * 256

    for n_in, n_out in ((1024, 128), (1024, 512), (512, 16), (37, 19), (64, 128), (1000, 95), (8192, 128)):
        for bic, f in ((True, _lib.OF_FILTER_BICUBIC), (False, _lib.OF_FILTER_BILINEAR)):
            k = ops._resize_taps(n_in, n_out, bic)
            assert L.of_resize_table_size(n_in, n_out, f) == up256(8 * n_out) + 8 * k * n_out, (n_in, n_out, bic)
    assert L.of_resize_table_size(0, 4, _lib.OF_FILTER_BICUBIC) == 0
    fake = ctypes.c_void_p(4096)  # never dereferenced: the checks fail first
    rc = L.of_resize_tabled(fake, 64, 64, 64, fake, 8, 8, 8, _lib.OF_FILTER_BICUBIC, None, fake, fake, 1 << 20, None)
    assert rc == -1 and "table" in _lib.last_error()
    rc = L.of_resize_tabled(fake, 64, 64, 64, fake, 8, 8, 8, _lib.OF_FILTER_BICUBIC, fake, fake, fake, 4 * 64 * 8 - 4,
                            None)
    assert rc == -3 and "workspace" in _lib.last_error()
