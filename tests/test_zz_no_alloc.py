"""The allocation-free Liu-Shen entry point (of_ls_solve_noalloc) against the regular one.

Callers that cannot allocate device memory at call time (a host framework that owns every
allocation, a plugin that must not touch the process's allocator, a real-time loop that
cannot afford cudaMalloc's synchronisation) use of_ls_solve_noalloc, whose scratch is a
fixed array inside the library.  These tests call both entry points through the C ABI
on the same inputs, twice in a row (the array keeps the previous call's contents, so the
second call checks that nothing stale leaks into it), and expect identical fields, sweep
counts and errors.  This file is collected last; it also passes on its own.
"""
import ctypes
import os
import re

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(REPO, "opticalflow-ri_b200", "ofb200", "libofb200.so")


def _header_scratch_bytes():
    """OF_LS_NOALLOC_SCRATCH_BYTES as include/ofb200.h defines it (the array's size)."""
    with open(os.path.join(REPO, "include", "ofb200.h")) as f:
        m = re.search(r"#define\s+OF_LS_NOALLOC_SCRATCH_BYTES\s+([0-9uUlL*+ ()]+)$", f.read(), re.M)
    assert m, "OF_LS_NOALLOC_SCRATCH_BYTES not found in include/ofb200.h"
    expr = re.sub(r"(?<=[0-9])[uUlL]+", "", m.group(1))
    return int(eval(expr, {"__builtins__": {}}))  # digits, *, +, parentheses only


SCRATCH_BYTES = _header_scratch_bytes()


@pytest.fixture(scope="module")
def env():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    L = ctypes.CDLL(LIB)
    P, I, F, D, Z = ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.c_double, ctypes.c_size_t
    L.of_ls_workspace_size.argtypes = [I, I, I, I]
    L.of_ls_workspace_size.restype = Z
    L.of_ls_solve.argtypes = [P, P, P, P, I, I, I, F, I, D, P, P, P, Z, P]
    L.of_ls_solve.restype = I
    L.of_ls_solve_noalloc.argtypes = [P, P, P, P, I, I, I, F, I, D, P, P, P]
    L.of_ls_solve_noalloc.restype = I
    L.of_last_error.argtypes = [ctypes.c_char_p, Z]
    return torch, L


def _frames(torch, H, W, seed):
    g = torch.Generator(device="cpu").manual_seed(seed)
    a = (torch.rand(H, W, generator=g) * 255).cuda()
    b = torch.roll(a, shifts=(1, 2), dims=(0, 1)) + (torch.rand(H, W, generator=g) * 4).cuda()
    return a.contiguous(), b.contiguous()


def _solve(torch, L, a, b, noalloc, tol=1e-8, maxnum=60):
    H, W = a.shape
    U = torch.zeros_like(a)
    V = torch.zeros_like(a)
    it = torch.full((), -7, dtype=torch.int32, device="cuda")
    er = torch.zeros((), dtype=torch.float64, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    if noalloc:
        rc = L.of_ls_solve_noalloc(a.data_ptr(), b.data_ptr(), U.data_ptr(), V.data_ptr(), H, W, W, 10.0, maxnum, tol,
                                   it.data_ptr(), er.data_ptr(), s)
    else:
        ws = torch.empty(L.of_ls_workspace_size(H, W, W, maxnum), dtype=torch.uint8, device="cuda")
        rc = L.of_ls_solve(a.data_ptr(), b.data_ptr(), U.data_ptr(), V.data_ptr(), H, W, W, 10.0, maxnum, tol,
                           it.data_ptr(), er.data_ptr(), ws.data_ptr(), ws.numel(), s)
    assert rc == 0
    torch.cuda.synchronize()
    return U.cpu().numpy(), V.cpu().numpy(), int(it.item()), float(er.item())


@pytest.mark.parametrize("shape", [(256, 256), (120, 200)])
def test_noalloc_matches_workspace_entry_point_twice(env, shape):
    torch, L = env
    assert L.of_ls_workspace_size(shape[0], shape[1], shape[1], 60) <= SCRATCH_BYTES
    for call, seed in enumerate((11, 12)):  # two calls in a row on the shared array
        a, b = _frames(torch, shape[0], shape[1], seed)
        ref = _solve(torch, L, a, b, noalloc=False)
        got = _solve(torch, L, a, b, noalloc=True)
        assert np.array_equal(got[0], ref[0]) and np.array_equal(got[1], ref[1]), call
        # the error is a sum of per-CTA double atomics: equal up to summation order
        assert got[2] == ref[2] and got[3] == pytest.approx(ref[3], rel=1e-9), call


def test_noalloc_early_stop_matches(env):
    torch, L = env
    a, b = _frames(torch, 96, 96, 13)
    for _ in range(2):
        ref = _solve(torch, L, a, b, noalloc=False, tol=1e-3)
        got = _solve(torch, L, a, b, noalloc=True, tol=1e-3)
        assert got[2] == ref[2] < 60
        assert np.array_equal(got[0], ref[0]) and np.array_equal(got[1], ref[1])


def test_noalloc_rejects_sizes_beyond_the_array(env):
    torch, L = env
    H, W = 1024, 1024
    assert L.of_ls_workspace_size(H, W, W, 60) > SCRATCH_BYTES
    a = torch.zeros(H, W, device="cuda")
    rc = L.of_ls_solve_noalloc(a.data_ptr(), a.data_ptr(), a.data_ptr(), a.data_ptr(), H, W, W, 10.0, 60, 1e-8, None,
                               None, torch.cuda.current_stream().cuda_stream)
    assert rc == -1
    buf = ctypes.create_string_buffer(512)
    L.of_last_error(buf, 512)
    assert b"fixed" in buf.value and b"of_ls_solve" in buf.value


def test_noalloc_boundary_of_the_array(env):
    """The widest 256-row image whose workspace fits is solved; one column more is rejected."""
    torch, L = env
    H = 256
    W = 256
    while L.of_ls_workspace_size(H, W + 1, W + 1, 60) <= SCRATCH_BYTES:
        W += 1
    assert L.of_ls_workspace_size(H, W + 1, W + 1, 60) > SCRATCH_BYTES
    a, b = _frames(torch, H, W, 21)
    ref = _solve(torch, L, a, b, noalloc=False)
    got = _solve(torch, L, a, b, noalloc=True)
    assert np.array_equal(got[0], ref[0]) and np.array_equal(got[1], ref[1]) and got[2] == ref[2]
    a2 = torch.zeros(H, W + 1, device="cuda")
    rc = L.of_ls_solve_noalloc(a2.data_ptr(), a2.data_ptr(), a2.data_ptr(), a2.data_ptr(), H, W + 1, W + 1, 10.0, 60,
                               1e-8, None, None, torch.cuda.current_stream().cuda_stream)
    assert rc == -1
