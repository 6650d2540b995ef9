"""Every device of the process: the kernels that opt into more than 48 KB of dynamic shared
memory do so per device, so a solve on a second GPU after one on the first launches and
gives the same fields.  Skipped when fewer than two devices are visible."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _solve_on(torch, dev, a, b):
    from ofb200 import ops
    with torch.cuda.device(dev):
        A = torch.from_numpy(a).to(dev)
        B = torch.from_numpy(b).to(dev)
        z = torch.zeros_like(A)
        Ul, Vl, it, _ = ops.ls_solve(A, B, z.clone(), z.clone(), 10.0, arithmetic="exact")
        Uh, Vh, _ = ops.hs_solve(A, B, z.clone(), z.clone(), 21.0, 40)
        Up, Vp, _ = ops.hs_solve(A, B, z.clone(), z.clone(), 21.0, 40, persistent=False)
        torch.cuda.synchronize(dev)
        return [t.cpu().numpy() for t in (Ul, Vl, Uh, Vh, Up, Vp)], int(it.item())


def test_second_device_after_first(cuda_ok):
    import torch
    if torch.cuda.device_count() < 2:
        pytest.skip("one CUDA device visible")
    from ofb200 import synthetic as S
    a, b, _, _ = S.config_pair("fbls1024", seed=13, size=160)
    a, b = a.astype(np.float32), b.astype(np.float32)
    first, it0 = _solve_on(torch, torch.device("cuda", 0), a, b)
    second, it1 = _solve_on(torch, torch.device("cuda", 1), a, b)
    assert it0 == it1
    for x, y in zip(first, second):
        assert np.array_equal(x, y)
