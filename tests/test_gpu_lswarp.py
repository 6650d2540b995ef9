"""The Liu-Shen optical-flow-equation warp (biLinear=False) and kLevels > 1 on the GPU:
bit-exact with the oracle and with the reference's golden warps, the same IndexErrors,
and the same in-place edit of the first frame."""
import numpy as np
import pytest

import oracle as O
from conftest import golden

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def test_warp_matches_reference_golden(torch_cuda):
    torch = torch_cuda
    import GenericPyramidalOpticalFlow as G
    g = golden("warp_liushen")
    for i in range(3):
        n1 = torch.from_numpy(g[f"I1_{i}"].copy()).cuda()
        G._liushen_warp(n1, torch.from_numpy(g[f"ua_{i}"]).cuda(), torch.from_numpy(g[f"va_{i}"]).cuda())
        assert np.array_equal(n1.cpu().numpy(), g[f"O1_{i}"]), i


def test_transition_matches_oracle(torch_cuda):
    import GenericPyramidalOpticalFlow as G
    g = golden("warp_liushen")
    for i in range(3):
        H, W, h, w, scale = (int(x) for x in g[f"spec_{i}"])
        z = np.zeros((h, w), np.float32)
        a = g[f"I1_{i}"].copy()
        got = G.updateNextPyramidalLevel(a, z, g[f"I2_{i}"], g[f"Ua_{i}"], g[f"Va_{i}"], z, z, True, False, bool(scale))
        b = g[f"I1_{i}"].copy()
        want = O._level_transition(b, (h, w), g[f"I2_{i}"], g[f"Ua_{i}"], g[f"Va_{i}"], True, False, bool(scale))
        for x, y in zip(got, want):
            assert np.array_equal(x, y), i
        assert np.array_equal(a, b)  # both edited the first frame in place


def test_index_errors_match_reference(torch_cuda):
    import GenericPyramidalOpticalFlow as G
    g = golden("warp_liushen")
    Ua = g["bad_Ua"]
    z8 = np.zeros_like(Ua)
    with pytest.raises(IndexError, match="index 8 is out of bounds for axis 1 with size 8"):
        G.updateNextPyramidalLevel(g["bad_I1"].copy(), g["bad_I1"], g["bad_I1"].copy(), Ua, z8, z8, z8, True, False,
                                   False)
    z = np.zeros((40, 30), np.float32)
    a = np.ones((40, 30), np.float32)
    with pytest.raises(IndexError) as e:
        G.updateNextPyramidalLevel(a, a.copy(), a.copy(), z, z, z, z, True, False, False)
    assert str(e.value) == str(g["small_msg"])
    rows = np.zeros((8, 8), np.float32)
    rows[0, 2] = -8.6  # destination row 0 + floor(-8.1) = -9 < -8; numpy checks rows before columns
    with pytest.raises(IndexError, match="index -9 is out of bounds for axis 0 with size 8"):
        G.updateNextPyramidalLevel(g["bad_I1"].copy(), g["bad_I1"], g["bad_I1"].copy(), Ua, rows, z8, z8, True,
                                   False, False)


def test_pipeline_liushen_warp_klevels(torch_cuda):
    """HS (adapter defaults off) with the Liu-Shen warp, 2 levels x 2 iterations, Liu-Shen
    refine: bit-exact with the oracle, within 1e-3 of the reference, and the caller's frame
    edited in place as both do."""
    import GenericPyramidalOpticalFlow as G
    import HornSchunck as HS
    import PhysicsBasedOpticalFlowLiuShen as LS
    g = golden("pyr_hs_lswarp")
    a = g["f0"].copy()
    U, V = G.genericPyramidalOpticalFlow(a, g["f1"], 3.4,
                                         HS.HSOpticalFlowAlgoAdapter([21, 45, 33, 17], 50,
                                                                     provideGenericPyramidalDefaults=False),
                                         2, 2, 0.48, LS.LiuShenOpticalFlowAlgoAdapter(10), True, False, True, True)
    b = g["f0"].copy()
    Uo, Vo = O.pyramid(b, g["f1"], 3.4, O.HS([21, 45, 33, 17], 50, provideGenericPyramidalDefaults=False), 2, 2, 0.48,
                       O.LS(10), True, False, True, True)
    assert np.array_equal(U, Uo) and np.array_equal(V, Vo)
    assert np.array_equal(a, b)
    assert np.abs(U - g["U"]).max() <= 1e-3 and np.abs(V - g["V"]).max() <= 1e-3


@pytest.mark.parametrize("method", ["hs", "fb"])
def test_pipeline_klevels_two(torch_cuda, method):
    """kLevels = 2 with the adapters' own defaults (HS: bilinear warp; Farneback: no warp)."""
    import Farneback_PyCL as F
    import GenericPyramidalOpticalFlow as G
    import HornSchunck as HS
    from ofb200 import synthetic as S
    a, b, _, _ = S.config_pair("fbls1024", seed=8, size=128)
    a, b = a.astype(np.float32), b.astype(np.float32)
    if method == "hs":
        U, V = G.genericPyramidalOpticalFlow(a, b, 3.4, HS.HSOpticalFlowAlgoAdapter([21, 45, 33, 17], 40), 2, 2)
        Uo, Vo = O.pyramid(a, b, 3.4, O.HS([21, 45, 33, 17], 40), 2, 2)
    else:
        U, V = G.genericPyramidalOpticalFlow(a, b, 0, F.Farneback_PyCL(), 2, 2)
        Uo, Vo = O.pyramid(a, b, 0, O.FB(), 2, 2)
    assert np.array_equal(U, Uo, equal_nan=True) and np.array_equal(V, Vo, equal_nan=True)
