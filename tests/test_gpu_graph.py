"""CUDA-graph replay of the pyramid gives the eager result and the adapters' visible
state changes as in the reference."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _pair(size=256, seed=9):
    from ofb200 import synthetic as S
    a, b, Ug, Vg = S.config_pair("fbls1024", seed=seed, size=size)
    return a.astype(np.float32), b.astype(np.float32)


def test_graph_matches_eager_fb_ls(torch_cuda):
    import Farneback_PyCL as F
    import GenericPyramidalOpticalFlow as G
    import PhysicsBasedOpticalFlowLiuShen as LS
    from ofb200 import graph
    a, b = _pair()
    graph.ENABLED = False
    Ue, Ve = G.genericPyramidalOpticalFlow(a, b, 0, F.Farneback_PyCL(), 2, 1, 0.48, LS.LiuShenOpticalFlowAlgoAdapter(10))
    graph.ENABLED = True
    for seed in (9, 10, 9):  # first call captures, later calls replay with new inputs
        a2, b2 = _pair(seed=seed)
        Ug, Vg = G.genericPyramidalOpticalFlow(a2, b2, 0, F.Farneback_PyCL(), 2, 1, 0.48,
                                               LS.LiuShenOpticalFlowAlgoAdapter(10))
        if seed == 9:
            assert np.array_equal(Ug, Ue) and np.array_equal(Vg, Ve)
            assert np.isfinite(Ug).all()


def test_graph_hs_pops_alphas(torch_cuda):
    import GenericPyramidalOpticalFlow as G
    import HornSchunck as HS
    from ofb200 import graph
    a, b = _pair(64, 3)
    graph.ENABLED = False
    ad = HS.HSOpticalFlowAlgoAdapter([7, 21, 45], 50)
    Ue, Ve = G.genericPyramidalOpticalFlow(a, b, 3.4, ad, 2, 1, None)
    assert ad.alphas == [7]
    graph.ENABLED = True
    for _ in range(2):
        ad = HS.HSOpticalFlowAlgoAdapter([7, 21, 45], 50)
        Ug, Vg = G.genericPyramidalOpticalFlow(a, b, 3.4, ad, 2, 1, None)
        assert ad.alphas == [7]
        assert np.array_equal(Ug, Ue) and np.array_equal(Vg, Ve)
    ad = HS.HSOpticalFlowAlgoAdapter([21], 50)
    with pytest.raises(IndexError):
        G.genericPyramidalOpticalFlow(a, b, 3.4, ad, 2, 1, None)
