"""The GPU's float32 fields against the float64 restatement of the algorithm
(oracle/oracle_f64.py) on the full-size single-pair workloads: max |GPU - float64| <= 1e-3
px, and the endpoint error against the analytic displacement no worse than float64's
(within 1e-5 px, the float32 rounding of the error itself)."""
import numpy as np
import pytest

import oracle_f64 as F

pytestmark = pytest.mark.gpu
TOL_PX = 1e-3


def _run(cfg):
    import Farneback_PyCL as FB
    import GenericPyramidalOpticalFlow as G
    import HornSchunck as HS
    import PhysicsBasedOpticalFlowLiuShen as LS
    from ofb200 import synthetic as S
    a8, b8, Ug, Vg = S.config_pair(cfg, seed=1)
    a, b = a8.astype(np.float32), b8.astype(np.float32)
    if cfg == "hs256":  # PyHSchunck_Fs3_4 calibration
        U, V = G.genericPyramidalOpticalFlow(a.copy(), b.copy(), 3.4, HS.HSOpticalFlowAlgoAdapter([21], 600), 1, 1, None)
        U6, V6 = F.pyramid(a, b, 3.4, F.HS([21], 600), 1, 1, None)
    else:  # LiuSE_Farneback_Fs0_0_PyrLvls2 calibration
        U, V = G.genericPyramidalOpticalFlow(a.copy(), b.copy(), 0, FB.Farneback_PyCL(), 2, 1, 0.48,
                                             LS.LiuShenOpticalFlowAlgoAdapter(10))
        U6, V6 = F.pyramid(a, b, 0, F.FB(), 2, 1, 0.48, F.LS(10))
    return U, V, U6, V6, Ug, Vg


@pytest.mark.parametrize("cfg", ["hs256", "fbls1024"])
def test_float32_gpu_within_1e3_px_of_float64(cuda_ok, cfg):
    from ofb200 import synthetic as S
    U, V, U6, V6, Ug, Vg = _run(cfg)
    d = max(np.abs(U - U6).max(), np.abs(V - V6).max())
    assert d <= TOL_PX, d
    e32 = S.epe(U, V, Ug, Vg, crop=16)
    e64 = S.epe(U6.astype(np.float32), V6.astype(np.float32), Ug, Vg, crop=16)
    assert e32 <= e64 + 1e-5, (e32, e64)
