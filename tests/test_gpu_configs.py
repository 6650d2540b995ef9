"""The single-pair workloads at their full sizes, GPU against the reference itself.

tests/golden/configs.npz (tests/golden/make_golden_cl.py --configs) holds SHA-256 digests
of the reference's U, V on seeded synthetic pairs -- the reference's own Python, scipy and
Pillow, with its OpenCL kernels compiled for the host -- for
  hs256    Horn-Schunck, PyHSchunck_Fs3_4 calibration (600 sweeps), 256 x 256;
  lk512    dense Lucas-Kanade pyr2, denseLK_Fs2_0_PyrLvls2 calibration, 512 x 512;
  fbls1024 Farneback pyr2 + Liu-Shen, LiuSE_Farneback_Fs0_0_PyrLvls2 calibration, 1024 x 1024.
The GPU drop-in must reproduce them bit for bit (the CPU oracle does too; its digest is
stored beside the reference's and equal to it)."""
import hashlib

import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def sha(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def _pipeline(cfg, a, b):
    import denseLucasKanade_PyCL as LK
    import Farneback_PyCL as FB
    import GenericPyramidalOpticalFlow as G
    import HornSchunck as HS
    import PhysicsBasedOpticalFlowLiuShen as LS
    if cfg == "hs256":
        return G.genericPyramidalOpticalFlow(a, b, 3.4, HS.HSOpticalFlowAlgoAdapter([21], 600), 1, 1, None)
    if cfg == "lk512":
        return G.genericPyramidalOpticalFlow(a, b, 2, LK.denseLucasKanade_PyCl(Niter=5, halfWindow=13), 2, 1, 0.48,
                                             None, warping=False)
    return G.genericPyramidalOpticalFlow(a, b, 0, FB.Farneback_PyCL(), 2, 1, 0.48, LS.LiuShenOpticalFlowAlgoAdapter(10))


@pytest.mark.parametrize("cfg", ["hs256", "lk512", "fbls1024"])
def test_config_bit_exact_with_reference(cuda_ok, cfg):
    from ofb200 import synthetic as S
    g = golden("configs")
    a8, b8, _, _ = S.config_pair(cfg, seed=1)
    assert sha(a8, b8) == str(g[f"{cfg}_frames"]), "synthetic generator drifted"
    U, V = _pipeline(cfg, a8.astype(np.float32), b8.astype(np.float32))
    if sha(U, V) != str(g[f"{cfg}_ref"]):
        d = max(np.abs(U[::8, ::8] - g[f"{cfg}_Uref8"]).max(), np.abs(V[::8, ::8] - g[f"{cfg}_Vref8"]).max())
        pytest.fail(f"{cfg}: GPU differs from the reference (max |diff| on every 8th pixel: {d:.3g} px)")
