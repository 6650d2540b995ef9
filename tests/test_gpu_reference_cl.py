"""The GPU drop-ins against the reference's own LK / Farneback code paths.

The fixtures (tests/golden/make_golden_cl.py) are outputs of the reference's unmodified
host modules -- denseLucasKanade_PyCl.compute, Farneback_PyCL.compute and
genericPyramidalOpticalFlow with those adapters -- running the reference's .cl kernels
compiled for the host CPU (exact float32 bilinear sampling in place of the device's
fixed-point texture filter).  Everything here is compared bit for bit.
"""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu
f32 = lambda a: np.ascontiguousarray(a, np.float32)  # noqa: E731


def test_lk_compute(cuda_ok):
    import denseLucasKanade_PyCL as LK
    g = golden("lk_ref")
    for i in range(int(g["n"])):
        hw, nit, vort = (int(x) for x in g[f"spec{i}"])
        ad = LK.denseLucasKanade_PyCl(Niter=nit, halfWindow=hw, enableVorticityEnhancement=bool(vort))
        if vort:  # the window masks the reference picked from the initial field's mean vorticity
            assert list(ad.evaluateVorticityEnhancement(g[f"U0_{i}"], g[f"V0_{i}"])) == [int(x) for x in g[f"asym{i}"]]
        U, V, ok = ad.compute(f32(g[f"I{i}"]), f32(g[f"J{i}"]), g[f"U0_{i}"].copy(), g[f"V0_{i}"].copy())
        assert ok is True
        assert np.array_equal(U, g[f"U{i}"]) and np.array_equal(V, g[f"V{i}"]), i


def test_farneback_compute(cuda_ok):
    import Farneback_PyCL as FB
    g = golden("fb_ref")
    for i in range(int(g["n"])):
        ws, nit, pn, ps, ug, pl = g[f"spec{i}"]
        fb = FB.Farneback_PyCL(windowSize=int(ws), Niters=int(nit), polyN=int(pn), polySigma=float(ps),
                               useGaussian=bool(ug), pyramidalLevels=int(pl))
        U, V, e = fb.compute(f32(g[f"I{i}"]), f32(g[f"J{i}"]), g[f"U0_{i}"].copy(), g[f"V0_{i}"].copy())
        assert e == "Unknown"
        assert np.array_equal(U, g[f"U{i}"]) and np.array_equal(V, g[f"V{i}"]), i


@pytest.mark.parametrize("name", ["pyr_lk_ref", "pyr_fb_ref", "pyr_fbls_ref"])
def test_pyramid_pipelines(cuda_ok, name):
    import denseLucasKanade_PyCL as LK
    import Farneback_PyCL as FB
    import GenericPyramidalOpticalFlow as G
    import PhysicsBasedOpticalFlowLiuShen as LS
    g = golden(name)
    a, b = f32(g["f0"]), f32(g["f1"])
    if name == "pyr_lk_ref":
        U, V = G.genericPyramidalOpticalFlow(a, b, 2, LK.denseLucasKanade_PyCl(Niter=5, halfWindow=13), 2, 1, 0.48, None,
                                             warping=False)
    elif name == "pyr_fb_ref":
        U, V = G.genericPyramidalOpticalFlow(a, b, 0, FB.Farneback_PyCL(), 2, 1, None, None)
    else:
        U, V = G.genericPyramidalOpticalFlow(a, b, 0, FB.Farneback_PyCL(), 2, 1, 0.48,
                                             LS.LiuShenOpticalFlowAlgoAdapter(10))
    assert np.array_equal(U, g["U"]) and np.array_equal(V, g["V"])
