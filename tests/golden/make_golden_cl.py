"""Golden fixtures for the reference's OpenCL paths: dense Lucas-Kanade and Farneback.

The reference's host modules (src/denseLucasKanade_PyCL.py, src/Farneback_PyCL.py, and the
pyramid driver src/GenericPyramidalOpticalFlow.py) are imported unmodified and run with a
stand-in `pyopencl` (oracle/clref.py) whose kernels are the reference's own .cl files
compiled for the host CPU (oracle/clref/: per-expression floating-point contraction as
OpenCL defines it, work-groups run as fibers with real barriers; the one substitution is
the image sampler, which uses exact float32 bilinear weights instead of the device's
fixed-point texture filter).  Run where the reference tree is present:

    PYTHONDONTWRITEBYTECODE=1 NUMBA_CACHE_DIR=/tmp/numba \\
        python tests/golden/make_golden_cl.py <reference>/src [--configs]

Writes tests/golden/{lk_ref,fb_ref,pyr_lk_ref,pyr_fb_ref,pyr_fbls_ref}.npz (small cases,
full arrays; the frames are stored as the uint8 values they hold).  With --configs it also writes tests/golden/configs.npz: the three
single-pair workloads at their full sizes (Horn-Schunck 256^2 600 sweeps, dense LK pyr2
512^2, Farneback pyr2 + Liu-Shen 1024^2), as SHA-256 digests of the frames, of the
reference's U, V and of the CPU oracle's U, V, plus every 8th row and column of both
outputs and the oracle-vs-reference differences (the full fields are megabytes).
"""
from __future__ import annotations

import hashlib
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(REPO, "oracle"))
sys.path.insert(0, os.path.join(REPO, "opticalflow-ri_b200"))

import make_golden as MG  # noqa: E402  (stubs, loader, quiet())

f32 = lambda a: np.ascontiguousarray(a, np.float32)  # noqa: E731


def sha(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def load(ref_src):
    import clref
    clref.build(ref_src)
    sys.modules.update(clref.fake_pyopencl(contract=True))
    MG.REF = ref_src
    R = MG.load_reference()
    import importlib
    R["denseLucasKanade_PyCL"] = importlib.import_module("denseLucasKanade_PyCL")
    return R


def rotation(H, W, omega):
    """Solid-body rotation field about the image centre (mean vorticity 2*omega)."""
    y, x = np.mgrid[0:H, 0:W].astype(np.float64)
    return f32(-omega * (y - H / 2)), f32(omega * (x - W / 2))


def small_cases(R):
    from ofb200 import synthetic as S
    rng = np.random.default_rng(977)
    LKm, FBm, G = R["denseLucasKanade_PyCL"], R["Farneback_PyCL"], R["GenericPyramidalOpticalFlow"]
    out = {}

    # --- A10/A11 + f3: denseLucasKanade_PyCl.compute
    d = {}
    cases = [(64, 64, 13, 5, "zero", False), (48, 64, 13, 5, "noise", False), (48, 56, 5, 5, "noise", False),
             (64, 64, 13, 3, "rot-", True), (64, 64, 13, 5, "rot+", True), (40, 40, 13, 5, "large", False)]
    for i, (H, W, hw, nit, init, vort) in enumerate(cases):
        a, b, _, _ = S.piv_pair(H, W, "lamb_oseen", seed=40 + i, core_radius=min(H, W) / 4, max_disp=2.0)
        a, b = f32(a), f32(b)
        if init == "zero":
            U0 = V0 = np.zeros((H, W), np.float32)
        elif init == "noise":
            U0, V0 = f32(rng.normal(0, 0.7, (H, W))), f32(rng.normal(0, 0.7, (H, W)))
        elif init == "large":  # some windows start outside the image: status 0 / early exit paths
            U0, V0 = f32(rng.uniform(-30, 30, (H, W))), f32(rng.uniform(-30, 30, (H, W)))
        else:
            U0, V0 = rotation(H, W, -0.02 if init == "rot-" else 0.02)
        ad = MG.quiet(LKm.denseLucasKanade_PyCl, Niter=nit, halfWindow=hw, enableVorticityEnhancement=vort)
        asym = np.array(ad.evaluateVorticityEnhancement(U0, V0), np.int32)
        U, V, err = MG.quiet(ad.compute, a, b, U0.copy(), V0.copy())
        d.update({f"I{i}": np.uint8(a), f"J{i}": np.uint8(b), f"U0_{i}": U0, f"V0_{i}": V0, f"U{i}": f32(U),
                  f"V{i}": f32(V), f"spec{i}": np.array([hw, nit, int(vort)]), f"asym{i}": asym})
    d["n"] = np.array(len(cases))
    out["lk_ref"] = d

    # --- A12-A19 + f2: Farneback_PyCL.compute (one pyramid level of the driver)
    d = {}
    cases = [dict(), dict(useGaussian=False), dict(polyN=5, polySigma=1.1), dict(pyramidalLevels=2, windowSize=21),
             dict(Niters=3, windowSize=15, useGaussian=False, polyN=5, polySigma=1.1)]
    shapes = [(128, 128), (96, 128), (96, 128), (128, 128), (64, 128)]
    for i, (kw, (H, W)) in enumerate(zip(cases, shapes)):
        a, b, _, _ = S.piv_pair(H, W, "fourier", seed=60 + i, max_disp=3.0)
        a, b = f32(a), f32(b)
        U0 = f32(rng.normal(0, 0.5, (H, W))) if i % 2 else np.zeros((H, W), np.float32)
        V0 = f32(rng.normal(0, 0.5, (H, W))) if i % 2 else np.zeros((H, W), np.float32)
        fb = MG.quiet(FBm.Farneback_PyCL, **kw)
        U, V, e = MG.quiet(fb.compute, a, b, U0.copy(), V0.copy())
        assert e == "Unknown"
        spec = [kw.get("windowSize", 33), kw.get("Niters", 5), kw.get("polyN", 7), kw.get("polySigma", 1.5),
                int(kw.get("useGaussian", True)), kw.get("pyramidalLevels", 1)]
        d.update({f"I{i}": np.uint8(a), f"J{i}": np.uint8(b), f"U0_{i}": U0, f"V0_{i}": V0, f"U{i}": f32(U),
                  f"V{i}": f32(V), f"spec{i}": np.array(spec, np.float64)})
    d["n"] = np.array(len(cases))
    out["fb_ref"] = d

    # --- A5 pipelines with the OpenCL adapters
    a, b, _, _ = S.piv_pair(128, 128, "lamb_oseen", seed=70, density=0.08, core_radius=15)
    a, b = f32(a), f32(b)
    lk = MG.quiet(LKm.denseLucasKanade_PyCl, Niter=5, halfWindow=13)
    U, V = MG.quiet(G.genericPyramidalOpticalFlow, a, b, 2, lk, 2, 1, 0.48, None, warping=False)
    out["pyr_lk_ref"] = dict(f0=np.uint8(a), f1=np.uint8(b), U=f32(U), V=f32(V))
    a, b, _, _ = S.piv_pair(128, 128, "fourier", seed=71)
    a, b = f32(a), f32(b)
    U, V = MG.quiet(G.genericPyramidalOpticalFlow, a, b, 0, MG.quiet(FBm.Farneback_PyCL), 2, 1, None, None)
    out["pyr_fb_ref"] = dict(f0=np.uint8(a), f1=np.uint8(b), U=f32(U), V=f32(V))
    ls = R["PhysicsBasedOpticalFlowLiuShen"]
    U, V = MG.quiet(G.genericPyramidalOpticalFlow, a, b, 0, MG.quiet(FBm.Farneback_PyCL), 2, 1, 0.48,
                    ls.LiuShenOpticalFlowAlgoAdapter(10))
    out["pyr_fbls_ref"] = dict(f0=np.uint8(a), f1=np.uint8(b), U=f32(U), V=f32(V))
    return out


def config_cases(R):
    """The three single-pair workloads at full size (seeds fixed here and in the GPU tests)."""
    import oracle as O
    from ofb200 import synthetic as S
    G, hs, ls = R["GenericPyramidalOpticalFlow"], R["HornSchunck"], R["PhysicsBasedOpticalFlowLiuShen"]
    LKm, FBm = R["denseLucasKanade_PyCL"], R["Farneback_PyCL"]
    out = {}
    runs = {
        "hs256": (lambda a, b: G.genericPyramidalOpticalFlow(a, b, 3.4, hs.HSOpticalFlowAlgoAdapter([21], 600), 1, 1,
                                                             None),
                  lambda a, b: O.pyramid(a, b, 3.4, O.HS([21], 600), 1, 1, None)),
        "lk512": (lambda a, b: G.genericPyramidalOpticalFlow(a, b, 2, LKm.denseLucasKanade_PyCl(Niter=5, halfWindow=13),
                                                             2, 1, 0.48, None, warping=False),
                  lambda a, b: O.pyramid(a, b, 2, O.LK(5, 13), 2, 1, 0.48, None, warping=False)),
        "fbls1024": (lambda a, b: G.genericPyramidalOpticalFlow(a, b, 0, FBm.Farneback_PyCL(), 2, 1, 0.48,
                                                                ls.LiuShenOpticalFlowAlgoAdapter(10)),
                     lambda a, b: O.pyramid(a, b, 0, O.FB(), 2, 1, 0.48, O.LS(10))),
    }
    for name, (ref_fn, ora_fn) in runs.items():
        a8, b8, Ug, Vg = S.config_pair(name, seed=1)
        a, b = f32(a8), f32(b8)
        t0 = time.time()
        Ur, Vr = MG.quiet(ref_fn, a.copy(), b.copy())
        t1 = time.time()
        Uo, Vo = ora_fn(a.copy(), b.copy())[:2]
        t2 = time.time()
        Ur, Vr, Uo, Vo = f32(Ur), f32(Vr), f32(Uo), f32(Vo)
        dmax = float(max(np.abs(Ur - Uo).max(), np.abs(Vr - Vo).max()))
        frac = float(np.mean(np.maximum(np.abs(Ur - Uo), np.abs(Vr - Vo)) > 1e-3))
        print(f"{name}: reference {t1 - t0:.1f} s, oracle {t2 - t1:.1f} s, max |oracle - reference| {dmax:.3g} px, "
              f"{100 * frac:.4f}% of pixels above 1e-3 px", flush=True)
        out.update({f"{name}_frames": np.array(sha(a8, b8)), f"{name}_ref": np.array(sha(Ur, Vr)),
                    f"{name}_oracle": np.array(sha(Uo, Vo)), f"{name}_Uref8": Ur[::8, ::8].copy(),
                    f"{name}_Vref8": Vr[::8, ::8].copy(), f"{name}_Uo8": Uo[::8, ::8].copy(),
                    f"{name}_Vo8": Vo[::8, ::8].copy(), f"{name}_maxdiff": np.array(dmax),
                    f"{name}_frac1e3": np.array(frac)})
    return {"configs": out}


def main():
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    ref = args[0] if args else os.environ.get("REFERENCE_SRC", "")
    if not ref or not os.path.isdir(ref):
        raise SystemExit("make_golden_cl.py: give the reference's src/ directory (argument or REFERENCE_SRC)")
    R = load(ref)
    out = config_cases(R) if "--configs" in sys.argv else small_cases(R)
    for name, d in out.items():
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **d)
        print("wrote", name, os.path.getsize(os.path.join(HERE, f"{name}.npz")))


if __name__ == "__main__":
    main()
