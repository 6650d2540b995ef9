"""The float64 restatement (oracle/oracle_f64.py) against the reference's float32 goldens:
the same algorithm, so the two agree to float32 rounding, and no closer (it is not a
copy of the float32 path)."""
import numpy as np
import pytest

import oracle as O
import oracle_f64 as F
from conftest import golden


def test_hs_ls_agree_with_float32_reference():
    g = golden("hs")
    u, v, _ = F.hs_solve(g["f0"], g["f1"], g["U0"], g["V0"], float(g["alpha"]), int(g["niter"]))
    assert np.abs(u - g["U"]).max() < 1e-5 and np.abs(v - g["V"]).max() < 1e-5
    assert not np.array_equal(u.astype(np.float32), g["U"])
    g = golden("ls")
    U, V, _, it = F.ls_solve(g["f0"], g["f1"], g["U0"], g["V0"], float(g["h"]))
    assert it == 60 and np.abs(U - g["U"]).max() < 1e-5 and np.abs(V - g["V"]).max() < 1e-5


def test_prefilter_and_resize_agree_with_float32_reference():
    g = golden("prefilter")
    for i, (s, K) in enumerate([(3.4, 3), (2.0, 3), (0.48, 5)]):
        ref = g[f"out{i}"]
        assert np.abs(F.prefilter(g["img"], s, K) - ref).max() <= 4e-7 * np.abs(ref).max()
    g = golden("resize")
    for i in range(6):
        Wd, Hd, bc = (int(x) for x in g[f"spec{i}"])
        ref = g[f"dst{i}"]
        assert np.abs(F.resize(g[f"src{i}"], (Wd, Hd), bool(bc)) - ref).max() <= 4e-7 * np.abs(ref).max() + 1e-6


@pytest.mark.parametrize("cfg", ["hs", "fbls"])
def test_pipelines_float32_within_tolerance_of_float64(cfg):
    """The reference's float32 pipeline (the oracle, bit-exact with it) stays within the
    1e-3 px bound of the float64 answer on small pairs of both HS and Farneback + Liu-Shen."""
    from ofb200 import synthetic as S
    if cfg == "hs":
        a8, b8, _, _ = S.config_pair("hs256", seed=2, size=96)
        a, b = a8.astype(np.float32), b8.astype(np.float32)
        U, V = O.pyramid(a, b, 3.4, O.HS([21], 200), 1, 1, None)
        U6, V6 = F.pyramid(a, b, 3.4, F.HS([21], 200), 1, 1, None)
    else:
        a8, b8, _, _ = S.config_pair("fbls1024", seed=2, size=128)
        a, b = a8.astype(np.float32), b8.astype(np.float32)
        U, V = O.pyramid(a, b, 0, O.FB(), 2, 1, 0.48, O.LS(10))
        U6, V6 = F.pyramid(a, b, 0, F.FB(), 2, 1, 0.48, F.LS(10))
    assert max(np.abs(U - U6).max(), np.abs(V - V6).max()) < 1e-3
