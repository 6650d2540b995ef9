"""Consistency of the full-size fixture (tests/golden/configs.npz): the synthetic pairs it
was made from are regenerated identically here, and the CPU oracle's digest equals the
reference's for every workload (both were recorded by make_golden_cl.py --configs)."""
import hashlib

import numpy as np
import pytest

from conftest import golden


@pytest.mark.parametrize("cfg", ["hs256", "lk512", "fbls1024"])
def test_fixture_frames_and_oracle_digest(cfg):
    from ofb200 import synthetic as S
    g = golden("configs")
    a8, b8, _, _ = S.config_pair(cfg, seed=1)
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(a8).tobytes())
    h.update(np.ascontiguousarray(b8).tobytes())
    assert h.hexdigest() == str(g[f"{cfg}_frames"])
    assert str(g[f"{cfg}_oracle"]) == str(g[f"{cfg}_ref"])
    assert float(g[f"{cfg}_maxdiff"]) == 0.0
