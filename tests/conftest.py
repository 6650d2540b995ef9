import os
import sys

import pytest

# The parity suites compare the Liu-Shen solver bit for bit, which only its 'exact'
# arithmetic promises; the float32 'fast' arithmetic (the library default) is tested on its
# own, explicitly, in test_gpu_ls_fast.py.
os.environ["OFB_LS_ARITHMETIC"] = "exact"
# autotuning choices made by tests go to a scratch file, not the user's cache
import tempfile  # noqa: E402

os.environ.setdefault("OFB_AUTOTUNE_CACHE", os.path.join(tempfile.mkdtemp(prefix="ofb200-tune-"), "autotune.json"))

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "opticalflow-ri_b200")
for p in (PKG, os.path.join(REPO, "oracle"), REPO):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(REPO, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def golden(name):
    import numpy as np
    return np.load(os.path.join(GOLDEN, f"{name}.npz"))


@pytest.fixture(scope="session")
def cuda_ok():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return True
