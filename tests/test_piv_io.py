"""TIFF ingest (8-bit and 16-bit containers) and the examples' .mat output."""
import numpy as np
import pytest


@pytest.mark.parametrize("bits", [8, 10, 12])
def test_read_frame_tiff(tmp_path, bits):
    from PIL import Image

    from ofb200.piv_io import read_frame, read_raw
    rng = np.random.default_rng(bits)
    a = rng.integers(0, 2 ** bits, (37, 53))
    a = a.astype(np.uint8 if bits == 8 else np.uint16)
    fn = str(tmp_path / f"f{bits}.tif")
    Image.fromarray(a).save(fn)
    raw = read_raw(fn)
    assert raw.dtype == a.dtype and np.array_equal(raw, a)
    f = read_frame(fn)
    assert f.dtype == np.float32 and np.array_equal(f, a.astype(np.float32))


def test_save_flow_structure(tmp_path):
    import scipy.io

    from ofb200.piv_io import load_flow, save_flow
    U = np.random.default_rng(0).normal(0, 1, (12, 17)).astype(np.float32)
    V = -U
    fn = str(tmp_path / "flow.mat")
    save_flow(U, V, fn)
    m = scipy.io.loadmat(fn)
    vel, par = m["velocities"][0, 0], m["parameters"][0, 0]
    assert set(vel.dtype.names) == {"u", "v", "iaWidth", "iaHeight", "margins"}
    assert set(vel["margins"][0, 0].dtype.names) == {"top", "left", "bottom", "right"}
    assert par["imageHeight"].item() == 12 and par["imageWidth"].item() == 17 and par["overlapFactor"].item() == 1.0
    u, v = load_flow(fn)
    assert np.array_equal(u, U) and np.array_equal(v, V)
