"""of_batch_run (the pyramid driver in C++, for callers outside Python) against the Python
drop-in on a mixed batch: Horn-Schunck (one level: its solves in the persistent launch; and
two levels with the warp), dense LK pyr2, Farneback pyr2 (Gaussian and box windows) and
Farneback pyr2 + Liu-Shen, uint8 and float32 frames, uneven sizes.  Bit for bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_batch_run_equals_python_driver(cuda_ok):
    import torch
    import denseLucasKanade_PyCL as LK
    import Farneback_PyCL as FB
    import HornSchunck as HS
    import PhysicsBasedOpticalFlowLiuShen as LS
    from ofb200 import _lib, synthetic as S
    from ofb200.batch import PairBatch, PairSpec, run_c
    specs = [
        PairSpec(3.4, lambda: HS.HSOpticalFlowAlgoAdapter([21], 600), 1, 1, key=("hs1",)),
        PairSpec(3.4, lambda: HS.HSOpticalFlowAlgoAdapter([21, 45], 100), 2, 1, key=("hs2",)),
        PairSpec(2.0, lambda: LK.denseLucasKanade_PyCl(Niter=5, halfWindow=13), 2, 1, 0.48, key=("lk",)),
        PairSpec(0, lambda: FB.Farneback_PyCL(), 2, 1, key=("fb",)),
        PairSpec(0, lambda: FB.Farneback_PyCL(useGaussian=False, windowSize=15), 2, 1, key=("fbbox",)),
        PairSpec(0, lambda: FB.Farneback_PyCL(), 2, 1, 0.48, lambda: LS.LiuShenOpticalFlowAlgoAdapter(10),
                 key=("fbls",)),
        PairSpec(3.4, lambda: HS.HSOpticalFlowAlgoAdapter([17], 40), 1, 1, key=("hs1b",)),
    ]
    sizes = [(128, 128), (96, 160), (256, 256), (128, 192), (128, 128), (256, 256), (64, 96)]
    frames = []
    for k, (H, W) in enumerate(sizes):
        a, b, _, _ = S.piv_pair(H, W, "lamb_oseen", seed=80 + k, core_radius=H / 6, max_disp=2.0)
        ta, tb = torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()
        if k % 2:  # float32 frames for some pairs
            ta, tb = ta.float(), tb.float()
        frames.append((ta, tb))
    want = PairBatch(specs, streams=1, use_graph=False).run(frames)
    want = [(U.clone(), V.clone()) for U, V in want]
    got, st = run_c(specs, frames, tile_shape=1)
    torch.cuda.synchronize()
    s = st.cpu().tolist()
    for k, ((U, V), (Uw, Vw)) in enumerate(zip(got, want)):
        assert torch.equal(U, Uw) and torch.equal(V, Vw), k
        assert s[k] & ~_lib.ST_NOT_CONVERGED == 0, (k, s[k])
