"""Concurrent multi-stream batches (ofb200.batch) give, pair for pair, the single-pair
result of the drop-in driver, for mixed sizes and methods, eager and graph-replayed."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _pair(size, seed):
    from ofb200 import synthetic as S
    a, b, _, _ = S.config_pair("fbls1024", seed=seed, size=size)
    return a.astype(np.float32), b.astype(np.float32)


def _specs():
    import Farneback_PyCL as F
    import HornSchunck as HS
    import PhysicsBasedOpticalFlowLiuShen as LS
    from ofb200.batch import PairSpec
    return [
        PairSpec(0, lambda: F.Farneback_PyCL(), 2, 1, 0.48, lambda: LS.LiuShenOpticalFlowAlgoAdapter(10),
                 key=("fbls",)),
        PairSpec(3.4, lambda: HS.HSOpticalFlowAlgoAdapter([7, 21, 45], 50), 2, 1, key=("hs",)),
        PairSpec(0, lambda: F.Farneback_PyCL(), 2, 1, 0.48, lambda: LS.LiuShenOpticalFlowAlgoAdapter(10),
                 key=("fbls",)),
        PairSpec(1.0, lambda: LS.LiuShenOpticalFlowAlgoAdapter(20), 1, 1, key=("ls",)),
    ], [(256, 1), (192, 2), (320, 3), (128, 4)]


def _single(spec, a, b):
    import GenericPyramidalOpticalFlow as G
    opt = spec.make_opt() if spec.make_opt is not None else None
    return G.genericPyramidalOpticalFlow(a, b, spec.FILTER, spec.make_main(), spec.pyramidalLevels, spec.kLevels,
                                         spec.FILTER_OPT, opt)


@pytest.mark.parametrize("use_graph", [False, True])
def test_batch_matches_single(torch_cuda, use_graph):
    torch = torch_cuda
    from ofb200 import graph
    from ofb200.batch import PairBatch
    specs, shapes = _specs()
    host = [_pair(s, seed) for s, seed in shapes]
    graph.ENABLED = False
    want = [_single(sp, a, b) for sp, (a, b) in zip(specs, host)]
    graph.ENABLED = True
    batch = PairBatch(specs, streams=3, use_graph=use_graph)
    dev = [(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()) for a, b in host]
    for _ in range(2):  # second run replays the captured graph
        got = batch.run(dev)
        torch.cuda.synchronize()
        for (Ug, Vg), (Uw, Vw) in zip(got, want):
            assert np.array_equal(Ug.cpu().numpy(), Uw)
            assert np.array_equal(Vg.cpu().numpy(), Vw)


def test_batch_new_inputs_replay(torch_cuda):
    """A replay on new frames of the same shapes gives those frames' results."""
    torch = torch_cuda
    from ofb200 import graph
    from ofb200.batch import PairBatch
    specs, shapes = _specs()
    batch = PairBatch(specs, streams=2)
    first = [_pair(s, seed) for s, seed in shapes]
    second = [_pair(s, seed + 50) for s, seed in shapes]
    batch.run([(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()) for a, b in first])
    got = batch.run([(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()) for a, b in second])
    got = [(u.cpu().numpy(), v.cpu().numpy()) for u, v in got]
    graph.ENABLED = False
    try:
        for sp, (a, b), (Ug, Vg) in zip(specs, second, got):
            Uw, Vw = _single(sp, a, b)
            assert np.array_equal(Ug, Uw) and np.array_equal(Vg, Vw)
    finally:
        graph.ENABLED = True


def test_batch_u8_frames(torch_cuda):
    torch = torch_cuda
    from ofb200 import synthetic as S
    from ofb200.batch import PairBatch
    specs, _ = _specs()
    a, b, _, _ = S.config_pair("fbls1024", seed=5, size=256)
    got = PairBatch(specs[:1], streams=1).run([(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda())])
    Uw, Vw = _single(specs[0], a.astype(np.float32), b.astype(np.float32))
    assert np.array_equal(got[0][0].cpu().numpy(), Uw) and np.array_equal(got[0][1].cpu().numpy(), Vw)


def test_batch_rejects_count_mismatch(torch_cuda):
    from ofb200.batch import PairBatch
    specs, _ = _specs()
    with pytest.raises(ValueError):
        PairBatch(specs).run([])


def ops_shapes():
    from ofb200 import ops
    return ops.hs_batch_shapes()


def test_config4_runner_matches_single_pairs(torch_cuda):
    """A small mixed manifest (all four methods, three sizes) through the chunked,
    autotuned runner gives each pair's single-call result."""
    torch = torch_cuda
    import GenericPyramidalOpticalFlow as G
    from ofb200 import graph
    from ofb200.batch import autotune, method_spec, render_entry
    entries = [{"size": s, "method": m, "flow": f, "seed": 70 + i}
               for i, (s, m, f) in enumerate([(128, "hs", "poiseuille"), (256, "lk", "lamb_oseen"),
                                              (256, "fb", "fourier"), (192, "ls", "fourier"),
                                              (128, "lk", "fourier"), (256, "hs", "lamb_oseen")])]
    rendered = [render_entry(e) for e in entries]
    frames = [(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()) for a, b, _, _ in rendered]
    runner, table = autotune(entries, frames, chunks=(2, 6), streams=(1, 3), reps=1)
    # chunk x streams candidates, the persistent Horn-Schunck kernel's tile shapes, and the
    # best candidate with the Horn-Schunck pairs back in the chunks
    assert len([k for k in table if isinstance(k[0], int)]) == 4
    assert len([k for k in table if k[0] == "hs_shape"]) == len(ops_shapes())
    assert len([k for k in table if k[0] == "hs_in_chunks"]) == 1
    outs = runner.run(frames)
    torch.cuda.synchronize()
    graph.ENABLED = False
    try:
        for e, (a, b, _, _), (U, V) in zip(entries, rendered, outs):
            sp = method_spec(e["method"])
            opt = sp.make_opt() if sp.make_opt is not None else None
            Uw, Vw = G.genericPyramidalOpticalFlow(a.astype(np.float32), b.astype(np.float32), sp.FILTER,
                                                   sp.make_main(), sp.pyramidalLevels, sp.kLevels, sp.FILTER_OPT, opt)
            assert np.array_equal(U.cpu().numpy(), Uw, equal_nan=True), e
            assert np.array_equal(V.cpu().numpy(), Vw, equal_nan=True), e
    finally:
        graph.ENABLED = True


def test_u16_frames_convert_on_device(torch_cuda):
    torch = torch_cuda
    from ofb200 import ops
    a = np.random.default_rng(3).integers(0, 4096, (33, 70)).astype(np.uint16)
    got = ops.u8_to_f32(torch.from_numpy(a).cuda())
    assert np.array_equal(got.cpu().numpy(), a.astype(np.float32))


def test_batch_status_words(cuda_ok):
    """Per-pair status words inside the batch graph: a host-injected NaN frame is reported
    (input and the NaN-polluted result), not a crash; clean pairs report only the Liu-Shen
    refine's use of all its sweeps (when the reference's tolerance 1e-8 is not reached), and the
    NaN pair does not disturb the other pairs' results."""
    import torch
    import Farneback_PyCL as FB
    import PhysicsBasedOpticalFlowLiuShen as LS
    from ofb200 import _lib, ops, synthetic as S
    from ofb200.batch import PairBatch, PairSpec
    frames = []
    for s in range(3):
        a, b, _, _ = S.config_pair("fbls1024", seed=50 + s, size=128)
        frames.append((ops.u8_to_f32(torch.from_numpy(a).cuda()), ops.u8_to_f32(torch.from_numpy(b).cuda())))
    spec = PairSpec(0, lambda: FB.Farneback_PyCL(), 2, 1, 0.48, lambda: LS.LiuShenOpticalFlowAlgoAdapter(10),
                    key=("fbls-status",))
    clean = PairBatch([spec] * 3, streams=3).run([(a.clone(), b.clone()) for a, b in frames])
    clean = [(U.clone(), V.clone()) for U, V in clean]
    bad = [(a.clone(), b.clone()) for a, b in frames]
    bad[1][1][40, 50] = float("nan")
    pb = PairBatch([spec] * 3, streams=3, status=True)
    for _ in range(2):  # eager capture run, then a graph replay
        out = pb.run(bad)
        st = pb.status.cpu().tolist()
        assert st[1] & _lib.ST_NONFINITE_INPUT and st[1] & _lib.ST_NONFINITE_OUTPUT
        for k in (0, 2):
            assert st[k] & ~_lib.ST_NOT_CONVERGED == 0
            assert torch.equal(out[k][0], clean[k][0]) and torch.equal(out[k][1], clean[k][1])


def test_host_batch_in_flight(torch_cuda):
    """HostBatch: host frames (numpy and pinned tensors) to host U, V with two batches in
    flight gives each batch's PairBatch result; a ticket whose slot was reused is refused."""
    torch = torch_cuda
    from ofb200.batch import HostBatch, PairBatch
    specs, shapes = _specs()
    batches = [[_pair(s, seed + 10 * k) for s, seed in shapes] for k in range(3)]
    want = []
    ref = PairBatch(specs, streams=2)
    for fr in batches:
        out = ref.run([(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()) for a, b in fr])
        want.append([(U.cpu().numpy(), V.cpu().numpy()) for U, V in out])
    hb = HostBatch(specs, streams=3, depth=2)
    pinned = [(torch.from_numpy(a).pin_memory(), torch.from_numpy(b).pin_memory()) for a, b in batches[1]]
    t0 = hb.submit(batches[0])
    t1 = hb.submit(pinned)
    got0 = [(U.copy(), V.copy()) for U, V in hb.result(t0)]
    t2 = hb.submit(batches[2])
    with pytest.raises(ValueError):
        hb.result(t0)
    got1, got2 = hb.result(t1), hb.result(t2)
    for got, exp in zip((got0, got1, got2), want):
        for (Ug, Vg), (Uw, Vw) in zip(got, exp):
            assert np.array_equal(Ug, Uw) and np.array_equal(Vg, Vw)
    with pytest.raises(ValueError):
        hb.submit(batches[0][:2])
