"""Horn-Schunck in one persistent launch (of_hs_batch), under both schedules: the device
work queue and the resident one (a CTA per tile for the whole solve, region on chip).

Bit-exact with the regular solver (of_hs_solve, itself bit-exact with the reference) for
one pair and for a batch of uneven pairs, with every tile shape; per-pair status words for
a NaN frame; and the bounded wait running out (a short wait limit) ends the launch with a
timeout status instead of hanging, leaving the context usable."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _pair(torch, H, W, seed):
    from ofb200 import synthetic as S
    a, b, _, _ = S.piv_pair(H, W, "poiseuille", seed=seed)
    return torch.from_numpy(a.astype(np.float32)).cuda(), torch.from_numpy(b.astype(np.float32)).cuda()


def _solve_ref(torch, a, b, U0, V0, alpha, niter):
    from ofb200 import ops
    U, V = U0.clone(), V0.clone()
    ops.hs_solve(a, b, U, V, alpha, niter, persistent=False)  # one launch per pass
    return U, V


@pytest.mark.parametrize("H,W,niter", [(256, 256, 600), (100, 300, 37), (17, 23, 9), (12, 40, 5), (64, 64, 0)])
def test_persistent_single_solve_equals_multi_launch(cuda_ok, H, W, niter):
    """of_hs_solve_persistent (the drop-in's single-pair form) against of_hs_solve: the
    same U, V bit for bit, and the same error value, from a non-zero initial flow."""
    import torch
    from ofb200 import ops
    a, b = _pair(torch, H, W, 31)
    g = torch.Generator().manual_seed(H + W)
    U0 = (torch.randn(H, W, generator=g) * 0.3).cuda()
    V0 = (torch.randn(H, W, generator=g) * 0.3).cuda()
    out = []
    for persistent in (False, True):
        U, V = U0.clone(), V0.clone()
        _, _, err = ops.hs_solve(a, b, U, V, 21.0, niter, persistent=persistent)
        out.append((U, V, float(err.item())))
    assert torch.equal(out[0][0], out[1][0]) and torch.equal(out[0][1], out[1][1])
    # the error's float64 sums are combined across CTAs by atomics (order-dependent last bit)
    assert out[0][2] == pytest.approx(out[1][2], rel=1e-12, abs=0.0)


SCHEDULES = ["queue", "resident"]


@pytest.mark.parametrize("schedule", SCHEDULES + ["cluster"])
@pytest.mark.parametrize("shape_index", [0, 1, 2, 3, 4])
def test_single_pair_config1_bit_exact(cuda_ok, shape_index, schedule):
    """256 x 256, alpha 21, 600 sweeps (the PyHSchunck_Fs3_4 calibration) in one launch."""
    import torch
    from ofb200 import ops
    a, b = _pair(torch, 256, 256, 1)
    z = torch.zeros_like(a)
    Ur, Vr = _solve_ref(torch, a, b, z, z, 21.0, 600)
    U, V = z.clone(), z.clone()
    st = ops.hs_batch([(a, b, U, V, 21.0, 600)], tile_shape=shape_index, schedule=schedule)
    torch.cuda.synchronize()
    assert int(st.item()) == 0
    assert torch.equal(U, Ur) and torch.equal(V, Vr)


@pytest.mark.parametrize("schedule,shape_index", [("queue", 0), ("resident", 0), ("queue", 4)])
def test_uneven_batch_bit_exact(cuda_ok, schedule, shape_index):
    """Uneven sizes and sweep counts (600, 37, 9, 0: a last pass of fewer sweeps than the
    shape's, and a pair with no sweep pass) in one launch, with 256- and 512-thread CTAs
    (the 573 tiles of shape 4 are more than the resident schedule's one CTA per SM)."""
    import torch
    from ofb200 import ops
    shapes = [(128, 128, 600), (256, 256, 600), (64, 200, 37), (512, 384, 120), (17, 23, 9), (16, 16, 0)]
    pairs, refs = [], []
    g = torch.Generator().manual_seed(4)
    for k, (H, W, n) in enumerate(shapes):
        a, b = _pair(torch, H, W, 10 + k)
        U0 = (torch.randn(H, W, generator=g) * 0.3).cuda()
        V0 = (torch.randn(H, W, generator=g) * 0.3).cuda()
        refs.append(_solve_ref(torch, a, b, U0, V0, 21.0 + k, n))
        pairs.append((a, b, U0.clone(), V0.clone(), 21.0 + k, n))
    st = ops.hs_batch(pairs, tile_shape=shape_index, schedule=schedule)
    torch.cuda.synchronize()
    assert st.cpu().tolist() == [0] * len(shapes)
    for (_, _, U, V, _, _), (Ur, Vr) in zip(pairs, refs):
        assert torch.equal(U, Ur) and torch.equal(V, Vr)


@pytest.mark.parametrize("schedule", SCHEDULES)
def test_nonfinite_frame_sets_status(cuda_ok, schedule):
    import torch
    from ofb200 import _lib, ops
    a, b = _pair(torch, 64, 64, 3)
    a2, b2 = _pair(torch, 64, 64, 4)
    b2[10, 20] = float("nan")
    z = torch.zeros_like(a)
    pairs = [(a, b, z.clone(), z.clone(), 21.0, 40), (a2, b2, z.clone(), z.clone(), 21.0, 40)]
    st = ops.hs_batch(pairs, schedule=schedule).cpu().tolist()
    assert st[0] == 0
    assert st[1] & _lib.ST_NONFINITE_INPUT and st[1] & _lib.ST_NONFINITE_OUTPUT


@pytest.mark.parametrize("schedule", SCHEDULES)
def test_bounded_wait_runs_out_and_returns(cuda_ok, schedule):
    """A wait limit of one poll: items that find their previous pass unfinished give up at
    once.  The launch ends, the failed pairs carry OF_ST_WAIT_TIMEOUT, and the pairs that
    report no error are bit-exact; afterwards the context works (a normal run follows)."""
    import torch
    from ofb200 import _lib, ops
    pairs, refs = [], []
    for k in range(4):
        a, b = _pair(torch, 256, 256, 20 + k)
        z = torch.zeros_like(a)
        refs.append(_solve_ref(torch, a, b, z, z, 21.0, 200))
        pairs.append((a, b, z.clone(), z.clone(), 21.0, 200))
    st = ops.hs_batch(pairs, wait_limit=1, schedule=schedule).cpu().tolist()
    assert any(s & _lib.ST_WAIT_TIMEOUT for s in st)
    for s, (_, _, U, V, _, _), (Ur, Vr) in zip(st, pairs, refs):
        assert s in (0, _lib.ST_WAIT_TIMEOUT)
        if s == 0:
            assert torch.equal(U, Ur) and torch.equal(V, Vr)
    for p in pairs:
        p[2].zero_()
        p[3].zero_()
    st = ops.hs_batch(pairs, schedule=schedule).cpu().tolist()
    assert st == [0] * 4
    for (_, _, U, V, _, _), (Ur, Vr) in zip(pairs, refs):
        assert torch.equal(U, Ur) and torch.equal(V, Vr)


def test_batch_runner_hs_group_equals_per_pair_graphs(cuda_ok):
    """The batched workload with its Horn-Schunck pairs in one persistent launch gives the
    same fields as with every pair in its own per-pair pipeline."""
    import torch
    from ofb200.batch import BatchRunner, config4_manifest, render_entry
    entries = [e for e in config4_manifest(40, seed=3) if e["size"] <= 512][:12]
    assert any(e["method"] == "hs" for e in entries)
    frames = []
    for e in entries:
        a, b, _, _ = render_entry(e)
        frames.append((torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()))
    ref = [(U.clone(), V.clone()) for U, V in BatchRunner(entries, chunk=8, streams=4).run(frames)]
    for shape in (0, 1):
        got = BatchRunner(entries, chunk=8, streams=4, hs_shape=shape).run(frames)
        for (U, V), (Ur, Vr) in zip(got, ref):
            assert torch.equal(U, Ur) and torch.equal(V, Vr)


def test_fast_arithmetic_within_float32_rounding(cuda_ok):
    """OF_HS_FAST (float32 averaging) stays within 1e-4 px of the bit-exact solver after
    600 sweeps at 256^2 (the reference's float64 answer is within a few 1e-6 px of both)."""
    import torch
    from ofb200 import ops
    a, b = _pair(torch, 256, 256, 1)
    z = torch.zeros_like(a)
    Ur, Vr = _solve_ref(torch, a, b, z, z, 21.0, 600)
    for shape in range(len(ops.hs_batch_shapes())):
        U, V = z.clone(), z.clone()
        st = ops.hs_batch([(a, b, U, V, 21.0, 600)], tile_shape=shape, arithmetic="fast")
        assert int(st.item()) == 0
        assert max((U - Ur).abs().max().item(), (V - Vr).abs().max().item()) <= 1e-4


def test_resident_schedule_refuses_more_tiles_than_ctas(cuda_ok):
    """A 2048^2 pair cut into 24 x 16 tiles has more tiles than resident CTAs: the resident
    schedule is refused with an error, and the automatic choice falls back to the queue."""
    import torch
    from ofb200 import _lib, ops
    a = torch.zeros(2048, 2048, device="cuda")
    U, V = torch.zeros_like(a), torch.zeros_like(a)
    with pytest.raises(_lib.OfError):
        ops.hs_batch([(a, a, U, V, 21.0, 4)], tile_shape=1, schedule="resident")
    st = ops.hs_batch([(a, a, U, V, 21.0, 4)], tile_shape=1, schedule="auto")
    assert int(st.item()) == 0 and float(U.abs().max()) == 0.0


@pytest.mark.parametrize("H,W,niter", [(256, 256, 601), (200, 130, 37), (64, 17, 9), (16, 16, 2), (100, 255, 0)])
def test_cluster_schedule_shapes(cuda_ok, H, W, niter):
    """The cluster schedule (one thread-block cluster, halos through distributed shared
    memory) on uneven tilings, odd sweep counts and the smallest images, from a non-zero
    initial flow, bit for bit against the multi-launch solver; float32 averaging within 1e-4."""
    import torch
    from ofb200 import ops
    a, b = _pair(torch, H, W, 41)
    g = torch.Generator().manual_seed(H * W)
    U0 = (torch.randn(H, W, generator=g) * 0.3).cuda()
    V0 = (torch.randn(H, W, generator=g) * 0.3).cuda()
    Ur, Vr = _solve_ref(torch, a, b, U0, V0, 21.0, niter)
    U, V = U0.clone(), V0.clone()
    st = ops.hs_batch([(a, b, U, V, 21.0, niter)], schedule="cluster")
    assert int(st.item()) == 0
    assert torch.equal(U, Ur) and torch.equal(V, Vr)
    U, V = U0.clone(), V0.clone()
    st = ops.hs_batch([(a, b, U, V, 21.0, niter)], schedule="cluster", arithmetic="fast")
    assert int(st.item()) == 0
    assert max((U - Ur).abs().max().item(), (V - Vr).abs().max().item()) <= 1e-4


def test_cluster_schedule_refusals_and_status(cuda_ok):
    """Two pairs, or an image beyond 16 tiles of 64 x 64, are refused; a NaN frame sets the
    status bits."""
    import torch
    from ofb200 import _lib, ops
    a, b = _pair(torch, 64, 64, 5)
    z = torch.zeros_like(a)
    with pytest.raises(_lib.OfError):
        ops.hs_batch([(a, b, z.clone(), z.clone(), 21.0, 4)] * 2, schedule="cluster")
    big = torch.zeros(300, 300, device="cuda")
    with pytest.raises(_lib.OfError):
        ops.hs_batch([(big, big, big.clone(), big.clone(), 21.0, 4)], schedule="cluster")
    b2 = b.clone()
    b2[10, 20] = float("nan")
    st = int(ops.hs_batch([(a, b2, z.clone(), z.clone(), 21.0, 40)], schedule="cluster").item())
    assert st & _lib.ST_NONFINITE_INPUT and st & _lib.ST_NONFINITE_OUTPUT


@pytest.mark.parametrize("shape_index", [3, 4])
def test_auto_schedule_runs_resident_on_an_idle_device(cuda_ok, shape_index):
    """The automatic schedule launches one CTA per tile; with the device to itself every CTA
    runs at once and they choose the resident schedule: bit-exact, and reported as such."""
    import torch
    from ofb200 import ops
    a, b = _pair(torch, 256, 256, 1)
    z = torch.zeros_like(a)
    Ur, Vr = _solve_ref(torch, a, b, z, z, 21.0, 600)
    pairs = [(a, b, z.clone(), z.clone(), 21.0, 600)]
    st = ops.hs_batch(pairs, tile_shape=shape_index, schedule="auto")
    assert int(st.item()) == 0
    assert torch.equal(pairs[0][2], Ur) and torch.equal(pairs[0][3], Vr)
    assert ops.hs_batch_schedule(pairs) == "resident"
    ops.hs_batch(pairs, tile_shape=shape_index, schedule="queue")
    assert ops.hs_batch_schedule(pairs) == "auto"  # an explicit schedule makes no decision


_OCCUPY_SRC = rb"""
extern "C" __global__ void occupy(unsigned long long ns) {
  extern __shared__ volatile int held[];
  unsigned long long t0, t = 0;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
  for (int k = 0; k < 200000; k++) {  // ends after ns, or after 200000 short sleeps
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    if (t - t0 > ns) break;
    __nanosleep(1000);
  }
  if (threadIdx.x == 0) held[0] = (int)(t - t0);
}
"""


def _occupy(torch, stream, ctas, smem_bytes, ns):
    """Launches `ctas` CTAs of one warp that each hold `smem_bytes` of shared memory (so an SM
    takes one) for about `ns` nanoseconds, on `stream`: other kernels find those SMs taken."""
    from cuda.bindings import driver, nvrtc
    err, prog = nvrtc.nvrtcCreateProgram(_OCCUPY_SRC, b"occupy.cu", 0, [], [])
    assert err == nvrtc.nvrtcResult.NVRTC_SUCCESS
    (err,) = nvrtc.nvrtcCompileProgram(prog, 1, [b"--gpu-architecture=sm_100a"])
    assert err == nvrtc.nvrtcResult.NVRTC_SUCCESS
    err, n = nvrtc.nvrtcGetCUBINSize(prog)
    cubin = b" " * n
    (err,) = nvrtc.nvrtcGetCUBIN(prog, cubin)
    assert err == nvrtc.nvrtcResult.NVRTC_SUCCESS
    err, mod = driver.cuModuleLoadData(cubin)
    assert err == driver.CUresult.CUDA_SUCCESS
    err, fn = driver.cuModuleGetFunction(mod, b"occupy")
    assert err == driver.CUresult.CUDA_SUCCESS
    (err,) = driver.cuFuncSetAttribute(fn, driver.CUfunction_attribute.CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES,
                                       smem_bytes)
    assert err == driver.CUresult.CUDA_SUCCESS
    arg = np.array([ns], dtype=np.uint64)
    params = np.array([arg.ctypes.data], dtype=np.uint64)
    (err,) = driver.cuLaunchKernel(fn, ctas, 1, 1, 32, 1, 1, smem_bytes, driver.CUstream(stream.cuda_stream),
                                   params.ctypes.data, 0)
    assert err == driver.CUresult.CUDA_SUCCESS
    return mod, arg, params


def test_auto_schedule_falls_back_to_the_queue_when_sms_are_taken(cuda_ok):
    """Another kernel holds all but 20 SMs for a few milliseconds when the automatic launch
    starts: its 256 CTAs cannot all run, they give up the resident schedule within their
    bounded poll and run the queue instead, and the result is still bit-exact."""
    import time
    import torch
    from ofb200 import ops
    a, b = _pair(torch, 256, 256, 1)
    z = torch.zeros_like(a)
    Ur, Vr = _solve_ref(torch, a, b, z, z, 21.0, 600)
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    side, main = torch.cuda.Stream(), torch.cuda.Stream()
    torch.cuda.synchronize()
    held = _occupy(torch, side, sms - 20, 200 * 1024, 5_000_000)
    time.sleep(0.001)  # the occupying CTAs are on their SMs
    with torch.cuda.stream(main):
        pairs = [(a, b, z.clone(), z.clone(), 21.0, 600)]
        st = ops.hs_batch(pairs, tile_shape=3, schedule="auto")
        mode = ops.hs_batch_schedule(pairs)
    torch.cuda.synchronize()
    del held
    assert int(st.item()) == 0
    assert torch.equal(pairs[0][2], Ur) and torch.equal(pairs[0][3], Vr)
    assert mode == "queue"
