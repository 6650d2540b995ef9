"""Benchmark of the dense pyramidal optical-flow hot path on B200.

Workload (the headline metric's plain arm): the LiuSE_Farneback_Fs0_0_PyrLvls2 calibration
(Farneback, 2 pyramid levels, no prefilter, then Liu-Shen refinement with h = 10 on
FILTER_OPT = 0.48 prefiltered frames) on 1024x1024 uint8 synthetic PIV pairs with a
divergence-free random-Fourier displacement (max 4 px, 0.05 particles/px, diameter 2-3 px,
noise 2 DN).  One step = `--pairs` frame pairs through the whole pipeline, spread over
`--streams` concurrent CUDA streams and replayed as one CUDA graph (ofb200.batch).

  value : pairs/s with the frames already resident in HBM (device-timed, CUDA events),
          aggregated over all ranks (pairs / max-over-ranks time).
  e2e   : pairs/s from host memory to host memory: the step's pairs as pinned uint8 frames
          through ofb200.batch.HostBatch (uploads, the batch graph and the downloads of U, V
          into pinned buffers, two steps in flight), wall clock; e2e.single_call is the
          one-pair drop-in call (genericPyramidalOpticalFlow, numpy float32 frames in, numpy
          U, V out) back to back.
  roofline : the Liu-Shen solves of one step (the dominant kernel): --pairs solves at
          1024^2 running concurrently on --streams streams, as they do in the step (their
          working set, 60 MB each, exceeds the 126 MB L2), algorithmic bytes = (24 B x
          sweeps + 8 B) per pixel per solve, against the measured HBM copy bandwidth.
  configs : the other workloads, each with its own device-timed pairs/s, roofline and CPU
          baseline: Horn-Schunck 256^2 (600 sweeps), dense LK pyr2 512^2, and the batch of
          256 uneven pairs (128^2-2048^2, four methods; --no-batch skips it).
  cpu_baseline : the CPU oracle (C restatement of the reference, 1 thread) on one pair.

--impl reference: the CPU restatement of the reference's path (the reference itself needs
OpenCL for Farneback and cannot run on the box), on all host cores, one pair per worker
per step.

Multi-GPU (torchrun): pairs are independent; every rank runs its own pairs (weak scaling),
no collective on the data path.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "opticalflow-ri_b200"))

METRIC = "pairs/s @1024^2 Liu-Shen (Farneback pyr2 + Liu-Shen, plain)"
WORKLOAD = "LiuSE_Farneback_Fs0_0_PyrLvls2 1024x1024 random-Fourier PIV pairs"
L2_BYTES = 126 * 2 ** 20
REF_BUDGET_S = 90.0
# DRAM bytes (read + write) of one 60-sweep Liu-Shen solve at 1024^2, summed over its
# launches from one ncu capture per arithmetic (profiles/ls_solve_traffic_1024.txt; cold cache
# per launch)
NCU_LS_TRAFFIC = {("exact", 1024): 663.48e6, ("fast", 1024): 663.49e6}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=50)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--pairs", type=int, default=8, help="frame pairs per step per GPU")
    p.add_argument("--size", type=int, default=1024)
    p.add_argument("--unique", type=int, default=4, help="distinct synthetic pairs (cycled)")
    p.add_argument("--streams", type=int, default=8,
                   help="concurrent CUDA streams per step (1: pairs one after another)")
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-learned", action="store_true", help="skip the learned warm-start arm")
    p.add_argument("--no-roofline", action="store_true", help="skip the Liu-Shen roofline block (profiling runs)")
    p.add_argument("--no-configs", action="store_true", help="skip the HS 256^2 / LK 512^2 / batch workloads")
    p.add_argument("--no-batch", action="store_true", help="skip the 256-pair batch inside the configs block")
    p.add_argument("--learned-weights", default=None, help="weights + calibration .npz (default: packaged)")
    p.add_argument("--learned-pairs", type=int, default=64, help="pairs per step of the learned arm (batch)")
    p.add_argument("--epe-pairs", type=int, default=32, help="distinct held-out pairs for the endpoint errors")
    p.add_argument("--batch-pairs", type=int, default=256, help="--mode batch: pairs in the manifest")
    p.add_argument("--mode", default="pipeline", choices=["pipeline", "ls", "batch", "cnn", "fb", "e2e", "hs", "lk",
                                                          "learned"],
                   help="ls: only the Liu-Shen solve of one pair, --steps times (for profiling)")
    return p.parse_args()


def run_ls_only(args):
    """Liu-Shen solve on one prefiltered --size pair, --warmup + --steps times."""
    import torch
    from gaussian_filter import prepareGaussianKernel
    from ofb200 import ops
    a, b, _, _ = make_pairs(1, args.size)[0]
    taps = prepareGaussianKernel(0.48, 5)
    fa = ops.prefilter(torch.from_numpy(a).cuda(), taps)
    fb = ops.prefilter(torch.from_numpy(b).cuda(), taps)
    ms = []
    for r in range(args.warmup + args.steps):
        U, V = torch.zeros_like(fa), torch.zeros_like(fa)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        _, _, it, _ = ops.ls_solve(fa, fb, U, V, 10.0)
        e1.record()
        e1.synchronize()
        if r >= args.warmup:
            ms.append(e0.elapsed_time(e1))
    print(json.dumps({"mode": "ls", "size": args.size, "sweeps": int(it.item()), "ms": float(np.mean(ms))}))


def run_hs_only(args):
    """Horn-Schunck, 600 sweeps at --size: the multi-launch solver (of_hs_solve) against the
    persistent one-launch solver (of_hs_batch) with every tile shape, one pair; CUDA events."""
    import torch
    from ofb200 import ops, synthetic as S
    a8, b8, _, _ = S.config_pair("hs256", seed=1, size=args.size)
    a = torch.from_numpy(a8.astype(np.float32)).cuda()
    b = torch.from_numpy(b8.astype(np.float32)).cuda()
    z = torch.zeros_like(a)

    def timeit(fn):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            fn()
        e1.record()
        e1.synchronize()
        return e0.elapsed_time(e1) / args.steps

    out = {"mode": "hs", "size": args.size, "sweeps": 600}
    U, V = z.clone(), z.clone()
    out["of_hs_solve_ms"] = timeit(lambda: ops.hs_solve(a, b, U.zero_(), V.zero_(), 21.0, 600))
    Um, Vm = z.clone(), z.clone()
    out["of_hs_solve_multilaunch_ms"] = timeit(lambda: ops.hs_solve(a, b, Um.zero_(), Vm.zero_(), 21.0, 600,
                                                                    persistent=False))
    for ar in ("exact", "fast"):  # one thread-block cluster (the tile shapes do not apply)
        U2, V2 = z.clone(), z.clone()
        out[f"of_hs_batch_cluster_{ar}_ms"] = timeit(lambda: ops.hs_batch(
            [(a, b, U2.zero_(), V2.zero_(), 21.0, 600)], arithmetic=ar, schedule="cluster"))
        out[f"cluster_{ar}_maxdiff"] = float(max((U2 - U).abs().max().item(), (V2 - V).abs().max().item()))
    for sched in ("queue", "resident"):
        for k, shp in enumerate(ops.hs_batch_shapes()):
            for ar in ("exact", "fast"):
                U2, V2 = z.clone(), z.clone()
                tag = f"{sched}_{ar}_shape{k}_{shp[0]}x{shp[1]}t{shp[2]}"
                out[f"of_hs_batch_{tag}_ms"] = timeit(lambda: ops.hs_batch(
                    [(a, b, U2.zero_(), V2.zero_(), 21.0, 600)], tile_shape=k, arithmetic=ar, schedule=sched))
                out[f"{tag}_maxdiff"] = float(max((U2 - U).abs().max().item(), (V2 - V).abs().max().item()))
    print(json.dumps(out))


def run_lk_only(args):
    """Dense LK (27 x 27 window, 5 Newton steps) on one --size pair from zero flow, and the
    LK pyr2 pipeline, --steps times after --warmup; CUDA events."""
    import torch
    import denseLucasKanade_PyCL as LK
    import GenericPyramidalOpticalFlow as G
    from ofb200 import ops, synthetic as S
    a8, b8, _, _ = S.config_pair("lk512", seed=1, size=args.size)
    I = torch.from_numpy(a8.astype(np.float32)).cuda()
    J = torch.from_numpy(b8.astype(np.float32)).cuda()
    U, V = torch.zeros_like(I), torch.zeros_like(I)
    ms = []
    for r in range(args.warmup + args.steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        ops.lk_dense(I, J, U.zero_(), V.zero_())
        e1.record()
        e1.synchronize()
        if r >= args.warmup:
            ms.append(e0.elapsed_time(e1))
    pm = []
    for r in range(args.warmup + args.steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        G.genericPyramidalOpticalFlow(I, J, 2, LK.denseLucasKanade_PyCl(Niter=5, halfWindow=13), 2, 1, 0.48, None,
                                      warping=False)
        e1.record()
        e1.synchronize()
        if r >= args.warmup:
            pm.append(e0.elapsed_time(e1))
    px = args.size * args.size
    t = float(np.mean(ms))
    print(json.dumps({"mode": "lk", "size": args.size, "lk_dense_ms": t, "pyr2_pipeline_ms": float(np.mean(pm)),
                      "tflops_at_7e4_flop_per_px": 7e4 * px / (t * 1e-3) / 1e12}))


def run_e2e_only(args):
    """The end-to-end figures alone: --pairs pairs per step through HostBatch (pinned uint8
    frames in, numpy U, V out, two steps in flight) and the one-pair drop-in call
    (genericPyramidalOpticalFlow, numpy float32 frames in and numpy U, V out); wall clock."""
    import torch
    pairs = make_pairs(args.unique, args.size)
    host = [(a.astype(np.float32), b.astype(np.float32)) for a, b, _, _ in pairs]
    dev = torch.device("cuda", torch.cuda.current_device())
    hb = e2e_host_batch(args, pairs, dev, 1, lambda: None)
    hb32 = e2e_host_batch(args, pairs, dev, 1, lambda: None, dtype=np.float32)
    one = e2e_single_call(host, 1, lambda: None, calls=max(2, args.steps))
    print(json.dumps({"mode": "e2e", "size": args.size, "host_batch": hb, "host_batch_float32": hb32,
                      "single_call": one}))


def run_fb_only(args):
    """One fused Farneback iteration (33-tap window, all 5 planes, updateFlow + updateMatrices)
    at --size on a synthetic pair's polynomial expansions, --warmup + --steps times."""
    import torch
    import Farneback_PyCL as F
    from ofb200 import ops
    a, b, _, _ = make_pairs(1, args.size)[0]
    fb = F.Farneback_PyCL()
    A, B = ops.u8_to_f32(torch.from_numpy(a).cuda()), ops.u8_to_f32(torch.from_numpy(b).cuda())
    RA, RB = ops.fb_polyexp(A, fb._poly), ops.fb_polyexp(B, fb._poly)
    cx, cy = torch.zeros_like(A), torch.zeros_like(A)
    M = ops.fb_update_matrices(cx, cy, RA, RB)
    Mb = torch.empty_like(M)
    fb.setGaussianBlurKernel(fb.windowSize, fb.windowSize / 2 * 0.3)
    wk = fb.matrixGKernel[0]
    ms = []
    for r in range(args.warmup + args.steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        ops.fb_iteration(M, Mb, RA, RB, cx, cy, wk, True)
        e1.record()
        e1.synchronize()
        if r >= args.warmup:
            ms.append(e0.elapsed_time(e1))
    px = args.size * args.size
    print(json.dumps({"mode": "fb", "size": args.size, "ms": float(np.mean(ms)),
                      "gbs_88B_per_px": 88.0 * px / (float(np.mean(ms)) * 1e-3) / 1e9}))


def run_learned_only(args):
    """The learned warm-start step alone (profiling): --learned-pairs pairs at --size through
    one LearnedBatch graph on --streams streams (the packaged network, its calibrated
    Farneback iterations and sweeps), four seeded pairs cycled; --warmup + --steps replays,
    CUDA events, no fallback pass."""
    import torch
    from ofb200.warmstart import LearnedBatch, load_trained
    net, meta = load_trained(**({"path": args.learned_weights} if args.learned_weights else {}), device="cuda")
    fr = [(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()) for a, b, _, _ in make_pairs(4, args.size)]
    frames = [fr[i % len(fr)] for i in range(args.learned_pairs)]
    lb = LearnedBatch(net, meta, args.learned_pairs, args.size, streams=args.streams)
    for _ in range(args.warmup):
        lb.run(frames)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        lb.run(frames)
    e1.record()
    e1.synchronize()
    ms = e0.elapsed_time(e1) / max(1, args.steps)
    print(json.dumps({"mode": "learned", "size": args.size, "pairs": args.learned_pairs, "ms_per_step": ms,
                      "pairs_per_s": args.learned_pairs / (ms * 1e-3)}))


def run_cnn(args):
    """The warm-start network alone: forward of --pairs frames at --size (the level it runs
    at), and one training step (16 x 256^2: forward, loss, backward, Adam), CUDA events."""
    import torch
    from ofb200.warmstart import LAYERS, WarmStartNet
    net = WarmStartNet(seed=0)

    def timeit(fn, reps):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        e1.synchronize()
        return e0.elapsed_time(e1) / reps

    n, S = args.pairs, args.size
    b = net.buffers(n, S)
    b["x0"][..., :2] = torch.rand((n, S, S, 2), device="cuda").to(torch.bfloat16)
    fwd = timeit(lambda: net.forward(b), args.steps)
    flops = sum(2 * 9 * ci * co * n * (S >> lvl) ** 2 for (name, ci, co), lvl in
                zip(LAYERS, [0, 0, 1, 1, 2, 2, 3, 3, 2, 1, 0, 0]))
    bt, gt = net.buffers(16, 256), net.grad_buffers(16, 256)
    bt["x0"][..., :2] = torch.rand((16, 256, 256, 2), device="cuda").to(torch.bfloat16)
    lab = torch.randn((16, 256, 256, 2), device="cuda")

    def train_step():
        net.forward(bt)
        net.loss(bt, gt, lab)
        net.backward(bt, gt)
        net.adam(1e-4)

    step = timeit(train_step, args.steps)
    net.check()
    print(json.dumps({"mode": "cnn", "size": S, "batch": n, "forward_ms": fwd, "forward_ms_per_pair": fwd / n,
                      "forward_tflops": flops / fwd / 1e9, "train_step_ms_16x256": step}))


def peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def make_pairs(n, size, seed0=100):
    from ofb200 import synthetic as S
    out = []
    for i in range(n):
        a, b, U, V = S.config_pair("fbls1024", seed=seed0 + i, size=size)
        out.append((a, b, U, V))
    return out


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, gpu_index):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={gpu_index}", f"--query-gpu={q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(5)
        except Exception:
            self.p.kill()
        self.f.seek(0)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.f.name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def pipeline_dev(a, b):
    """One pair on device tensors through the drop-in driver (no host synchronisation)."""
    import Farneback_PyCL as F
    import GenericPyramidalOpticalFlow as G
    import PhysicsBasedOpticalFlowLiuShen as LS
    return G.genericPyramidalOpticalFlow(a, b, 0, F.Farneback_PyCL(), 2, 1, 0.48, LS.LiuShenOpticalFlowAlgoAdapter(10))


def e2e_host_batch(args, pairs, dev, world, barrier, dtype=np.uint8):
    """pairs/s of --steps steps of --pairs pairs from pinned host frames (uint8, the camera's
    format, or float32 as the reference's examples cast them) to numpy U, V through
    ofb200.batch.HostBatch, wall clock, max over ranks."""
    import torch
    import torch.distributed as dist
    import Farneback_PyCL as F
    import PhysicsBasedOpticalFlowLiuShen as LS
    from ofb200.batch import HostBatch, PairSpec
    spec = PairSpec(0, lambda: F.Farneback_PyCL(), 2, 1, 0.48, lambda: LS.LiuShenOpticalFlowAlgoAdapter(10),
                    key=("fbls",))
    hb = HostBatch([spec] * args.pairs, streams=max(1, args.streams), depth=2)
    pinned = [(torch.from_numpy(a.astype(dtype)).pin_memory(), torch.from_numpy(b.astype(dtype)).pin_memory())
              for a, b, _, _ in pairs]
    step_host = [pinned[i % len(pinned)] for i in range(args.pairs)]
    for _ in range(max(3, args.warmup)):
        hb.run(step_host)
    torch.cuda.synchronize()
    barrier()
    t0 = time.perf_counter()
    prev = None
    for _ in range(args.steps):
        t = hb.submit(step_host)
        if prev is not None:
            hb.result(prev)
        prev = t
    hb.result(prev)
    dt = torch.tensor([time.perf_counter() - t0], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(dt, op=dist.ReduceOp.MAX)
    N = args.size * args.size
    name = np.dtype(dtype).name
    return {"value": args.pairs * args.steps * world / float(dt.item()), "unit": "pairs/s",
            "h2d_bytes_per_step": sum(a.numel() * a.element_size() + b.numel() * b.element_size() for a, b in step_host),
            "d2h_bytes_per_step": 2 * N * 4 * args.pairs,
            "api": f"ofb200.batch.HostBatch: pinned {name} frames in, numpy float32 U, V out, 2 steps in flight",
            "timing": "wall clock over the steps, max over ranks"}


def e2e_single_call(host_frames, world, barrier, calls):
    """pairs/s of the one-pair drop-in call (genericPyramidalOpticalFlow with numpy float32
    frames in and numpy U, V out), called back to back, wall clock."""
    import torch
    import torch.distributed as dist
    import Farneback_PyCL as F
    import GenericPyramidalOpticalFlow as G
    import PhysicsBasedOpticalFlowLiuShen as LS
    for i in range(2):
        G.genericPyramidalOpticalFlow(*host_frames[i % len(host_frames)], 0, F.Farneback_PyCL(), 2, 1, 0.48,
                                      LS.LiuShenOpticalFlowAlgoAdapter(10))
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i in range(calls):
        G.genericPyramidalOpticalFlow(*host_frames[i % len(host_frames)], 0, F.Farneback_PyCL(), 2, 1, 0.48,
                                      LS.LiuShenOpticalFlowAlgoAdapter(10))
    dt = torch.tensor([time.perf_counter() - t0], dtype=torch.float64, device=torch.cuda.current_device())
    if world > 1:
        dist.all_reduce(dt, op=dist.ReduceOp.MAX)
    N = host_frames[0][0].size
    return {"value": calls * world / float(dt.item()), "unit": "pairs/s", "h2d_bytes_per_call": 2 * N * 4,
            "d2h_bytes_per_call": 2 * N * 4,
            "api": "GenericPyramidalOpticalFlow.genericPyramidalOpticalFlow, numpy float32 frames in, numpy out"}


def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from ofb200 import _lib, ops

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    pairs = make_pairs(args.unique, args.size, seed0=100 + 1000 * rank)
    frames = [(torch.from_numpy(a).to(dev), torch.from_numpy(b).to(dev)) for a, b, _, _ in pairs]
    host_frames = [(a.astype(np.float32), b.astype(np.float32)) for a, b, _, _ in pairs]
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device=dev)
    N = args.size * args.size

    step_frames = [frames[i % len(frames)] for i in range(args.pairs)]
    batch = None
    if args.streams > 1:
        import Farneback_PyCL as F
        import PhysicsBasedOpticalFlowLiuShen as LS
        from ofb200.batch import PairBatch, PairSpec
        spec = PairSpec(0, lambda: F.Farneback_PyCL(), 2, 1, 0.48, lambda: LS.LiuShenOpticalFlowAlgoAdapter(10),
                        key=("fbls",))
        batch = PairBatch([spec] * args.pairs, streams=args.streams)

    def step():
        if batch is not None:
            return batch.run(step_frames)[-1]
        for a8, b8 in step_frames:
            U, V = pipeline_dev(ops.u8_to_f32(a8), ops.u8_to_f32(b8))
        return U, V

    def barrier():
        if world > 1:
            dist.barrier()

    # warm-up
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    barrier()

    # device-timed steps (L2 flushed between steps, outside the events)
    clocks = Clocks(local_rank) if rank == 0 else None
    from ofb200 import graph as _graph
    lc0 = _lib.lib().of_launch_count() + _graph.replayed_kernels()
    total_ms = 0.0
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        step()
        e1.record()
        e1.synchronize()
        total_ms += e0.elapsed_time(e1)
    launches = _lib.lib().of_launch_count() + _graph.replayed_kernels() - lc0
    clk = clocks.stop() if clocks else None
    t = torch.tensor([total_ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    total_ms = float(t.item())
    barrier()

    # roofline of the dominant kernel: the step's Liu-Shen solves (--pairs of them at full
    # size, concurrently on --streams streams, as in the step), graph-replayed
    roof = None if args.no_roofline else ls_step_roofline(args, frames, flush)

    # end to end from host buffers to host results: the step's pairs as pinned uint8 frames
    # through HostBatch (frames up on one copy stream, the batch graph, U and V down into
    # pinned buffers on another; two steps in flight), wall clock over --steps steps
    e2e = None
    if not args.no_e2e:
        e2e = e2e_host_batch(args, pairs, dev, world, barrier)
        e2e["float32_frames"] = e2e_host_batch(args, pairs, dev, world, barrier, dtype=np.float32)
        e2e["single_call"] = e2e_single_call(host_frames, world, barrier, calls=max(2, args.pairs))
    learned = None if args.no_learned else run_learned(args, step_frames, pairs, dev, flush, world,
                                                           pairs_total_ms=total_ms)
    configs = None if args.no_configs else run_configs(args, rank, world, dev, flush)
    if rank != 0:
        return None
    pairs_total = args.pairs * args.steps * world
    line = {
        "metric": METRIC, "value": pairs_total / (total_ms * 1e-3), "unit": "pairs/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "pairs_per_step_per_gpu": args.pairs, "size": args.size,
                   "unique_pairs": args.unique, "streams": args.streams,
                   "l2": "flushed between steps (256 MB write)",
                   "parallelism": f"pairs sharded over {world} rank(s)"},
        "clocks": clk, "e2e": e2e, "gpu_launches": int(launches), "learned": learned, "roofline": roof,
    }
    if configs is not None:
        line["configs"] = configs
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(pairs[0])
    return line


def _graph_of(fn):
    """fn (enqueues work on the current stream, may fork to other streams and join) run once
    eagerly, then captured into a CUDA graph.  Returns (graph, outputs of the capture)."""
    import torch
    fn()
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.graph(g, stream=side):
        out = fn()
    torch.cuda.synchronize()
    return g, out


def _time_graph(g, flush, reps, warm=2):
    """Mean CUDA-event time (ms) of g.replay() with L2 flushed before each replay."""
    import torch
    ms = []
    for r in range(warm + reps):
        flush.zero_()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        g.replay()
        e1.record()
        e1.synchronize()
        if r >= warm:
            ms.append(e0.elapsed_time(e1))
    return float(np.mean(ms))


def _fork_join(streams, jobs):
    """Runs jobs[i]() on streams[i % len(streams)] after the current stream's work, and
    makes the current stream wait for all of them (capturable)."""
    import torch
    cur = torch.cuda.current_stream()
    for st in streams:
        st.wait_stream(cur)
    outs = []
    for i, job in enumerate(jobs):
        with torch.cuda.stream(streams[i % len(streams)]):
            outs.append(job())
    for st in streams:
        cur.wait_stream(st)
    return outs


def ls_step_roofline(args, frames, flush):
    """The step's Liu-Shen solves alone: --pairs prefiltered 1024^2 pairs solved concurrently
    on --streams streams (one CUDA graph), L2 flushed before each replay."""
    import torch
    from gaussian_filter import prepareGaussianKernel
    from ofb200 import ops
    taps = prepareGaussianKernel(0.48, 5)
    N = args.size * args.size
    pre = []
    for i in range(args.pairs):
        a8, b8 = frames[i % len(frames)]
        pre.append((ops.prefilter(ops.u8_to_f32(a8), taps), ops.prefilter(ops.u8_to_f32(b8), taps)))
    zero = torch.zeros_like(pre[0][0])
    streams = [torch.cuda.Stream() for _ in range(max(1, args.streams))]
    arith = ops.ls_arithmetic()

    def solve(fa, fb):
        return lambda: ops.ls_solve(fa, fb, zero.clone(), zero.clone(), 10.0, arithmetic=arith)

    g, outs = _graph_of(lambda: _fork_join(streams, [solve(fa, fb) for fa, fb in pre]))
    ms = _time_graph(g, flush, reps=5)
    iters = [int(o[2].item()) for o in outs]
    alg = float(sum((24.0 * k + 8.0) * N for k in iters))
    peak, peak_kind = peaks()
    achieved = alg / (ms * 1e-3) / 1e9
    per_solve = NCU_LS_TRAFFIC.get((arith, args.size))
    del g
    return {"kernel": f"Liu-Shen solve {args.size}^2 (set-up + sweeps), {args.pairs} concurrent on {len(streams)} "
                      f"streams as in the step, working set {args.pairs * 60} MB > L2",
            "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "peak_kind": peak_kind, "traffic": per_solve * args.pairs if per_solve and set(iters) == {60} else None,
            "traffic_note": "ncu DRAM bytes of one solve's launches (cold cache per launch) x solves",
            "sweeps": iters[0] if len(set(iters)) == 1 else iters, "ms": ms, "solves": args.pairs,
            "algorithmic_bytes": alg, "arithmetic": arith}


FP32_LANES_PER_SM = 128


def _fp32_peak_tflops(clk):
    """Nominal FP32 rate at the sampled max SM clock: 148 SMs x 128 lanes x 2 flop."""
    mhz = (clk or {}).get("sm_max_mhz") or 1965.0
    return 148 * FP32_LANES_PER_SM * 2 * mhz * 1e6 / 1e12


def _pair_throughput(spec_fn, frames, nstreams, flush, reps=5, hs_shape=None):
    """Device pairs/s of a list of uint8 frame pairs through PairBatch (one CUDA graph), or,
    with hs_shape, through HsGroup (every Horn-Schunck solve in one persistent launch)."""
    from ofb200.batch import HsGroup, PairBatch
    if hs_shape is None:
        batch = PairBatch([spec_fn() for _ in frames], streams=nstreams)
    else:
        batch = HsGroup([spec_fn() for _ in frames], tile_shape=hs_shape)
    for _ in range(3):
        batch.run(frames)
    import torch
    ms = []
    for r in range(reps):
        flush.zero_()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        batch.run(frames)
        e1.record()
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    return len(frames) / (float(np.mean(ms)) * 1e-3), float(np.mean(ms))


def _single_pair_ms(spec_fn, frames, flush, reps=5):
    """Device time of one pair through the drop-in driver (genericPyramidalOpticalFlow on
    device frames, its own CUDA graph), the latency a one-pair-per-call user sees."""
    import torch
    import GenericPyramidalOpticalFlow as G
    from ofb200 import ops
    a, b = ops.u8_to_f32(frames[0]), ops.u8_to_f32(frames[1])

    def once():
        sp = spec_fn()
        opt = sp.make_opt() if sp.make_opt is not None else None
        return G.genericPyramidalOpticalFlow(a, b, sp.FILTER, sp.make_main(), sp.pyramidalLevels, sp.kLevels,
                                             sp.FILTER_OPT, opt)
    for _ in range(3):
        once()
    ms = []
    for _ in range(reps):
        flush.zero_()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        once()
        e1.record()
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    return float(np.median(ms))


def _oracle_cfg(args):
    cfg, size = args
    O = _oracle()
    from ofb200 import synthetic as S
    a8, b8, _, _ = S.config_pair(cfg, seed=7, size=size)
    a, b = a8.astype(np.float32), b8.astype(np.float32)
    t0 = time.perf_counter()
    if cfg == "hs256":
        O.pyramid(a, b, 3.4, O.HS([21], 600), 1, 1, None)
    else:
        O.pyramid(a, b, 2, O.LK(5, 13), 2, 1, 0.48, None, warping=False)
    return time.perf_counter() - t0


def run_configs(args, rank, world, dev, flush):
    """Configs 1, 2 and 4 with their own device-timed numbers (each rank runs its own pairs:
    weak scaling; pairs/s summed over ranks)."""
    import torch
    import torch.distributed as dist
    import denseLucasKanade_PyCL as LK
    import HornSchunck as HS
    from ofb200 import synthetic as S
    from ofb200.batch import PairSpec
    from ofb200.shard import max_over_ranks
    out = {}
    n_hs, n_lk, nst = 16, 8, 8
    hs_frames, lk_frames = [], []
    for i in range(n_hs):
        a, b, _, _ = S.config_pair("hs256", seed=200 + 1000 * rank + i)
        hs_frames.append((torch.from_numpy(a).to(dev), torch.from_numpy(b).to(dev)))
    for i in range(n_lk):
        a, b, _, _ = S.config_pair("lk512", seed=300 + 1000 * rank + i)
        lk_frames.append((torch.from_numpy(a).to(dev), torch.from_numpy(b).to(dev)))
    clocks = Clocks(dev.index) if rank == 0 else None
    hs_spec = lambda: PairSpec(3.4, lambda: HS.HSOpticalFlowAlgoAdapter([21], 600), 1, 1, key=("hs",))  # noqa: E731
    lk_spec = lambda: PairSpec(2.0, lambda: LK.denseLucasKanade_PyCl(Niter=5, halfWindow=13), 2, 1, 0.48,  # noqa
                               key=("lk",))
    # Horn-Schunck: the batch runner's path (every solve in one persistent launch, tile shape
    # tuned on these pairs), beside per-pair graphs on 8 streams for comparison
    from ofb200.batch import tune_hs_shape
    hs_shape, _ = tune_hs_shape(hs_frames, reps=2)
    _, hs_ms = _pair_throughput(hs_spec, hs_frames, nst, flush, hs_shape=hs_shape)
    _, hs_graph_ms = _pair_throughput(hs_spec, hs_frames, nst, flush)
    hs_single_ms = _single_pair_ms(hs_spec, hs_frames[0], flush)
    _, lk_ms = _pair_throughput(lk_spec, lk_frames, nst, flush)
    lk_single_ms = _single_pair_ms(lk_spec, lk_frames[0], flush)
    clk = clocks.stop() if clocks else None
    hs_ms, lk_ms = max_over_ranks(hs_ms, dev), max_over_ranks(lk_ms, dev)
    hs_graph_ms = max_over_ranks(hs_graph_ms, dev)
    peak, peak_kind = peaks()
    hs_bytes = (600 * 24.0 + 20.0 + 8.0) * 256 * 256  # sweeps, derivatives, prefilter (per pair)
    lk_px = 512 * 512 + 256 * 256
    lk_flop = 7.0e4 * lk_px
    fp32 = _fp32_peak_tflops(clk)
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        import multiprocessing as mp
        with mp.get_context("spawn").Pool(2) as pool:
            t_hs, t_lk = pool.map(_oracle_cfg, [("hs256", 256), ("lk512", 256)])
        cpu = {"hs256": {"value": 1.0 / t_hs, "unit": "pairs/s", "cores": 1, "kind": "port",
                         "sample": f"1 pair 256x256, full pipeline, {t_hs:.1f} s"},
               "lk512": {"value": 0.25 / t_lk, "unit": "pairs/s", "cores": 1, "kind": "port",
                         "sample": f"1 pair at 256x256 (a quarter of the pixels), full LK pyr2 pipeline, {t_lk:.1f} s; "
                                   "pairs/s scaled by the pixel ratio"}}
    # the faster of the two paths is the configuration's number; both are reported
    best_ms = min(hs_ms, hs_graph_ms)
    path = (f"one persistent launch (tile shape {hs_shape})" if hs_ms <= hs_graph_ms
            else "per-pair graphs on 8 streams (one launch per 4 sweeps)")
    out["hs256"] = {"workload": "PyHSchunck_Fs3_4 Horn-Schunck, 256x256 Poiseuille pairs, 600 sweeps",
                    "value": n_hs * world / (best_ms * 1e-3), "unit": "pairs/s", "ms_per_step": best_ms,
                    "pairs_per_step_per_gpu": n_hs, "path": path,
                    "persistent_one_launch": {"value": n_hs * world / (hs_ms * 1e-3), "ms_per_step": hs_ms,
                                              "tile_shape": hs_shape},
                    "per_pair_graphs_8_streams": {"value": n_hs * world / (hs_graph_ms * 1e-3), "ms_per_step": hs_graph_ms},
                    "single_pair_ms": hs_single_ms,
                    "roofline": {"bound": "hbm", "achieved": n_hs * hs_bytes / (best_ms * 1e-3) / 1e9, "peak": peak,
                                 "unit": "GB/s", "frac": n_hs * hs_bytes / (best_ms * 1e-3) / 1e9 / peak,
                                 "peak_kind": peak_kind, "algorithmic_bytes_per_pair": hs_bytes},
                    "cpu_baseline": cpu["hs256"] if cpu else None}
    out["lk512"] = {"workload": "denseLK_Fs2_0_PyrLvls2 dense LK pyr2, 512x512 Lamb-Oseen pairs",
                    "value": n_lk * world / (lk_ms * 1e-3), "unit": "pairs/s", "ms_per_step": lk_ms,
                    "pairs_per_step_per_gpu": n_lk, "streams": nst, "single_pair_ms": lk_single_ms,
                    "roofline": {"bound": "fp32", "achieved": n_lk * lk_flop / (lk_ms * 1e-3) / 1e12, "peak": fp32,
                                 "unit": "TFLOP/s", "frac": n_lk * lk_flop / (lk_ms * 1e-3) / 1e12 / fp32,
                                 "peak_kind": "nominal (148 SMs x 128 FP32 lanes x 2 x max SM clock)",
                                 "algorithmic_flop_per_pair": lk_flop,
                                 "flop_model": "7e4 FP32 flop per pixel (27x27 window, 5 Newton steps), both levels"},
                    "cpu_baseline": cpu["lk512"] if cpu else None}
    out["clocks"] = clk
    if not args.no_batch:
        out["batch256"] = run_batch_inline(args, rank, world, dev, flush)
    return out


def _cand(k):
    """Autotune table key -> label: ('hs_shape', i) -> 'hs_shape_i', (chunk, streams) -> 'CxS',
    ('hs_in_chunks', chunk, streams) -> 'CxS_hs_in_chunks'."""
    if k[0] == "hs_shape":
        return f"hs_shape_{k[1]}"
    if k[0] == "hs_in_chunks":
        return f"{k[1]}x{k[2]}_hs_in_chunks"
    return f"{k[0]}x{k[1]}"


def run_batch_inline(args, rank, world, dev, flush):
    """Config 4 inside the default bench: the seeded 256-pair manifest, autotuned over a
    short candidate list, one timed pass (device events, L2 flushed before it)."""
    import multiprocessing as mp
    import torch
    from ofb200.batch import autotune, config4_manifest, pair_cost_of, render_entry
    from ofb200.shard import max_over_ranks, shard_by_cost
    manifest = config4_manifest(args.batch_pairs, seed=0)
    mine = shard_by_cost([pair_cost_of(e) for e in manifest], world)[rank]
    entries = [manifest[i] for i in mine]
    try:
        ncores = len(os.sched_getaffinity(0))
    except Exception:
        ncores = os.cpu_count() or 1
    with mp.get_context("spawn").Pool(max(1, min(32, ncores // world))) as pool:
        rendered = pool.map(render_entry, entries)
    frames = [(torch.from_numpy(a).to(dev), torch.from_numpy(b).to(dev)) for a, b, _, _ in rendered]
    runner, table = autotune(entries, frames, chunks=(64, 256), streams=(8,), reps=1)
    ms = []
    for _ in range(2):
        flush.zero_()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        runner.run(frames)
        e1.record()
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    t = max_over_ranks(float(np.mean(ms)), dev)
    runner_key, hs_shape = runner.key, runner.hs_shape
    del runner
    return {"workload": f"{len(manifest)} pairs, sizes 128^2-2048^2, HS / LK pyr2 / FB pyr2 / FB pyr2 + LS, "
                        "Poiseuille / Lamb-Oseen / random-Fourier, max 4 px",
            "value": len(manifest) / (t * 1e-3), "unit": "pairs/s", "ms_per_pass": t, "scaling": "strong",
            "autotuned": {"chunk": runner_key[-2], "streams": runner_key[-1], "hs_tile_shape": hs_shape,
                          "candidates_ms": {_cand(k): round(v, 2) for k, v in table.items()}}}


def _render_eval(seed):
    from ofb200 import synthetic as S
    return S.config_pair("fbls1024", seed=seed)


LARGE_DISP_PX = 12.0


def _render_eval_large(seed):
    """The workload's pairs with displacements up to LARGE_DISP_PX, where a zero start at
    full size needs the pyramid's coarse level."""
    from ofb200 import synthetic as S
    return S.piv_pair(1024, 1024, "fourier", seed, density=0.05, diameter=(2.0, 3.0), noise=2.0,
                      max_disp=LARGE_DISP_PX)


def _events_ms(fn, flush, steps, warmup):
    """Mean device time of fn() (CUDA events, L2 flushed before each timed call)."""
    import torch
    for _ in range(warmup):
        fn()
    ms = []
    for _ in range(steps):
        flush.zero_()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    return float(np.mean(ms))


def learned_large_disp(args, net, meta, dev, flush, npairs=8):
    """Held-out pairs with displacements up to LARGE_DISP_PX: interior EPE of the plain
    pyramid, of the packaged network's start (trained on max 4 px) and of the no-network
    ablation; and, when the package holds a network trained on larger displacements
    (warmstart_weights_12px.npz, calibrated on this kind of pair), that network's arm and
    its ablation with pairs/s for each arm (CUDA events over --steps batches of the pairs)."""
    import multiprocessing as mp
    import torch
    import Farneback_PyCL as F
    import PhysicsBasedOpticalFlowLiuShen as LS
    from ofb200 import ops, synthetic as S
    from ofb200.batch import PairBatch, PairSpec
    from ofb200.warmstart import WEIGHTS, LearnedBatch, load_trained
    seeds = [970_000 + i for i in range(npairs)]
    with mp.get_context("spawn").Pool(min(8, max(1, (os.cpu_count() or 2) // 2))) as pool:
        evals = pool.map(_render_eval_large, seeds)
    frames = [(torch.from_numpy(a).to(dev), torch.from_numpy(b).to(dev)) for a, b, _, _ in evals]
    epe_of = lambda res: float(np.mean([S.epe(U.cpu().numpy(), V.cpu().numpy(), e[2], e[3], crop=16)  # noqa: E731
                                        for (U, V), e in zip(res, evals)]))
    spec = PairSpec(0, lambda: F.Farneback_PyCL(), 2, 1, 0.48, lambda: LS.LiuShenOpticalFlowAlgoAdapter(10),
                    key=("fbls",))
    pb = PairBatch([spec] * npairs, streams=max(1, args.streams))
    out = {"max_disp_px": LARGE_DISP_PX, "pairs": npairs, "crop_px": 16,
           "epe_plain": epe_of(pb.run(frames)),
           "plain_pairs_per_s": npairs / (_events_ms(lambda: pb.run(frames), flush, args.steps, 2) * 1e-3)}
    del pb

    def arms(net_, meta_, tag, timed):
        for start, key in (("cnn", "learned"), ("zero", "no_network_ablation")):
            lb = LearnedBatch(net_, meta_, npairs, args.size, streams=args.streams, start=start)
            res, errs = lb.run(frames)
            if start == "cnn":
                out[f"{tag}epe_learned_before_fallback"] = epe_of(res)
                res, nfb = lb.fallback(frames, res, errs.cpu())
                out[f"{tag}learned_fallback_pairs"] = int(nfb)
            out[f"{tag}epe_{key}"] = epe_of(res)
            if timed:
                def step():
                    r, e = lb.run(frames)
                    if start == "cnn":
                        lb.fallback(frames, r, e.cpu())
                out[f"{tag}{key}_pairs_per_s"] = npairs / (_events_ms(step, flush, args.steps, 2) * 1e-3)
            del lb

    arms(net, meta, "", False)
    large = os.path.join(os.path.dirname(WEIGHTS), "warmstart_weights_12px.npz")
    if os.path.exists(large):
        net2, meta2 = load_trained(path=large, device=dev)
        out["large_network"] = {k: meta2.get(k) for k in ("train_max_disp", "eval_max_disp", "mode", "fb_iters",
                                                           "sweeps", "zero_fb_iters", "zero_sweeps", "train_pairs")}
        arms(net2, meta2, "large_network_", True)
        net2.check()
    return out


def run_learned(args, step_frames, pairs, dev, flush, world, pairs_total_ms):
    """The learned warm start (config 5: batch --learned-pairs at 1024^2): one network
    forward over the step's pairs (at the network's level), Farneback at full size from that
    start, then the calibrated number of Liu-Shen sweeps; pairs whose last update norm exceeds
    the calibrated threshold are recomputed by the plain pyramid inside the timed region.
    The step's frames are --epe-pairs distinct held-out pairs (seeds outside the training and
    calibration sets), cycled; the endpoint errors of all arms against the analytic ground
    truth (16 px interior) are taken over those distinct pairs."""
    import multiprocessing as mp
    import torch
    import torch.distributed as dist
    from ofb200 import ops, synthetic as S
    from ofb200.warmstart import LearnedBatch, load_trained
    net, meta = load_trained(**({"path": args.learned_weights} if args.learned_weights else {}), device=dev)
    seeds = [960_000 + 1000 * (dist.get_rank() if world > 1 else 0) + i for i in range(args.epe_pairs)]
    with mp.get_context("spawn").Pool(min(16, max(1, (os.cpu_count() or 2) // 2))) as pool:
        evals = pool.map(_render_eval, seeds)
    eval_frames = [(torch.from_numpy(a).to(dev), torch.from_numpy(b).to(dev)) for a, b, _, _ in evals]
    nb = args.learned_pairs
    lframes = [eval_frames[i % len(eval_frames)] for i in range(nb)]
    nu = min(len(eval_frames), nb)
    plain_value = args.pairs * args.steps * world / (pairs_total_ms * 1e-3)
    epe_p = []
    for i in range(nu):
        a, b, Ug, Vg = evals[i]
        Up, Vp = pipeline_dev(ops.u8_to_f32(lframes[i][0]), ops.u8_to_f32(lframes[i][1]))
        epe_p.append(S.epe(Up.cpu().numpy(), Vp.cpu().numpy(), Ug, Vg, crop=16))
    step_frames = lframes
    pairs = evals

    def arm(start):
        lb = LearnedBatch(net, meta, nb, args.size, streams=args.streams, start=start)

        def step():
            res, errs = lb.run(step_frames)  # uint8 frames, converted inside the graph
            if start == "zero":
                return list(res), 0
            return lb.fallback(step_frames, res, errs.cpu())

        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        total_ms, fallbacks = 0.0, 0
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            _, nfb = step()
            e1.record()
            e1.synchronize()
            total_ms += e0.elapsed_time(e1)
            fallbacks += nfb
        t = torch.tensor([total_ms], dtype=torch.float64, device=dev)
        if world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
        out, _ = step()  # accuracy on the distinct pairs, outside the timed region
        epe = [S.epe(out[i][0].cpu().numpy(), out[i][1].cpu().numpy(), pairs[i][2], pairs[i][3], crop=16)
               for i in range(nu)]
        value = nb * args.steps * world / (total_ms * 1e-3)
        ll = lb.ll
        return {"value": value, "unit": "pairs/s", "ms_per_step": total_ms / args.steps,
                "speedup_vs_plain": value / plain_value, "fb_iters": ll.fb_iters if ll.mode == "fb" else 0,
                "sweeps": ll.sweeps, "fallback_pairs": fallbacks, "epe": float(np.mean(epe))}

    learned = arm("cnn")
    ablation = arm("zero")
    large = learned_large_disp(args, net, meta, dev, flush)
    net.check()
    learned.update({"mode": meta["mode"], "threshold": meta["threshold"], "epe_plain": float(np.mean(epe_p)),
                    "epe_pairs": nu, "epe_crop_px": 16, "pairs_per_step": nb,
                    "network": f"encoder-decoder CNN at the {meta.get('level', 512)}^2 level, 1.75M params, bf16 tcgen05 convs, "
                               "f32 accumulate",
                    "trained": {k: meta[k] for k in ("train_pairs", "steps", "batch", "crop", "level", "eval_pairs")},
                    "no_network_ablation": ablation, "large_displacement": large})
    return learned


def run_batch(args, rank, world, local_rank):
    """Config 4: a seeded manifest of pairs of uneven sizes (128^2-2048^2), methods (HS,
    LK pyr2, Farneback pyr2, Farneback pyr2 + Liu-Shen) and flows, sharded over the ranks by
    cost, rendered on the host cores, run as autotuned chunks of multi-stream CUDA graphs.
    value = pairs of the whole manifest / max-over-ranks time of one pass."""
    import multiprocessing as mp
    from ofb200.batch import config4_manifest, pair_cost_of, render_entry
    from ofb200.shard import gather_objects, max_over_ranks, shard_by_cost
    manifest = config4_manifest(args.batch_pairs, seed=0)
    mine = shard_by_cost([pair_cost_of(e) for e in manifest], world)[rank]
    entries = [manifest[i] for i in mine]
    try:
        ncores = len(os.sched_getaffinity(0))
    except Exception:
        ncores = os.cpu_count() or 1
    with mp.get_context("spawn").Pool(max(1, min(32, ncores // world))) as pool:  # before CUDA is touched
        rendered = pool.map(render_entry, entries)
    import torch
    import torch.distributed as dist
    from ofb200 import synthetic as S
    from ofb200.batch import autotune
    dev = torch.device("cuda", local_rank)
    frames = [(torch.from_numpy(a).to(dev), torch.from_numpy(b).to(dev)) for a, b, _, _ in rendered]
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device=dev)
    runner, table = autotune(entries, frames)
    for _ in range(args.warmup):
        runner.run(frames)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = Clocks(local_rank) if rank == 0 else None
    total = 0.0
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        outs = runner.run(frames)
        e1.record()
        e1.synchronize()
        total += e0.elapsed_time(e1)
    clk = clocks.stop() if clocks else None
    total = max_over_ranks(total, dev)
    per = {}
    for e, (U, V), (_, _, Ug, Vg) in zip(entries, outs, rendered):
        ep = S.epe(U.cpu().numpy(), V.cpu().numpy(), Ug, Vg, crop=16 if e["size"] > 64 else 0)
        per.setdefault(e["method"], []).append(ep)
    per = gather_objects(per)
    if rank != 0:
        return None
    merged = {}
    for d in per:
        for k, v in d.items():
            merged.setdefault(k, []).extend(v)
    epe = {k: {"mean": float(np.nanmean(v)) if np.isfinite(v).any() else None, "pairs": len(v),
               "nonfinite": int(np.sum(~np.isfinite(v)))} for k, v in merged.items()}
    return {"metric": "pairs/s, batched uneven pairs (config 4)", "value": len(manifest) * args.steps / (total * 1e-3),
            "unit": "pairs/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": total / args.steps, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"{len(manifest)} pairs, sizes 128^2-2048^2, HS / LK pyr2 / FB pyr2 / FB pyr2 + LS, "
                                   "Poiseuille / Lamb-Oseen / random-Fourier, max 4 px",
                       "l2": "flushed between steps (256 MB write)", "parallelism": f"pairs sharded by cost over {world}",
                       "autotuned": {"chunk": runner.key[-2], "streams": runner.key[-1], "hs_tile_shape": runner.hs_shape,
                                     "candidates_ms": {_cand(k): round(v, 2) for k, v in table.items()}}},
            "clocks": clk, "epe_interior": epe}


def _oracle():
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle as O
    return O


def _oracle_pair(args):
    a, b = args
    O = _oracle()
    return O.pyramid(a, b, 0, O.FB(), 2, 1, 0.48, O.LS(10))


def cpu_baseline(pair):
    """The oracle (scalar C port, 1 thread) on one 1024^2 pair."""
    a, b = pair[0].astype(np.float32), pair[1].astype(np.float32)
    t0 = time.perf_counter()
    _oracle_pair((a, b))
    dt = time.perf_counter() - t0
    return {"value": 1.0 / dt, "unit": "pairs/s", "cores": 1, "kind": "port",
            "sample": f"1 pair {a.shape[0]}x{a.shape[1]}, full pipeline, {dt:.1f} s"}


def run_reference(args, rank, world):
    """The reference arm: the oracle (the reference's path restated in C, one thread per
    pair) on the GPU arm's workload, --pairs pairs per step, on every host core.  Steps are
    handed to a pool of one process per core in groups of cores // pairs steps, so every core
    works while a step's pairs run in parallel; the run stops after REF_BUDGET_S seconds
    (whole groups), and value = pairs done / time."""
    if rank != 0:
        return None
    import multiprocessing as mp
    try:
        ncores = len(os.sched_getaffinity(0))
    except Exception:
        ncores = os.cpu_count() or 1
    pairs = make_pairs(args.unique, args.size)  # the same distinct pairs as the GPU arm's step
    work = [(p[0].astype(np.float32), p[1].astype(np.float32)) for p in pairs]
    ctx = mp.get_context("spawn")
    per_step = args.pairs
    group = max(1, ncores // per_step)  # steps per pool call
    steps = 0
    with ctx.Pool(ncores) as pool:
        for _ in range(min(args.warmup, 1)):
            pool.map(_oracle_pair, [work[i % len(work)] for i in range(min(ncores, per_step * group))])
        t0 = time.perf_counter()
        # a step takes several seconds of CPU time: stop after REF_BUDGET_S so the run stays short
        while steps < args.steps and (steps == 0 or time.perf_counter() - t0 < REF_BUDGET_S):
            g = min(group, args.steps - steps)
            pool.map(_oracle_pair, [work[i % len(work)] for i in range(per_step * g)])
            steps += g
        dt = time.perf_counter() - t0
    v = per_step * steps / dt
    return {"metric": METRIC, "value": v, "unit": "pairs/s", "n_gpus": world, "steps": steps,
            "warmup": args.warmup, "ms_per_step": dt / steps * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOAD, "pairs_per_step_per_gpu": per_step, "size": args.size,
                       "unique_pairs": args.unique,
                       "parallelism": f"one pair per host process, {ncores} processes, {group} step(s) at a time"},
            "cpu_baseline": {"value": v, "unit": "pairs/s", "cores": ncores, "kind": "port",
                             "sample": f"{per_step} pairs per step, one per process, {steps} of "
                                       f"{args.steps} steps (capped at {REF_BUDGET_S:.0f} s)"},
            "e2e": {"value": v, "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    args = parse()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        line = run_reference(args, rank, world)
        if line:
            print(json.dumps(line))
        return
    if args.mode == "ls":
        run_ls_only(args)
        return
    if args.mode == "cnn":
        run_cnn(args)
        return
    if args.mode == "fb":
        run_fb_only(args)
        return
    if args.mode == "e2e":
        run_e2e_only(args)
        return
    if args.mode == "hs":
        run_hs_only(args)
        return
    if args.mode == "lk":
        run_lk_only(args)
        return
    if args.mode == "learned":
        run_learned_only(args)
        return
    if args.mode == "batch":
        if world > 1:
            import datetime

            import torch
            import torch.distributed as dist
            torch.cuda.set_device(local_rank)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        line = run_batch(args, rank, world, local_rank)
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
            dist.destroy_process_group()
        if line:
            print(json.dumps(line))
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    line = run_ours(args, rank, world, local_rank)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if line:
        print(json.dumps(line))


if __name__ == "__main__":
    main()
