"""Training and calibration of the learned Liu-Shen warm start.

    python -m ofb200.warmstart_train --pairs 2000 --steps 3000 --out warmstart.npz

1. Training pairs (1024^2, seeded; random-Fourier or Lamb-Oseen flow with a random core
   radius, 0.02-0.1 particles/px, noise sigma 0-5 DN, diameter 2-3 px, max displacement
   4 px or drawn from --max-disp) are rendered on the host cores by a spawn process pool.
2. Each pair is labelled by the plain pipeline on the GPU (Farneback pyr2 + Liu-Shen h = 10,
   the package's converged output); frames and label are taken to the --level size (the
   pyramid's bicubic downsample; the label scaled by level / 1024 in magnitude).  The
   packaged weights: --level 128 --crop 128.
3. The network is trained on random --crop crops (Adam, mean squared flow error) with the
   package's own forward / backward kernels.
4. On held-out pairs of the 1024^2 benchmark workload (disjoint seeds; with
   --eval-max-disp, the same flows scaled to that maximum displacement) the plain pipeline,
   the network's start followed by each full-size stage (Liu-Shen alone with K sweeps, or
   Farneback with 1-5 iterations then K sweeps), and the same stages from a zero field
   (the no-network ablation) are compared by interior endpoint error against the analytic
   ground truth.  The cheapest network configuration whose mean EPE is at most the plain
   mean is kept, with a fallback threshold on the solve's last update norm set from the
   pairs that met the plain EPE; the cheapest such zero-start stage is recorded too.
Weights, the configuration, the threshold and the evaluation table go to one .npz;
--calibrate redoes step 4 for existing weights.
"""
from __future__ import annotations

import argparse
import functools
import json
import multiprocessing as mp
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
if PKG not in sys.path:
    sys.path.insert(0, PKG)

TRAIN_SEED0 = 10_000
EVAL_SEED0 = 900_000
LEVEL = 512
CROP = 256


def _train_pair(seed, disp=(4.0, 4.0)):
    """disp: the range the pair's maximum displacement is drawn from (px)."""
    from ofb200 import synthetic as S
    rng = np.random.default_rng(seed)
    kind = "fourier" if rng.uniform() < 0.5 else "lamb_oseen"
    kw = {"core_radius": float(rng.uniform(40, 160))} if kind == "lamb_oseen" else {}
    md = float(rng.uniform(disp[0], disp[1])) if disp[1] > disp[0] else float(disp[0])
    a, b, U, V = S.piv_pair(1024, 1024, kind, seed=seed, density=float(rng.uniform(0.02, 0.1)), diameter=(2.0, 3.0),
                            noise=float(rng.uniform(0.0, 5.0)), max_disp=md, **kw)
    return a, b


def _eval_pair(seed, max_disp=4.0):
    """The benchmark workload's pairs (max 4 px), or the same flows scaled to max_disp."""
    from ofb200 import synthetic as S
    if max_disp == 4.0:
        return S.config_pair("fbls1024", seed=seed)
    return S.piv_pair(1024, 1024, "fourier", seed, density=0.05, diameter=(2.0, 3.0), noise=2.0, max_disp=max_disp)


def generate(fn, seeds, workers):
    ctx = mp.get_context("spawn")
    with ctx.Pool(workers) as pool:
        return pool.map(fn, seeds, chunksize=max(1, len(seeds) // (4 * workers)))


def plain(a, b):
    import Farneback_PyCL as F
    import GenericPyramidalOpticalFlow as G
    import PhysicsBasedOpticalFlowLiuShen as LS
    return G.genericPyramidalOpticalFlow(a, b, 0, F.Farneback_PyCL(), 2, 1, 0.48, LS.LiuShenOpticalFlowAlgoAdapter(10))


def build_level_data(pairs, dev, level=LEVEL):
    """(N, level, level, 2) bf16 inputs (each frame / its max) and (N, level, level, 2) f32
    labels (the plain output resized to the level, displacements scaled by level / 1024)."""
    import torch
    from ofb200 import ops
    from ofb200._lib import call
    from ofb200.warmstart import _p, _sp
    N = len(pairs)
    X = torch.empty((N, level, level, 2), dtype=torch.bfloat16, device=dev)
    Y = torch.empty((N, level, level, 2), dtype=torch.float32, device=dev)
    tmp = torch.empty((level, level, 16), dtype=torch.bfloat16, device=dev)
    mx = torch.zeros(2, dtype=torch.int32, device=dev)
    for i, (a, b) in enumerate(pairs):
        A = ops.u8_to_f32(torch.from_numpy(a).to(dev))
        B = ops.u8_to_f32(torch.from_numpy(b).to(dev))
        U, V = plain(A, B)
        a2 = ops.resize(A, (level, level), bicubic=True)
        b2 = ops.resize(B, (level, level), bicubic=True)
        call("of_cnn_pack_pair", _p(a2), _p(b2), level, level, level, _p(mx), _p(tmp), 16, _sp())
        X[i] = tmp[..., :2]
        sc = level / float(A.shape[0])
        Y[i, ..., 0] = ops.scale(ops.resize(U, (level, level), bicubic=True), sc)
        Y[i, ..., 1] = ops.scale(ops.resize(V, (level, level), bicubic=True), sc)
    torch.cuda.synchronize()
    return X, Y


def train(net, X, Y, steps, batch=16, lr=1e-3, seed=0, log=print, sync=None, crop=CROP):
    """Adam on random crops.  `sync(grads)` (data-parallel training) averages the flat
    gradient vector over the ranks between backward and the optimizer step."""
    import torch
    N, level = X.shape[0], X.shape[1]
    g = torch.Generator(device="cpu").manual_seed(seed)
    b = net.buffers(batch, crop)
    gb = net.grad_buffers(batch, crop)
    b["x0"].zero_()
    lab = torch.empty((batch, crop, crop, 2), dtype=torch.float32, device=X.device)
    hist = []
    t0 = time.time()
    for s in range(steps):
        idx = torch.randint(0, N, (batch,), generator=g)
        oy = torch.randint(0, level - crop + 1, (batch,), generator=g)
        ox = torch.randint(0, level - crop + 1, (batch,), generator=g)
        for j in range(batch):
            i, y, x = int(idx[j]), int(oy[j]), int(ox[j])
            b["x0"][j, ..., :2] = X[i, y:y + crop, x:x + crop]
            lab[j] = Y[i, y:y + crop, x:x + crop]
        net.forward(b)
        loss = net.loss(b, gb, lab)
        net.backward(b, gb)
        if sync is not None:
            sync(net.grads)
        cur = lr * 0.5 * (1 + np.cos(np.pi * s / steps))  # cosine decay
        net.adam(cur)
        if s % 100 == 0 or s == steps - 1:
            lv = float(loss.item())
            hist.append((s, lv))
            log(f"step {s} loss {lv:.5f} lr {cur:.2e} {time.time() - t0:.1f}s")
    net.check()
    return hist


FB_ITERS = (1, 2, 3, 5)
FB_SWEEPS = (4, 8)


def _configs(sweeps_list):
    """Full-size stages in increasing cost: Liu-Shen alone (by sweeps), then Farneback
    (by iterations, then sweeps) followed by Liu-Shen."""
    cfg = [("ls", 0, K) for K in sorted(sweeps_list)]
    cfg += [("fb", it, K) for it in FB_ITERS for K in FB_SWEEPS]
    return cfg


def evaluate(net, pairs, sweeps_list, dev, log=print, level=LEVEL):
    """Interior EPE (16 px crop) against the analytic ground truth of the plain pyramid,
    of the network's start followed by each full-size stage, and of the same stages from
    a zero field (no network).  The cheapest network configuration whose mean EPE is at
    most the plain mean is kept; its fallback threshold is 1.5 x the largest update norm
    among the pairs within 2% of their plain EPE."""
    import torch
    from ofb200 import synthetic as S
    from ofb200.warmstart import LearnedLiuShen
    cfgs = _configs(sweeps_list)
    rows = []
    for a, b, Ug, Vg in pairs:
        A = torch.from_numpy(a.astype(np.float32)).to(dev)
        B = torch.from_numpy(b.astype(np.float32)).to(dev)
        Up, Vp = plain(A, B)
        row = {"plain": S.epe(Up.cpu().numpy(), Vp.cpu().numpy(), Ug, Vg, crop=16)}
        f = A.shape[0] // level
        base = LearnedLiuShen(net, factor=f)
        U0, V0 = base.predict(A, B)
        row["cnn"] = S.epe(U0.cpu().numpy(), V0.cpu().numpy(), Ug, Vg, crop=16)
        for mode, it, K in cfgs:
            ll = LearnedLiuShen(net, sweeps=K, mode=mode, fb_iters=max(it, 1), factor=f)
            U, V, _, err = ll.refine(A, B, U0.clone(), V0.clone())
            row[("cnn", mode, it, K)] = (S.epe(U.cpu().numpy(), V.cpu().numpy(), Ug, Vg, crop=16), float(err.item()))
            if mode == "fb":
                Z = torch.zeros_like(A)
                U, V, _, err = ll.refine(A, B, Z, Z.clone())
                row[("zero", mode, it, K)] = (S.epe(U.cpu().numpy(), V.cpu().numpy(), Ug, Vg, crop=16),
                                              float(err.item()))
        rows.append(row)
    plain_m = float(np.mean([r["plain"] for r in rows]))
    table = {"plain_epe": plain_m, "cnn_epe": float(np.mean([r["cnn"] for r in rows])), "configs": {}}
    best = {"cnn": None, "zero": None}
    for start in ("cnn", "zero"):
        for mode, it, K in cfgs:
            key = (start, mode, it, K)
            if key not in rows[0]:
                continue
            e = [r[key][0] for r in rows]
            name = f"{start}:{mode}:fb{it}:ls{K}"
            table["configs"][name] = {"epe": float(np.mean(e)), "err_max": float(np.max([r[key][1] for r in rows])),
                                      "worse_pairs": int(sum(x > r["plain"] for x, r in zip(e, rows)))}
            log(f"{name}: EPE {np.mean(e):.4f} (plain {plain_m:.4f})")
            if best[start] is None and np.mean(e) <= plain_m:
                best[start] = key
    key = best["cnn"] or ("cnn", "fb", FB_ITERS[-1], FB_SWEEPS[-1])
    good = [r[key][1] for r in rows if r[key][0] <= r["plain"] * 1.02]
    thr = float(np.max(good)) * 1.5 if good else 0.0
    zkey = best["zero"] or ("zero", "fb", FB_ITERS[-1], FB_SWEEPS[-1])
    sel = {"mode": key[1], "fb_iters": key[2], "sweeps": key[3], "threshold": thr, "zero_fb_iters": zkey[2],
           "zero_sweeps": zkey[3]}
    return sel, table, rows


def calibrate_only(args):
    """New calibration (configuration, threshold, table) for existing weights."""
    workers = args.workers or max(1, min(64, len(os.sched_getaffinity(0))))
    eval_pairs = generate(functools.partial(_eval_pair, max_disp=args.eval_max_disp),
                          [EVAL_SEED0 + i for i in range(args.eval)], workers)
    import torch
    from ofb200.warmstart import WarmStartNet
    d = np.load(args.calibrate)
    old = json.loads(str(d["meta"]))
    net = WarmStartNet(seed=0).load(args.calibrate)
    sweeps = [int(s) for s in args.sweeps.split(",")]
    sel, table, _ = evaluate(net, eval_pairs, sweeps, torch.device("cuda", 0), log=lambda m: print(m, flush=True),
                             level=int(old.get("level", LEVEL)))
    meta = {**{k: v for k, v in old.items() if k not in ("table",)}, **sel, "table": table, "eval_pairs": args.eval}
    np.savez_compressed(args.out, meta=json.dumps(meta), params=d["params"], layers=d["layers"])
    print(json.dumps({k: v for k, v in meta.items() if k not in ("loss_history", "table")}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--pairs", type=int, default=2000)
    ap.add_argument("--eval", type=int, default=16)
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--workers", type=int, default=0)
    ap.add_argument("--sweeps", default="4,8,12,16,24,32,60")
    ap.add_argument("--out", default="warmstart.npz")
    ap.add_argument("--calibrate", default=None, help="recalibrate the weights in this .npz (no training)")
    ap.add_argument("--level", type=int, default=LEVEL, help="size the network runs at (1024 / 2^k)")
    ap.add_argument("--crop", type=int, default=CROP, help="training crop (<= level)")
    ap.add_argument("--max-disp", default="4,4", help="range of the training pairs' maximum displacement (px)")
    ap.add_argument("--eval-max-disp", type=float, default=4.0,
                    help="maximum displacement of the calibration pairs (4: the benchmark workload)")
    args = ap.parse_args()
    if args.calibrate:
        return calibrate_only(args)
    # data-parallel under torchrun: each rank renders and labels its share of the pairs
    # and the gradients are averaged every step (one all-reduce of the flat vector)
    from ofb200.shard import average_gradients, shard_range
    rank, world = int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    workers = args.workers or max(1, min(64, len(os.sched_getaffinity(0)) // world))
    t0 = time.time()
    # host rendering first, in spawned workers, before this process touches CUDA
    mine = [TRAIN_SEED0 + i for i in shard_range(args.pairs, rank, world)]
    disp = tuple(float(x) for x in args.max_disp.split(","))
    train_pairs = generate(functools.partial(_train_pair, disp=disp), mine, workers)
    eval_pairs = (generate(functools.partial(_eval_pair, max_disp=args.eval_max_disp),
                           [EVAL_SEED0 + i for i in range(args.eval)], workers) if rank == 0 else [])
    print(f"rank {rank}: generated {len(train_pairs)} + {len(eval_pairs)} pairs on {workers} workers in "
          f"{time.time() - t0:.0f}s", flush=True)
    import torch
    from ofb200.warmstart import WarmStartNet
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    t1 = time.time()
    X, Y = build_level_data(train_pairs, dev, args.level)
    del train_pairs
    print(f"rank {rank}: labelled in {time.time() - t1:.0f}s", flush=True)
    net = WarmStartNet(seed=0, device=dev)  # the same initial weights on every rank
    t2 = time.time()
    hist = train(net, X, Y, args.steps, args.batch, args.lr, seed=rank,
                 log=(lambda m: print(m, flush=True)) if rank == 0 else (lambda m: None),
                 sync=average_gradients if world > 1 else None, crop=min(args.crop, args.level))
    print(f"rank {rank}: trained in {time.time() - t2:.0f}s", flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    sweeps = [int(s) for s in args.sweeps.split(",")]
    sel, table, rows = evaluate(net, eval_pairs, sweeps, dev, log=lambda m: print(m, flush=True), level=args.level)
    meta = {**sel, "table": table, "train_pairs": args.pairs, "steps": args.steps, "ranks": world,
            "batch": args.batch, "crop": min(args.crop, args.level), "level": args.level, "eval_pairs": args.eval,
            "train_max_disp": list(disp), "eval_max_disp": args.eval_max_disp,
            "train_seed0": TRAIN_SEED0, "eval_seed0": EVAL_SEED0, "loss_history": hist}
    np.savez(args.out, meta=json.dumps(meta), **net.state())
    print(json.dumps({k: v for k, v in meta.items() if k != "loss_history"}), flush=True)


if __name__ == "__main__":
    main()
