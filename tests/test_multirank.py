"""Multi-rank host logic on CPU ranks (gloo, world size 2): the pair assignment, the
max-over-ranks step time, the metric gather and the gradient average used by the learned
warm start's data-parallel training."""
import os
import socket
import sys

import pytest

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "opticalflow-ri_b200"))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime

    import torch
    import torch.distributed as dist
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "opticalflow-ri_b200"))
    from ofb200 import shard
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        t = shard.max_over_ranks(1.5 + rank)
        g = torch.full((5,), float(rank + 1))
        shard.average_gradients(g)
        got = shard.gather_objects({"rank": rank, "pairs": list(shard.shard_range(7, rank, world))})
        out.put((rank, t, g.tolist(), got))
    finally:
        dist.destroy_process_group()


def test_collectives_on_two_cpu_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, t, g, got in res:
        assert t == 2.5                      # the slower rank's time
        assert g == [1.5] * 5                # mean of 1 and 2
        assert got == [{"rank": 0, "pairs": [0, 1, 2, 3]}, {"rank": 1, "pairs": [4, 5, 6]}]


def test_shard_by_cost_covers_and_balances():
    from ofb200 import shard
    import numpy as np
    rng = np.random.default_rng(0)
    sizes = rng.choice([128, 256, 512, 1024, 2048], 256)
    methods = rng.choice(["hs", "lk", "fb", "ls"], 256)
    costs = [shard.pair_cost(int(s), str(m)) for s, m in zip(sizes, methods)]
    for world in (1, 2, 4, 8):
        parts = shard.shard_by_cost(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(256))
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(costs)   # LPT bound
    assert list(shard.shard_range(10, 2, 3)) == [7, 8, 9]
    assert sum(len(shard.shard_range(10, r, 3)) for r in range(3)) == 10
