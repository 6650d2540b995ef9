"""CUDA-graph capture of whole device pipelines.

A pipeline here is a function of device tensors that only enqueues kernels (no host
synchronisation, no data-dependent host control flow: the Liu-Shen stop rule is decided
on the device).  The first call with a given key runs the function eagerly (which also
sizes every workspace), then captures it into a CUDA graph on static input buffers; every
later call copies the inputs into those buffers and replays the graph: one launch per
call instead of hundreds.  Outputs are the graph's static tensors (overwritten by the next
replay of the same key) - copy them if they must survive.
"""
from __future__ import annotations

import threading

import numpy as np
import torch

from . import par_copyto

ENABLED = True

_lock = threading.Lock()
_replayed_kernels = 0


def replayed_kernels() -> int:
    """Kernels of this library launched through graph replays so far (the C library's
    of_launch_count() sees only direct launches, including those recorded at capture)."""
    return _replayed_kernels


class GraphCache:
    def __init__(self, max_entries: int = 32):
        self.entries = {}
        self.max_entries = max_entries

    def run(self, key, fn, inputs, device=None):
        """inputs: CUDA tensors, or float32 numpy planes (host frames) that are staged through
        pinned buffers and copied asynchronously into the graph's input tensors."""
        global _replayed_kernels
        from ._lib import lib
        with _lock:
            e = self.entries.get(key)
            if e is None or not ENABLED:
                dev = torch.device("cuda", torch.cuda.current_device() if device is None else device)
                inputs = [torch.from_numpy(x).to(dev) if isinstance(x, np.ndarray) else x for x in inputs]
                if not ENABLED:
                    return fn(*inputs)
                static_in = [t.clone() for t in inputs]
                side = torch.cuda.Stream()
                side.wait_stream(torch.cuda.current_stream())
                with torch.cuda.stream(side):
                    fn(*static_in)  # eager warm-up on the capture stream sizes the workspaces
                torch.cuda.current_stream().wait_stream(side)
                g = torch.cuda.CUDAGraph()
                n0 = lib().of_launch_count()
                with torch.cuda.graph(g, stream=side):
                    static_out = fn(*static_in)
                nk = lib().of_launch_count() - n0
                if len(self.entries) >= self.max_entries:
                    self.entries.pop(next(iter(self.entries)))
                e = (g, static_in, static_out, nk, {})
                self.entries[key] = e
            g, static_in, static_out, nk, pinned = e
            for i, (s, t) in enumerate(zip(static_in, inputs)):
                if isinstance(t, np.ndarray):
                    if i not in pinned:
                        pinned[i] = (torch.empty(s.shape, dtype=s.dtype, pin_memory=True), torch.cuda.Event())
                    p, done = pinned[i]
                    done.synchronize()  # the previous asynchronous copy out of this buffer has finished
                    par_copyto(p.numpy(), t)
                    s.copy_(p, non_blocking=True)
                    done.record()
                else:
                    s.copy_(t)
            g.replay()
            _replayed_kernels += nk
            return static_out


CACHE = GraphCache()
