"""Many frame pairs at once: per-pair pyramids on several CUDA streams, captured into one
CUDA graph.

A single pair leaves the GPU partly idle (the coarse level's kernels have fewer tiles than
the GPU has CTA slots, and every kernel ends in a partial wave).  `PairBatch` runs the
pyramids of a list of pairs concurrently, pair i on stream i mod S, joins them, and
captures the whole fork/join into one graph on its first call: later calls with the
same shapes and settings are one graph launch.  Pairs may differ in size and method; each
entry carries its own settings.  Each stream gets its own workspaces (ofb200.ops keys
them by stream), so concurrent pairs never share scratch memory.
"""
from __future__ import annotations

import threading
from dataclasses import dataclass, field

import torch

from . import graph as _graph
from . import ops

__all__ = ["PairSpec", "PairBatch"]


@dataclass
class PairSpec:
    """One pair's pipeline: genericPyramidalOpticalFlow arguments without the frames.

    make_main / make_opt build fresh adapters for every execution (adapters such as
    Horn-Schunck consume state per call)."""
    FILTER: float
    make_main: object
    pyramidalLevels: int = 1
    kLevels: int = 1
    FILTER_OPT: float | None = None
    make_opt: object = None
    warping: bool = True
    biLinear: bool = True
    pyramidalIntermediateScaling: bool = True
    pyramidalScaling: bool = False
    key: tuple = field(default=())  # settings identity for graph reuse


def _cfg_for(spec: PairSpec, main):
    warping, biLinear = spec.warping, spec.biLinear
    inter, last = spec.pyramidalIntermediateScaling, spec.pyramidalScaling
    if main.hasGenericPyramidalDefaults():
        dm = main.getGenericPyramidalDefaults() or {}
        warping = dm.get("warping", warping) if dm.get("warping") is not None else warping
        biLinear = dm.get("biLinear") if dm.get("biLinear") is not None else biLinear
        inter = dm.get("intermediateScaling") if dm.get("intermediateScaling") is not None else inter
        last = dm.get("scaling") if dm.get("scaling") is not None else last
    return (float(spec.FILTER), int(spec.pyramidalLevels), int(spec.kLevels),
            None if spec.FILTER_OPT is None else float(spec.FILTER_OPT), bool(warping), bool(biLinear), bool(inter),
            bool(last))


class PairBatch:
    """Runs len(specs) pairs concurrently on `streams` CUDA streams (graph-captured)."""

    def __init__(self, specs, streams: int = 4, use_graph: bool = True):
        self.specs = list(specs)
        self.nstreams = max(1, int(streams))
        self.use_graph = use_graph
        self._graphs = {}
        self._lock = threading.Lock()
        self._streams = None

    def _pipelines(self, frames):
        import GenericPyramidalOpticalFlow as G
        cur = torch.cuda.current_stream()
        if self._streams is None:
            self._streams = [torch.cuda.Stream() for _ in range(self.nstreams)]
        outs = [None] * len(frames)
        for s in self._streams:
            s.wait_stream(cur)
        for i, ((a, b), spec) in enumerate(zip(frames, self.specs)):
            st = self._streams[i % self.nstreams]
            with torch.cuda.stream(st):
                main = spec.make_main()
                opt = spec.make_opt() if spec.make_opt is not None else None
                if a.dtype == torch.uint8:
                    a, b = ops.u8_to_f32(a), ops.u8_to_f32(b)
                outs[i] = G._pyramid_dev(a, b, _cfg_for(spec, main), main, opt)
        for s in self._streams:
            cur.wait_stream(s)
        return outs

    def run(self, frames):
        """frames: list of (frame1, frame2) CUDA tensors (uint8 or float32) matching specs.
        Returns a list of (U, V) CUDA tensors (graph-owned: overwritten by the next run)."""
        if len(frames) != len(self.specs):
            raise ValueError("one frame pair per spec")
        if not (self.use_graph and _graph.ENABLED):
            return self._pipelines(frames)
        key = tuple((tuple(a.shape), a.dtype, s.key) for (a, _), s in zip(frames, self.specs))
        with self._lock:
            e = self._graphs.get(key)
            if e is None:
                static_in = [(a.clone(), b.clone()) for a, b in frames]
                self._pipelines(static_in)  # eager warm-up: sizes every stream's workspaces
                torch.cuda.synchronize()
                from ._lib import lib
                n0 = lib().of_launch_count()
                g = torch.cuda.CUDAGraph()
                side = torch.cuda.Stream()
                side.wait_stream(torch.cuda.current_stream())
                with torch.cuda.graph(g, stream=side):
                    static_out = self._pipelines(static_in)
                nk = lib().of_launch_count() - n0
                e = (g, static_in, static_out, nk)
                self._graphs[key] = e
            g, static_in, static_out, nk = e
            for (sa, sb), (a, b) in zip(static_in, frames):
                sa.copy_(a)
                sb.copy_(b)
            g.replay()
            _graph._replayed_kernels += nk
            return static_out
