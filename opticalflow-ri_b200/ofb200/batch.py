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

import contextlib
import ctypes
import threading
from dataclasses import dataclass, field

import torch

from . import _lib
from . import graph as _graph
from . import ops

__all__ = ["PairSpec", "PairBatch", "HostBatch", "HsGroup", "method_spec", "config4_manifest", "render_entry", "pair_cost_of",
           "BatchRunner", "autotune", "tune_hs_shape", "pair_descriptors", "run_c"]


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

    def __init__(self, specs, streams=4, use_graph: bool = True, status: bool = False):
        """streams: a count, or a list of torch.cuda.Stream to share with other batches
        (their workspaces are shared too: batches sharing streams must not overlap).
        status: also compute per-pair status words (self.status, device int32, bits
        ofb200._lib.ST_*: non-finite frames, non-finite results, a Liu-Shen refine that
        used all its sweeps above its tolerance), inside the same graph."""
        self.specs = list(specs)
        self.want_status = status
        self.status = None
        if isinstance(streams, (list, tuple)):
            self._streams, self.nstreams = list(streams), len(streams)
        else:
            self._streams, self.nstreams = None, max(1, int(streams))
        self.use_graph = use_graph
        self._graphs = {}
        self._lock = threading.Lock()

    def _pipelines(self, frames):
        cur = torch.cuda.current_stream()
        if self._streams is None:
            self._streams = [torch.cuda.Stream() for _ in range(self.nstreams)]
        outs = [None] * len(frames)
        if self.want_status:
            if self.status is None or self.status.numel() != len(frames):
                self.status = torch.zeros(len(frames), dtype=torch.int32, device=frames[0][0].device)
            self.status.zero_()
        for s in self._streams:
            s.wait_stream(cur)
        conc = ops.concurrent_streams() if self.nstreams > 1 else contextlib.nullcontext()
        with conc:
            self._enqueue(frames, outs)
        for s in self._streams:
            cur.wait_stream(s)
        return outs

    def _enqueue(self, frames, outs):
        import GenericPyramidalOpticalFlow as G
        for i, ((a, b), spec) in enumerate(zip(frames, self.specs)):
            st = self._streams[i % self.nstreams]
            with torch.cuda.stream(st):
                main = spec.make_main()
                opt = spec.make_opt() if spec.make_opt is not None else None
                if a.dtype in (torch.uint8, torch.uint16):
                    a, b = ops.u8_to_f32(a), ops.u8_to_f32(b)
                elif self.want_status:
                    self._check(a, i, _lib.ST_NONFINITE_INPUT)
                    self._check(b, i, _lib.ST_NONFINITE_INPUT)
                outs[i] = G._pyramid_dev(a, b, _cfg_for(spec, main), main, opt)
                if self.want_status:
                    self._check(outs[i][0], i, _lib.ST_NONFINITE_OUTPUT)
                    self._check(outs[i][1], i, _lib.ST_NONFINITE_OUTPUT)
                    if getattr(opt, "last_iterations", None) is not None:
                        import PhysicsBasedOpticalFlowLiuShen as LS
                        _lib.call("of_ls_status", ctypes.c_void_p(opt.last_iterations.data_ptr()),
                                  ctypes.c_void_p(opt.last_error.data_ptr()), LS.MAXNUM, LS.TOL,
                                  ctypes.c_void_p(self.status[i:].data_ptr()), ops.stream_ptr())

    def _check(self, t, i, bit):
        H, W = t.shape
        _lib.call("of_check_finite", ctypes.c_void_p(t.data_ptr()), H, W, t.stride(0),
                  ctypes.c_void_p(self.status[i:].data_ptr()), bit, ops.stream_ptr())

    def run(self, frames):
        """frames: list of (frame1, frame2) CUDA tensors (uint8 or float32) matching specs.
        Returns a list of (U, V) CUDA tensors (graph-owned: overwritten by the next run)."""
        if len(frames) != len(self.specs):
            raise ValueError("one frame pair per spec")
        if not (self.use_graph and _graph.ENABLED):
            return self._pipelines(frames)
        with self._lock:
            g, static_in, static_out, nk = self._entry(frames)
            # all inputs into the graph's buffers with one multi-tensor copy
            torch._foreach_copy_([t for p in static_in for t in p], [t for p in frames for t in p])
            g.replay()
            _graph._replayed_kernels += nk
            return static_out

    def _entry(self, frames):
        """The graph for these frames' shapes, dtypes and settings, captured on first use
        (frames: CUDA tensors whose values feed the eager warm-up run)."""
        key = tuple((tuple(a.shape), a.dtype, s.key) for (a, _), s in zip(frames, self.specs))
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
        return e


class HostBatch:
    """Frame pairs from host memory to flow fields in host memory, `depth` batches in flight.

    submit() copies a batch's frames host -> device on a copy stream, replays the batch's
    graph (a PairBatch per slot, so that the batches in flight own distinct device buffers;
    the slots share the compute streams and run one after another), then copies every U, V
    device -> host into the slot's pinned buffers on the copy stream.  result() waits for
    those copies and returns numpy views of the pinned buffers.  While the GPU computes
    batch k the host prepares batch k+1, and batch k's results cross PCIe while batch k+1
    computes.  A slot's results stay valid until its next submit, `depth` submits later.
    Frames given as pinned CPU tensors are copied from directly (keep them unchanged until
    their result is taken); other host arrays go through the slot's pinned staging first."""

    def __init__(self, specs, streams=8, depth=2, status: bool = False):
        self.specs = list(specs)
        self.depth = max(1, int(depth))
        shared = [torch.cuda.Stream() for _ in range(max(1, int(streams)))]
        self._slots = [PairBatch(self.specs, streams=shared, status=status) for _ in range(self.depth)]
        # separate copy streams: batch k+1's inputs go up while batch k computes and while
        # batch k-1's results come down
        self._up, self._down = torch.cuda.Stream(), torch.cuda.Stream()
        self._state = [None] * self.depth
        self._submitted = 0

    @staticmethod
    def _host(x):
        return x if isinstance(x, torch.Tensor) else torch.from_numpy(x)

    def _first_use(self, slot, frames):
        dev = torch.device("cuda", torch.cuda.current_device())
        pb = self._slots[slot]
        d = [(self._host(a).to(dev), self._host(b).to(dev)) for a, b in frames]
        g, static_in, static_out, nk = pb._entry(d)
        pin = lambda t: torch.empty(t.shape, dtype=t.dtype, pin_memory=True)  # noqa: E731
        st = {"entry": (g, static_in, static_out, nk),
              "stage": [(pin(a), pin(b)) for a, b in static_in],
              "out": [(pin(U), pin(V)) for U, V in static_out],
              "status": pin(pb.status) if pb.status is not None else None,
              "h2d": torch.cuda.Event(), "done": torch.cuda.Event(), "d2h": torch.cuda.Event(), "ticket": -1}
        self._state[slot] = st
        return st

    def submit(self, frames):
        """frames: list of (frame1, frame2) host arrays / CPU tensors (uint8, uint16 or
        float32) matching the specs.  Returns a ticket for result()."""
        if len(frames) != len(self.specs):
            raise ValueError("one frame pair per spec")
        ticket = self._submitted
        slot = ticket % self.depth
        st = self._state[slot] or self._first_use(slot, frames)
        g, static_in, static_out, nk = st["entry"]
        for (a, b), (sa, sb) in zip(frames, static_in):
            if tuple(a.shape) != tuple(sa.shape) or tuple(b.shape) != tuple(sb.shape):
                raise ValueError("HostBatch: frame shapes differ from the first batch's")
        st["h2d"].synchronize()  # the staging buffers' previous copy has left the host
        srcs = []
        for (a, b), (pa, pb_) in zip(frames, st["stage"]):
            for x, p in ((a, pa), (b, pb_)):
                t = self._host(x)
                if t.is_pinned() and t.dtype == p.dtype:
                    srcs.append(t)
                else:
                    p.copy_(t)
                    srcs.append(p)
        cur, up, down = torch.cuda.current_stream(), self._up, self._down
        up.wait_event(st["done"])  # the slot's previous replay has read its inputs
        with torch.cuda.stream(up):
            torch._foreach_copy_([t for p in static_in for t in p], srcs, non_blocking=True)
        st["h2d"].record(up)
        cur.wait_event(st["h2d"])
        cur.wait_event(st["d2h"])  # the slot's previous results have left the device
        g.replay()
        _graph._replayed_kernels += nk
        st["done"].record(cur)
        down.wait_event(st["done"])
        with torch.cuda.stream(down):
            torch._foreach_copy_([t for p in st["out"] for t in p], [t for p in static_out for t in p],
                                 non_blocking=True)
            if st["status"] is not None:
                st["status"].copy_(self._slots[slot].status, non_blocking=True)
        st["d2h"].record(down)
        st["ticket"] = ticket
        self._submitted += 1
        return ticket

    def result(self, ticket):
        """[(U, V)] numpy float32 views of the slot's pinned buffers for a submitted batch
        (and, with status=True, self.last_status: the batch's status words)."""
        st = self._state[ticket % self.depth] if 0 <= ticket < self._submitted else None
        if st is None or st["ticket"] != ticket:
            raise ValueError(f"HostBatch: ticket {ticket} is not in flight (its slot was reused)")
        st["d2h"].synchronize()
        if st["status"] is not None:
            self.last_status = st["status"].numpy().copy()
        return [(U.numpy(), V.numpy()) for U, V in st["out"]]

    def run(self, frames):
        """submit + result: one batch from host frames to host flow fields."""
        return self.result(self.submit(frames))


# ----------------------------------------------------------------------------- config 4
# The batched workload: pairs of uneven sizes and methods, each method with its reference
# calibration (examples/PyHSchunck_Fs3_4.py, denseLK_Fs2_0_PyrLvls2.py,
# Farneback_Fs0_0_PyrLvls2.py, LiuSE_Farneback_Fs0_0_PyrLvls2.py).
CONFIG4_SIZES = (128, 256, 512, 1024, 2048)
CONFIG4_METHODS = ("hs", "lk", "fb", "ls")
CONFIG4_FLOWS = ("poiseuille", "lamb_oseen", "fourier")


def method_spec(method: str) -> PairSpec:
    import Farneback_PyCL as F
    import HornSchunck as HS
    import PhysicsBasedOpticalFlowLiuShen as LS
    import denseLucasKanade_PyCL as LK
    if method == "hs":
        return PairSpec(3.4, lambda: HS.HSOpticalFlowAlgoAdapter([21], 600), 1, 1, key=("hs",))
    if method == "lk":
        return PairSpec(2.0, lambda: LK.denseLucasKanade_PyCl(), 2, 1, key=("lk",))
    if method == "fb":
        return PairSpec(0, lambda: F.Farneback_PyCL(), 2, 1, key=("fb",))
    if method == "ls":  # Liu-Shen as the refiner of Farneback pyr2 (it cannot be the main adapter)
        return PairSpec(0, lambda: F.Farneback_PyCL(), 2, 1, 0.48, lambda: LS.LiuShenOpticalFlowAlgoAdapter(10),
                        key=("ls",))
    raise ValueError(method)


def config4_manifest(n=256, seed=0):
    """n entries {size, method, flow, seed}, each field drawn uniformly from its set."""
    import numpy as np
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        out.append({"size": int(rng.choice(CONFIG4_SIZES)), "method": str(rng.choice(CONFIG4_METHODS)),
                    "flow": str(rng.choice(CONFIG4_FLOWS)), "seed": int(seed * 100_000 + i)})
    return out


def pair_cost_of(e) -> float:
    from .shard import pair_cost
    return pair_cost(e["size"], e["method"])


def render_entry(e):
    """(frame1 u8, frame2 u8, U_gt, V_gt) of one manifest entry (max 4 px displacement;
    the vortex core scales with the image, 60 px at 512^2)."""
    from . import synthetic as S
    n = e["size"]
    density, diameter = {"hs": (0.05, 2.5), "lk": (0.08, 2.5)}.get(e["method"], (0.05, (2.0, 3.0)))
    kw = {"core_radius": 60.0 * n / 512.0} if e["flow"] == "lamb_oseen" else {}
    return S.piv_pair(n, n, e["flow"], e["seed"], density=density, diameter=diameter, noise=2.0, **kw)


class HsGroup:
    """The Horn-Schunck pairs of a batch (one pyramid level, as method_spec("hs") sets them
    up: prefilter, then the solve) with every solve in ONE persistent launch (of_hs_batch,
    bit-exact with the per-pair path).  The prefilters, the launch and the accumulation into
    the result are captured into one CUDA graph on the first run."""

    def __init__(self, specs, tile_shape=0, schedule="auto"):
        """schedule: ops.hs_batch's ('auto', 'queue' or 'resident').  The resident schedule
        needs every tile's CTA resident at once: with other kernels running beside the
        group (BatchRunner's chunks) use 'queue', whose items only wait for running CTAs."""
        self.specs, self.tile_shape, self.schedule = list(specs), int(tile_shape), schedule
        for sp in self.specs:
            if sp.pyramidalLevels != 1 or sp.kLevels != 1 or sp.make_opt is not None:
                raise ValueError("HsGroup takes single-level Horn-Schunck pairs")
        self._graph = None
        self.status = None

    def _pipelines(self, frames):
        from gaussian_filter import prepareGaussianKernel
        pairs, outs = [], []
        for (a, b), sp in zip(frames, self.specs):
            hs = sp.make_main()
            if a.dtype in (torch.uint8, torch.uint16):
                a, b = ops.u8_to_f32(a), ops.u8_to_f32(b)
            if sp.FILTER > 1e-3:
                taps = prepareGaussianKernel(sp.FILTER, 3)
                a, b = ops.prefilter(a, taps), ops.prefilter(b, taps)
            U, V = torch.zeros_like(a), torch.zeros_like(a)
            pairs.append((a, b, U, V, hs.alphas[-1], hs.Niter))
            outs.append((U, V))
        self.status = ops.hs_batch(pairs, tile_shape=self.tile_shape, schedule=self.schedule)
        # the driver's Uaccum = 0 + U (the sign of a zero result is the accumulation's)
        return [(ops.accumulate(torch.zeros_like(U), U), ops.accumulate(torch.zeros_like(V), V)) for U, V in outs]

    def run(self, frames):
        if not _graph.ENABLED:
            return self._pipelines(frames)
        if self._graph is None:
            static_in = [(a.clone(), b.clone()) for a, b in frames]
            self._pipelines(static_in)
            torch.cuda.synchronize()
            g = torch.cuda.CUDAGraph()
            side = torch.cuda.Stream()
            side.wait_stream(torch.cuda.current_stream())
            with torch.cuda.graph(g, stream=side):
                static_out = self._pipelines(static_in)
            self._graph = (g, static_in, static_out)
        g, static_in, static_out = self._graph
        torch._foreach_copy_([t for p in static_in for t in p], [t for p in frames for t in p])
        g.replay()
        _graph._replayed_kernels += 1
        return static_out


class BatchRunner:
    """A manifest in chunks of `chunk` pairs, ordered by decreasing cost, each chunk one
    multi-stream CUDA graph (PairBatch) on `streams` shared streams.  With hs_shape set,
    the Horn-Schunck pairs leave the chunks and run as one persistent launch (HsGroup with
    that tile shape) on a stream of their own, overlapping the chunks.  run() returns every
    pair's (U, V) in manifest order."""

    def __init__(self, entries, chunk=32, streams=4, hs_shape=None):
        self.entries = list(entries)
        self.hs_shape = hs_shape
        hs_idx = [i for i, e in enumerate(self.entries) if e["method"] == "hs"] if hs_shape is not None else []
        rest = [i for i in range(len(self.entries)) if i not in set(hs_idx)]
        self.order = sorted(rest, key=lambda i: (-pair_cost_of(self.entries[i]), i))
        self.chunk, self.nstreams = int(chunk), int(streams)
        self._streams = [torch.cuda.Stream() for _ in range(self.nstreams)]
        self._hs = (hs_idx, HsGroup([method_spec("hs") for _ in hs_idx], hs_shape, schedule="queue")) if hs_idx else None
        self._hs_stream = torch.cuda.Stream() if hs_idx else None
        self._batches = []
        for c in range(0, len(self.order), self.chunk):
            idx = self.order[c:c + self.chunk]
            specs = [method_spec(self.entries[i]["method"]) for i in idx]
            self._batches.append((idx, PairBatch(specs, streams=self._streams)))

    def run(self, frames):
        outs = [None] * len(self.entries)
        cur = torch.cuda.current_stream()
        if self._hs is not None:
            idx, grp = self._hs
            self._hs_stream.wait_stream(cur)
            with torch.cuda.stream(self._hs_stream):
                res = grp.run([frames[i] for i in idx])
            for i, r in zip(idx, res):
                outs[i] = r
        for idx, pb in self._batches:
            res = pb.run([frames[i] for i in idx])
            for i, r in zip(idx, res):
                outs[i] = r
        if self._hs is not None:
            cur.wait_stream(self._hs_stream)
        return outs


def _time_runner(r, frames, reps):
    r.run(frames)  # capture
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        r.run(frames)
    e1.record()
    e1.synchronize()
    return e0.elapsed_time(e1) / reps


def _cache_path():
    import os
    return os.environ.get("OFB_AUTOTUNE_CACHE", os.path.join(os.path.expanduser("~"), ".cache", "ofb200",
                                                             "autotune.json"))


def tune_hs_shape(frames_hs, reps=2, log=None, use_cache=True, schedule="auto"):
    """The persistent Horn-Schunck kernel's tile shape (region and sweeps per pass) for a set
    of Horn-Schunck pairs under `schedule`: every shape of ops.hs_batch_shapes() timed on
    them; the choice is cached per (GPU, method, schedule, sizes) in a JSON file
    (OFB_AUTOTUNE_CACHE, default ~/.cache/ofb200/autotune.json).  Returns (shape index,
    {shape: ms})."""
    import json
    import os
    key = "|".join([torch.cuda.get_device_name(), "hs", schedule,
                    ",".join(sorted(f"{a.shape[0]}x{a.shape[1]}" for a, _ in frames_hs))])
    path = _cache_path()
    cache = {}
    if use_cache and os.path.exists(path):
        try:
            with open(path) as f:
                cache = json.load(f)
        except (OSError, ValueError):
            cache = {}
    if key in cache:
        return int(cache[key]["shape"]), {int(k): v for k, v in cache[key]["ms"].items()}
    specs = [method_spec("hs") for _ in frames_hs]
    table = {}
    for k in range(len(ops.hs_batch_shapes())):
        g = HsGroup(specs, tile_shape=k, schedule=schedule)
        table[k] = _time_runner(g, frames_hs, reps)
        if log:
            log(f"hs tile shape {k} {ops.hs_batch_shapes()[k]}: {table[k]:.2f} ms")
        del g
    best = min(table, key=table.get)
    if use_cache:
        cache[key] = {"shape": best, "ms": table}
        try:
            os.makedirs(os.path.dirname(path), exist_ok=True)
            with open(path, "w") as f:
                json.dump(cache, f, indent=1)
        except OSError:
            pass
    return best, table


def autotune(entries, frames, chunks=(16, 64, 256), streams=(2, 4, 8), reps=2, log=None, hs_persistent=True):
    """Times every (chunk, streams) candidate on the manifest (after its capture run) and
    returns (best runner, {candidate: ms}).  With hs_persistent, the Horn-Schunck pairs run
    in one persistent launch whose tile shape is tuned first (tune_hs_shape); the best
    candidate is then timed once more with the Horn-Schunck pairs back in the chunks
    (key ('hs_in_chunks', chunk, streams)), and the faster of the two is returned."""
    import gc
    best, table = None, {}
    hs_shape = None
    if hs_persistent:
        hs = [frames[i] for i, e in enumerate(entries) if e["method"] == "hs"]
        if hs:
            hs_shape, hs_table = tune_hs_shape(hs, reps=reps, log=log, schedule="queue")
            table.update({("hs_shape", k): v for k, v in hs_table.items()})
    for c in chunks:
        for s in streams:
            r = BatchRunner(entries, chunk=min(c, len(entries)), streams=s, hs_shape=hs_shape)
            r.key = (c, s)
            ms = _time_runner(r, frames, reps)
            table[(c, s)] = ms
            if log:
                log(f"chunk {c} streams {s}: {ms:.1f} ms")
            if best is None or ms < table[best.key]:
                best = r
            else:
                del r
                gc.collect()
    if hs_shape is not None:
        c, s = best.key
        r = BatchRunner(entries, chunk=min(c, len(entries)), streams=s, hs_shape=None)
        r.key = ("hs_in_chunks", c, s)
        ms = _time_runner(r, frames, reps)
        table[r.key] = ms
        if log:
            log(f"chunk {c} streams {s}, Horn-Schunck in the chunks: {ms:.1f} ms")
        if ms < table[best.key]:
            best = r
        else:
            del r
            gc.collect()
    return best, table


# ----------------------------------------------------------------------------- C driver
def pair_descriptors(specs, frames, outs, keep):
    """OfPairDesc entries for of_batch_run from PairSpecs (this package's HS / LK / Farneback
    adapters, optional Liu-Shen refine), CUDA frames (uint8 or float32) and output planes.
    Host constants (taps, Farneback kernels) are appended to `keep`, which must outlive the
    call."""
    import numpy as np
    import denseLucasKanade_PyCL as LKm
    import Farneback_PyCL as FBm
    import HornSchunck as HSm
    import PhysicsBasedOpticalFlowLiuShen as LSm
    from gaussian_filter import prepareGaussianKernel
    arr = (_lib.OfPairDesc * len(specs))()

    def host(a):
        a = np.ascontiguousarray(a, np.float32)
        keep.append(a)
        return a.ctypes.data

    for k, (sp, (a, b), (U, V)) in enumerate(zip(specs, frames, outs)):
        main = sp.make_main()
        opt = sp.make_opt() if sp.make_opt is not None else None
        FILTER, L, kL, FOPT, warping, biLinear, inter, last = _cfg_for(sp, main)
        if kL != 1 or not biLinear:
            raise ValueError("of_batch_run takes kLevels = 1 and the bilinear warp")
        d = arr[k]
        d.frame_u8 = int(a.dtype == torch.uint8)
        d.I0, d.I1, d.in_pitch = a.data_ptr(), b.data_ptr(), a.stride(0)
        d.U, d.V, d.out_pitch = U.data_ptr(), V.data_ptr(), U.stride(0)
        d.H, d.W = a.shape
        d.filter = FILTER
        d.filter_taps = host(prepareGaussianKernel(FILTER, 3)) if FILTER > 1e-3 else None
        d.levels = L
        d.warping, d.intermediate_scaling, d.scaling = int(warping), int(inter), int(last)
        if opt is not None:
            if not isinstance(opt, LSm.LiuShenOpticalFlowAlgoAdapter):
                raise ValueError("of_batch_run refines with Liu-Shen only")
            d.refine_ls = 1
            d.filter_opt = float(FOPT) if FOPT is not None else 0.0
            d.filter_opt_taps = host(prepareGaussianKernel(FOPT, 5)) if FOPT is not None and FOPT > 1e-3 else None
            d.ls_h = float(np.float32(opt.alpha))
            d.ls_arithmetic = 1 if opt.arithmetic == "fast" else 0
        if isinstance(main, HSm.HSOpticalFlowAlgoAdapter):
            d.method = _lib.OF_METHOD_HS
            al = list(main.alphas)[-8:]
            for i, x in enumerate(al):
                d.hs_alphas[i] = float(np.float32(x))
            d.hs_nalphas, d.hs_niter = len(al), int(main.Niter)
        elif isinstance(main, LKm.denseLucasKanade_PyCl):
            if main.enableVorticityEnhancement:
                raise ValueError("of_batch_run: no vorticity-enhanced windows")
            d.method = _lib.OF_METHOD_LK
            d.lk_half_win, d.lk_niter = int(main.windowHalfWidth), int(main.Niter)
        elif isinstance(main, FBm.Farneback_PyCL):
            d.method = _lib.OF_METHOD_FB
            p = _lib.OfFbParams()
            p.window_size, p.niters, p.use_gaussian = int(main.windowSize), int(main.numIters), int(main.useGaussianFilter)
            p.levels, p.pyr_scale, p.poly = int(main.pyramidalLevels) + 1, float(main.pyrScale), main._poly
            main.setGaussianBlurKernel(main.windowSize, main.windowSize / 2 * 0.3)
            p.window_taps, p.window_kh = host(main.matrixGKernel[0]), len(main.matrixGKernel[0]) - 1
            scale = 1.0
            for lev in range(_lib.OF_FB_MAX_LEVELS):
                sigma = (1.0 / scale - 1.0) * 0.5
                smooth = max(int(round(sigma * 5)) | 1, 3)
                main.setGaussianBlurKernel(smooth, sigma)
                p.level_taps[lev], p.level_kh[lev] = host(main.matrixGKernel[0]), smooth // 2
                scale *= main.pyrScale
            keep.append(p)
            d.fb = ctypes.addressof(p)
        else:
            raise ValueError("of_batch_run: unsupported main adapter")
    return arr


def run_c(specs, frames, tile_shape: int = 0, status: bool = True):
    """The pairs through the C driver of_batch_run (one call, the current stream).  Returns
    ([(U, V)], status words or None)."""
    outs = [(torch.empty(a.shape, dtype=torch.float32, device=a.device),
             torch.empty(a.shape, dtype=torch.float32, device=a.device)) for a, _ in frames]
    keep = []
    arr = pair_descriptors(specs, frames, outs, keep)
    n = len(specs)
    tun = _lib.OfTuning(int(tile_shape), 0, 0, 0)
    st = torch.zeros(n, dtype=torch.int32, device=frames[0][0].device) if status else None
    need = _lib.lib().of_batch_workspace_size(arr, n, ctypes.byref(tun))
    if need == 0:
        raise ValueError("of_batch_run: invalid descriptors")
    ws, wn = ops.workspace(need, "batch_c")
    _lib.call("of_batch_run", arr, n, ctypes.byref(tun), ctypes.c_void_p(st.data_ptr()) if st is not None else None,
              ws, wn, ops.stream_ptr())
    return outs, st
