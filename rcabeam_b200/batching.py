"""Batching form: a queue of uneven ensembles under one CUDA graph.

``BatchQueue`` holds device-resident ensembles (packed RC/CR channels, grid,
geometry, traversal order, method).  The queue is split by method into
sub-queues; each runs either as one launch of the persistent batch kernel
(``rcabeam_batch_run_device`` with 1-3 CTAs per SM: persistent CTAs take
(tile, frame chunk) items from a global counter in queue order, so small and
large ensembles share the GPU without launch gaps or per-ensemble tails, with
a kernel compiled for that method alone) or as per-ensemble launches of the
single-ensemble kernels (``ctas_per_sm`` 0), whichever ``autotune`` measures
faster for that method on bounded samples of its ensembles (it also picks the
staged pipeline's frame chunk per shape class).  Ensembles that fill the GPU
alone run the single-ensemble kernels faster than the persistent loop for
OPW and DMAS-CCF-ACF; XDoppler's persistent kernel is the faster one.  The
sub-queues run one after another on one stream (run concurrently, their
sample windows compete for L2) and the whole queue is captured into one CUDA
graph.  Per-ensemble completion times come from the device's global timer.

Methods: "opw" (power of the coherent sum), "xdoppler" (|mean r conj(q)|) and
"dmas" (DMAS-CCF-ACF), as in ``ensemble_pd_from_channels`` (reference
src/rcabeam/ensemble.py:133-218).
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np
import torch

from rcabeam_b200 import _cuda_impl, _lib
from rcabeam_b200.sim import RCAGeometry, scan_coords

METHODS = {"opw": 0, "xdoppler": 1, "dmas": 3}
FRAME_CHUNKS = (16, 32, 64)


class BatchEnsembleC(ctypes.Structure):
    """ctypes mirror of ``rcabeam_batch_ensemble`` (include/rcabeam.h)."""

    _fields_ = [("rc", ctypes.c_void_p), ("cr", ctypes.c_void_p), ("scan", ctypes.c_void_p),
                ("order", ctypes.c_void_p), ("xe", ctypes.c_void_p), ("ye", ctypes.c_void_p),
                ("angles", ctypes.c_void_p), ("starts", ctypes.c_void_p), ("pd", ctypes.c_void_p),
                ("ns", ctypes.c_size_t), ("nc", ctypes.c_size_t), ("na", ctypes.c_size_t), ("nt", ctypes.c_size_t),
                ("nv", ctypes.c_size_t), ("c", ctypes.c_float), ("fs", ctypes.c_float), ("fd", ctypes.c_float),
                ("fn", ctypes.c_float), ("method", ctypes.c_int), ("frames_per_chunk", ctypes.c_int)]


def _declare():
    lib = _lib.lib()
    if getattr(lib, "_batch_declared", False):
        return lib
    P, Z, I = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int  # noqa: E741
    arr = ctypes.POINTER(BatchEnsembleC)
    lib.rcabeam_batch_table_bytes.argtypes = [Z, arr, ctypes.POINTER(Z)]
    lib.rcabeam_batch_prepare.argtypes = [Z, arr, P, Z]
    lib.rcabeam_batch_run_device.argtypes = [Z, arr, P, Z, P, I, P]
    for fn in (lib.rcabeam_batch_table_bytes, lib.rcabeam_batch_prepare, lib.rcabeam_batch_run_device):
        fn.restype = I
    lib._batch_declared = True
    return lib


@dataclass
class Ensemble:
    """One device-resident ensemble of the queue."""

    rc: torch.Tensor            # packed (c, a, s, t) complex64 channels, as bytes or complex
    cr: torch.Tensor
    shape: tuple                # (ns, nc, na, nt)
    grid: tuple
    geom: RCAGeometry
    angles: np.ndarray
    t_start: object
    method: str = "opw"
    frames_per_chunk: int = 64
    tensors: dict = field(default_factory=dict)

    def build(self, device, order: bool = True) -> None:
        ns, nc, na, nt = self.shape
        if self.method not in METHODS:
            raise ValueError("method must be opw, xdoppler or dmas")
        f32 = lambda v: torch.from_numpy(np.ascontiguousarray(v, np.float32)).to(device)  # noqa: E731
        scan = f32(scan_coords(self.grid))
        nv = scan.shape[0]
        t = dict(scan=scan, xe=f32(self.geom.x_el), ye=f32(self.geom.y_el), angles=f32(self.angles),
                 starts=f32(np.broadcast_to(np.asarray(self.t_start, np.float32), (na,))),
                 pd=torch.zeros((nv, 2), dtype=torch.float32, device=device), order=None)
        if order and nv >= 128:  # every method's 64-voxel tiles want compact (Morton) voxel sets
            size = ctypes.c_size_t(0)
            _lib.check(_lib.lib().rcabeam_voxel_order_workspace_bytes(nv, ctypes.byref(size)), "voxel_order")
            ws = torch.empty(int(size.value), dtype=torch.uint8, device=device)
            t["order"] = torch.empty(nv, dtype=torch.int32, device=device)
            _lib.call("rcabeam_voxel_order_device", scan.data_ptr(), nv, t["order"].data_ptr(), ws.data_ptr(),
                      ws.numel())
        self.tensors = t

    @property
    def voxels(self) -> int:
        return self.tensors["scan"].shape[0]

    def units(self) -> int:
        ns, nc, na, nt = self.shape
        return self.voxels * 2 * nc * na * nt

    def descriptor(self, frames_per_chunk: int | None = None, voxels: int | None = None) -> BatchEnsembleC:
        ns, nc, na, nt = self.shape
        t = self.tensors
        g = self.geom
        return BatchEnsembleC(
            self.rc.data_ptr(), self.cr.data_ptr(), t["scan"].data_ptr(),
            None if t["order"] is None else t["order"].data_ptr(), t["xe"].data_ptr(), t["ye"].data_ptr(),
            t["angles"].data_ptr(), t["starts"].data_ptr(), t["pd"].data_ptr(), ns, nc, na, nt,
            self.voxels if voxels is None else voxels, float(g.c), float(g.fs), float(g.f_demod),
            -1.0 if g.fnumber is None else float(g.fnumber), METHODS[self.method],
            int(frames_per_chunk or self.frames_per_chunk))

    def power(self) -> torch.Tensor:
        return self.tensors["pd"][:, 0]


class _SubQueue:
    """The ensembles of one method: device table, completion times, and how it runs:
    ``ctas_per_sm`` 1-3 is the persistent kernel at that many CTAs per SM, 0 the
    single-ensemble kernels launched per ensemble on the sub-queue's stream."""

    def __init__(self, lib, indices, ensembles, ctas_per_sm: int, voxel_limit: int | None, device):
        self.lib = lib
        self.indices = indices
        n = len(ensembles)
        self.list = (BatchEnsembleC * n)(*[e.descriptor(voxels=None if voxel_limit is None else
                                                       min(voxel_limit, e.voxels)) for e in ensembles])
        size = ctypes.c_size_t(0)
        _lib.check(lib.rcabeam_batch_table_bytes(n, self.list, ctypes.byref(size)), "batch_table_bytes")
        self.table = torch.empty(int(size.value) + 256, dtype=torch.uint8, device=device)
        self.base = (256 - self.table.data_ptr() % 256) % 256
        self.table_bytes = int(size.value)
        _lib.check(lib.rcabeam_batch_prepare(n, self.list, self.table.data_ptr() + self.base, self.table_bytes),
                   "batch_prepare")
        self.times = torch.zeros(n + 1, dtype=torch.int64, device=device)
        self.ctas_per_sm = ctas_per_sm
        self.ensembles = ensembles

    def kernel_launches(self) -> int:
        """Kernels one launch() enqueues: the persistent kernel, or per ensemble its
        single-ensemble kernels (64-frame chunks plus a tail launch; XDoppler's
        magnitude pass; DMAS one) and a completion stamp, plus the start stamp."""
        if self.ctas_per_sm:
            return 1
        total = 1
        for e in self.ensembles:
            nt = e.shape[3]
            das = 1 if e.method == "dmas" else (nt >= 64) + (nt % 64 > 0) + (e.method == "xdoppler")
            total += das + 1
        return total

    def launch(self, stream) -> None:
        _lib.check(self.lib.rcabeam_batch_run_device(len(self.indices), self.list, self.table.data_ptr() + self.base,
                                                     self.table_bytes, self.times.data_ptr(), self.ctas_per_sm,
                                                     ctypes.c_void_p(stream.cuda_stream)), "batch_run")


class BatchQueue:
    """A prepared queue: one sub-queue per method, completion-time buffers, optional CUDA graph.

    ``ctas_per_sm`` is an int (every method) or a {method: int} map (the autotuner's choice)."""

    def __init__(self, ensembles, *, ctas_per_sm=1, voxel_limit: int | None = None):
        self.lib = _declare()
        self.ensembles = list(ensembles)
        device = self.ensembles[0].rc.device
        budget = ctas_per_sm if isinstance(ctas_per_sm, dict) else {m: int(ctas_per_sm) for m in METHODS}
        # One sub-queue after another on one stream: run concurrently, the methods'
        # sample windows compete for L2 (measured 129.7 s against 109.6 s for the
        # sequential launches on the 48-ensemble queue, with the same kernels).
        self.parts = []
        for method in ("dmas", "opw", "xdoppler"):
            idx = [i for i, e in enumerate(self.ensembles) if e.method == method]
            if idx:
                self.parts.append(_SubQueue(self.lib, idx, [self.ensembles[i] for i in idx], int(budget[method]),
                                            voxel_limit, device))
        self.graph = None

    def launch(self, stream: torch.cuda.Stream | None = None) -> None:
        """Enqueue the sub-queues one after another on ``stream`` (default: the current stream)."""
        main = torch.cuda.current_stream() if stream is None else stream
        for part in self.parts:
            part.launch(main)

    def capture(self) -> None:
        """Record the launches into one CUDA graph (the first run warms up outside the capture)."""
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            self.launch(side)
        torch.cuda.current_stream().wait_stream(side)
        torch.cuda.synchronize()
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self.launch()

    def run(self) -> None:
        if self.graph is not None:
            self.graph.replay()
        else:
            self.launch()

    def completion_ms(self) -> np.ndarray:
        """Per-ensemble completion time since the first sub-queue kernel started (device clock), ms."""
        times = [part.times.cpu().numpy().astype(np.int64) for part in self.parts]
        start = min(t[0] for t in times)
        out = np.empty(len(self.ensembles))
        for part, t in zip(self.parts, times):
            out[part.indices] = (t[1:] - start) / 1e6
        return out


def _sample(e: Ensemble, tiles: int) -> int:
    return min(e.voxels, 64 * tiles)


def autotune(ensembles, *, sample_tiles: int = 148 * 2, repeats: int = 2, cache: dict | None = None) -> dict:
    """Frame chunk per shape class (staged methods) and CTAs per SM per method.

    Each candidate runs the persistent kernel on a bounded sample (the first
    ``sample_tiles`` tiles of one ensemble of the class in traversal order) and
    is timed with CUDA events; the fastest per class is written back into the
    ensembles.  Returns {class: frames_per_chunk, "ctas_per_sm": {method: k}}.
    """
    cache = {} if cache is None else cache
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(queue):
        queue.launch()
        torch.cuda.synchronize()
        best = float("inf")
        for _ in range(repeats):
            start.record()
            queue.launch()
            stop.record()
            torch.cuda.synchronize()
            best = min(best, start.elapsed_time(stop))
        return best

    classes = {}
    for e in ensembles:
        key = (e.method, e.shape[2], e.shape[3])
        classes.setdefault(key, e)
    for key, e in classes.items():
        if key in cache:
            continue
        if e.method == "dmas":
            cache[key] = 64
            continue
        results = {}
        for fpc in FRAME_CHUNKS:
            e.frames_per_chunk = fpc
            results[fpc] = timed(BatchQueue([e], ctas_per_sm=3, voxel_limit=_sample(e, sample_tiles)))
        cache[key] = min(results, key=results.get)
    for e in ensembles:
        e.frames_per_chunk = cache[(e.method, e.shape[2], e.shape[3])]
    if "ctas_per_sm" not in cache:
        # Register budget per method, on that method's shape classes.
        budgets = {}
        for method in METHODS:
            reps = [e for key, e in classes.items() if key[0] == method]
            if not reps:
                budgets[method] = 1
                continue
            # Persistent kernel at 2 or 3 CTAs per SM, or per-ensemble grids (0): which one wins
            # depends on the ensembles' size, so the sample is eight times the frame-chunk one.
            results = {k: timed(BatchQueue(reps, ctas_per_sm=k, voxel_limit=8 * 64 * sample_tiles))
                       for k in (0, 2, 3)}
            budgets[method] = min(results, key=results.get)
        cache["ctas_per_sm"] = budgets
    return {**{str(k): v for k, v in cache.items() if k != "ctas_per_sm"}, "ctas_per_sm": cache["ctas_per_sm"]}


def sequential(ensembles) -> np.ndarray:
    """The plain path: one rcabeam_ensemble_device launch per ensemble in queue
    order on the default stream.  Returns each ensemble's completion time since
    the first launch (ms, CUDA events)."""
    events = [torch.cuda.Event(enable_timing=True) for _ in range(len(ensembles) + 1)]
    work = {}
    for e in ensembles:
        ns, nc, na, _ = e.shape
        key = e.voxels
        if key not in work:
            work[key] = torch.empty(_cuda_impl.workspace_bytes(e.voxels, nc, na), dtype=torch.uint8,
                                    device=e.rc.device)
    torch.cuda.synchronize()
    events[0].record()
    for i, e in enumerate(ensembles):
        ns, nc, na, nt = e.shape
        t = e.tensors
        g = e.geom
        t["pd"].zero_()
        _lib.call("rcabeam_ensemble_device", e.rc.data_ptr(), e.cr.data_ptr(), t["scan"].data_ptr(),
                  t["xe"].data_ptr(), t["ye"].data_ptr(), t["angles"].data_ptr(), t["starts"].data_ptr(),
                  t["pd"].data_ptr(), None, None, None, work[e.voxels].data_ptr(), ns, nc, na, nt, e.voxels,
                  float(g.c), float(g.fs), float(g.f_demod), -1.0 if g.fnumber is None else float(g.fnumber),
                  METHODS[e.method], 2)
        events[i + 1].record()
    torch.cuda.synchronize()
    return np.array([events[0].elapsed_time(ev) for ev in events[1:]])
