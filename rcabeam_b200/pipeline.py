"""End-to-end filtered OPW power Doppler on one GPU.

``FilteredOpw`` is the resident form of the reference's filtered-OPW
composition (examples/_support/clutter_pipeline.py:18-146): pack RC/CR ->
OPW IQ (kept on the device) -> scaled temporal Gram -> float64 EVD ->
clutter-filtered power Doppler.  All buffers are allocated once; ``run``
launches every stage on the default stream without host synchronization
except the final solver-status check, and records CUDA events per stage.
``run_host`` adds the pinned host -> device upload of the channels and the
device -> host read of the power, the boundary a host caller sees.

``domain="channel"`` is the reference's channel-domain variant
(clutter_pipeline.py:85-91, 121-123): one temporal basis estimated over the
channel Casorati rows of both apertures ((samples x channels x angles) x
frames each), both apertures filtered before packing, then OPW and the mean
|IQ|^2 from the DAS kernel's power output (no IQ ensemble is stored).  DAS is
linear and acts on every frame alike, so for a given basis both domains give
the same filtered IQ; they differ in the rows the basis is estimated from.  With a
process group, each rank reconstructs its x slab of the grid
(``sharded.shard_grid``) and the clutter basis is estimated over every rank's
rows (one MAX and one SUM all-reduce, ``rcabeam_b200.sharded``).
"""

from __future__ import annotations

import numpy as np
import torch

from rcabeam_b200 import _cuda_impl, _lib
from rcabeam_b200.gpu_clutter import Gram
from rcabeam_b200.sim import RCAGeometry, scan_coords

_STAGES = ("pack", "das", "gram", "eig", "power")
_CHANNEL_STAGES = ("gram", "eig", "filter", "pack", "das")


class FilteredOpw:
    """Fixed-shape filtered-OPW pipeline: ``run(rc, cr) -> (nx, nz, ny)`` float64 filtered power.

    ``refine=True`` corrects the discarded leading vectors of a tensor-core Gram
    (``"tf32"``, ``"bf16x3"``) by a float64 Rayleigh-Ritz step on its 16 leading
    eigenvectors against the exact Gram (one extra pass over the IQ; when the
    smaller projector is ranks [0, rank_start)).
    ``iq_storage="bf16x2"`` runs the tensor-core DAS on split-BF16 planes; with
    ``deterministic=True`` every tile starts its channel walk at the same slot
    (by default each tile starts where the other SMs are, which keeps their
    windows in L2 together but makes the order of the float32 sums timing
    dependent); the builder warps' interleaving remains timing dependent, so
    reruns agree to 2e-6 - 1e-5 in filtered power instead of up to 5e-5, at about
    10 % more DAS time (measured 921 against 834 ms at the full-size workload)."""

    def __init__(self, channel_shape, angles, t_start, grid, geom: RCAGeometry, *, rank_start: int = 3,
                 rank_stop: int | None = None, precision: str = "complex128", iq_storage: str = "float32",
                 group=None, domain: str = "beamformed", deterministic: bool = False, refine: bool = False):
        ns, nc, na, nt = (int(n) for n in channel_shape)
        self.shape = (len(grid[0]), len(grid[1]), len(grid[2]))
        self.channel_shape = (ns, nc, na, nt)
        stop = nt if rank_stop is None else int(rank_stop)
        if not 0 <= rank_start <= stop <= nt:
            raise ValueError("Require 0 <= rank_start <= rank_stop <= number of frames")
        self.rank = (int(rank_start), stop)
        self.precision = precision
        self.group = group  # process group whose ranks hold the other x slabs (rcabeam_b200.sharded)
        if domain not in ("beamformed", "channel"):
            raise ValueError("Unknown filter domain")
        if domain == "channel" and group is not None:
            raise ValueError("Channel-domain filtering runs on one device")
        self.domain = domain
        if iq_storage not in ("float32", "float16", "bf16x2"):
            raise ValueError("IQ storage must be float32, float16 or bf16x2")
        if iq_storage == "bf16x2" and nt % 4:
            raise ValueError("bf16x2 storage requires a frame count divisible by 4")
        self.storage = iq_storage
        self.half = iq_storage == "float16"
        # Tensor-core DAS: fixed channel walk (bit-identical reruns) instead of the L2-aligned one.
        self.deterministic = bool(deterministic)
        dev = torch.device("cuda", torch.cuda.current_device())
        self.device = dev
        scan = scan_coords(grid)
        self.nv = len(scan)
        f32 = lambda v: torch.from_numpy(np.array(v, dtype=np.float32)).to(dev)  # noqa: E731
        self.scan = f32(scan)
        self.xe, self.ye, self.angles = f32(geom.x_el), f32(geom.y_el), f32(angles)
        self.starts = f32(np.broadcast_to(np.asarray(t_start, dtype=np.float32), (na,)))
        self.consts = (float(geom.c), float(geom.fs), float(geom.f_demod),
                       -1.0 if geom.fnumber is None else float(geom.fnumber))
        elem = 8 if iq_storage == "float32" else 4
        self.packed = [torch.empty(ns * nc * na * nt * elem, dtype=torch.uint8, device=dev) for _ in range(2)]
        self.packed_lo = ([torch.empty(ns * nc * na * nt * elem, dtype=torch.uint8, device=dev) for _ in range(2)]
                          if iq_storage == "bf16x2" else None)
        self.range_error = torch.zeros(1, dtype=torch.int32, device=dev)
        self.geometry = torch.empty(_cuda_impl.workspace_bytes(self.nv, nc, na), dtype=torch.uint8, device=dev)
        self.pd = torch.empty((self.nv, 2), dtype=torch.float32, device=dev)
        # Beamformed domain: the IQ ensemble (Casorati rows); channel domain: the filtered channels.
        self.iq = torch.empty((self.nv, nt), dtype=torch.complex64, device=dev) if domain == "beamformed" else None
        self.filtered = ([torch.empty(self.channel_shape, dtype=torch.complex64, device=dev) for _ in range(2)]
                         if domain == "channel" else None)
        self.gram = Gram(nt, dev)
        self.power = torch.empty(self.nv, dtype=torch.float64, device=dev)
        self.host_power = torch.empty(self.nv, dtype=torch.float64, pin_memory=True)
        self.inputs = [torch.empty(self.channel_shape, dtype=torch.complex64, device=dev) for _ in range(2)]
        start, stop = self.rank
        self.subtract = stop - start > nt - (stop - start)
        self.k = (start + nt - stop) if self.subtract else (stop - start)
        self.vectors = torch.empty((max(self.k, 1), nt), dtype=torch.complex128, device=dev)
        # Optional float64 Rayleigh-Ritz correction of the discarded leading vectors (one pass
        # over the IQ) for tensor-core Gram precisions; only when the smaller projector is
        # the leading ranks [0, rank_start) (subtract mode, rank_stop = nt).
        leading = self.subtract and stop == nt and 0 < self.k <= 4
        self.refine = bool(refine) and leading
        if self.refine and (domain != "beamformed" or group is not None):
            self.refine = False
        # Rayleigh-Ritz subspace: the m leading eigenvectors (m = k + 13, at most 16 and T).
        self.ritz_m = min(nt, self.k + 13, 16)
        self.ritz_basis = torch.empty((self.ritz_m, nt), dtype=torch.complex128, device=dev)
        self.ritz = Gram(self.ritz_m, dev) if self.refine else None
        self.events = [torch.cuda.Event(enable_timing=True) for _ in range(len(_STAGES) + 1)]
        self.last_das_event_ms = None

    def _select_vectors(self) -> None:
        """Column-major (T x k) vectors of the smaller projector from the ascending eigenvectors."""
        nt = self.channel_shape[3]
        start, stop = self.rank
        vt = torch.view_as_complex(self.gram.matrix.view(nt, nt, 2))  # row e = e-th eigenvector (ascending)
        desc = torch.arange(nt - 1, -1, -1, device=self.device)     # descending rank r -> eigenvector nt-1-r
        ranks = torch.cat((desc[:start], desc[stop:])) if self.subtract else desc[start:stop]
        if self.k:
            torch.index_select(vt, 0, ranks, out=self.vectors[: self.k])

    def _refine(self) -> None:
        """Float64 Rayleigh-Ritz on the m leading eigenvectors of the reduced-precision Gram:
        H = (X V_m)^H (X V_m) in float64 (one pass over the IQ), H's eigenvectors rotate V_m,
        and the k with the largest Ritz values replace the discarded vectors (no host sync)."""
        nt, m, k = self.channel_shape[3], self.ritz_m, self.k
        vt = torch.view_as_complex(self.gram.matrix.view(nt, nt, 2))  # row e: e-th eigenvector (ascending)
        torch.index_select(vt, 0, torch.arange(nt - 1, nt - 1 - m, -1, device=self.device), out=self.ritz_basis)
        _lib.call("rcabeam_ritz_matrix_device", self.iq.data_ptr(), self.nv, nt, self.ritz_basis.data_ptr(), m,
                  self.ritz.matrix.data_ptr())
        self.ritz.decompose()  # ascending Ritz values; row c of the view = c-th Ritz vector's coefficients
        u = torch.view_as_complex(self.ritz.matrix.view(m, m, 2))[m - k:].flip(0)  # k largest, descending
        torch.matmul(u, self.ritz_basis, out=self.vectors[:k])

    def run(self, rc: torch.Tensor, cr: torch.Tensor, after_inputs=None) -> torch.Tensor:
        """Filtered power of resident complex64 RC/CR channels ``(ns, nc, na, nt)``.

        ``after_inputs`` (optional) is called once the work that reads ``rc`` / ``cr`` has
        been queued (packing; in the channel domain, filtering), before the rest of the
        step: a caller may queue the next ensemble's upload into them there.
        """
        if self.domain == "channel":
            return self._run_channel(rc, cr, after_inputs)
        ev = self.events
        ev[0].record()
        self._pack(rc, cr)
        ev[1].record()
        if after_inputs is not None:
            after_inputs()
        self._das(self.iq)
        ev[2].record()
        self.gram.accumulate((self.iq,), self.precision, self.group)
        ev[3].record()
        self.gram.decompose()
        ev[4].record()
        if self.rank[0] == self.rank[1]:
            self.power.zero_()
        else:
            self._select_vectors()
            if self.refine:
                self._refine()
            _lib.call("rcabeam_project_device", self.iq.data_ptr(), None, self.power.data_ptr(), self.nv,
                      self.channel_shape[3], 0, self.vectors.data_ptr(), self.k, 1 if self.subtract else 0, None)
        ev[5].record()
        self.last_das_event_ms = (ev[1], ev[2])
        return self.power.view(self.shape)

    def _run_channel(self, rc: torch.Tensor, cr: torch.Tensor, after_inputs=None) -> torch.Tensor:
        """Channel domain: shared basis of the RC and CR channel rows, filter, pack, OPW power."""
        ns, nc, na, nt = self.channel_shape
        ev = self.events
        ev[0].record()
        self.gram.accumulate((rc, cr), self.precision)
        ev[1].record()
        self.gram.decompose()
        ev[2].record()
        rows = ns * nc * na
        if self.rank[0] != self.rank[1]:
            self._select_vectors()
            for src, dst in zip((rc, cr), self.filtered):
                _lib.call("rcabeam_project_device", src.data_ptr(), dst.data_ptr(), None, rows, nt, 0,
                          self.vectors.data_ptr(), self.k, (1 if self.subtract else 0) | 2, None)
        ev[3].record()
        if after_inputs is not None:
            after_inputs()
        if self.rank[0] == self.rank[1]:
            self.power.zero_()
            for e in ev[4:]:
                e.record()
        else:
            self._pack(*self.filtered)
            ev[4].record()
            self._das(None)
            self.power.copy_(self.pd[:, 0])
            ev[5].record()
        self.last_das_event_ms = (ev[4], ev[5])
        return self.power.view(self.shape)

    def _pack(self, rc: torch.Tensor, cr: torch.Tensor) -> None:
        ns, nc, na, nt = self.channel_shape
        if self.storage == "float16":
            self.range_error.zero_()
            for src, dst in zip((rc, cr), self.packed):
                _lib.call("rcabeam_pack_ensemble_fp16_device", src.data_ptr(), dst.data_ptr(),
                          self.range_error.data_ptr(), ns, nc, na, nt)
        elif self.storage == "bf16x2":
            self.range_error.zero_()
            for src, hi, lo in zip((rc, cr), self.packed, self.packed_lo):
                _lib.call("rcabeam_pack_ensemble_split_device", src.data_ptr(), hi.data_ptr(), lo.data_ptr(),
                          self.range_error.data_ptr(), ns, nc, na, nt)
        else:
            for src, dst in zip((rc, cr), self.packed):
                _lib.call("rcabeam_pack_ensemble_device", src.data_ptr(), dst.data_ptr(), ns, nc, na, nt)

    def _das(self, iq: torch.Tensor | None) -> None:
        """OPW of the packed channels: power into pd, IQ into ``iq`` when given."""
        ns, nc, na, nt = self.channel_shape
        signal = None if iq is None else iq.data_ptr()
        if self.storage == "bf16x2":
            _lib.call("rcabeam_opw_tc_device", self.packed[0].data_ptr(), self.packed_lo[0].data_ptr(),
                      self.packed[1].data_ptr(), self.packed_lo[1].data_ptr(), self.scan.data_ptr(),
                      self.xe.data_ptr(), self.ye.data_ptr(), self.angles.data_ptr(), self.starts.data_ptr(),
                      self.pd.data_ptr(), signal, self.geometry.data_ptr(), ns, nc, na, nt, self.nv,
                      *self.consts, 1 | (2 if self.deterministic else 0))
        else:
            _cuda_impl.opw_from_packed(self.packed[0], self.packed[1], self.scan, self.xe, self.ye, self.angles,
                                       self.starts, self.pd, iq, self.geometry, ns, nc, na, nt, *self.consts,
                                       self.half, synchronize=False)

    def check(self) -> None:
        """Synchronize and raise on solver or staging-pipeline failures."""
        torch.cuda.synchronize()
        if int(self.gram.info.item()):
            raise np.linalg.LinAlgError("cuSOLVER eigendecomposition failed")
        if self.storage != "float32" and int(self.range_error.item()):
            raise ValueError("packed IQ storage requires finite components (within +/-65504 for FP16)")
        if _lib.device_error():
            raise _lib.RcabeamCudaError("a reconstruction kernel timed out waiting on its staging pipeline")

    def run_host(self, rc_host: torch.Tensor, cr_host: torch.Tensor) -> torch.Tensor:
        """Pinned host channels -> pinned host float64 filtered power (upload and download included)."""
        self.inputs[0].copy_(rc_host, non_blocking=True)
        self.inputs[1].copy_(cr_host, non_blocking=True)
        self.run(self.inputs[0], self.inputs[1])
        self.host_power.copy_(self.power, non_blocking=True)
        return self.host_power

    def run_host_sequence(self, pairs, outputs=None) -> list[torch.Tensor]:
        """Filtered power of a sequence of pinned host ``(rc, cr)`` ensembles, each uploaded,
        reconstructed and read back (pinned float64 host arrays, one per ensemble).

        Each ensemble's upload runs on a side stream as soon as the previous ensemble no
        longer reads the raw channels (after packing; after filtering in the channel
        domain), so it overlaps that ensemble's reconstruction, the way an acquisition
        stream feeds the pipeline.  ``outputs`` may pass preallocated pinned arrays.
        """
        pairs = list(pairs)
        if outputs is None:
            outputs = [torch.empty(self.nv, dtype=torch.float64, pin_memory=True) for _ in pairs]
        if len(outputs) != len(pairs):
            raise ValueError("one output per ensemble is required")
        if not hasattr(self, "_copy_stream"):
            self._copy_stream = torch.cuda.Stream(self.device)
            self._uploaded = torch.cuda.Event()
        # Raw channels are last read by the packing (beamformed) or the filter (channel domain).
        consumed = self.events[3] if self.domain == "channel" else self.events[1]
        main = torch.cuda.current_stream(self.device)
        self._copy_stream.wait_stream(main)  # no upload before the work already queued

        def upload(i: int) -> None:
            rc_host, cr_host = pairs[i]
            with torch.cuda.stream(self._copy_stream):
                self._copy_stream.wait_event(consumed)
                self.inputs[0].copy_(rc_host, non_blocking=True)
                self.inputs[1].copy_(cr_host, non_blocking=True)
                self._uploaded.record(self._copy_stream)

        if pairs:
            upload(0)
        for i, out in enumerate(outputs):
            main.wait_event(self._uploaded)
            # The next upload is queued as soon as this step's reads of the inputs are queued,
            # i.e. before the step's later stages (whose eigensolver may block the host).
            nxt = (lambda j=i + 1: upload(j)) if i + 1 < len(pairs) else None
            self.run(self.inputs[0], self.inputs[1], after_inputs=nxt)
            out.copy_(self.power.view(-1), non_blocking=True)
        torch.cuda.synchronize(self.device)
        return outputs

    @staticmethod
    def collect_das_ms(pair) -> float:
        return pair[0].elapsed_time(pair[1])

    def stage_ms(self) -> dict:
        torch.cuda.synchronize()
        names = _CHANNEL_STAGES if self.domain == "channel" else _STAGES
        return {name: round(self.events[i].elapsed_time(self.events[i + 1]), 3) for i, name in enumerate(names)}

    def launches_per_step(self) -> int:
        """Kernels of this library launched per ``run``: pack x2, voxel order (bounding box,
        Morton codes, 4 radix-sort passes), DAS (one persistent tensor-core launch, or main +
        tail staged launches), scale, Gram, Gram finish, projection (channel domain: per
        aperture scale, Gram and projection)."""
        das = 1 if self.storage != "float32" and self.channel_shape[3] % 4 == 0 else 2
        if self.domain == "channel":  # scale x2, Gram x2, finish, projection x2, pack x2, order, DAS
            return 5 + 2 + 2 + 6 + das
        return 2 + 6 + das + 4 + (1 if self.refine else 0)


def synthetic_channels(shape, *, generator: torch.Generator, device, scale: float = 1.0):
    """Seeded complex Gaussian channel IQ ``(ns, nc, na, nt)`` for both apertures, made on the device."""
    out = []
    for _ in range(2):
        re = torch.randn(shape, generator=generator, device=device, dtype=torch.float32)
        im = torch.randn(shape, generator=generator, device=device, dtype=torch.float32)
        out.append(torch.complex(re, im).mul_(scale))
    return out
