"""Reusable OPW buffers on one CUDA device: ``OpwWorkspace`` (reference src/rcabeam/gpu.py:16-209).

The reference keeps CuPy arrays; this implementation keeps ``torch.Tensor``
CUDA buffers under the same ownership contract: the acquisition is validated
and copied to the device at construction, ``pack`` copies (and optionally
FP16-converts) channels into owned packed buffers, ``reconstruct`` returns
borrowed IQ that the next call overwrites, ``power`` returns borrowed power.
The workspace is a small state machine (empty -> packed -> reconstructed);
calls are synchronous, serialized by a lock, and only accepted on the
construction device with the default stream current.  Warmed reconstruction
allocates no device memory.
"""

from __future__ import annotations

import enum
from contextlib import contextmanager
from threading import Lock

import torch

from rcabeam_b200 import _cuda_impl, _inputs
from rcabeam_b200.ensemble import IQStorage
from rcabeam_b200.sim import RCAGeometry

_PACKED_BYTES = {"float32": 8, "float16": 4}  # bytes per packed complex sample


class _State(enum.Enum):
    EMPTY = 0          # no valid packed channels (fresh, or the last pack failed)
    PACKED = 1         # packed channels ready; no output for them yet
    RECONSTRUCTED = 2  # IQ / power of the packed channels are valid


class OpwWorkspace:
    """Own fixed-shape packed channels, scratch and GPU IQ/power outputs.

    The acquisition is checked by the same validator as the frame-batched
    functions.  ``spatial_order`` is accepted for interface compatibility: the
    kernels always traverse voxels in spatially compact tiles and write
    canonical order, so both settings return identical canonical outputs.
    """

    def __init__(self, channel_shape, angles, t_start, grid, geom: RCAGeometry, *, iq_storage: IQStorage = "float32",
                 spatial_order: bool = False) -> None:
        acq = _inputs.acquisition(channel_shape, angles, t_start, grid, geom)
        if iq_storage not in _PACKED_BYTES:
            raise ValueError("IQ storage must be float32 or float16 for the workspace")
        if not torch.cuda.is_available():
            raise ValueError("OpwWorkspace requires a CUDA device")
        self._device = torch.cuda.current_device()
        self._require_context()
        self._acq = acq
        self._storage = iq_storage
        self._spatial_order = bool(spatial_order)
        self._lock = Lock()
        self._state = _State.EMPTY
        dev = torch.device("cuda", self._device)
        on_device = lambda a: torch.from_numpy(a).to(dev)  # noqa: E731
        self._geometry_vectors = tuple(on_device(a) for a in (acq.scan, acq.x_el, acq.y_el, acq.angles, acq.starts))
        ns, nc, na, nt = acq.channel_shape
        packed = ns * nc * na * nt * _PACKED_BYTES[iq_storage]
        self._packed = (torch.empty(packed, dtype=torch.uint8, device=dev),
                        torch.empty(packed, dtype=torch.uint8, device=dev))
        self._range_error = torch.zeros(1, dtype=torch.int32, device=dev)
        self._scratch = torch.empty(_cuda_impl.workspace_bytes(acq.voxels, nc, na), dtype=torch.uint8, device=dev)
        self._pd = torch.empty((acq.voxels, 2), dtype=torch.float32, device=dev)
        self._signal = torch.empty((acq.voxels, nt), dtype=torch.complex64, device=dev)
        torch.cuda.synchronize(dev)

    def _require_context(self) -> None:
        """Only the construction device with its default stream current may run work."""
        if torch.cuda.current_device() != self._device or torch.cuda.current_stream().cuda_stream != 0:
            raise ValueError("Workspace requires its construction device and the default CUDA stream")

    @contextmanager
    def _serialized(self):
        with self._lock:
            self._require_context()
            yield

    @property
    def power(self) -> torch.Tensor:
        """Borrowed float32 ``(nx, nz, ny)`` unfiltered power of the last reconstruction."""
        with self._lock:
            if self._state is not _State.RECONSTRUCTED:
                raise RuntimeError("Reconstruct valid channels before reading power")
            return self._pd[:, 0].view(self._acq.grid_shape)

    def pack(self, rc: torch.Tensor, cr: torch.Tensor) -> None:
        """Synchronously copy GPU IQ into the owned packed buffers, invalidating any output."""
        with self._lock:
            self._state = _State.EMPTY  # a failed pack leaves nothing to reconstruct
            self._require_context()
            for data in (rc, cr):
                self._check_channels(data)
            _cuda_impl.pack_opw_channels(rc, cr, *self._packed, self._range_error, self._storage == "float16")
            self._state = _State.PACKED

    def _check_channels(self, data) -> None:
        if not (isinstance(data, torch.Tensor) and data.is_cuda and data.dtype == torch.complex64
                and tuple(data.shape) == self._acq.channel_shape):
            raise ValueError("Inputs must be matching complex64 CUDA IQ arrays")
        if data.device.index != self._device or not data.is_contiguous():
            raise ValueError("Inputs must be contiguous and on the workspace device")

    def reconstruct(self) -> torch.Tensor:
        """Reconstruct the packed IQ without allocation; returns borrowed ``(nx, nz, ny, frames)`` IQ."""
        with self._serialized():
            if self._state is _State.EMPTY:
                raise RuntimeError("Pack valid channels before reconstructing")
            self._state = _State.PACKED  # the previous output is overwritten from here on
            scan, xe, ye, angles, starts = self._geometry_vectors
            _cuda_impl.opw_from_packed(*self._packed, scan, xe, ye, angles, starts, self._pd, self._signal,
                                       self._scratch, *self._acq.channel_shape, *self._acq.constants,
                                       self._storage == "float16")
            self._state = _State.RECONSTRUCTED
            return self._signal.view(*self._acq.grid_shape, self._acq.channel_shape[3])
