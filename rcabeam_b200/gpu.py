"""Reusable OPW buffers on one CUDA device: ``OpwWorkspace`` (reference src/rcabeam/gpu.py:16-209).

The reference keeps CuPy arrays; this implementation keeps ``torch.Tensor``
CUDA buffers with the same ownership rules: metadata is snapshotted at
construction, ``pack`` copies (and optionally FP16-converts) channels into
owned packed buffers, ``reconstruct`` returns borrowed IQ that the next call
overwrites, ``power`` returns borrowed power.  Calls are synchronous,
serialized by a lock, and only accepted on the construction device with the
default stream current.  Warmed reconstruction allocates no device memory.
"""

from __future__ import annotations

from operator import index
from threading import Lock

import numpy as np
import torch

from rcabeam_b200 import _cuda_impl
from rcabeam_b200.ensemble import IQStorage
from rcabeam_b200.sim import RCAGeometry, scan_coords


class OpwWorkspace:
    """Own fixed-shape packed channels, scratch and GPU IQ/power outputs.

    ``spatial_order`` is accepted for interface compatibility: the kernels
    always traverse voxels in spatially compact tiles and write canonical
    order, so both settings return identical canonical outputs.
    """

    def __init__(self, channel_shape, angles, t_start, grid, geom: RCAGeometry, *, iq_storage: IQStorage = "float32",
                 spatial_order: bool = False) -> None:
        if len(channel_shape) != 4 or any(index(n) < 1 for n in channel_shape) or channel_shape[0] < 2:
            raise ValueError("Expected nonempty (samples, channels, angles, frames), samples >=2")
        if iq_storage not in ("float32", "float16"):
            raise ValueError("IQ storage must be float32 or float16")
        self._channel_shape = tuple(index(n) for n in channel_shape)
        ns, nc, na, nt = self._channel_shape
        if any(np.ndim(v) != 1 for v in (angles, geom.x_el, geom.y_el)):
            raise ValueError("Geometry must contain coordinate/angle vectors")
        if len(angles) != na or len(geom.x_el) != nc or len(geom.y_el) != nc:
            raise ValueError("Geometry must match channel/angle dimensions")
        if len(grid) != 3 or any(np.ndim(axis) != 1 or not len(axis) for axis in grid):
            raise ValueError("Grid axes must be nonempty coordinate vectors")
        starts = np.broadcast_to(np.asarray(t_start, dtype=np.float32), (na,))
        scan = scan_coords(grid)
        vectors = [np.array(v, dtype=np.float32) for v in (geom.x_el, geom.y_el, angles, starts)]
        fn = -1.0 if geom.fnumber is None else geom.fnumber
        constants = np.asarray([geom.c, geom.fs, geom.f_demod, fn], dtype=np.float32)
        if not all(np.isfinite(v).all() for v in (scan, *vectors, constants)) or min(constants[:2]) <= 0:
            raise ValueError("Geometry must be finite with positive sound speed/sampling frequency")
        if geom.fnumber is not None and fn <= 0:
            raise ValueError("F-number must be positive or None")
        if not torch.cuda.is_available():
            raise ValueError("OpwWorkspace requires a CUDA device")
        self._device = torch.cuda.current_device()
        self._check_context()
        self._lock = Lock()
        self._ready = False
        self._has_output = False
        self._half = iq_storage == "float16"
        self._constants = tuple(float(v) for v in constants)
        self._shape = (len(grid[0]), len(grid[1]), len(grid[2]))
        self._spatial_order = bool(spatial_order)
        dev = torch.device("cuda", self._device)
        nv = len(scan)
        self._scan = torch.from_numpy(scan).to(dev)
        self._xe, self._ye, self._angles, self._starts = (torch.from_numpy(v).to(dev) for v in vectors)
        size = ns * nc * na * nt * (4 if self._half else 8)
        self._rc = torch.empty(size, dtype=torch.uint8, device=dev)
        self._cr = torch.empty(size, dtype=torch.uint8, device=dev)
        self._range_error = torch.zeros(1, dtype=torch.int32, device=dev)
        self._geometry = torch.empty(_cuda_impl.workspace_bytes(nv, nc, na), dtype=torch.uint8, device=dev)
        self._pd = torch.empty((nv, 2), dtype=torch.float32, device=dev)
        self._signal = torch.empty((nv, nt), dtype=torch.complex64, device=dev)
        self._iq = self._signal.view(*self._shape, nt)
        torch.cuda.synchronize(dev)

    def _check_context(self) -> None:
        """Reject a different CUDA device or a nondefault stream before any work."""
        if torch.cuda.current_device() != self._device or torch.cuda.current_stream().cuda_stream != 0:
            raise ValueError("Workspace requires its construction device and the default CUDA stream")

    @property
    def power(self) -> torch.Tensor:
        """Borrowed float32 ``(nx, nz, ny)`` unfiltered power of the last reconstruction."""
        with self._lock:
            if not self._has_output:
                raise RuntimeError("Reconstruct valid channels before reading power")
            return self._pd[:, 0].reshape(self._shape)

    def pack(self, rc: torch.Tensor, cr: torch.Tensor) -> None:
        """Synchronously copy GPU IQ into the owned packed buffers, invalidating output."""
        with self._lock:
            self._ready = False
            self._has_output = False
            self._check_context()
            for data in (rc, cr):
                if (not isinstance(data, torch.Tensor) or not data.is_cuda or tuple(data.shape) != self._channel_shape
                        or data.dtype != torch.complex64):
                    raise ValueError("Inputs must be matching complex64 CUDA IQ arrays")
                if not data.is_contiguous() or data.device.index != self._device:
                    raise ValueError("Inputs must be contiguous and on the workspace device")
            _cuda_impl.pack_opw_channels(rc, cr, self._rc, self._cr, self._range_error, self._half)
            self._ready = True

    def reconstruct(self) -> torch.Tensor:
        """Reconstruct packed IQ without allocation; returns borrowed ``(nx, nz, ny, frames)`` IQ."""
        with self._lock:
            self._check_context()
            if not self._ready:
                raise RuntimeError("Pack valid channels before reconstructing")
            self._has_output = False
            ns, nc, na, nt = self._channel_shape
            _cuda_impl.opw_from_packed(self._rc, self._cr, self._scan, self._xe, self._ye, self._angles,
                                       self._starts, self._pd, self._signal, self._geometry, ns, nc, na, nt,
                                       *self._constants, self._half)
            self._has_output = True
            return self._iq
