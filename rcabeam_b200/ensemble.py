"""Frame-batched RCA reconstruction: the public entry points of ``rcabeam.ensemble``.

Same signatures, validation and error messages as the reference
(src/rcabeam/ensemble.py:52-287); the work runs through the C ABI on the GPU.
Host NumPy arrays are uploaded and results downloaded, as in the reference.
"""

from __future__ import annotations

from typing import Literal, TypedDict

import numpy as np
from numpy.typing import NDArray

from rcabeam_b200 import _cuda_impl
from rcabeam_b200.sim import RCAGeometry, scan_coords

Method = Literal["opw", "xdoppler", "rc_fmas", "dmas", "st_sw"]
IQStorage = Literal["float32", "float16", "bf16x2"]
_METHODS = {"opw": 0, "xdoppler": 1, "rc_fmas": 2, "dmas": 3, "st_sw": 4, "apertures": 5}


class EnsembleTiming(TypedDict):
    """Host wall time for completed raw RC/CR uploads, excluding allocation."""

    raw_upload_seconds: float


def opw_voxel_order(shape: tuple[int, int, int]) -> NDArray[np.intp]:
    """Canonical voxel indices in 2 x 4 lateral patches, tails last (reference ensemble.py:24-49).

    Patches of 2 x-rows by 4 y-columns are visited for every depth; the y tail
    (ny mod 4 columns) of the even-x part follows, then the odd x row.  The
    GPU kernels choose their own spatial traversal, so this order is only
    provided for callers that reorder voxels themselves.
    """
    nx, nz, ny = (int(s) for s in shape)
    if min(nx, nz, ny) < 1:
        raise ValueError("Grid dimensions must be positive")
    bx, by = nx - nx % 2, ny - ny % 4
    # Index arithmetic over (x-pair, z, y-quad, x-in-pair, y-in-quad).
    xp = np.arange(bx // 2)[:, None, None, None, None]
    zz = np.arange(nz)[None, :, None, None, None]
    yq = np.arange(by // 4)[None, None, :, None, None]
    xi = np.arange(2)[None, None, None, :, None]
    yi = np.arange(4)[None, None, None, None, :]
    core = (((2 * xp + xi) * nz + zz) * ny + 4 * yq + yi).ravel()
    ids = np.arange(nx * nz * ny, dtype=np.intp).reshape(nx, nz, ny)
    return np.concatenate((core.astype(np.intp), ids[:bx, :, by:].ravel(), ids[bx:].ravel()))


def _run(rc, cr, angles, t_start, grid, geom: RCAGeometry, method, k: int, return_signal: bool,
         timings: EnsembleTiming | None, iq_storage: IQStorage):
    """Validate ensemble inputs and execute the frame-batched CUDA path (reference ensemble.py:52-130)."""
    if method not in _METHODS or (method == "apertures" and not return_signal):
        raise ValueError(f"Unknown method: {method}")
    if iq_storage not in ("float32", "float16", "bf16x2") or (iq_storage != "float32" and method != "opw"):
        raise ValueError("IQ storage must be float32, or float16 / bf16x2 for OPW only")
    rc, cr = np.asarray(rc), np.asarray(cr)
    if rc.ndim != 4 or cr.shape != rc.shape or any(n == 0 for n in rc.shape) or rc.shape[0] < 2:
        raise ValueError("RC/CR must have matching nonempty (samples, channels, angles, frames) shapes")
    if len(angles) != rc.shape[2] or len(geom.x_el) != rc.shape[1] or len(geom.y_el) != rc.shape[1]:
        raise ValueError("Geometry must match the channel/angle dimensions")
    if any(np.ndim(axis) != 1 or not len(axis) or not np.isfinite(axis).all() for axis in grid):
        raise ValueError("Grid axes must be nonempty finite coordinate vectors")
    if not np.isfinite([geom.c, geom.fs, geom.f_demod]).all() or geom.c <= 0 or geom.fs <= 0:
        raise ValueError("Sound speed and sampling frequency must be finite and positive")
    if geom.fnumber is not None and (not np.isfinite(geom.fnumber) or geom.fnumber <= 0):
        raise ValueError("F-number must be positive or None")
    if method == "st_sw" and (k < 2 or k > 4 or len(angles) < k):
        raise ValueError("St-SW requires 2 <= k <= 4 and at least k angles")
    starts = np.ascontiguousarray(np.broadcast_to(np.asarray(t_start, dtype=np.float32), (len(angles),)))
    if not all(np.isfinite(a).all() for a in (angles, starts, geom.x_el, geom.y_el)):
        raise ValueError("Geometry and sample starts must be finite")
    scan = scan_coords(grid)
    nv, nt = len(scan), rc.shape[-1]
    shape = (len(grid[0]), len(grid[1]), len(grid[2]))
    pd = np.empty((nv, 2), dtype=np.float32)
    planes = 2 if method == "apertures" else 1
    signal = np.empty((nv * planes if return_signal else 0, nt), dtype=np.complex64)
    weights = np.empty(nv if method == "st_sw" else 0, dtype=np.float32)
    raw_upload_seconds = _cuda_impl.ensemble_from_channels(
        np.ascontiguousarray(rc, dtype=np.complex64),
        np.ascontiguousarray(cr, dtype=np.complex64),
        scan,
        np.ascontiguousarray(geom.x_el, dtype=np.float32),
        np.ascontiguousarray(geom.y_el, dtype=np.float32),
        np.ascontiguousarray(angles, dtype=np.float32),
        starts,
        pd,
        signal,
        weights,
        float(geom.c),
        float(geom.fs),
        float(geom.f_demod),
        -1.0 if geom.fnumber is None else float(geom.fnumber),
        _METHODS[method],
        k,
        iq_storage,
    )
    if timings is not None:
        timings["raw_upload_seconds"] = raw_upload_seconds
    if method == "st_sw":
        # Raw weights normalized by the full-volume peak (reference ensemble.py:127-129).
        peak = weights.max()
        pd[:, 0] *= weights / peak if peak > 0 else 0
    if return_signal:
        signal_shape = (*shape, 2, nt) if method == "apertures" else (*shape, nt)
        return pd[:, 0].reshape(shape), signal.reshape(signal_shape)
    return np.ascontiguousarray(pd[:, 0]).reshape(shape), signal


def ensemble_pd_from_channels(rc, cr, angles, t_start, grid, geom: RCAGeometry, *, method: Method = "opw", k: int = 2,
                              timings: EnsembleTiming | None = None,
                              iq_storage: IQStorage = "float32") -> NDArray[np.float32]:
    """Reconstruct a channel ensemble and reduce it without exporting IQ (reference ensemble.py:133-218).

    OPW / RC-FMAS return the mean squared magnitude over frames, XDoppler the
    magnitude of the mean RC x conj(CR) product, DMAS the mean DMAS-CCF-ACF
    response.  ``iq_storage="float16"`` (OPW only) packs channels to FP16;
    interpolation and accumulation stay float32.  ``iq_storage="bf16x2"``
    (OPW only, extension) packs float32 channels into BF16 hi/lo planes for the
    three-product tensor-core path.
    """
    return _run(rc, cr, angles, t_start, grid, geom, method, k, False, timings, iq_storage)[0]


def beamform_ensemble(rc, cr, angles, t_start, grid, geom: RCAGeometry, *,
                      method: Literal["opw", "xdoppler", "rc_fmas"] = "opw", timings: EnsembleTiming | None = None,
                      iq_storage: IQStorage = "float32") -> NDArray[np.complex64]:
    """Complex64 ``(nx, nz, ny, frames)`` OPW IQ or nonlinear slow-time signal (reference ensemble.py:221-270)."""
    if method not in ("opw", "xdoppler", "rc_fmas"):
        raise ValueError("Only OPW, XDoppler and RC-FMAS have complex signal outputs")
    return _run(rc, cr, angles, t_start, grid, geom, method, 2, True, timings, iq_storage)[1]


def beamform_apertures(rc, cr, angles, t_start, grid, geom: RCAGeometry):
    """Separately compounded RC and CR IQ, each ``(nx, nz, ny, frames)`` (reference ensemble.py:273-287)."""
    _, iq = _run(rc, cr, angles, t_start, grid, geom, "apertures", 2, True, None, "float32")
    return iq[..., 0, :], iq[..., 1, :]
