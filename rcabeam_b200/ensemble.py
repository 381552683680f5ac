"""Frame-batched RCA reconstruction: the public entry points of ``rcabeam.ensemble``.

Same signatures and argument contract as the reference
(src/rcabeam/ensemble.py:52-287), checked by the shared validator
``rcabeam_b200._inputs``; the work runs through the C ABI on the GPU.
Host NumPy arrays are uploaded and results downloaded, as in the reference.
"""

from __future__ import annotations

from typing import Literal, TypedDict

import numpy as np
from numpy.typing import NDArray

from rcabeam_b200 import _cuda_impl, _inputs
from rcabeam_b200.sim import RCAGeometry

Method = Literal["opw", "xdoppler", "rc_fmas", "dmas", "st_sw"]
IQStorage = Literal["float32", "float16", "bf16x2"]


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
    """Check the inputs once (``_inputs.acquisition``), reconstruct on the GPU, shape the outputs.

    The argument contract is the reference's (ensemble.py:52-130): same accepted inputs, the
    contract's message substrings.  Power comes back in canonical voxel order (the kernels
    write canonical positions from their own traversal), so no host un-permutation is needed.
    """
    rc, cr = np.asarray(rc), np.asarray(cr)
    code = _inputs.method_code(method, iq_storage, wants_signal=return_signal)
    acq = _inputs.acquisition(_inputs.channel_pair_shape(rc, cr), angles, t_start, grid, geom)
    _inputs.check_subsets(method, k, acq.channel_shape[2])
    nv, nt = acq.voxels, acq.channel_shape[3]
    planes = 2 if method == "apertures" else 1
    pd = np.empty((nv, 2), dtype=np.float32)
    signal = np.empty((nv * planes if return_signal else 0, nt), dtype=np.complex64)
    weights = np.empty(nv if method == "st_sw" else 0, dtype=np.float32)
    upload_s = _cuda_impl.ensemble_from_channels(
        np.ascontiguousarray(rc, dtype=np.complex64), np.ascontiguousarray(cr, dtype=np.complex64), acq.scan,
        acq.x_el, acq.y_el, acq.angles, acq.starts, pd, signal, weights, *acq.constants, code, k, iq_storage)
    if timings is not None:
        timings["raw_upload_seconds"] = upload_s
    power = pd[:, 0]
    if method == "st_sw":
        # Raw weights normalized by the whole volume's peak (reference ensemble.py:127-129).
        peak = weights.max()
        power = power * (weights / peak if peak > 0 else 0)
    power = np.ascontiguousarray(power).reshape(acq.grid_shape)
    if not return_signal:
        return power, signal
    return power, signal.reshape((*acq.grid_shape, 2, nt) if planes == 2 else (*acq.grid_shape, nt))


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
