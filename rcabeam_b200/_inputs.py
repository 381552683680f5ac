"""One validator for every reconstruction entry point.

``acquisition()`` checks a channel shape, steering angles, sample starts, grid
and geometry once and returns them normalized to what the C ABI consumes
(float32 vectors, float32 scan coordinates, the four scalar constants).  The
frame-batched functions (``rcabeam_b200.ensemble``) and the resident
``OpwWorkspace`` both go through it, so they accept and reject the same inputs.

Errors are ``ValueError`` with messages that keep the substrings the
reference's tests match on ("nonempty", "F-number", "IQ storage", "OPW only",
"complex signal", "St-SW requires"; reference tests/test_ensemble.py:80-82,
tests/test_gpu_workspace.py:53-90).
"""

from __future__ import annotations

from dataclasses import dataclass
from operator import index

import numpy as np

from rcabeam_b200.sim import RCAGeometry, scan_coords

# Method name -> C ABI method code (reference ensemble.py:15; "apertures" is method 5).
METHOD_CODES = {"opw": 0, "xdoppler": 1, "rc_fmas": 2, "dmas": 3, "st_sw": 4, "apertures": 5}
# Packed IQ storages and the methods that may use them.
STORAGE_METHODS = {"float32": tuple(METHOD_CODES), "float16": ("opw",), "bf16x2": ("opw",)}


@dataclass(frozen=True)
class Acquisition:
    """Validated acquisition metadata in the C ABI's types."""

    channel_shape: tuple[int, int, int, int]  # (samples, channels, angles, frames)
    grid_shape: tuple[int, int, int]          # (nx, nz, ny)
    scan: np.ndarray                          # (nv, 3) float32 (x, z, y)
    x_el: np.ndarray                          # float32 vectors
    y_el: np.ndarray
    angles: np.ndarray
    starts: np.ndarray
    constants: tuple[float, float, float, float]  # c, fs, f_demod, f-number (-1 = full aperture)

    @property
    def voxels(self) -> int:
        return len(self.scan)


def _shape_of(channel_shape) -> tuple[int, int, int, int]:
    try:
        dims = tuple(index(n) for n in channel_shape)
    except TypeError:
        dims = ()
    if len(dims) != 4 or min(dims) < 1 or dims[0] < 2:
        raise ValueError("Channel data must be nonempty (samples, channels, angles, frames) with at least 2 samples")
    return dims  # type: ignore[return-value]


def channel_pair_shape(rc: np.ndarray, cr: np.ndarray) -> tuple[int, int, int, int]:
    """Shape shared by the RC and CR channel arrays."""
    if rc.shape != cr.shape:
        raise ValueError("RC and CR must be nonempty arrays of one (samples, channels, angles, frames) shape")
    return _shape_of(rc.shape)


def acquisition(channel_shape, angles, t_start, grid, geom: RCAGeometry) -> Acquisition:
    """Validate and normalize one acquisition (raises ``ValueError``)."""
    ns, nc, na, nt = _shape_of(channel_shape)
    vectors = {"angles": angles, "x_el": geom.x_el, "y_el": geom.y_el}
    if any(np.ndim(v) != 1 for v in vectors.values()):
        raise ValueError("Geometry must hold one-dimensional element and angle vectors")
    counts = (len(angles), len(geom.x_el), len(geom.y_el))
    if counts != (na, nc, nc):
        raise ValueError(f"Geometry must match the channel/angle dimensions: got {counts[0]} angles and "
                         f"{counts[1]} / {counts[2]} elements for {na} angles and {nc} channels")
    if len(grid) != 3 or any(np.ndim(a) != 1 or len(a) == 0 or not np.isfinite(a).all() for a in grid):
        raise ValueError("Grid must be three nonempty finite (x, z, y) coordinate vectors")
    speed, rate, demod = (float(v) for v in (geom.c, geom.fs, geom.f_demod))
    if not (np.isfinite(demod) and np.isfinite(speed) and np.isfinite(rate) and speed > 0 and rate > 0):
        raise ValueError("Sound speed and sampling frequency must be finite and positive (finite f_demod)")
    fnumber = geom.fnumber
    if fnumber is not None and not (np.isfinite(fnumber) and fnumber > 0):
        raise ValueError("F-number must be positive or None")
    as32 = {name: np.ascontiguousarray(v, dtype=np.float32) for name, v in vectors.items()}
    starts = np.ascontiguousarray(np.broadcast_to(np.asarray(t_start, dtype=np.float32), (na,)))
    if not all(np.isfinite(v).all() for v in (*as32.values(), starts)):
        raise ValueError("Element positions, angles and sample starts must be finite")
    scan = scan_coords(grid)
    if not np.isfinite(scan).all():
        raise ValueError("Grid must be three nonempty finite (x, z, y) coordinate vectors")
    constants = (speed, rate, demod, -1.0 if fnumber is None else float(fnumber))
    return Acquisition((ns, nc, na, nt), tuple(len(a) for a in grid), scan, as32["x_el"], as32["y_el"],
                       as32["angles"], starts, constants)  # type: ignore[arg-type]


def method_code(method, storage: str, *, wants_signal: bool) -> int:
    """C ABI code of a reconstruction method, checked against the storage and output asked for."""
    code = METHOD_CODES.get(method)
    if code is None or (method == "apertures" and not wants_signal):
        raise ValueError(f"Unknown method: {method}")
    if method not in STORAGE_METHODS.get(storage, ()):
        raise ValueError("IQ storage must be float32, or float16 / bf16x2 for OPW only")
    return code


def check_subsets(method, k: int, angles: int) -> None:
    """St-SW angle subsets: 2 <= k <= 4 and at least k angles (reference ensemble.py:80-81)."""
    if method == "st_sw" and not (2 <= k <= 4 and angles >= k):
        raise ValueError("St-SW requires 2 <= k <= 4 and at least k angles")
