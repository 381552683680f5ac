"""Complex128 restatement of the global temporal SVD clutter filter (TEST INFRASTRUCTURE).

Follows src/rcabeam/clutter.py:

* rows = all axes but the last, frames last (clutter.py:10-15);
* ``svd``: direct complex128 SVD, singular values padded to T (clutter.py:20-26);
* ``gram``: X^H X accumulated over 16384-row chunks in complex128, Hermitian
  EVD, negative eigenvalues beyond 64 eps T max|lambda| rejected, order reversed
  to descending (clutter.py:27-39);
* the filter keeps the zero-based rank interval [start, stop) (clutter.py:65-109).
"""

from __future__ import annotations

import numpy as np


def _matrix(iq: np.ndarray) -> np.ndarray:
    iq = np.asarray(iq)
    if iq.dtype not in (np.complex64, np.complex128):
        raise ValueError("IQ must be a complex64 or complex128 NumPy array")
    if iq.ndim == 0 or iq.size == 0 or not np.isfinite(iq).all():
        raise ValueError("IQ must be nonempty and finite, with frames on the last axis")
    return iq.reshape(-1, iq.shape[-1])


def gram(matrix: np.ndarray, chunk: int = 16384) -> np.ndarray:
    """Complex128 X^H X summed over row chunks."""
    frames = matrix.shape[-1]
    g = np.zeros((frames, frames), dtype=np.complex128)
    for first in range(0, len(matrix), chunk):
        block = matrix[first : first + chunk].astype(np.complex128)
        g += block.conj().T @ block
    return g


def temporal_basis(iq: np.ndarray, *, method: str = "svd") -> tuple[np.ndarray, np.ndarray]:
    """Descending singular values (T,) and column temporal vectors V (T, T)."""
    matrix = _matrix(iq)
    frames = matrix.shape[-1]
    if method == "svd":
        _, values, vh = np.linalg.svd(matrix.astype(np.complex128), full_matrices=matrix.shape[0] < frames)
        values = np.pad(values, (0, frames - len(values)))
        basis = vh.conj().T
    elif method == "gram":
        g = gram(matrix)
        if not np.isfinite(g).all():
            raise np.linalg.LinAlgError("Nonfinite Gram matrix; rescale the IQ input")
        lam, vec = np.linalg.eigh(g)
        tolerance = 64 * np.finfo(np.float64).eps * frames * np.max(np.abs(lam))
        if np.any(lam < -tolerance):
            raise np.linalg.LinAlgError("Gram matrix has significantly negative eigenvalues")
        values = np.sqrt(np.maximum(lam[::-1], 0))
        basis = vec[:, ::-1]
    else:
        raise ValueError("Method must be 'svd' or 'gram'")
    return values, basis


def rank_interval(frames: int, rank_start, rank_stop) -> tuple[int, int]:
    stop = frames if rank_stop is None else rank_stop
    for v in (rank_start, stop):
        if isinstance(v, (bool, np.bool_)) or not isinstance(v, (int, np.integer)):
            raise ValueError("Rank bounds must be integers")
    if not 0 <= rank_start <= stop <= frames:
        raise ValueError("Require 0 <= rank_start <= rank_stop <= number of frames")
    return int(rank_start), int(stop)


def svd_clutter_filter(iq: np.ndarray, *, rank_start: int, rank_stop: int | None = None, method: str = "svd") -> np.ndarray:
    """Retain ranks [start, stop); complex128 result (not cast back)."""
    matrix = _matrix(iq)
    frames = matrix.shape[-1]
    start, stop = rank_interval(frames, rank_start, rank_stop)
    if method == "svd":
        u, values, vh = np.linalg.svd(matrix.astype(np.complex128), full_matrices=False)
        values = values.copy()
        values[:start] = 0
        values[stop:] = 0
        out = (u * values) @ vh
    else:
        _, basis = temporal_basis(matrix, method=method)
        kept = basis[:, start:stop]
        out = (matrix.astype(np.complex128) @ kept) @ kept.conj().T
    return out.reshape(np.asarray(iq).shape)


def filtered_power(iq: np.ndarray, basis: np.ndarray, rank_start: int, rank_stop: int | None = None) -> np.ndarray:
    """Power Doppler of the filtered IQ, denominator = original frame count."""
    matrix = _matrix(iq).astype(np.complex128)
    frames = matrix.shape[-1]
    start, stop = rank_interval(frames, rank_start, rank_stop)
    kept = basis[:, start:stop]
    coords = matrix @ kept
    power = np.sum(coords.real**2 + coords.imag**2, axis=-1) / frames
    return power.reshape(np.asarray(iq).shape[:-1])
