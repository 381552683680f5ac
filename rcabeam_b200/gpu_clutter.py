"""Resident GPU global temporal clutter filtering (reference src/rcabeam/gpu_clutter.py).

Same functions, arguments and failure policy as the reference CuPy module, on
``torch.Tensor`` CUDA arrays: a scaled Gram matrix accumulated in row tiles,
a float64 Hermitian eigendecomposition on the GPU, the smaller of the
retained / discarded projectors, and float64 power accumulation.  No silent
precision fallback.

Precision of the Gram matrix (``precision=``):

* ``"complex128"`` (default): float64 CUDA-core accumulation, as the reference;
* ``"complex64"``: float32 CUDA-core accumulation (the reference's complex64 mode);
* ``"tf32"`` / ``"bf16x3"``: tensor-core (tcgen05) Gram in TF32 or three-term
  split BF16 products with float32 accumulation.

The eigendecomposition and every projection run in float64 whatever the Gram
precision; the returned basis is complex128 except for ``"complex64"``.
"""

from __future__ import annotations

import ctypes
from time import perf_counter

import numpy as np
import torch

from rcabeam_b200 import _lib, sharded

_GRAM_PRECISION = {"complex128": 0, "complex64": 1, "tf32": 2, "bf16x3": 3}
# Machine epsilon of the Gram's products, for the negative-eigenvalue tolerance
# 64 eps T max|lambda| (gpu_clutter.py:171 uses the eigenvalue dtype's eps):
# float64, float32, TF32 (10-bit mantissa) and the 3xBF16 split (whose dropped
# lo x lo term is about 2^-16 of a product).
_GRAM_EPS = {"complex128": 2.0 ** -52, "complex64": 2.0 ** -23, "tf32": 2.0 ** -10, "bf16x3": 2.0 ** -16}


def _inputs(iq, *, check_finite: bool = True) -> tuple[torch.Tensor, ...]:
    """The reference's input checks (gpu_clutter.py:25-40).  Callers whose kernel
    flags non-finite samples itself pass check_finite=False and raise the same
    error from the flag, which saves a separate pass over the input."""
    arrays = iq if isinstance(iq, tuple) else (iq,)
    if not arrays:
        raise ValueError("At least one IQ array is required")
    for a in arrays:
        if not isinstance(a, torch.Tensor) or not a.is_cuda or a.dtype not in (torch.complex64, torch.complex128):
            raise ValueError("IQ must contain complex64 or complex128 CUDA tensors")
        if a.dim() == 0 or a.numel() == 0:
            raise ValueError("IQ must be nonempty with frames on the last axis")
        if a.device.index != torch.cuda.current_device():
            raise ValueError("IQ must be on the current CUDA device")
        if check_finite and not bool(torch.isfinite(torch.view_as_real(a)).all()):
            raise ValueError("IQ must be finite")
    if any(a.shape[-1] != arrays[0].shape[-1] for a in arrays):
        raise ValueError("All IQ arrays must share the frame count")
    return arrays


def _rank_interval(frames: int, rank_start, rank_stop) -> tuple[int, int]:
    stop = frames if rank_stop is None else rank_stop
    for v in (rank_start, stop):
        if isinstance(v, (bool, np.bool_)) or not isinstance(v, (int, np.integer)):
            raise ValueError("Rank bounds must be integers")
    if not 0 <= rank_start <= stop <= frames:
        raise ValueError("Require 0 <= rank_start <= rank_stop <= number of frames")
    return int(rank_start), int(stop)


def _rows(a: torch.Tensor) -> torch.Tensor:
    """Contiguous (rows, T) view of an IQ array."""
    return a.reshape(-1, a.shape[-1]).contiguous()


def _is128(a: torch.Tensor) -> int:
    return int(a.dtype == torch.complex128)


class Gram:
    """Device buffers of one Gram / eigendecomposition of T frames (reusable across ensembles)."""

    def __init__(self, frames: int, device: torch.device):
        self.frames = frames
        self.scale = torch.zeros(1, dtype=torch.float64, device=device)
        self.upper = torch.zeros(frames * frames * 2, dtype=torch.float64, device=device)
        self.matrix = torch.empty(frames * frames * 2, dtype=torch.float64, device=device)
        self.eigenvalues = torch.empty(frames, dtype=torch.float64, device=device)
        self.info = torch.zeros(1, dtype=torch.int32, device=device)
        size = ctypes.c_size_t(0)
        _lib.check(_lib.lib().rcabeam_heevd_workspace_bytes(frames, ctypes.byref(size)), "heevd_workspace")
        self.workspace = torch.empty(max(int(size.value), 16), dtype=torch.uint8, device=device)

    def accumulate(self, arrays, precision: str, group=None) -> int:
        """Scale, then Gram of every array into one shared matrix; returns total rows.

        With a process group the rows are spread over its ranks: the scale is
        the maximum and the Gram the sum over all ranks (rcabeam_b200.sharded).
        """
        prec = _GRAM_PRECISION[precision]
        if prec >= 2 and (any(a.dtype != torch.complex64 for a in arrays) or self.frames % 2 or self.frames > 1024):
            raise ValueError(f"Precision {precision} requires complex64 IQ with an even frame count <= 1024")
        self.scale.zero_()
        self.upper.zero_()
        for a in arrays:
            _lib.call("rcabeam_clutter_scale_device", a.data_ptr(), a.numel(), _is128(a), self.scale.data_ptr())
        sharded.reduce_scale(self.scale, group)
        rows = 0
        for a in arrays:
            m = _rows(a)
            _lib.call("rcabeam_gram_accumulate_device", m.data_ptr(), m.shape[0], self.frames, _is128(m),
                      self.scale.data_ptr(), prec, self.upper.data_ptr())
            rows += m.shape[0]
        rows = sharded.reduce_gram(self.upper, rows, group)
        _lib.call("rcabeam_gram_finish_device", self.upper.data_ptr(), self.matrix.data_ptr(), self.frames, rows)
        return rows

    def decompose(self) -> None:
        """Float64 eigendecomposition in place: ascending eigenvalues, column eigenvectors."""
        _lib.call("rcabeam_heevd_device", self.matrix.data_ptr(), self.eigenvalues.data_ptr(), self.frames,
                  self.workspace.data_ptr(), self.workspace.numel(), self.info.data_ptr())

    def vectors(self) -> torch.Tensor:
        """Eigenvectors as a (T, T) complex128 tensor with column k = k-th eigenvector (ascending)."""
        t = self.frames
        # The solver writes column-major: row-major (T, T) storage holds V^T.
        return torch.view_as_complex(self.matrix.view(t, t, 2)).transpose(0, 1)


def temporal_basis(iq, *, method: str = "gram", precision: str = "complex128", timings: dict | None = None,
                   diagnostics: dict | None = None, group=None) -> tuple[torch.Tensor, torch.Tensor]:
    """Descending singular values (T,) and column temporal vectors V (T, T) (gpu_clutter.py:112-193).

    A tuple of arrays estimates one shared basis over all of their rows; with a
    torch.distributed process group, over the rows of every rank of the group.
    """
    # Without a group the Casorati scale pass certifies finite input (a non-finite
    # component gives a non-finite scale), so the input is read once less.
    arrays = _inputs(iq, check_finite=group is not None)
    frames = arrays[0].shape[-1]
    if precision not in _GRAM_PRECISION:
        raise ValueError("Precision must be complex64, complex128, tf32 or bf16x3")
    if method != "gram":
        raise ValueError("Method must be 'gram'")
    begin = perf_counter()
    gram = Gram(frames, arrays[0].device)
    rows = gram.accumulate(arrays, precision, group)
    if not np.isfinite(float(gram.scale.item())):
        raise ValueError("IQ must be finite")
    matrix = torch.view_as_real(gram.vectors())
    if not bool(torch.isfinite(matrix).all()):
        raise np.linalg.LinAlgError("Nonfinite Gram matrix; rescale the IQ input")
    if timings is not None:
        torch.cuda.synchronize()
        timings["matrix_seconds"] = perf_counter() - begin
    begin = perf_counter()
    gram.decompose()
    info = int(gram.info.item())
    if timings is not None:
        timings["decomposition_seconds"] = perf_counter() - begin
    if info != 0:
        raise np.linalg.LinAlgError(f"cuSOLVER eigendecomposition failed (info={info})")
    lam = gram.eigenvalues
    eps = _GRAM_EPS[precision]
    tolerance = float(64 * eps * frames * lam.abs().max().item())
    minimum = float(lam[0].item())
    scale = float(gram.scale.item())
    if diagnostics is not None:
        diagnostics.update(precision=precision, input_scale=scale, gram_rows=rows, minimum_eigenvalue=minimum,
                           negative_eigenvalues=int((lam < 0).sum().item()), negative_tolerance=tolerance)
    if minimum < -tolerance:
        raise np.linalg.LinAlgError(
            f"Gram matrix has significantly negative eigenvalues (minimum={minimum:.6g}, tolerance={tolerance:.6g})"
        )
    values = torch.sqrt(torch.clamp(lam.flip(0), min=0)) * (scale or 1.0) * np.sqrt(rows)
    basis = gram.vectors().flip(1).contiguous()
    if precision == "complex64":
        basis = basis.to(torch.complex64)
    if not bool(torch.isfinite(values).all()) or not bool(torch.isfinite(torch.view_as_real(basis)).all()):
        raise np.linalg.LinAlgError("Nonfinite temporal decomposition")
    return values, basis


def _filter_vectors(basis, frames: int, start: int, stop: int) -> tuple[torch.Tensor, bool]:
    """Validated column-major (T x k) complex128 vectors of the smaller projector (gpu_clutter.py:196-209)."""
    if not isinstance(basis, torch.Tensor) or not basis.is_cuda or basis.dtype not in (torch.complex64,
                                                                                         torch.complex128):
        raise ValueError("Basis must be a complex CUDA tensor")
    if basis.device.index != torch.cuda.current_device() or tuple(basis.shape) != (frames, frames):
        raise ValueError("Basis must have shape (frames, frames) on the current device")
    checked = basis.to(torch.complex128)
    eps = 2.0**-52 if basis.dtype == torch.complex128 else 2.0**-23
    tol = max(1e-12, 32 * eps)
    eye = torch.eye(frames, dtype=torch.complex128, device=basis.device)
    if not bool(torch.isfinite(torch.view_as_real(checked)).all()) or not bool(
            torch.allclose(checked.conj().T @ checked, eye, rtol=tol, atol=tol)):
        raise ValueError("Basis must be finite and orthonormal")
    subtract = stop - start > frames - (stop - start)
    vectors = torch.cat((checked[:, :start], checked[:, stop:]), dim=1) if subtract else checked[:, start:stop]
    return vectors.transpose(0, 1).contiguous(), subtract


def _project(matrix: torch.Tensor, vectors_cm: torch.Tensor, k: int, mode: int, out: torch.Tensor | None,
             power: torch.Tensor | None, flags: torch.Tensor | None = None) -> None:
    _lib.call("rcabeam_project_device", matrix.data_ptr(), None if out is None else out.data_ptr(),
              None if power is None else power.data_ptr(), matrix.shape[0], matrix.shape[1], _is128(matrix),
              vectors_cm.data_ptr() if k else None, k, mode, None if flags is None else flags.data_ptr())


def apply_temporal_filter(iq, basis, *, rank_start: int, rank_stop: int | None = None):
    """Filtered IQ keeping ranks [start, stop) via the smaller projector (gpu_clutter.py:219-241)."""
    arrays = _inputs(iq)
    frames = arrays[0].shape[-1]
    start, stop = _rank_interval(frames, rank_start, rank_stop)
    vectors, subtract = _filter_vectors(basis, frames, start, stop)
    k = vectors.shape[0]
    result = []
    for a in arrays:
        m = _rows(a)
        out = torch.empty_like(m)
        _project(m, vectors, k, (1 if subtract else 0) | 2, out, None)
        if not bool(torch.isfinite(torch.view_as_real(out)).all()):
            raise np.linalg.LinAlgError("Nonfinite filtered IQ; rescale the input")
        result.append(out.reshape(a.shape))
    return tuple(result) if isinstance(iq, tuple) else result[0]


def filtered_power(iq, basis, *, rank_start: int, rank_stop: int | None = None) -> torch.Tensor:
    """Float64 filtered power without materializing filtered IQ (gpu_clutter.py:244-273)."""
    if not isinstance(iq, torch.Tensor):
        raise ValueError("Power requires one coherent beamformed IQ array")
    arrays = _inputs(iq, check_finite=False)  # the projection flags non-finite samples
    frames = arrays[0].shape[-1]
    start, stop = _rank_interval(frames, rank_start, rank_stop)
    vectors, subtract = _filter_vectors(basis, frames, start, stop)
    if start == stop:
        _inputs(iq)
        return torch.zeros(iq.shape[:-1], dtype=torch.float64, device=iq.device)
    m = _rows(iq)
    power = torch.empty(m.shape[0], dtype=torch.float64, device=iq.device)
    flags = torch.zeros(1, dtype=torch.int32, device=iq.device)
    _project(m, vectors, vectors.shape[0], 1 if subtract else 0, None, power, flags)
    bits = int(flags.item())
    if bits & 1:
        raise ValueError("IQ must be finite")
    if bits & 2:
        raise np.linalg.LinAlgError("Nonfinite filtered power; rescale the input")
    return power.reshape(iq.shape[:-1])


def svd_clutter_filter(iq, *, rank_start: int, rank_stop: int | None = None, method: str = "gram",
                       precision: str = "complex128"):
    """Gram-EVD temporal filter keeping ranks [start, stop); no silent precision fallback (gpu_clutter.py:322-336)."""
    arrays = _inputs(iq)
    _rank_interval(arrays[0].shape[-1], rank_start, rank_stop)
    _, basis = temporal_basis(iq, method=method, precision=precision)
    return apply_temporal_filter(iq, basis, rank_start=rank_start, rank_stop=rank_stop)


def power_doppler(signal):
    """Mean |x|^2 over the last (frame) axis, float64 accumulation (reference src/rcabeam/power.py:8-21).

    CUDA tensors are reduced in place; NumPy arrays are uploaded, reduced on the
    GPU and returned as NumPy.
    """
    host = not isinstance(signal, torch.Tensor)
    x = torch.from_numpy(np.ascontiguousarray(signal)).cuda() if host else signal
    if x.dtype not in (torch.complex64, torch.complex128):
        x = x.to(torch.complex128)
    m = _rows(x)
    power = torch.empty(m.shape[0], dtype=torch.float64, device=x.device)
    _project(m, m.new_zeros(0), 0, 1, None, power)
    power = power.reshape(x.shape[:-1])
    return power.cpu().numpy() if host else power
