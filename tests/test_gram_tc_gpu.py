"""Tensor-core (tcgen05) Gram in TF32 and 3xBF16 against float64.

The Gram of a complex64 Casorati matrix is formed as the real symmetric
product of its (rows, 2T) float32 view.  Bars (relative Frobenius error of the
finished Gram against float64, tolerances in the tests):
  * TF32 (10-bit mantissa operands, round to nearest): <= 1e-3;
  * 3xBF16 (hi/lo split, three products): <= 3e-5;
both with float32 accumulation flushed to float64 every 2048 rows.
Shapes cover frame counts that are not multiples of 64 (ragged last block),
row counts that are not multiples of 16 (ragged last stage), more than one
flush per CTA, and data scaled far from 1 (the power-of-two prescale).
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from oracle import clutter as oc
from rcabeam_b200 import _lib, gpu_clutter, scenes

pytestmark = pytest.mark.gpu

TOL = {"tf32": 1e-3, "bf16x3": 3e-5}


@pytest.fixture(autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs CUDA")
    yield
    assert _lib.device_error() == 0


def _gram(iq: torch.Tensor, precision: str) -> np.ndarray:
    g = gpu_clutter.Gram(iq.shape[-1], iq.device)
    rows = g.accumulate((iq,), precision)
    torch.cuda.synchronize()
    t = iq.shape[-1]
    m = torch.view_as_complex(g.matrix.view(t, t, 2)).transpose(0, 1).cpu().numpy()  # column-major storage
    return m, rows


def _reference(host: np.ndarray) -> np.ndarray:
    x = host.astype(np.complex128)
    s = max(np.abs(x.real).max(), np.abs(x.imag).max())
    xs = x / s if s > 0 else x
    return (xs.conj().T @ xs) / x.shape[0]


def _fro(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("precision", ["tf32", "bf16x3"])
@pytest.mark.parametrize("rows,frames", [(1, 2), (37, 16), (1000, 64), (5003, 66), (40000, 200), (2048, 400),
                                         (777, 1024),
                                         # every unit shape of the block planner: 3, 5, 6, 8, 10, 13 blocks
                                         (300, 130), (300, 320), (300, 384), (300, 512), (200, 600), (200, 832)])
def test_gram_matches_float64(precision, rows, frames):
    rng = np.random.default_rng(rows + frames)
    host = (rng.normal(size=(rows, frames)) + 1j * rng.normal(size=(rows, frames))).astype(np.complex64)
    got, total = _gram(torch.from_numpy(host).cuda(), precision)
    assert total == rows
    want = _reference(host)
    np.testing.assert_allclose(got, got.conj().T, rtol=0, atol=1e-15 * np.abs(want).max())
    assert _fro(got, want) <= TOL[precision]


@pytest.mark.parametrize("scale", [1e-30, 3.7e-3, 1.0, 6.5e4, 1e30])
def test_gram_prescale_keeps_products_in_range(scale):
    rng = np.random.default_rng(3)
    host = (rng.normal(size=(3000, 32)) + 1j * rng.normal(size=(3000, 32))).astype(np.complex64)
    scaled = (host * np.float32(scale)).astype(np.complex64)
    want = _reference(scaled)
    for precision in ("tf32", "bf16x3"):
        got, _ = _gram(torch.from_numpy(scaled).cuda(), precision)
        assert np.isfinite(got).all()
        assert _fro(got, want) <= TOL[precision]


def test_zero_matrix_gives_zero_gram():
    iq = torch.zeros((100, 8), dtype=torch.complex64, device="cuda")
    for precision in ("tf32", "bf16x3"):
        got, _ = _gram(iq, precision)
        assert not np.any(got)


def test_tensor_core_precisions_reject_unsupported_inputs():
    g = gpu_clutter.Gram(7, torch.device("cuda"))
    with pytest.raises(ValueError, match="Precision"):
        g.accumulate((torch.zeros((4, 7), dtype=torch.complex64, device="cuda"),), "tf32")
    g = gpu_clutter.Gram(8, torch.device("cuda"))
    with pytest.raises(ValueError, match="Precision"):
        g.accumulate((torch.zeros((4, 8), dtype=torch.complex128, device="cuda"),), "bf16x3")


@pytest.mark.parametrize("frames", [64, 200])
def test_filtered_power_of_clutter_scene_against_float64_oracle(frames):
    """Rank-3 tissue (0/-6/-12 dB) + blood -40 dB + noise -50 dB: filtered power vs the complex128 oracle.

    The filtered power keeps about 1e-5 of the energy, so an eigenvector error
    d of the removed tissue subspace shows up to first order as ~2 d sqrt(1e5):
    bars 2e-5 (3xBF16) and 5e-4 (TF32) at 20000 rows (errors shrink with the
    square root of the row count)."""
    gen = torch.Generator(device="cuda").manual_seed(5)
    iq = scenes.clutter_casorati(20000, frames, generator=gen, device="cuda")
    host = iq.cpu().numpy()
    _, basis = oc.temporal_basis(host, method="gram")
    expected = oc.filtered_power(host, basis, 3)
    errors = {}
    for precision in ("complex128", "complex64", "tf32", "bf16x3"):
        _, basis_gpu = gpu_clutter.temporal_basis(iq, precision=precision)
        got = gpu_clutter.filtered_power(iq, basis_gpu, rank_start=3).cpu().numpy()
        errors[precision] = float(np.linalg.norm(got - expected) / np.linalg.norm(expected))
    print(f"\nfiltered power rel. L2 vs float64 oracle, {frames} frames: {errors}")
    assert errors["complex128"] <= 1e-8
    assert errors["bf16x3"] <= 2e-5
    assert errors["tf32"] <= 5e-4
