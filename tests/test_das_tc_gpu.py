"""Tensor-core (tcgen05) OPW against the float64 oracle.

FP16 storage: the FP16-quantized channels are the exact operand; the bar is
relative L2 <= 5e-5 against the oracle on quantized inputs.  bf16x2 storage:
three split products; bar relative L2 <= 5e-5 against the oracle on the raw
float32 channels (the target for filtered power is 1e-4).
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

import rcabeam_b200 as rb
from oracle import das
from rcabeam_b200 import _lib
from rcabeam_b200.sim import RCAGeometry, simulate_point
from tests._cases import oracle_inputs, random_case, rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs CUDA")
    yield
    assert _lib.device_error() == 0


def _oracle(rc, cr, angles, starts, grid, geom):
    o = oracle_inputs(angles, starts, grid, geom)
    return das.opw_iq(rc, cr, o["scan"], o["xe"], o["ye"], o["angles"], o["starts"], o["c"], o["fs"], o["fd"],
                      o["fnumber"])


def _quant(z):
    return (z.real.astype(np.float16).astype(np.float32) + 1j * z.imag.astype(np.float16).astype(np.float32)
            ).astype(np.complex64)


@pytest.mark.parametrize("storage", ["float16", "bf16x2"])
@pytest.mark.parametrize("frames", [4, 8, 136, 200, 256, 300])
@pytest.mark.parametrize("fnumber", [None, 1.0])
def test_tc_small_random(storage, frames, fnumber):
    grid = (np.array([0.0, 0.008]), np.array([0.001, 0.007, 0.03]), np.array([0.0]))
    rc, cr, angles, starts, grid, geom = random_case(44, 16, 2, 4, frames, grid, fnumber=fnumber)
    ref_in = (_quant(rc), _quant(cr)) if storage == "float16" else (rc, cr)
    expected = _oracle(*ref_in, angles, starts, grid, geom).reshape(2, 3, 1, frames)
    actual = rb.beamform_ensemble(rc, cr, angles, starts, grid, geom, iq_storage=storage)
    tol = 5e-5
    assert rel_l2(actual, expected) <= tol
    pd = rb.ensemble_pd_from_channels(rc, cr, angles, starts, grid, geom, iq_storage=storage)
    assert rel_l2(pd, das.power_doppler(expected)) <= 2 * tol


@pytest.mark.parametrize("storage", ["float16", "bf16x2"])
@pytest.mark.parametrize("fnumber", [None, 1.0])
def test_tc_physical_volume(storage, fnumber):
    """3-D 15 MHz volume, many 64-voxel tiles and 16-row windows (sub-window splits included)."""
    el = (np.arange(64) - 31.5) * 0.2e-3
    geom = RCAGeometry(el, el, c=1540.0, fs=20e6, f_demod=15e6, fnumber=fnumber)
    angles = np.deg2rad(np.linspace(-8, 8, 5))
    t0 = 2 * 3e-3 / 1540.0 - 0.5e-6
    rng = np.random.default_rng(3)
    frames = 8
    chans = []
    for config in ("RC", "CR"):
        data = sum(a * simulate_point(geom, angles, p, 256, t0, config)
                   for p, a in [((0.0, 5e-3, 0.0), 1.0), ((-1.2e-3, 4.2e-3, 0.8e-3), 0.7)])
        noise = 0.05 * (rng.normal(size=(256, 64, 5, frames)) + 1j * rng.normal(size=(256, 64, 5, frames)))
        chans.append((data[..., None] * np.exp(2j * np.pi * rng.random(frames)) + noise).astype(np.complex64))
    grid = (np.linspace(-3.2e-3, 3.2e-3, 12), np.linspace(3e-3, 7e-3, 24), np.linspace(-3.2e-3, 3.2e-3, 10))
    ref_in = [_quant(c) for c in chans] if storage == "float16" else chans
    expected = _oracle(*ref_in, angles, t0, grid, geom).reshape(12, 24, 10, frames)
    actual = rb.beamform_ensemble(chans[0], chans[1], angles, t0, grid, geom, iq_storage=storage)
    assert rel_l2(actual, expected) <= 5e-5


def test_tc_long_line_and_empty_tiles():
    """16385 voxels on a line; most tiles see no sample (window outside the record) -> exact zeros."""
    el = np.array([-0.05e-3, 0.05e-3])
    geom = RCAGeometry(x_el=el, y_el=el, fs=20e6, f_demod=15e6, fnumber=1)
    grid = (np.zeros(1), np.array([8e-3]), np.linspace(-1e-3, 1e-3, 16385))
    angles = np.array([-0.08, -0.02, 0.05, 0.09])
    rng = np.random.default_rng(7)
    rc = (rng.normal(size=(368, 2, 4, 4)) + 1j * rng.normal(size=(368, 2, 4, 4))).astype(np.complex64)
    cr = (rng.normal(size=rc.shape) + 1j * rng.normal(size=rc.shape)).astype(np.complex64)
    expected = _oracle(rc, cr, angles, 2e-6, grid, geom).reshape(1, 1, 16385, 4)
    actual = rb.beamform_ensemble(rc, cr, angles, 2e-6, grid, geom, iq_storage="bf16x2")
    assert rel_l2(actual, expected) <= 5e-5
    # Voxels with no valid tap are exact zeros in both.
    dead = np.all(expected == 0, axis=-1)
    assert np.all(actual[dead] == 0)


@pytest.mark.parametrize("storage", ["float16", "bf16x2"])
@pytest.mark.parametrize("angles", [15, 24])
def test_tc_many_angles_shallow_ring(storage, angles):
    """200 frames with 15 angles still fits the five-stage ring (five builders); with 24 angles the
    per-tile transmit tables leave room for a three-stage ring (three builders)."""
    grid = (np.linspace(-1e-3, 1e-3, 6), np.linspace(3e-3, 6e-3, 7), np.linspace(-1e-3, 1e-3, 5))
    rc, cr, _, starts, grid, geom = random_case(31, 96, 8, angles, 200, grid, fnumber=None, fs=20e6, fd=15e6,
                                                starts=np.full(angles, 2e-6))
    ang = np.deg2rad(np.linspace(-10, 10, angles))
    ref_in = (_quant(rc), _quant(cr)) if storage == "float16" else (rc, cr)
    expected = _oracle(*ref_in, ang, starts, grid, geom).reshape(6, 7, 5, 200)
    actual = rb.beamform_ensemble(rc, cr, ang, starts, grid, geom, iq_storage=storage)
    assert rel_l2(actual, expected) <= 5e-5
