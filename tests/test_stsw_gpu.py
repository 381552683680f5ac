"""GPU parity of St-SW (method 4) against the float64 oracle.

The oracle restates the reference's st_sw_weights / st_sw_pd (stsw.py:10-107)
and is pinned to the reference's own outputs in tests/test_oracle.py.  Cases
follow the reference's tests: the small random ensemble of
tests/test_ensemble.py:17-69 (frames 1 to 300, both apertures, k = 2, 3, 4)
and the 4097-voxel line of tests/test_ensemble_targets.py:46-65 with a silent
RC angle (zero-energy correlation series).  Bar: relative L2 <= 1e-4 and
elementwise |err| <= 2e-4 * max|ref| on the peak-normalized St-SW power (the
reference's own test tolerance is 1e-3).
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

import rcabeam_b200 as rb
from oracle import methods
from rcabeam_b200 import _cuda_impl, _lib
from rcabeam_b200.sim import RCAGeometry
from tests._cases import oracle_inputs, random_case, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-4


@pytest.fixture(autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs CUDA")
    yield
    assert _lib.device_error() == 0


def _oracle(rc, cr, angles, starts, grid, geom, k):
    o = oracle_inputs(angles, starts, grid, geom)
    return methods.st_sw_power(rc, cr, o["scan"], o["xe"], o["ye"], o["angles"], o["starts"], o["c"], o["fs"],
                               o["fd"], o["fnumber"], k)


def _check(actual, expected):
    expected = np.asarray(expected).reshape(np.shape(actual))
    assert rel_l2(actual, expected) <= TOL
    np.testing.assert_allclose(actual, expected, rtol=0, atol=2 * TOL * max(np.abs(expected).max(), 1e-30))


@pytest.mark.parametrize("frames", [1, 33, 200, 300])
@pytest.mark.parametrize("fnumber", [None, 1.0])
@pytest.mark.parametrize("k", [2, 3, 4])
def test_st_sw_matches_oracle(frames, fnumber, k):
    grid = (np.array([0.0, 0.008]), np.array([0.001, 0.007, 0.03]), np.array([0.0]))
    rc, cr, angles, starts, grid, geom = random_case(44, 16, 2, 4, frames, grid, fnumber=fnumber)
    actual = rb.ensemble_pd_from_channels(rc, cr, angles, starts, grid, geom, method="st_sw", k=k)
    _check(actual, _oracle(rc, cr, angles, starts, grid, geom, k))


@pytest.mark.parametrize("k", [2, 3, 4])
def test_st_sw_line_silent_angle_and_tiles(k, monkeypatch):
    """4097 voxels, RC angle 0 silent; the scratch tile loop must not change the
    full-volume peak normalization (reference test_ensemble_targets.py:46-65)."""
    geom = RCAGeometry(x_el=np.array([-0.001, 0.001]), y_el=np.array([-0.001, 0.001]), fs=1e6, f_demod=0.1e6)
    grid = (np.zeros(1), np.array([0.007]), np.linspace(-0.001, 0.001, 4097))
    angles = np.array([-0.08, -0.02, 0.05, 0.09])
    rng = np.random.default_rng(42)
    rc = (rng.normal(size=(16, 2, 4, 3)) + 1j * rng.normal(size=(16, 2, 4, 3))).astype(np.complex64)
    cr = (rng.normal(size=rc.shape) + 1j * rng.normal(size=rc.shape)).astype(np.complex64)
    rc[:, :, 0] = 0
    expected = _oracle(rc, cr, angles, 1e-6, grid, geom, k)
    whole = rb.ensemble_pd_from_channels(rc, cr, angles, 1e-6, grid, geom, method="st_sw", k=k)
    _check(whole, expected)
    # Scratch for 1000 voxels at a time: five tiles, the last one ragged.
    monkeypatch.setattr(_cuda_impl, "_STSW_SCRATCH_BYTES", 1000 * k * k * 3 * 8)
    tiled = rb.ensemble_pd_from_channels(rc, cr, angles, 1e-6, grid, geom, method="st_sw", k=k)
    np.testing.assert_array_equal(tiled, whole)


def test_st_sw_zero_input_and_arguments():
    grid = (np.array([0.0, 0.008]), np.array([0.001, 0.007, 0.03]), np.array([0.0]))
    rc, cr, angles, starts, grid, geom = random_case(44, 16, 2, 4, 8, grid)
    zeros = np.zeros_like(rc)
    for k in (2, 3, 4):
        assert not rb.ensemble_pd_from_channels(zeros, zeros, angles, starts, grid, geom, method="st_sw", k=k).any()
    for k in (1, 5):
        with pytest.raises(ValueError, match="St-SW"):
            rb.ensemble_pd_from_channels(rc, cr, angles, starts, grid, geom, method="st_sw", k=k)
    with pytest.raises(ValueError, match="St-SW"):
        rb.ensemble_pd_from_channels(rc[:, :, :3], cr[:, :, :3], angles[:3], starts[:3], grid, geom, method="st_sw",
                                     k=4)
