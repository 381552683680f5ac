"""GPU parity of the frame-batched reconstruction against the float64 oracle.

Every case runs the CUDA path through the public API / C ABI and the oracle on
the float32-quantized geometry the C ABI receives.  Bar: relative L2 <= 1e-5
and elementwise |err| <= 2e-5 * max|ref| for IQ; the same on power.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

import rcabeam_b200 as rb
from oracle import das, methods
from rcabeam_b200 import _lib
from rcabeam_b200.sim import RCAGeometry, scan_coords, simulate_point
from tests._cases import oracle_inputs, random_case, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _oracle_apertures(rc, cr, angles, starts, grid, geom):
    o = oracle_inputs(angles, starts, grid, geom)
    return das.apertures_iq(rc, cr, o["scan"], o["xe"], o["ye"], o["angles"], o["starts"], o["c"], o["fs"], o["fd"],
                            o["fnumber"])


def _check(actual, expected, tol=TOL):
    expected = np.asarray(expected)
    assert rel_l2(actual, expected) <= tol
    scale = max(np.abs(expected).max(), 1e-30)
    np.testing.assert_allclose(actual, expected, rtol=0, atol=2 * tol * scale)


@pytest.fixture(autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs CUDA")
    yield
    assert _lib.device_error() == 0


@pytest.mark.parametrize("frames", [1, 2, 3, 8, 33, 64, 66, 70, 200, 300])
@pytest.mark.parametrize("fnumber", [None, 1.0])
def test_opw_iq_and_power_match_oracle(frames, fnumber):
    """Frame tails, odd frame counts (plain staging) and both aperture modes."""
    grid = (np.array([0.0, 0.008]), np.array([0.001, 0.007, 0.03]), np.array([0.0]))
    rc, cr, angles, starts, grid, geom = random_case(44, 16, 2, 4, frames, grid, fnumber=fnumber)
    r, q = _oracle_apertures(rc, cr, angles, starts, grid, geom)
    expected = (r + q).reshape(2, 3, 1, frames)
    timing = {"raw_upload_seconds": -1.0}
    actual = rb.beamform_ensemble(rc, cr, angles, starts, grid, geom, timings=timing)
    assert actual.dtype == np.complex64 and actual.shape == expected.shape
    assert timing["raw_upload_seconds"] > 0
    _check(actual, expected)
    pd = rb.ensemble_pd_from_channels(rc, cr, angles, starts, grid, geom)
    assert pd.dtype == np.float32
    _check(pd, das.power_doppler(expected))


@pytest.mark.parametrize("frames", [2, 4, 8, 66, 200])
@pytest.mark.parametrize("channels", [1, 17])
def test_channel_tails(frames, channels):
    """Reference tests/test_ensemble_targets.py:177-203 shapes."""
    el = np.array([0.001]) if channels == 1 else np.linspace(-0.006, 0.001, channels)
    grid = (np.zeros(1), np.array([0.007]), np.array([-0.001, 0.0, 0.001]))
    rc, cr, angles, starts, grid, geom = random_case(19, 16, channels, 3, frames, grid, x_el=el, y_el=el,
                                                     starts=np.array([1e-6, 2e-6, 3e-6]))
    r, q = _oracle_apertures(rc, cr, angles, starts, grid, geom)
    expected = (r + q).reshape(1, 1, 3, frames)
    _check(rb.beamform_ensemble(rc, cr, angles, starts, grid, geom), expected)


@pytest.mark.parametrize("frames", [3, 4])
def test_long_line_of_voxels(frames):
    """16385 voxels on one lateral line at 15 MHz (reference test_ensemble_targets.py:151-174)."""
    el = np.array([-0.05e-3, 0.05e-3])
    geom = RCAGeometry(x_el=el, y_el=el, fs=20e6, f_demod=15e6, fnumber=1)
    grid = (np.zeros(1), np.array([8e-3]), np.linspace(-1e-3, 1e-3, 16385))
    angles = np.array([-0.08, -0.02, 0.05, 0.09])
    rng = np.random.default_rng(7)
    rc = (rng.normal(size=(368, 2, 4, frames)) + 1j * rng.normal(size=(368, 2, 4, frames))).astype(np.complex64)
    cr = (rng.normal(size=rc.shape) + 1j * rng.normal(size=rc.shape)).astype(np.complex64)
    r, q = _oracle_apertures(rc, cr, angles, 2e-6, grid, geom)
    expected = (r + q).reshape(1, 1, 16385, frames)
    _check(rb.beamform_ensemble(rc, cr, angles, 2e-6, grid, geom), expected)
    _check(rb.ensemble_pd_from_channels(rc, cr, angles, 2e-6, grid, geom), das.power_doppler(expected))


def _physical_scene(frames, fnumber=1.0, grid_shape=(12, 24, 10)):
    el = (np.arange(64) - 31.5) * 0.2e-3
    geom = RCAGeometry(el, el, c=1540.0, fs=20e6, f_demod=15e6, fnumber=fnumber)
    angles = np.deg2rad(np.linspace(-8, 8, 5))
    t0 = 2 * 3e-3 / 1540.0 - 0.5e-6
    rng = np.random.default_rng(3)
    phases = np.exp(2j * np.pi * rng.random(frames))
    chans = []
    for config in ("RC", "CR"):
        data = sum(a * simulate_point(geom, angles, p, 256, t0, config)
                   for p, a in [((0.0, 5e-3, 0.0), 1.0), ((-1.2e-3, 4.2e-3, 0.8e-3), 0.7), ((1e-3, 6e-3, -6e-4), 0.5)])
        noise = 0.05 * (rng.normal(size=(256, 64, 5, frames)) + 1j * rng.normal(size=(256, 64, 5, frames)))
        chans.append((data[..., None] * phases + noise).astype(np.complex64))
    nx, nz, ny = grid_shape
    grid = (np.linspace(-3.2e-3, 3.2e-3, nx), np.linspace(3e-3, 7e-3, nz), np.linspace(-3.2e-3, 3.2e-3, ny))
    return chans[0], chans[1], angles, t0, grid, geom


@pytest.mark.parametrize("fnumber", [None, 1.0])
def test_physical_volume_with_spatial_tiles(fnumber):
    """3-D 15 MHz volume: many Morton tiles, full and f-number apertures."""
    rc, cr, angles, t0, grid, geom = _physical_scene(8, fnumber)
    r, q = _oracle_apertures(rc, cr, angles, t0, grid, geom)
    expected = (r + q).reshape(12, 24, 10, 8)
    _check(rb.beamform_ensemble(rc, cr, angles, t0, grid, geom), expected)
    _check(rb.ensemble_pd_from_channels(rc, cr, angles, t0, grid, geom), das.power_doppler(expected))


@pytest.mark.parametrize("frames", [1, 3, 8, 66, 200])
def test_fp16_storage_matches_quantized_oracle(frames):
    """FP16 packing: exact against an FP16-quantized oracle; within 4 % of unquantized (test_opw_fp16.py:11-44)."""
    rng = np.random.default_rng(111)
    shape = (48, 3, 4, frames)
    rc = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)
    cr = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)
    el = np.linspace(-0.001, 0.001, 3)
    angles = np.linspace(-0.1, 0.1, 4)
    geom = RCAGeometry(el, el, fs=2e6, f_demod=1e6)
    grid = (np.linspace(-0.001, 0.001, 3), np.array([0.005, 0.007]), np.linspace(-0.001, 0.003, 5))
    for scale in (0.0, 1.0, 1e-4):
        a, b = rc * scale, cr * scale
        quant = lambda z: (z.real.astype(np.float16).astype(np.float32)  # noqa: E731
                           + 1j * z.imag.astype(np.float16).astype(np.float32)).astype(np.complex64)
        r, q = _oracle_apertures(quant(a), quant(b), angles, 1e-6, grid, geom)
        expected = (r + q).reshape(3, 2, 5, frames)
        actual = rb.beamform_ensemble(a, b, angles, 1e-6, grid, geom, iq_storage="float16")
        pd = rb.ensemble_pd_from_channels(a, b, angles, 1e-6, grid, geom, iq_storage="float16")
        if scale == 0:
            assert not actual.any() and not pd.any()
            continue
        _check(actual, expected)
        _check(pd, das.power_doppler(expected))
        original = rb.beamform_ensemble(a, b, angles, 1e-6, grid, geom)
        assert rel_l2(actual, original) < 0.04


def test_fp16_rejects_out_of_range_values():
    data = np.zeros((48, 1, 2, 3), dtype=np.complex64)
    geom = RCAGeometry(np.zeros(1), np.zeros(1), fs=2e6, f_demod=1e6)
    grid = (np.zeros(1), np.array([0.005]), np.zeros(1))
    for value in (70000.0, 70000j, float("inf"), float("nan")):
        bad = data.copy()
        bad[0, 0, 0, 0] = value
        with pytest.raises(ValueError, match="FP16 IQ requires"):
            rb.ensemble_pd_from_channels(bad, data, np.array([0.0, 0.05]), 1e-6, grid, geom, iq_storage="float16")


@pytest.mark.parametrize("frames", [1, 33, 200])
def test_apertures_xdoppler_fmas_dmas(frames):
    """Separate apertures (method 5), XDoppler (1), RC-FMAS (2), DMAS-CCF-ACF (3)."""
    grid = (np.array([0.0, 0.008]), np.array([0.001, 0.007, 0.03]), np.array([0.0]))
    rc, cr, angles, starts, grid, geom = random_case(44, 16, 2, 4, frames, grid, fnumber=1.0)
    r, q = _oracle_apertures(rc, cr, angles, starts, grid, geom)
    ar, aq = rb.beamform_apertures(rc, cr, angles, starts, grid, geom)
    _check(ar, r.reshape(ar.shape))
    _check(aq, q.reshape(aq.shape))
    xd = r * np.conj(q)
    _check(rb.beamform_ensemble(rc, cr, angles, starts, grid, geom, method="xdoppler"), xd.reshape(2, 3, 1, frames))
    _check(rb.ensemble_pd_from_channels(rc, cr, angles, starts, grid, geom, method="xdoppler"),
           methods.xdoppler_power(r, q).reshape(2, 3, 1))
    o = oracle_inputs(angles, starts, grid, geom)
    args = (o["scan"], o["xe"], o["ye"], o["angles"], o["starts"], o["c"], o["fs"], o["fd"], o["fnumber"])
    _, per_r, _ = methods.aperture_terms(rc, o["scan"], o["xe"], o["angles"], o["starts"], o["c"], o["fs"], o["fd"],
                                         o["fnumber"], "RC")
    _, per_q, _ = methods.aperture_terms(cr, o["scan"], o["ye"], o["angles"], o["starts"], o["c"], o["fs"], o["fd"],
                                         o["fnumber"], "CR")
    fmas = methods.signed_sqrt(per_r).sum(axis=1) * methods.signed_sqrt(per_q).sum(axis=1)
    _check(rb.beamform_ensemble(rc, cr, angles, starts, grid, geom, method="rc_fmas"), fmas.reshape(2, 3, 1, frames))
    dmas = methods.dmas_ccf_acf_power(rc, cr, *args)
    np.testing.assert_allclose(rb.ensemble_pd_from_channels(rc, cr, angles, starts, grid, geom, method="dmas"),
                               dmas.reshape(2, 3, 1), rtol=1e-4, atol=1e-4 * np.abs(dmas).max())
    zeros = np.zeros_like(rc)
    for method in ("opw", "xdoppler", "rc_fmas", "dmas"):
        assert not rb.ensemble_pd_from_channels(zeros, zeros, angles, starts, grid, geom, method=method).any()


def test_single_frame_api_closed_receive_window():
    """Reference tests/test_iq_sampling.py:255-266 through rcabeam_delay_rca_channel_data_device."""
    zero = np.zeros(1, np.float32)
    scan = scan_coords((zero, np.array([0, 1.5, 2, 2.25]), zero))
    raw = torch.arange(1, 4, dtype=torch.float32).to(torch.complex64).cuda()
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()  # noqa: E731
    ds, de, dz = d(scan), d(zero), d(zero)
    angle_sum = torch.zeros(4, dtype=torch.complex64, device="cuda")
    ch_sum = torch.zeros(4, dtype=torch.complex64, device="cuda")
    active = torch.zeros(4, dtype=torch.float32, device="cuda")
    _lib.call("rcabeam_delay_rca_channel_data_device", raw.data_ptr(), ds.data_ptr(), de.data_ptr(), dz.data_ptr(),
              dz.data_ptr(), ch_sum.data_ptr(), angle_sum.data_ptr(), active.data_ptr(), 3, 1, 1, 4, 0, 2.0, 1.0,
              0.0, -1.0)
    np.testing.assert_array_equal(angle_sum.cpu().numpy(), [1, 2.5, 3, 0])
    np.testing.assert_array_equal(ch_sum.cpu().numpy(), [1, 2.5, 3, 0])
    np.testing.assert_array_equal(active.cpu().numpy(), [1, 1, 1, 1])


def test_single_frame_api_matches_oracle():
    """Per-frame OPW / XDoppler / RC-FMAS / DMAS power and angle sums (reference core.cu)."""
    grid = (np.array([0.0, 0.008]), np.array([0.001, 0.007, 0.03]), np.array([0.0]))
    rc, cr, angles, starts, grid, geom = random_case(44, 16, 2, 4, 1, grid, fnumber=1.0)
    o = oracle_inputs(angles, starts, grid, geom)
    args = (o["scan"], o["xe"], o["ye"], o["angles"], o["starts"], o["c"], o["fs"], o["fd"], o["fnumber"])
    r, q = _oracle_apertures(rc, cr, angles, starts, grid, geom)
    dev = lambda a, dt=torch.float32: torch.from_numpy(np.ascontiguousarray(a)).to("cuda", dt)  # noqa: E731
    f_rc, f_cr = dev(rc[..., 0], torch.complex64), dev(cr[..., 0], torch.complex64)
    scan = dev(scan_coords(grid))
    xe, ye, an, st = dev(geom.x_el), dev(geom.y_el), dev(angles), dev(np.asarray(starts, np.float32))
    outs = [torch.zeros(6, device="cuda") for _ in range(4)]
    consts = (16, 2, 4, 6, float(geom.c), float(geom.fs), float(geom.f_demod), float(geom.fnumber))
    ptrs = (f_rc.data_ptr(), f_cr.data_ptr(), scan.data_ptr(), xe.data_ptr(), ye.data_ptr(), an.data_ptr(),
            st.data_ptr())
    _lib.call("rcabeam_fast_pd_from_channels_device", *ptrs, outs[0].data_ptr(), outs[1].data_ptr(),
              outs[2].data_ptr(), *consts)
    _lib.call("rcabeam_dmas_ccf_acf_from_channels_device", *ptrs, outs[3].data_ptr(), *consts)
    _check(outs[0].cpu().numpy(), np.abs(r[:, 0] + q[:, 0]) ** 2)
    _check(outs[1].cpu().numpy(), np.abs(r[:, 0] * np.conj(q[:, 0])))
    _, per_r, _ = methods.aperture_terms(rc[..., :1], o["scan"], o["xe"], o["angles"], o["starts"], o["c"], o["fs"],
                                         o["fd"], o["fnumber"], "RC")
    _, per_q, _ = methods.aperture_terms(cr[..., :1], o["scan"], o["ye"], o["angles"], o["starts"], o["c"], o["fs"],
                                         o["fd"], o["fnumber"], "CR")
    fmas = np.abs(methods.signed_sqrt(per_r).sum(axis=1) * methods.signed_sqrt(per_q).sum(axis=1))[:, 0] ** 2
    _check(outs[2].cpu().numpy(), fmas)
    dmas = methods.dmas_ccf_acf_power(rc[..., :1], cr[..., :1], *args)
    np.testing.assert_allclose(outs[3].cpu().numpy(), dmas, rtol=1e-4, atol=1e-4 * np.abs(dmas).max())
