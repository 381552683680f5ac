"""Differentiation form: hand-written adjoint of the OPW power Doppler on the GPU.

* The offset-extended forward against the float64 oracle (oracle/adjoint.py).
* The GPU adjoint (autograd backward) against the float64 NumPy adjoint:
  complex128 channels (float64 kernels) within 1e-10, complex64 within 2e-4.
* The full differentiation workload -- grid 64 x 128 x 64, channels
  (384, 128, 7, 32), loss = sum of PD over a 1 mm sphere around a point
  target, delay offsets ~ N(0, 5 ns), sound speed 1523 m/s -- against central
  finite differences with a relative step of 1e-3, within 1e-3 (float64
  kernels), and the frame-chunk invariance of the result.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from oracle import adjoint as oa
from rcabeam_b200 import _lib
from rcabeam_b200.autograd import DasGeometry, OpwPowerDoppler, opw_power_doppler
from rcabeam_b200.sim import RCAGeometry, scan_coords, simulate_point
from tests._cases import rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs CUDA")
    yield
    assert _lib.device_error() == 0


def _small(seed=4, fnumber=None, nt=11):
    rng = np.random.default_rng(seed)
    ns, nc, na = 96, 8, 3
    el = (np.arange(nc) - 3.5) * 0.2e-3
    geom = RCAGeometry(el, el * 0.95, c=1540.0, fs=20e6, f_demod=15e6, fnumber=fnumber)
    angles = np.deg2rad([-7.0, 1.0, 8.0])
    grid = (np.linspace(-0.6e-3, 0.6e-3, 4) + 1.3e-5, np.linspace(3e-3, 4e-3, 5) + 0.7e-5,
            np.linspace(-0.5e-3, 0.5e-3, 3) + 2.1e-5)
    rc = rng.normal(size=(ns, nc, na, nt)) + 1j * rng.normal(size=(ns, nc, na, nt))
    cr = rng.normal(size=(ns, nc, na, nt)) + 1j * rng.normal(size=(ns, nc, na, nt))
    offsets = rng.normal(scale=5e-9, size=(2, nc))
    return rc, cr, offsets, geom, angles, 3e-6, grid


def _oracle_kwargs(geometry: DasGeometry, offsets, c):
    f64 = lambda t: t.cpu().numpy().astype(np.float64)  # noqa: E731
    return dict(scan=f64(geometry.scan), xe=f64(geometry.xe), ye=f64(geometry.ye), angles=f64(geometry.angles),
                starts=f64(geometry.starts), offsets=offsets, c=c, fs=geometry.fs, fd=geometry.fd,
                fnumber=None if geometry.fn <= 0 else geometry.fn)


@pytest.mark.parametrize("dtype", [torch.complex128, torch.complex64])
@pytest.mark.parametrize("fnumber", [None, 1.0])
def test_forward_power_matches_oracle(dtype, fnumber):
    rc, cr, offsets, geom, angles, t0, grid = _small(fnumber=fnumber)
    geometry = DasGeometry.build(grid, geom, angles, t0)
    drc, dcr = torch.from_numpy(rc).to(dtype).cuda(), torch.from_numpy(cr).to(dtype).cuda()
    if dtype == torch.complex64:
        rc, cr = rc.astype(np.complex64), cr.astype(np.complex64)
    off = torch.from_numpy(offsets).cuda()
    pd = opw_power_doppler(drc, dcr, off, torch.tensor(1531.0, dtype=torch.float64, device="cuda"), geometry)
    want = oa.power(rc, cr, **_oracle_kwargs(geometry, offsets, 1531.0))
    assert rel_l2(pd.cpu().numpy().ravel(), want) <= (1e-12 if dtype == torch.complex128 else 2e-6)


@pytest.mark.parametrize("dtype,tol", [(torch.complex128, 1e-10), (torch.complex64, 2e-4)])
@pytest.mark.parametrize("chunk", [8, 3])
def test_adjoint_matches_float64_numpy_adjoint(dtype, tol, chunk):
    rc, cr, offsets, geom, angles, t0, grid = _small(fnumber=1.0)
    geometry = DasGeometry.build(grid, geom, angles, t0)
    nv = geometry.voxels
    rng = np.random.default_rng(9)
    g = rng.uniform(0.5, 1.5, size=nv) * (rng.random(nv) < 0.6)  # sparse upstream gradient
    drc = torch.from_numpy(rc).to(dtype).cuda().requires_grad_()
    dcr = torch.from_numpy(cr).to(dtype).cuda().requires_grad_()
    off = torch.from_numpy(offsets).cuda().requires_grad_()
    c = torch.tensor(1528.0, dtype=torch.float64, device="cuda", requires_grad=True)
    pd = OpwPowerDoppler.apply(drc, dcr, off, c, geometry, chunk)
    (pd * torch.from_numpy(g).cuda()).sum().backward()
    if dtype == torch.complex64:
        rc, cr = rc.astype(np.complex64), cr.astype(np.complex64)
    w_rc, w_cr, w_off, w_c = oa.adjoint(rc, cr, **_oracle_kwargs(geometry, offsets, 1528.0), grad_pd=g)
    assert rel_l2(drc.grad.cpu().numpy(), w_rc) <= tol
    assert rel_l2(dcr.grad.cpu().numpy(), w_cr) <= tol
    assert rel_l2(off.grad.cpu().numpy(), w_off) <= tol
    assert abs(c.grad.item() - w_c) <= tol * abs(w_c)


def _differentiation_workload(dtype):
    """Grid 64 x 128 x 64 over +-7 mm x 4-12 mm, channels (384, 128, 7, 32), one point target."""
    ns, nc, na, nt = 384, 128, 7, 32
    pitch = 0.11e-3
    el = (np.arange(nc) - (nc - 1) / 2) * pitch
    half = (nc - 1) / 2 * pitch
    geom_true = RCAGeometry(el, el, c=1540.0, fs=20e6, f_demod=15e6, fnumber=None)
    angles = np.deg2rad(np.linspace(-10, 10, na))
    t0 = 4e-6
    target = (0.35e-3, 8.0e-3, -0.22e-3)
    rng = np.random.default_rng(21)
    phases = np.exp(2j * np.pi * rng.random(nt))
    chans = []
    for config in ("RC", "CR"):
        data = simulate_point(geom_true, angles, target, ns, t0, config)
        noise = 0.01 * (rng.normal(size=(ns, nc, na, nt)) + 1j * rng.normal(size=(ns, nc, na, nt)))
        chans.append(torch.from_numpy(data[..., None] * phases + noise).to(dtype).cuda())
    grid = (np.linspace(-half, half, 64), np.linspace(4e-3, 12e-3, 128), np.linspace(-half, half, 64))
    geometry = DasGeometry.build(grid, geom_true, angles, t0)
    scan = scan_coords(grid).astype(np.float64)
    roi = np.sum((scan - np.array([target[0], target[1], target[2]])) ** 2, axis=1) <= (1e-3) ** 2
    offsets = torch.from_numpy(rng.normal(scale=5e-9, size=(2, nc))).cuda()
    return chans[0], chans[1], offsets, geometry, torch.from_numpy(roi.astype(np.float64)).cuda()


def _roi_loss(rc, cr, offsets, c, geometry, roi):
    pd = OpwPowerDoppler.apply(rc, cr, offsets, torch.tensor(c, dtype=torch.float64, device="cuda"), geometry, 8)
    return float((pd * roi).sum().item())


def test_differentiation_workload_against_finite_differences():
    rc, cr, offsets, geometry, roi = _differentiation_workload(torch.complex128)
    c0 = 1523.0
    assert int(roi.sum().item()) > 500
    rc.requires_grad_()
    off = offsets.clone().requires_grad_()
    c = torch.tensor(c0, dtype=torch.float64, device="cuda", requires_grad=True)
    before = torch.cuda.max_memory_allocated()
    pd = OpwPowerDoppler.apply(rc, cr, off, c, geometry, 8)
    (pd * roi).sum().backward()
    # Beyond the two channel-gradient buffers (outputs, the size of the inputs)
    # the passes keep one 8-frame IQ chunk of the ROI voxels, not the ensemble.
    ensemble_bytes = geometry.voxels * rc.shape[3] * 16
    extra = torch.cuda.max_memory_allocated() - before - 2 * rc.numel() * 16
    assert extra < ensemble_bytes / 16
    table = []
    # Sound speed.  Every sample crossing of the ~2.5M ROI taps is a kink of the
    # linearly interpolated loss, and a 1e-3 relative step (1.5 m/s) moves every
    # tap by ~0.2 samples: the secant then differs from the local derivative by
    # a few 1e-3 whatever the gradient code.  So check (a) the secant against
    # the adjoint averaged over the same interval (trapezoid, 33 nodes), and
    # (b) the local derivative against a central difference small enough to
    # resolve it (relative step 3e-6).
    h = 1e-3 * c0
    fd = (_roi_loss(rc.detach(), cr, offsets, c0 + h, geometry, roi)
          - _roi_loss(rc.detach(), cr, offsets, c0 - h, geometry, roi)) / (2 * h)
    nodes = np.linspace(c0 - h, c0 + h, 33)
    slopes = []
    for cn in nodes:
        cc = torch.tensor(float(cn), dtype=torch.float64, device="cuda", requires_grad=True)
        (OpwPowerDoppler.apply(rc.detach(), cr, offsets, cc, geometry, 8) * roi).sum().backward()
        slopes.append(cc.grad.item())
    mean_slope = float(np.trapezoid(slopes, nodes) / (2 * h))
    table.append(("c: mean adjoint", mean_slope, fd))
    h_small = 3e-6 * c0
    fd_small = (_roi_loss(rc.detach(), cr, offsets, c0 + h_small, geometry, roi)
                - _roi_loss(rc.detach(), cr, offsets, c0 - h_small, geometry, roi)) / (2 * h_small)
    table.append(("c: local", c.grad.item(), fd_small))
    print(f"\nsound speed: adjoint {c.grad.item():.6e}, central difference at 1e-3 relative step {fd:.6e} "
          f"(relative difference {abs(c.grad.item() - fd) / abs(fd):.2e}, interpolation kinks)")
    # Delay offsets of a few elements of both apertures.
    for a, ch in ((0, 10), (0, 64), (1, 33), (1, 100)):
        h = 1e-3 * max(abs(float(offsets[a, ch])), 5e-9)
        op, om = offsets.clone(), offsets.clone()
        op[a, ch] += h
        om[a, ch] -= h
        fd = (_roi_loss(rc.detach(), cr, op, c0, geometry, roi) - _roi_loss(rc.detach(), cr, om, c0, geometry, roi)) / (
            2 * h)
        table.append((f"offset[{a},{ch}]", off.grad[a, ch].item(), fd))
    # Channel samples with the largest gradients (real and imaginary directions).
    grad = rc.grad.detach()
    for idx in torch.topk(grad.abs().flatten(), 2).indices.tolist():
        for direction in (1.0, 1j):
            x = rc.detach().flatten()
            h = 1e-3 * float(x[idx].abs())
            xp, xm = x.clone(), x.clone()
            xp[idx] += h * direction
            xm[idx] -= h * direction
            fd = (_roi_loss(xp.view_as(rc), cr, offsets, c0, geometry, roi)
                  - _roi_loss(xm.view_as(rc), cr, offsets, c0, geometry, roi)) / (2 * h)
            g = grad.flatten()[idx]
            table.append((f"rc[{idx}] {'re' if direction == 1.0 else 'im'}",
                          float(g.real if direction == 1.0 else g.imag), fd))
    print("\ngradient check (adjoint, central difference, relative error):")
    for name, adj, fd in table:
        print(f"  {name:18s} {adj: .6e} {fd: .6e} {abs(adj - fd) / abs(fd):.2e}")
    for name, adj, fd in table:
        assert abs(adj - fd) <= 1e-3 * abs(fd), name


def test_single_precision_gradients_track_double():
    rc, cr, offsets, geometry, roi = _differentiation_workload(torch.complex128)
    grads = {}
    for dtype in (torch.complex128, torch.complex64):
        a = rc.detach().to(dtype).clone().requires_grad_()
        b = cr.to(dtype)
        off = offsets.clone().requires_grad_()
        c = torch.tensor(1523.0, dtype=torch.float64, device="cuda", requires_grad=True)
        pd = OpwPowerDoppler.apply(a, b, off, c, geometry, 8)
        (pd * roi).sum().backward()
        grads[dtype] = (a.grad.to(torch.complex128), off.grad, c.grad)
    g64, g32 = grads[torch.complex128], grads[torch.complex64]
    assert float(torch.linalg.vector_norm(g32[0] - g64[0]) / torch.linalg.vector_norm(g64[0])) <= 1e-4
    assert float(torch.linalg.vector_norm(g32[1] - g64[1]) / torch.linalg.vector_norm(g64[1])) <= 1e-3
    assert abs(float(g32[2] - g64[2])) <= 1e-3 * abs(float(g64[2]))


def test_frame_chunks_do_not_change_the_result():
    rc, cr, offsets, geom, angles, t0, grid = _small(nt=13)
    geometry = DasGeometry.build(grid, geom, angles, t0)
    drc, dcr = torch.from_numpy(rc).cuda(), torch.from_numpy(cr).cuda()
    c = torch.tensor(1540.0, dtype=torch.float64, device="cuda")
    off = torch.from_numpy(offsets).cuda()
    ref = OpwPowerDoppler.apply(drc, dcr, off, c, geometry, 8)
    for chunk in (1, 2, 5):
        got = OpwPowerDoppler.apply(drc, dcr, off, c, geometry, chunk)
        assert rel_l2(got.cpu().numpy(), ref.cpu().numpy()) <= 1e-13


def test_invalid_arguments():
    rc, cr, offsets, geom, angles, t0, grid = _small()
    geometry = DasGeometry.build(grid, geom, angles, t0)
    drc, dcr = torch.from_numpy(rc).cuda(), torch.from_numpy(cr).cuda()
    c = torch.tensor(1540.0, dtype=torch.float64, device="cuda")
    with pytest.raises(ValueError, match="offsets"):
        OpwPowerDoppler.apply(drc, dcr, torch.zeros(3, device="cuda", dtype=torch.float64), c, geometry, 8)
    with pytest.raises(ValueError, match="frame_chunk"):
        OpwPowerDoppler.apply(drc, dcr, torch.from_numpy(offsets).cuda(), c, geometry, 9)
    with pytest.raises(ValueError, match="share"):
        OpwPowerDoppler.apply(drc, dcr.to(torch.complex64), torch.from_numpy(offsets).cuda(), c, geometry, 8)
