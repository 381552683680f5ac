"""Seeded reconstruction cases shared by the GPU parity tests."""

from __future__ import annotations

import numpy as np

from rcabeam_b200.sim import RCAGeometry, scan_coords


def random_case(seed, ns, nc, na, nt, grid, *, fs=1e6, fd=0.1e6, fnumber=1.0, starts=None, x_el=None, y_el=None):
    rng = np.random.default_rng(seed)
    x_el = np.linspace(-0.001, 0.001, nc) if x_el is None else x_el
    y_el = np.linspace(-0.0008, 0.0007, nc) if y_el is None else y_el
    geom = RCAGeometry(x_el=x_el, y_el=y_el, fs=fs, f_demod=fd, fnumber=fnumber)
    angles = np.linspace(-0.08, 0.09, na)
    if starts is None:
        starts = 1e-6 * (1 + np.arange(na) % 3)
    rc = (rng.normal(size=(ns, nc, na, nt)) + 1j * rng.normal(size=(ns, nc, na, nt))).astype(np.complex64)
    cr = (rng.normal(size=rc.shape) + 1j * rng.normal(size=rc.shape)).astype(np.complex64)
    return rc, cr, angles, starts, grid, geom


def oracle_inputs(angles, starts, grid, geom):
    """The float32-quantized geometry the C ABI sees, as float64 oracle inputs."""
    f32 = lambda v: np.asarray(v, dtype=np.float32).astype(np.float64)  # noqa: E731
    na = len(angles)
    return dict(
        scan=scan_coords(grid).astype(np.float64),
        xe=f32(geom.x_el),
        ye=f32(geom.y_el),
        angles=f32(angles),
        starts=f32(np.broadcast_to(starts, (na,))),
        c=float(np.float32(geom.c)),
        fs=float(np.float32(geom.fs)),
        fd=float(np.float32(geom.f_demod)),
        fnumber=None if geom.fnumber is None else float(np.float32(geom.fnumber)),
    )


def rel_l2(actual, expected):
    expected = np.asarray(expected)
    denom = np.linalg.norm(expected.ravel())
    return np.linalg.norm((np.asarray(actual) - expected).ravel()) / (denom if denom > 0 else 1.0)
