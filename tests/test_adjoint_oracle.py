"""The float64 adjoint oracle against central finite differences of its own forward (CPU)."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import adjoint


def _case(seed=3, fnumber=None):
    rng = np.random.default_rng(seed)
    ns, nc, na, nt = 48, 4, 3, 5
    rc = rng.normal(size=(ns, nc, na, nt)) + 1j * rng.normal(size=(ns, nc, na, nt))
    cr = rng.normal(size=(ns, nc, na, nt)) + 1j * rng.normal(size=(ns, nc, na, nt))
    el = np.linspace(-0.6e-3, 0.6e-3, nc)
    scan = np.array([[0.1e-3, 3.0e-3, -0.2e-3], [0.37e-3, 3.3e-3, 0.21e-3], [-0.5e-3, 3.7e-3, 0.05e-3]])
    angles = np.deg2rad([-6.0, 0.5, 7.0])
    starts = np.full(na, 3.0e-6)
    offsets = rng.normal(scale=5e-9, size=(2, nc))
    return dict(rc=rc, cr=cr, scan=scan, xe=el, ye=el * 0.9, angles=angles, starts=starts, offsets=offsets,
                c=1540.0, fs=20e6, fd=15e6, fnumber=fnumber)


def _loss(k, g):
    return float(np.dot(g, adjoint.power(**k)))


@pytest.mark.parametrize("fnumber", [None, 1.0])
def test_adjoint_matches_central_differences(fnumber):
    k = _case(fnumber=fnumber)
    g = np.array([1.0, 0.5, 2.0])
    d_rc, d_cr, d_off, d_c = adjoint.adjoint(**k, grad_pd=g)
    # Sound speed (relative step 1e-6; the loss is smooth between sample crossings).
    h = 1e-6 * k["c"]
    kp, km = dict(k, c=k["c"] + h), dict(k, c=k["c"] - h)
    fd = (_loss(kp, g) - _loss(km, g)) / (2 * h)
    assert abs(fd - d_c) <= 1e-5 * abs(fd)
    # Delay offsets.
    for a, c in ((0, 1), (1, 2), (0, 3)):
        h = 1e-13
        op, om = k["offsets"].copy(), k["offsets"].copy()
        op[a, c] += h
        om[a, c] -= h
        fd = (_loss(dict(k, offsets=op), g) - _loss(dict(k, offsets=om), g)) / (2 * h)
        assert abs(fd - d_off[a, c]) <= 1e-5 * max(abs(fd), 1e-3 * np.abs(d_off).max())
    # Channel samples: real and imaginary directions of a few entries.
    flat = np.flatnonzero(np.abs(d_rc) > 0.1 * np.abs(d_rc).max())[:3]
    for idx in flat:
        for direction in (1.0, 1j):
            xp, xm = k["rc"].copy(), k["rc"].copy()
            xp.flat[idx] += 1e-6 * direction
            xm.flat[idx] -= 1e-6 * direction
            fd = (_loss(dict(k, rc=xp), g) - _loss(dict(k, rc=xm), g)) / 2e-6
            want = d_rc.flat[idx].real if direction == 1.0 else d_rc.flat[idx].imag
            assert abs(fd - want) <= 1e-6 * np.abs(d_rc).max()


def test_adjoint_is_zero_without_upstream_gradient():
    k = _case()
    d_rc, d_cr, d_off, d_c = adjoint.adjoint(**k, grad_pd=np.zeros(3))
    assert not d_rc.any() and not d_cr.any() and not d_off.any() and d_c == 0.0
