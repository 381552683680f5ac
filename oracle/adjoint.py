"""Float64 adjoint of the OPW power-Doppler forward model -- TEST INFRASTRUCTURE ONLY.

Forward (the reference DAS of src/rcabeam/sim.py:344-393 summed over both
apertures, src/rcabeam/opw.py:8-21, and power Doppler src/rcabeam/power.py:21),
extended with a per-receive-element delay offset d[A][c] (A = RC, CR):

    tau(v,c,a)  = (z cos(th_a) + u sin(th_a)) / c_s + sqrt(z^2 + (w - e_c)^2) / c_s + d[A][c]
    s           = (tau - start_a) fs,  valid iff 0 <= s <= ns - 1 (and |w - e_c| <= z / (2 fn))
    y(v,c,a,t)  = ((1 - f) X[i0,c,a,t] + f X[i1,c,a,t]) exp(+j 2 pi fd tau),  i0 = floor(s),
                  f = s - i0, i1 = min(i0 + 1, ns - 1)
    IQ(v,t)     = sum over A, c, a of y;   PD(v) = mean_t |IQ(v,t)|^2

with (u, w) = (y, x) for RC and (x, y) for CR.  For a loss L = sum_v g_v PD(v)
the gradients (complex gradients in the dL/dRe + j dL/dIm convention) are

    G(v,t)           = (2 / nt) g_v IQ(v,t)
    dL/dX[i0,c,a,t] += (1 - f) conj(phase) G(v,t),   dL/dX[i1,c,a,t] += f conj(phase) G(v,t)
    dL/dtau(v,c,a)   = Re sum_t conj(G(v,t)) (fs (X[i1] - X[i0]) phase + j 2 pi fd y)
    dL/dd[A][c]      = sum_{v,a} dL/dtau,      dL/dc_s = sum dL/dtau (-(tau - d[A][c]) / c_s).

Everything here is float64 / complex128; the GPU kernels are checked against
it and it is checked against central finite differences of its own forward.
"""

from __future__ import annotations

import numpy as np


def _taps(scan, elements, angles, starts, c, fs, fd, fnumber, ns, offsets, config):
    """Per (voxel, channel, angle): tau, i0, i1, f, phase, mask."""
    x, z, y = scan[:, 0], scan[:, 1], scan[:, 2]
    rx, tx = (x, y) if config == "RC" else (y, x)
    dist = rx[:, None] - elements[None, :]
    receive = np.sqrt(z[:, None] ** 2 + dist**2) / c                      # (nv, nc)
    active = np.ones_like(dist, dtype=bool) if fnumber is None else np.abs(dist) <= z[:, None] / (2 * fnumber)
    transmit = (z[:, None] * np.cos(angles)[None, :] + tx[:, None] * np.sin(angles)[None, :]) / c   # (nv, na)
    tau = transmit[:, None, :] + receive[:, :, None] + offsets[None, :, None]                     # (nv, nc, na)
    sample = (tau - starts[None, None, :]) * fs
    valid = (sample >= 0) & (sample <= ns - 1) & active[:, :, None]
    sample = np.clip(sample, 0, ns - 1)
    i0 = np.floor(sample).astype(np.intp)
    i1 = np.minimum(i0 + 1, ns - 1)
    f = sample - i0
    phase = np.exp(2j * np.pi * fd * tau) * valid
    return tau, i0, i1, f, phase, valid


def forward(rc, cr, scan, xe, ye, angles, starts, offsets, c, fs, fd, fnumber):
    """IQ (nv, nt) complex128 of the offset-extended OPW model."""
    ns, nc, na, nt = rc.shape
    iq = np.zeros((len(scan), nt), np.complex128)
    ch = np.arange(nc)[None, :, None]
    an = np.arange(na)[None, None, :]
    for k, (data, el, cfg) in enumerate(((rc, xe, "RC"), (cr, ye, "CR"))):
        x = np.asarray(data, np.complex128)
        _, i0, i1, f, phase, _ = _taps(scan, el, angles, starts, c, fs, fd, fnumber, ns, offsets[k], cfg)
        y = ((1 - f)[..., None] * x[i0, ch, an] + f[..., None] * x[i1, ch, an]) * phase[..., None]
        iq += y.sum(axis=(1, 2))
    return iq


def power(rc, cr, scan, xe, ye, angles, starts, offsets, c, fs, fd, fnumber):
    iq = forward(rc, cr, scan, xe, ye, angles, starts, offsets, c, fs, fd, fnumber)
    return np.mean(np.abs(iq) ** 2, axis=1)


def adjoint(rc, cr, scan, xe, ye, angles, starts, offsets, c, fs, fd, fnumber, grad_pd):
    """Gradients (dRC, dCR, d offsets (2, nc), d c) of L = sum_v grad_pd[v] PD[v]."""
    ns, nc, na, nt = rc.shape
    iq = forward(rc, cr, scan, xe, ye, angles, starts, offsets, c, fs, fd, fnumber)
    g = (2.0 / nt) * np.asarray(grad_pd, np.float64)[:, None] * iq          # (nv, nt)
    ch = np.arange(nc)[None, :, None]
    an = np.arange(na)[None, None, :]
    grads, d_off, d_c = [], np.zeros((2, nc)), 0.0
    for k, (data, el, cfg) in enumerate(((rc, xe, "RC"), (cr, ye, "CR"))):
        x = np.asarray(data, np.complex128)
        tau, i0, i1, f, phase, valid = _taps(scan, el, angles, starts, c, fs, fd, fnumber, ns, offsets[k], cfg)
        x0, x1 = x[i0, ch, an], x[i1, ch, an]                                # (nv, nc, na, nt)
        y = ((1 - f)[..., None] * x0 + f[..., None] * x1) * phase[..., None]
        dy = fs * (x1 - x0) * phase[..., None] + 2j * np.pi * fd * y
        dtau = np.real(np.sum(np.conj(g)[:, None, None, :] * dy, axis=3)) * valid   # (nv, nc, na)
        d_off[k] = dtau.sum(axis=(0, 2))
        d_c += float(np.sum(dtau * (-(tau - offsets[k][None, :, None]) / c)))
        gx = np.zeros_like(x)
        w0 = ((1 - f) * np.conj(phase))[..., None] * g[:, None, None, :]
        w1 = (f * np.conj(phase))[..., None] * g[:, None, None, :]
        idx_c = np.broadcast_to(ch, i0.shape)
        idx_a = np.broadcast_to(an, i0.shape)
        np.add.at(gx, (i0, idx_c, idx_a), w0)
        np.add.at(gx, (i1, idx_c, idx_a), w1)
        grads.append(gx)
    return grads[0], grads[1], d_off, d_c
