"""Float64 restatement of rcabeam's RCA delay-and-sum (TEST INFRASTRUCTURE).

Follows the reference NumPy DAS ``_delay_numpy`` (src/rcabeam/sim.py:344-393):

* receive delay  tau_rx = sqrt(z^2 + (v - e)^2) / c, v = x for RC, y for CR
  (sim.py:369-371);
* transmit delay tau_tx = (z cos(theta) + u sin(theta)) / c, u = y for RC,
  x for CR (sim.py:369, 377);
* sample = (tau - t_start[angle]) * fs, valid iff 0 <= sample <= ns - 1
  (sim.py:379-380);
* linear interpolation between floor(sample) and min(floor + 1, ns - 1)
  (sim.py:381-384);
* rotation by exp(+j 2 pi f_demod tau), masked by the f-number aperture
  |v - e| <= z / (2 fnumber) (sim.py:373, 385);
* sums over channels per angle (sim.py:386); OPW sums angles and both
  apertures (src/rcabeam/opw.py:8-21, ensemble.cu:444); power Doppler is
  mean |x|^2 over frames (src/rcabeam/power.py:21).

Everything is evaluated in float64 / complex128 -- including the
interpolation weight, which the reference keeps in float32 (sim.py:383) --
so this is the FP64 oracle that the CUDA path is measured against.  An
optional per-element delay offset (seconds) is added to the receive delay;
it is the differentiation parameter of the adjoint form and defaults to zero,
which reproduces the reference exactly.
"""

from __future__ import annotations

import numpy as np

# Voxel x channel x frame elements per gathered temporary.
_BLOCK_ELEMENTS = 1 << 21


def scan_coords(grid) -> np.ndarray:
    """Flatten a Cartesian ``(x, z, y)`` grid into float32 ``(nv, 3)`` rows.

    Same traversal as the reference ``_scan_coords`` (sim.py:192-199): x-major,
    then z, y innermost.
    """
    x, z, y = (np.asarray(a, dtype=np.float64) for a in grid)
    out = np.empty((len(x), len(z), len(y), 3), dtype=np.float32)
    out[..., 0] = x[:, None, None]
    out[..., 1] = z[None, :, None]
    out[..., 2] = y[None, None, :]
    return out.reshape(-1, 3)


def _as_frames(iq: np.ndarray) -> np.ndarray:
    iq = np.asarray(iq)
    return iq[..., None] if iq.ndim == 3 else iq


def aperture_das(
    iq: np.ndarray,
    scan: np.ndarray,
    elements: np.ndarray,
    angles: np.ndarray,
    starts: np.ndarray,
    c: float,
    fs: float,
    fd: float,
    fnumber: float | None,
    config: str,
    *,
    per_angle: bool = False,
    offsets: np.ndarray | None = None,
) -> np.ndarray:
    """Delay-and-sum one aperture (``config`` "RC" or "CR") in complex128.

    Parameters
    ----------
    iq
        Channel IQ ``(ns, nc, na[, nt])``.
    scan
        Voxel coordinates ``(nv, 3)`` as ``(x, z, y)``.
    elements
        Receive element positions of this aperture (x_el for RC, y_el for CR).
    angles, starts
        Steering angles (rad) and first-sample times (s), one per angle.
    c, fs, fd
        Sound speed, sampling and demodulation frequencies.
    fnumber
        Receive f-number; ``None`` (or a value <= 0) keeps the full aperture.
    per_angle
        Return ``(nv, na, nt)`` instead of the angle sum ``(nv, nt)``.
    offsets
        Optional per-element receive delay offsets in seconds.
    """
    if config not in ("RC", "CR"):
        raise ValueError("config must be 'RC' or 'CR'")
    iq = _as_frames(iq)
    ns, nc, na, nt = iq.shape
    if ns < 2:
        raise ValueError("need at least two samples")
    scan = np.asarray(scan, dtype=np.float64).reshape(-1, 3)
    elements = np.asarray(elements, dtype=np.float64)
    angles = np.asarray(angles, dtype=np.float64)
    starts = np.broadcast_to(np.asarray(starts, dtype=np.float64), (na,))
    delta = np.zeros(nc) if offsets is None else np.asarray(offsets, dtype=np.float64)
    full = fnumber is None or fnumber <= 0
    nv = len(scan)
    x, z, y = scan[:, 0], scan[:, 1], scan[:, 2]
    v_rx, u_tx = (x, y) if config == "RC" else (y, x)
    out = np.zeros((nv, na, nt) if per_angle else (nv, nt), dtype=np.complex128)
    block = max(1, _BLOCK_ELEMENTS // (nc * nt))
    channels = np.arange(nc)
    cos_t, sin_t = np.cos(angles), np.sin(angles)
    for first in range(0, nv, block):
        sl = slice(first, min(first + block, nv))
        depth = z[sl, None]
        distance = v_rx[sl, None] - elements[None, :]
        receive = np.sqrt(depth * depth + distance * distance) / c + delta[None, :]
        active = np.ones_like(distance, dtype=bool) if full else np.abs(distance) <= depth / (2 * fnumber)
        for m in range(na):
            transmit = (z[sl] * cos_t[m] + u_tx[sl] * sin_t[m]) / c
            tau = transmit[:, None] + receive
            sample = (tau - starts[m]) * fs
            valid = active & (sample >= 0) & (sample <= ns - 1)
            clipped = np.clip(sample, 0, ns - 1)
            lower = np.floor(clipped).astype(np.intp)
            upper = np.minimum(lower + 1, ns - 1)
            w = (clipped - lower)[..., None]
            a = iq[lower, channels, m].astype(np.complex128)
            b = iq[upper, channels, m].astype(np.complex128)
            value = (1 - w) * a + w * b
            phase = np.exp(2j * np.pi * fd * tau) * valid
            summed = np.einsum("vct,vc->vt", value, phase)
            if per_angle:
                out[sl, m] = summed
            else:
                out[sl] += summed
    return out


def opw_iq(rc, cr, scan, xe, ye, angles, starts, c, fs, fd, fnumber, *, offsets=None) -> np.ndarray:
    """Coherent OPW IQ ``(nv, nt)``: RC + CR, each summed over angles and channels."""
    off_rc = None if offsets is None else offsets[0]
    off_cr = None if offsets is None else offsets[1]
    r = aperture_das(rc, scan, xe, angles, starts, c, fs, fd, fnumber, "RC", offsets=off_rc)
    q = aperture_das(cr, scan, ye, angles, starts, c, fs, fd, fnumber, "CR", offsets=off_cr)
    return r + q


def apertures_iq(rc, cr, scan, xe, ye, angles, starts, c, fs, fd, fnumber):
    """Separately compounded RC and CR IQ (the reference's method 5, ensemble.cu:278-287)."""
    r = aperture_das(rc, scan, xe, angles, starts, c, fs, fd, fnumber, "RC")
    q = aperture_das(cr, scan, ye, angles, starts, c, fs, fd, fnumber, "CR")
    return r, q


def power_doppler(signal: np.ndarray) -> np.ndarray:
    """Mean squared magnitude over the last (frame) axis (src/rcabeam/power.py:8-21)."""
    s = np.asarray(signal)
    return np.mean(s.real.astype(np.float64) ** 2 + s.imag.astype(np.float64) ** 2, axis=-1)


def opw_voxel_order(shape) -> np.ndarray:
    """Lateral 2 x 4 patch traversal with tails (src/rcabeam/ensemble.py:24-49)."""
    nx, nz, ny = (int(s) for s in shape)
    if min(nx, nz, ny) < 1:
        raise ValueError("Grid dimensions must be positive")
    ids = np.arange(nx * nz * ny, dtype=np.intp).reshape(nx, nz, ny)
    bx, by = nx - nx % 2, ny - ny % 4
    core = ids[:bx, :, :by].reshape(bx // 2, 2, nz, by // 4, 4).transpose(0, 2, 3, 1, 4).ravel()
    return np.concatenate((core, ids[:bx, :, by:].ravel(), ids[bx:].ravel()))
