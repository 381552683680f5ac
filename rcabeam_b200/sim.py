"""RCA geometry, scan coordinates and synthetic channel data.

``RCAGeometry``, ``depth_axis`` and ``simulate_point`` keep the interface of
the reference module ``rcabeam.sim`` (src/rcabeam/sim.py:12-189): a flat
row-column array whose RC acquisitions receive on the column elements
(positions ``x_el``) and CR acquisitions on the row elements (``y_el``).
Scene synthesis here is test/benchmark input generation, not part of the
reconstruction path.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Literal

import numpy as np


@dataclass(frozen=True)
class RCAGeometry:
    """Flat row-column-array geometry (reference sim.py:12-37).

    x_el, y_el: receive element positions (m) of the RC and CR apertures;
    c: sound speed (m/s); fs: IQ sampling rate (Hz); f_demod: demodulation
    frequency (Hz); fnumber: receive f-number, ``None`` = full aperture.
    """

    x_el: np.ndarray
    y_el: np.ndarray
    c: float = 1540.0
    fs: float = 24e6
    f_demod: float = 6e6
    fnumber: float | None = 1.0


def depth_axis(start: float, stop: float, frequency: float, *, sound_speed: float = 1540.0,
               spacing: float | None = None) -> np.ndarray:
    """Uniform depths from ``start`` to ``stop`` inclusive, step <= lambda/2 (sim.py:40-77)."""
    if (
        not np.isfinite([start, stop, frequency, sound_speed]).all()
        or start < 0
        or stop < start
        or min(frequency, sound_speed) <= 0
    ):
        raise ValueError("Require finite ordered nonnegative depths and positive frequency/sound speed")
    step = sound_speed / (2 * frequency) if spacing is None else spacing
    if not np.isfinite(step) or step <= 0:
        raise ValueError("Depth spacing must be finite and positive")
    return np.linspace(start, stop, int(np.ceil((stop - start) / step)) + 1)


def scan_coords(grid) -> np.ndarray:
    """Float32 ``(nv, 3)`` voxel coordinates ``(x, z, y)``, x-major and y innermost (sim.py:192-199)."""
    x, z, y = (np.asarray(a, dtype=np.float32).ravel() for a in grid)
    nx, nz, ny = len(x), len(z), len(y)
    out = np.empty((nx, nz, ny, 3), dtype=np.float32)
    out[..., 0] = x.reshape(nx, 1, 1)
    out[..., 1] = z.reshape(1, nz, 1)
    out[..., 2] = y.reshape(1, 1, ny)
    return out.reshape(nx * nz * ny, 3)


def simulate_point(geom: RCAGeometry, angles: np.ndarray, point: tuple[float, float, float], nsamp: int,
                   t_start: float, config: Literal["RC", "CR"], *, sigma_t: float = 0.15e-6) -> np.ndarray:
    """Baseband channel IQ ``(nsamp, channels, angles)`` of one point scatterer (sim.py:131-189).

    Two-way delay tau = plane-wave transmit + element receive; a Gaussian
    envelope exp(-((t - tau) / sigma_t)^2) demodulated by exp(-j 2 pi f_demod tau).
    """
    xp, zp, yp = point
    el = np.asarray(geom.x_el if config == "RC" else geom.y_el, dtype=np.float64)
    v_rx, u_tx = (xp, yp) if config == "RC" else (yp, xp)
    t = t_start + np.arange(nsamp) / geom.fs
    receive = np.sqrt(zp * zp + (v_rx - el) ** 2) / geom.c
    out = np.empty((nsamp, len(el), len(angles)), dtype=np.complex64)
    for m, theta in enumerate(np.asarray(angles, dtype=np.float64)):
        tau = (zp * np.cos(theta) + u_tx * np.sin(theta)) / geom.c + receive
        envelope = np.exp(-(((t[:, None] - tau[None, :]) / sigma_t) ** 2))
        out[:, :, m] = envelope * np.exp(-2j * np.pi * geom.f_demod * tau)[None, :]
    return out
