"""Float64 forward model of moving point-scatterer scenes -- TEST INFRASTRUCTURE ONLY.

Restates, scatterer by scatterer, the model that ``rcabeam_simulate_scene_device``
evaluates on the GPU: the Gaussian-pulse channel IQ of the reference's
``simulate_point`` (src/rcabeam/sim.py:131-189, the ``sigma_t`` branch: envelope
exp(-((t - tau) / sigma_t)^2) demodulated by exp(-j 2 pi f_demod tau), two-way
delay = plane-wave transmit + element receive, sim.py:176-188) summed over
scatterers, each at its frame's position o + d * s(t), s(t) = s0 + speed * t
wrapped into [0, period) when period > 0, and evaluated only where
|t - tau| <= half_width (the reference's envelope is untruncated; with
half_width = 4 sigma_t the difference is below exp(-16) ~ 1e-7).
"""

from __future__ import annotations

import numpy as np

FIELDS = ("ox", "oz", "oy", "dx", "dz", "dy", "s0", "speed", "period", "amp_re", "amp_im")


def positions(scatterers: np.ndarray, t: float) -> np.ndarray:
    """(n, 3) float64 (x, z, y) positions at time t."""
    s = np.asarray(scatterers, dtype=np.float64)
    along = s[:, 6] + s[:, 7] * t
    period = s[:, 8]
    wrap = period > 0
    along[wrap] -= period[wrap] * np.floor(along[wrap] / period[wrap])
    return s[:, 0:3] + s[:, 3:6] * along[:, None]


def simulate(scatterers, elements, angles, starts, ns: int, nt: int, *, prf: float, c: float, fs: float, fd: float,
             sigma_t: float, half_width: float, config: str) -> np.ndarray:
    """Channel IQ ``(ns, nc, na, nt)`` complex128 of one aperture ("RC" or "CR")."""
    s = np.asarray(scatterers, dtype=np.float32).astype(np.float64)  # the device reads float32 fields
    el = np.asarray(elements, dtype=np.float32).astype(np.float64)
    ang = np.asarray(angles, dtype=np.float32).astype(np.float64)
    st = np.asarray(starts, dtype=np.float32).astype(np.float64)
    amp = s[:, 9] + 1j * s[:, 10]
    out = np.zeros((ns, len(el), len(ang), nt), dtype=np.complex128)
    rows = np.arange(ns, dtype=np.float64)
    for f in range(nt):
        pos = positions(s, f / prf)
        x, z, y = pos[:, 0], pos[:, 1], pos[:, 2]
        v, u = (x, y) if config == "RC" else (y, x)
        receive = np.sqrt(z[:, None] ** 2 + (v[:, None] - el[None, :]) ** 2) / c  # (n, nc)
        for a, theta in enumerate(ang):
            tau = (z * np.cos(theta) + u * np.sin(theta))[:, None] / c + receive  # (n, nc)
            t = st[a] + rows / fs  # (ns,)
            r = (t[:, None, None] - tau[None]) / sigma_t  # (ns, n, nc)
            env = np.where(np.abs(t[:, None, None] - tau[None]) <= half_width, np.exp(-r * r), 0.0)
            rot = amp[:, None] * np.exp(-2j * np.pi * fd * tau)  # (n, nc)
            out[:, :, a, f] = np.einsum("snc,nc->sc", env, rot)
    return out
