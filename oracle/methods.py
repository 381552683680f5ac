"""Float64 oracles for the batching-form methods (TEST INFRASTRUCTURE).

* XDoppler, method 1: |mean_t r_t conj(q_t)| with r, q the RC and CR
  compounded IQ (src/rcabeam/xdoppler.py:33-51; ensemble.cu:236-315, 596-627).
* St-SW, method 4: interleaved angle subsets s::k of each aperture, per-frame
  subset means and variances, the k x k cross-correlation series, their
  energies over frames and the normalized pair sum, times XDoppler power
  (src/rcabeam/stsw.py:10-107; the C ABI returns the raw weights and the
  caller normalizes by the full-volume peak, ensemble.py:127-129).
* DMAS-CCF-ACF, method 3: per frame, signed-square-root channel DMAS, the
  cross-coherence factor over active channels and the angular coherence factor,
  then the mean over frames (src/rcabeam/dmas.py:32-85 evaluated on per-frame
  channel and angle sums as tests/test_ensemble.py:31-37 does; the frame
  batching itself is ensemble.cu:143-232).
"""

from __future__ import annotations

import numpy as np

from oracle.das import _as_frames


def aperture_terms(iq, scan, elements, angles, starts, c, fs, fd, fnumber, config):
    """Per-channel (angle-summed) and per-angle (channel-summed) DAS terms in complex128.

    Returns ``per_channel (nv, nc, nt)``, ``per_angle (nv, na, nt)`` and the
    active channel count ``(nv,)`` (sim.py:362-388).
    """
    iq = _as_frames(iq)
    ns, nc, na, nt = iq.shape
    scan = np.asarray(scan, dtype=np.float64).reshape(-1, 3)
    elements = np.asarray(elements, dtype=np.float64)
    angles = np.asarray(angles, dtype=np.float64)
    starts = np.broadcast_to(np.asarray(starts, dtype=np.float64), (na,))
    full = fnumber is None or fnumber <= 0
    x, z, y = scan[:, 0], scan[:, 1], scan[:, 2]
    v_rx, u_tx = (x, y) if config == "RC" else (y, x)
    depth = z[:, None]
    distance = v_rx[:, None] - elements[None, :]
    receive = np.sqrt(depth * depth + distance * distance) / c
    active = np.ones_like(distance, dtype=bool) if full else np.abs(distance) <= depth / (2 * fnumber)
    channels = np.arange(nc)
    per_channel = np.zeros((len(scan), nc, nt), np.complex128)
    per_angle = np.zeros((len(scan), na, nt), np.complex128)
    for m in range(na):
        tau = ((z * np.cos(angles[m]) + u_tx * np.sin(angles[m])) / c)[:, None] + receive
        sample = (tau - starts[m]) * fs
        valid = active & (sample >= 0) & (sample <= ns - 1)
        clipped = np.clip(sample, 0, ns - 1)
        lower = np.floor(clipped).astype(np.intp)
        upper = np.minimum(lower + 1, ns - 1)
        w = (clipped - lower)[..., None]
        value = (1 - w) * iq[lower, channels, m] + w * iq[upper, channels, m]
        value = value * (np.exp(2j * np.pi * fd * tau) * valid)[..., None]
        per_channel += value
        per_angle[:, m] = value.sum(axis=1)
    return per_channel, per_angle, active.sum(axis=1).astype(np.float64)


def signed_sqrt(x: np.ndarray) -> np.ndarray:
    """x / sqrt(|x|), zero where x == 0 (src/rcabeam/fmas.py:11-30)."""
    mag = np.abs(x)
    out = np.zeros_like(x)
    nz = mag > 0
    out[nz] = x[nz] / np.sqrt(mag[nz])
    return out


def xdoppler_power(r: np.ndarray, q: np.ndarray) -> np.ndarray:
    """|mean over frames of r conj(q)|."""
    return np.abs(np.mean(r * np.conj(q), axis=-1))


def dmas_ccf_acf_power(rc, cr, scan, xe, ye, angles, starts, c, fs, fd, fnumber):
    """Mean over frames of DMAS * CCF * ACF (dmas.py:32-85 per frame)."""
    sr, ar, nr = aperture_terms(rc, scan, xe, angles, starts, c, fs, fd, fnumber, "RC")
    sq, aq, nq = aperture_terms(cr, scan, ye, angles, starts, c, fs, fd, fnumber, "CR")
    s = np.concatenate([sr, sq], axis=1)  # (nv, 2nc, nt)
    st = signed_sqrt(s)
    y_dmas = np.abs(st.sum(axis=1)) ** 2 - np.sum(np.abs(st) ** 2, axis=1)
    norm = (nr + nq)[:, None]
    with np.errstate(divide="ignore", invalid="ignore"):
        w_ccf = np.maximum(y_dmas, 0) / norm / np.sum(np.abs(s), axis=1)
    mu_r, mu_q = ar.mean(axis=1), aq.mean(axis=1)
    var_r = np.mean(np.abs(ar - mu_r[:, None]) ** 2, axis=1)
    var_q = np.mean(np.abs(aq - mu_q[:, None]) ** 2, axis=1)
    num = np.abs(mu_r * np.conj(mu_q))
    den = np.abs(mu_r) ** 2 + np.abs(mu_q) ** 2 + (var_r + var_q) / 2 - num
    with np.errstate(divide="ignore", invalid="ignore"):
        w_acf = num / den
    y_dmas = np.where(np.isfinite(y_dmas), y_dmas, 0)
    w_ccf = np.where(np.isfinite(w_ccf), w_ccf, 0)
    w_acf = np.where(np.isfinite(w_acf) & (den > 0), w_acf, 0)
    return np.mean(y_dmas * w_ccf * w_acf, axis=-1)


def _subset_stats(per_angle: np.ndarray, k: int):
    """Means and mean squared deviations over angles s::k, per frame (stsw.py:45-53)."""
    means, variances = [], []
    for subset in range(k):
        group = per_angle[:, subset::k, :]
        mu = group.mean(axis=1)
        means.append(mu)
        variances.append(np.mean(np.abs(group - mu[:, None, :]) ** 2, axis=1))
    return means, variances


def st_sw_raw_weights(per_angle_rc: np.ndarray, per_angle_cr: np.ndarray, k: int) -> np.ndarray:
    """Unnormalized St-SW weights ``|acc|`` per voxel from per-angle IQ ``(nv, na, nt)`` (stsw.py:54-79)."""
    m_rc, v_rc = _subset_stats(per_angle_rc, k)
    m_cr, v_cr = _subset_stats(per_angle_cr, k)
    ccf, energy = {}, {}
    for ir in range(k):
        for ic in range(k):
            num = m_rc[ir] * np.conj(m_cr[ic])
            den = np.abs(m_rc[ir]) ** 2 + np.abs(m_cr[ic]) ** 2 + (v_rc[ir] + v_cr[ic]) / 2 - np.abs(num)
            with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
                value = num / den
            value[~np.isfinite(value)] = 0
            ccf[ir, ic] = value
            energy[ir, ic] = np.sum(np.abs(value) ** 2, axis=-1)
    acc = np.zeros(per_angle_rc.shape[0], dtype=np.complex128)
    for ir1 in range(k):
        for ic1 in range(k):
            for ir2 in range(ir1 + 1, k):
                for ic2 in range(k):
                    if ic2 == ic1:
                        continue
                    den = np.sqrt(energy[ir1, ic1] * energy[ir2, ic2])
                    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
                        corr = np.sum(ccf[ir1, ic1] * np.conj(ccf[ir2, ic2]), axis=-1) / den
                    corr[~np.isfinite(corr)] = 0
                    acc += corr
    return np.abs(acc)


def st_sw_terms(rc, cr, scan, xe, ye, angles, starts, c, fs, fd, fnumber, k):
    """(raw weights, XDoppler power) per voxel: the two outputs of C ABI method 4."""
    _, ar, _ = aperture_terms(rc, scan, xe, angles, starts, c, fs, fd, fnumber, "RC")
    _, aq, _ = aperture_terms(cr, scan, ye, angles, starts, c, fs, fd, fnumber, "CR")
    return st_sw_raw_weights(ar, aq, k), xdoppler_power(ar.sum(axis=1), aq.sum(axis=1))


def st_sw_power(rc, cr, scan, xe, ye, angles, starts, c, fs, fd, fnumber, k):
    """St-SW power Doppler: peak-normalized weights times XDoppler power (stsw.py:82-107)."""
    weights, power = st_sw_terms(rc, cr, scan, xe, ye, angles, starts, c, fs, fd, fnumber, k)
    peak = weights.max()
    return (weights / peak if peak > 0 else weights) * power
