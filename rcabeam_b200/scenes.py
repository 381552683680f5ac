"""Seeded synthetic inputs: point-scatterer scenes and a Casorati clutter model.

Scenes (``config1_scene``, ``flow_scene``) are channel data: seeded scatterer
lists (positions, motion, complex amplitudes) rendered on the GPU by the
forward-model kernel ``rcabeam_simulate_scene_device`` -- the Gaussian-pulse
model of the reference's ``simulate_point`` (src/rcabeam/sim.py:131-189) summed
over moving scatterers -- plus complex white noise at a stated level.

* ``config1_scene``: 64 + 64 elements at 0.2 mm, 5 angles in [-8, 8] deg,
  (256 samples, 64 channels, 5 angles, 16 frames), 32 x 64 x 32 grid over
  +-6.4 mm and 3-15 mm; 5 static unit point targets, 2000 uniformly placed
  speckle scatterers with N(0, 1) complex amplitudes, complex white noise at
  20 dB SNR.
* ``flow_scene``: the full-size filtered-OPW scene -- tissue speckle moving
  rigidly at 1 mm/s (0 dB), blood scatterers at -40 dB flowing at 10-30 mm/s
  (parabolic profile) through a 1 mm-radius tube, complex noise at -50 dB --
  at any aperture / grid size.

``clutter_casorati`` is a Casorati-matrix model of a power-Doppler ensemble:
rigidly moving tissue (a strong, temporally coherent component), blood flowing
in a tube (weak, fast-rotating phases), and complex white noise.  It is a
model of beamformed IQ, not a beamformed scene: it gives the clutter filter
the spectrum it meets in practice (a few dominant tissue singular values, a
blood band 40 dB lower, a noise floor) at any size, on the device.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import torch

from rcabeam_b200 import _lib
from rcabeam_b200.sim import RCAGeometry

SIGMA_T = 0.15e-6  # Gaussian pulse width of the reference's simulate_point (sim.py:139)
PRF = 500.0        # slow-time rate of the flow scenes (frames per second)

# Five point targets (x, z, y) in metres: the reference examples' target layout
# (examples/_support/scene.py:12-18), all inside the config-1 volume.
TARGETS = ((0.0, 8.0e-3, 0.0), (-2.2e-3, 6.0e-3, 1.8e-3), (2.0e-3, 9.5e-3, -1.5e-3),
           (-1.2e-3, 11.2e-3, -2.4e-3), (2.6e-3, 7.2e-3, 2.5e-3))


@dataclass
class Scene:
    """Channel data of both apertures (complex64 ``(ns, nc, na, nt)`` on the device) and their acquisition."""

    rc: torch.Tensor
    cr: torch.Tensor
    angles: np.ndarray
    t_start: float
    grid: tuple
    geom: RCAGeometry
    info: dict = field(default_factory=dict)


def scatterer_table(pos, *, amplitude, direction=None, speed=None, s0=None, period=None) -> np.ndarray:
    """(n, 11) float32 rows (ox, oz, oy, dx, dz, dy, s0, speed, period, amp_re, amp_im)."""
    pos = np.asarray(pos, dtype=np.float64).reshape(-1, 3)
    n = len(pos)
    out = np.zeros((n, 11), dtype=np.float32)
    out[:, 0:3] = pos
    if direction is not None:
        out[:, 3:6] = np.broadcast_to(np.asarray(direction, dtype=np.float64), (n, 3))
    for col, val in ((6, s0), (7, speed), (8, period)):
        if val is not None:
            out[:, col] = np.broadcast_to(np.asarray(val, dtype=np.float64), (n,))
    amp = np.broadcast_to(np.asarray(amplitude, dtype=np.complex128), (n,))
    out[:, 9], out[:, 10] = amp.real, amp.imag
    return out


def render(table: np.ndarray, geom: RCAGeometry, angles, t_start, ns: int, nt: int, *, device=None,
           prf: float = PRF, sigma_t: float = SIGMA_T, half_width: float | None = None):
    """Noise-free channel IQ ``(rc, cr)`` of the scatterers, rendered by the forward-model kernel."""
    dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
    angles = np.asarray(angles, dtype=np.float32)
    na = len(angles)
    f32 = lambda v: torch.from_numpy(np.ascontiguousarray(v, dtype=np.float32)).to(dev)  # noqa: E731
    scat = f32(table)
    ang = f32(angles)
    starts = f32(np.broadcast_to(np.asarray(t_start, dtype=np.float32), (na,)))
    hw = 4.0 * sigma_t if half_width is None else half_width
    out = []
    for config, el in enumerate((geom.x_el, geom.y_el)):
        elem = f32(el)
        data = torch.empty((ns, len(el), na, nt), dtype=torch.complex64, device=dev)
        _lib.call("rcabeam_simulate_scene_device", scat.data_ptr(), len(table), elem.data_ptr(), ang.data_ptr(),
                  starts.data_ptr(), data.data_ptr(), ns, len(el), na, nt, config, float(prf), float(geom.c),
                  float(geom.fs), float(geom.f_demod), float(sigma_t), float(hw))
        out.append(data)
    return out[0], out[1]


def add_noise(channels, level_db: float, generator: torch.Generator) -> float:
    """Adds circular complex white noise of power 10^(level_db / 10) x the mean signal power of all
    arrays (in place); returns the noise standard deviation per complex sample."""
    power = sum(float(torch.sum(torch.view_as_real(c).double() ** 2)) for c in channels)
    power /= sum(c.numel() for c in channels)
    std = math.sqrt(power * 10 ** (level_db / 10))
    for c in channels:
        re = torch.randn(c.shape, generator=generator, device=c.device, dtype=torch.float32)
        im = torch.randn(c.shape, generator=generator, device=c.device, dtype=torch.float32)
        c += torch.complex(re, im) * (std / math.sqrt(2))
    return std


def config1_scene(seed: int = 0, *, device=None, fnumber: float | None = None) -> Scene:
    """The small plain-OPW scene: 5 unit targets + 2000 N(0, 1) speckle + 20 dB noise, static over 16 frames.

    t_start = 2 x 3 mm / c - 0.5 us: the 256-sample window (12.8 us) then spans two-way
    delays of 3.4-16.2 us, so on-axis depths up to ~12.5 mm are in the window (all five
    targets; speckle deeper than that falls outside, as in a real acquisition)."""
    el = (np.arange(64) - 31.5) * 0.2e-3
    geom = RCAGeometry(el, el, c=1540.0, fs=20e6, f_demod=15e6, fnumber=fnumber)
    angles = np.deg2rad(np.linspace(-8, 8, 5))
    grid = (np.linspace(-6.4e-3, 6.4e-3, 32), np.linspace(3e-3, 15e-3, 64), np.linspace(-6.4e-3, 6.4e-3, 32))
    t_start = 2 * 3e-3 / 1540.0 - 0.5e-6
    rng = np.random.default_rng(seed)
    speckle = rng.uniform([-6.4e-3, 3e-3, -6.4e-3], [6.4e-3, 15e-3, 6.4e-3], (2000, 3))
    amp = (rng.standard_normal(2000) + 1j * rng.standard_normal(2000)) / math.sqrt(2)
    table = np.concatenate((scatterer_table(TARGETS, amplitude=1.0), scatterer_table(speckle, amplitude=amp)))
    rc, cr = render(table, geom, angles, t_start, 256, 16, device=device)
    gen = torch.Generator(device=rc.device).manual_seed(seed)
    std = add_noise((rc, cr), -20.0, gen)
    return Scene(rc, cr, angles, t_start, grid, geom,
                 {"scene": "config 1: 5 targets, 2000 speckle, 20 dB SNR", "seed": seed, "noise_std": std})


def flow_scene(*, channels: int = 128, pitch: float = 0.11e-3, samples: int = 512, angles: int = 11,
               max_angle_deg: float = 10.0, frames: int = 200, grid_shape=(128, 256, 128),
               depth=(4e-3, 12e-3), t_start: float = 4e-6, n_tissue: int = 20000, n_blood: int = 5000,
               tube_radius: float = 1e-3, tube_tilt_deg: float = 20.0, blood_db: float = -40.0,
               noise_db: float = -50.0, seed: int = 0, device=None) -> Scene:
    """Tissue / blood / noise scene of the full-size filtered-OPW workload (any size).

    Tissue: ``n_tissue`` speckle scatterers (N(0, 1) complex amplitudes, 0 dB) uniform in
    the grid volume (padded by 0.5 mm), moving rigidly at 1 mm/s along depth.  Blood:
    ``n_blood`` scatterers at ``blood_db`` in a straight tube of ``tube_radius`` through
    the grid centre, tilted ``tube_tilt_deg`` from x toward depth; speed 10-30 mm/s with a
    parabolic radial profile, re-entering at the tube start (periodic along its axis).
    Noise: complex white at ``noise_db`` of the mean channel power.  PRF 500 Hz."""
    el = (np.arange(channels) - (channels - 1) / 2) * pitch
    geom = RCAGeometry(el, el, c=1540.0, fs=20e6, f_demod=15e6, fnumber=None)
    ang = np.deg2rad(np.linspace(-max_angle_deg, max_angle_deg, angles))
    half = (channels - 1) / 2 * pitch
    grid = (np.linspace(-half, half, grid_shape[0]), np.linspace(depth[0], depth[1], grid_shape[1]),
            np.linspace(-half, half, grid_shape[2]))
    rng = np.random.default_rng(seed)
    pad = 0.5e-3
    tissue = rng.uniform([-half - pad, depth[0] - pad, -half - pad], [half + pad, depth[1] + pad, half + pad],
                         (n_tissue, 3))
    t_amp = (rng.standard_normal(n_tissue) + 1j * rng.standard_normal(n_tissue)) / math.sqrt(2)
    tilt = math.radians(tube_tilt_deg)
    axis = np.array([math.cos(tilt), math.sin(tilt), 0.0])   # (x, z, y)
    e1 = np.array([-math.sin(tilt), math.cos(tilt), 0.0])
    e2 = np.array([0.0, 0.0, 1.0])
    centre = np.array([0.0, 0.5 * (depth[0] + depth[1]), 0.0])
    length = min(2 * 0.85 * half / math.cos(tilt), (depth[1] - depth[0] - 2 * tube_radius) / max(math.sin(tilt), 1e-9))
    r = tube_radius * np.sqrt(rng.uniform(size=n_blood))
    phi = rng.uniform(0, 2 * math.pi, n_blood)
    origin = centre - axis * length / 2 + r[:, None] * (np.cos(phi)[:, None] * e1 + np.sin(phi)[:, None] * e2)
    speed = 10e-3 + 20e-3 * (1 - (r / tube_radius) ** 2)
    b_amp = (rng.standard_normal(n_blood) + 1j * rng.standard_normal(n_blood)) / math.sqrt(2) * 10 ** (blood_db / 20)
    table = np.concatenate((
        scatterer_table(tissue, amplitude=t_amp, direction=(0.0, 1.0, 0.0), speed=1e-3),
        scatterer_table(origin, amplitude=b_amp, direction=axis, speed=speed, s0=rng.uniform(0, length, n_blood),
                        period=length)))
    rc, cr = render(table, geom, ang, t_start, samples, frames, device=device)
    gen = torch.Generator(device=rc.device).manual_seed(seed)
    std = add_noise((rc, cr), noise_db, gen)
    return Scene(rc, cr, ang, t_start, grid, geom,
                 {"scene": f"flow: {n_tissue} tissue (1 mm/s, 0 dB) + {n_blood} blood ({blood_db:g} dB, 10-30 mm/s, "
                           f"{tube_radius * 1e3:g} mm tube) + {noise_db:g} dB noise", "seed": seed, "noise_std": std,
                  "tube_length_m": length})


def clutter_casorati(rows: int, frames: int, *, generator: torch.Generator, device, prf: float = 500.0,
                     f0: float = 15e6, c: float = 1540.0, tissue_speed: float = 1e-3,
                     tissue_db=(0.0, -6.0, -12.0), blood_speeds=(10e-3, 30e-3), blood_fraction: float = 0.02,
                     blood_db: float = -40.0, noise_db: float = -50.0) -> torch.Tensor:
    """complex64 ``(rows, frames)``: tissue + blood + noise, powers relative to the strongest tissue term.

    Tissue: ``len(tissue_db)`` components, each a per-row complex Gaussian
    speckle amplitude times a temporal mode -- the axial Doppler phase ramp of
    a rigid motion at ``tissue_speed`` (2 v f0 / c) modulated by the k-th
    slow cosine (k = 0, 1, 2, ...), the first terms of a decorrelating speckle
    -- so the tissue subspace has exactly that rank.  Blood: ``blood_fraction``
    of the rows (a contiguous band, the tube) with per-row Doppler frequencies
    from axial speeds drawn uniformly in ``blood_speeds``.  Noise: circular
    complex Gaussian.
    """
    def randn(*shape):
        return torch.randn(*shape, generator=generator, device=device, dtype=torch.float32)

    def rand(*shape):
        return torch.rand(*shape, generator=generator, device=device, dtype=torch.float32)

    t = torch.arange(frames, device=device, dtype=torch.float32)
    w_tis = 2 * math.pi * (2 * tissue_speed * f0 / c) / prf
    ramp = torch.polar(torch.ones_like(t), w_tis * t)
    out = torch.zeros((rows, frames), dtype=torch.complex64, device=device)
    for k, level in enumerate(tissue_db):
        mode = ramp * torch.cos(math.pi * k * (t + 0.5) / frames)
        mode = mode / torch.linalg.vector_norm(mode) * math.sqrt(frames)
        amp = torch.complex(randn(rows, 1), randn(rows, 1)) * (10 ** (level / 20) / math.sqrt(2))
        out += amp * mode[None, :]
    n_blood = max(1, int(rows * blood_fraction))
    start = (rows - n_blood) // 2
    speed = blood_speeds[0] + (blood_speeds[1] - blood_speeds[0]) * rand(n_blood, 1)
    w_blood = 2 * math.pi * (2 * speed * f0 / c) / prf
    phase0 = 2 * math.pi * rand(n_blood, 1)
    b_amp = torch.complex(randn(n_blood, 1), randn(n_blood, 1)) * (10 ** (blood_db / 20) / math.sqrt(2))
    out[start:start + n_blood] += b_amp * torch.polar(torch.ones_like(w_blood), phase0 + w_blood * t[None, :])
    out += torch.complex(randn(rows, frames), randn(rows, frames)) * (10 ** (noise_db / 20) / math.sqrt(2))
    return out
