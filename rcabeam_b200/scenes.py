"""Seeded synthetic inputs shaped like the workloads' scenes.

``clutter_casorati`` is a Casorati-matrix model of a power-Doppler ensemble:
rigidly moving tissue (a strong, temporally coherent component), blood flowing
in a tube (weak, fast-rotating phases), and complex white noise.  It is a
model of beamformed IQ, not a beamformed scene: it gives the clutter filter
the spectrum it meets in practice (a few dominant tissue singular values, a
blood band 40 dB lower, a noise floor) at any size, on the device.
"""

from __future__ import annotations

import math

import torch


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
