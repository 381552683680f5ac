"""Generate golden vectors from the reference's own NumPy implementation.

Run in a container where the reference checkout is available:

    python tests/golden/make_golden.py /path/to/rcabeam    (or RCABEAM_REFERENCE=/path/to/rcabeam)

It imports ``rcabeam`` from ``<reference>/src`` (NumPy modules only: sim,
clutter, power, opw, ensemble.opw_voxel_order, dmas, fmas, stsw) and writes
``tests/golden/*.npz``.  The fixtures hold the exact inputs next to the
reference outputs, so the tests never need the reference at run time.
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def _import_reference(root: str):
    sys.path.insert(0, str(Path(root) / "src"))
    import rcabeam.clutter as clutter
    import rcabeam.dmas as dmas
    import rcabeam.ensemble as ensemble
    import rcabeam.sim as sim

    return sim, clutter, ensemble, dmas


def das_cases(sim):
    """Per-angle / per-channel DAS from the reference ``_delay_numpy``."""
    cases = {}
    rng = np.random.default_rng(44)
    # Shapes and geometry of tests/test_ensemble.py:21-29 (5 frames).
    geo = dict(x_el=np.array([-0.001, 0.001]), y_el=np.array([-0.0008, 0.0007]), fs=1e6, f_demod=0.1e6)
    angles = np.array([-0.08, -0.02, 0.05, 0.09])
    starts = np.array([1e-6, 2e-6, 1e-6, 3e-6])
    grid = (np.array([0.0, 0.008]), np.array([0.001, 0.007, 0.03]), np.array([0.0]))
    rc = (rng.normal(size=(16, 2, 4, 5)) + 1j * rng.normal(size=(16, 2, 4, 5))).astype(np.complex64)
    cr = (rng.normal(size=rc.shape) + 1j * rng.normal(size=rc.shape)).astype(np.complex64)
    for fnumber in (None, 1.0):
        geom = sim.RCAGeometry(fnumber=fnumber, **geo)
        tag = "full" if fnumber is None else "f1"
        for config, iq in (("RC", rc), ("CR", cr)):
            ch, ang, cnt = sim._delay_numpy(iq, angles, starts, grid, geom, config, channels_out=True)
            cases[f"small_{tag}_{config}_per_angle"] = ang
            cases[f"small_{tag}_{config}_per_channel"] = ch
            cases[f"small_{tag}_{config}_count"] = cnt
    cases.update(
        small_rc=rc, small_cr=cr, small_angles=angles, small_starts=starts, small_x=grid[0], small_z=grid[1],
        small_y=grid[2], small_xe=geo["x_el"], small_ye=geo["y_el"], small_fs=geo["fs"], small_fd=geo["f_demod"],
    )

    # A physical 15 MHz / 20 MS/s case with simulated point targets (sim.py:131-189):
    # 64 + 64 elements at 0.2 mm pitch, 5 angles in [-8, 8] deg, 4 frames.
    el = (np.arange(64) - 31.5) * 0.2e-3
    geom = sim.RCAGeometry(el, el, c=1540.0, fs=20e6, f_demod=15e6, fnumber=1.0)
    angles = np.deg2rad(np.linspace(-8, 8, 5))
    t0 = 2 * 3e-3 / 1540.0 - 0.5e-6
    targets = [((0.0, 5.0e-3, 0.0), 1.0), ((-1.2e-3, 4.2e-3, 0.8e-3), 0.7), ((1.0e-3, 6.0e-3, -0.6e-3), 0.5)]
    phases = np.exp(2j * np.pi * np.arange(4) / 7.0)
    chans = []
    for config in ("RC", "CR"):
        data = sum(a * sim.simulate_point(geom, angles, p, 256, t0, config) for p, a in targets)
        chans.append((data[..., None] * phases).astype(np.complex64))
    grid = (np.linspace(-1.6e-3, 1.6e-3, 6), np.linspace(3.5e-3, 6.5e-3, 9), np.linspace(-1.2e-3, 1.2e-3, 5))
    for config, iq in zip(("RC", "CR"), chans):
        _, ang, _ = sim._delay_numpy(iq, angles, t0, grid, geom, config, channels_out=False)
        cases[f"target_{config}_per_angle"] = ang
    cases.update(
        target_rc=chans[0], target_cr=chans[1], target_angles=angles, target_t0=t0, target_x=grid[0],
        target_z=grid[1], target_y=grid[2], target_el=el,
    )
    # The simulated channels alone (checks the product's scene synthesizer).
    cases["point_rc"] = sim.simulate_point(geom, angles, (0.3e-3, 5.0e-3, -0.2e-3), 256, t0, "RC")[::2]
    cases["point_cr"] = sim.simulate_point(geom, angles, (0.3e-3, 5.0e-3, -0.2e-3), 256, t0, "CR")[::2]

    # Closed receive window known answer (tests/test_iq_sampling.py:255-266).
    zero = np.zeros(1)
    geom = sim.RCAGeometry(zero, zero, c=2, fs=1, f_demod=0, fnumber=None)
    raw = np.arange(1, 4, dtype=np.complex64).reshape(3, 1, 1)
    _, ang, _ = sim._delay_numpy(raw, zero, 0, (zero, np.array([0, 1.5, 2, 2.25]), zero), geom, "RC",
                                 channels_out=True)
    cases["closed_window"] = ang.ravel()
    return cases


def clutter_cases(clutter):
    cases = {}
    rng = np.random.default_rng(47)
    values = np.array([20.0, 8.0, 3.0, 1.0, 0.2, 0.03])
    left, _ = np.linalg.qr(rng.normal(size=(18, 6)) + 1j * rng.normal(size=(18, 6)))
    right, _ = np.linalg.qr(rng.normal(size=(6, 6)) + 1j * rng.normal(size=(6, 6)))
    matrix = (left * values) @ right.conj().T
    cases["spectrum_matrix"] = matrix
    cases["spectrum_values"] = values
    for method in ("svd", "gram"):
        s, v = clutter.temporal_basis(matrix.reshape(3, 6, 6), method=method)
        cases[f"spectrum_{method}_values"] = s
        cases[f"spectrum_{method}_filtered"] = clutter.svd_clutter_filter(
            matrix.reshape(3, 6, 6), rank_start=1, rank_stop=4, method=method
        )
    # A tissue-dominated slow-time matrix: rank-3 strong clutter + weak noise.
    rng = np.random.default_rng(5)
    rows, frames = 300, 24
    t = np.arange(frames)
    clutter_part = sum(
        (rng.normal(size=(rows, 1)) + 1j * rng.normal(size=(rows, 1))) * 100 * np.exp(2j * np.pi * f * t)
        for f in (0.0, 0.01, -0.02)
    )
    weak = rng.normal(size=(rows, frames)) + 1j * rng.normal(size=(rows, frames))
    iq = (clutter_part + weak).astype(np.complex64)
    cases["tissue_iq"] = iq
    for method in ("svd", "gram"):
        cases[f"tissue_{method}_filtered"] = clutter.svd_clutter_filter(iq, rank_start=3, method=method)
        cases[f"tissue_{method}_values"] = clutter.temporal_basis(iq, method=method)[0]
    return cases


def order_cases(ensemble):
    cases = {}
    for shape in ((4, 3, 8), (3, 2, 5), (1, 2, 1), (2, 1, 4), (5, 3, 2), (7, 2, 11)):
        cases["order_" + "x".join(map(str, shape))] = ensemble.opw_voxel_order(shape)
    return cases


def dmas_cases(sim, dmas):
    """Per-frame DMAS-CCF-ACF on the small case, as tests/test_ensemble.py:30-37 builds it."""
    rng = np.random.default_rng(44)
    x_el, y_el = np.array([-0.001, 0.001]), np.array([-0.0008, 0.0007])
    geom = sim.RCAGeometry(x_el=x_el, y_el=y_el, fs=1e6, f_demod=0.1e6, fnumber=1.0)
    angles = np.array([-0.08, -0.02, 0.05, 0.09])
    starts = np.array([1e-6, 2e-6, 1e-6, 3e-6])
    grid = (np.array([0.0, 0.008]), np.array([0.001, 0.007, 0.03]), np.array([0.0]))
    rc = (rng.normal(size=(16, 2, 4, 5)) + 1j * rng.normal(size=(16, 2, 4, 5))).astype(np.complex64)
    cr = (rng.normal(size=rc.shape) + 1j * rng.normal(size=rc.shape)).astype(np.complex64)
    out = []
    for t in range(rc.shape[-1]):
        sr, r, nr = sim.delay_rca_channel_data(rc[..., t], angles, starts, grid, geom, "RC", use_cuda=False)
        sq, q, nq = sim.delay_rca_channel_data(cr[..., t], angles, starts, grid, geom, "CR", use_cuda=False)
        dm, wc, wa = dmas.dmas_ccf_acf_core(sr, sq, r, q, ccf_norm=nr + nq)
        out.append(dm * wc * wa)
    return {"dmas_f1_power": np.mean(out, axis=0)}


def stsw_cases(sim, stsw):
    """St-SW power from per-frame per-angle DAS, as tests/test_ensemble.py:30-69 and
    tests/test_ensemble_targets.py:46-65 build it (k = 2, 3, 4)."""
    cases = {}
    # Small case of test_ensemble.py (full aperture, 5 frames).
    rng = np.random.default_rng(44)
    geom = sim.RCAGeometry(x_el=np.array([-0.001, 0.001]), y_el=np.array([-0.0008, 0.0007]), fs=1e6, f_demod=0.1e6)
    angles = np.array([-0.08, -0.02, 0.05, 0.09])
    starts = np.array([1e-6, 2e-6, 1e-6, 3e-6])
    grid = (np.array([0.0, 0.008]), np.array([0.001, 0.007, 0.03]), np.array([0.0]))
    rc = (rng.normal(size=(16, 2, 4, 5)) + 1j * rng.normal(size=(16, 2, 4, 5))).astype(np.complex64)
    cr = (rng.normal(size=rc.shape) + 1j * rng.normal(size=rc.shape)).astype(np.complex64)
    # A lateral line of 257 voxels, 3 frames, RC angle 0 silent (zero-norm series for k = 4).
    line_grid = (np.zeros(1), np.array([0.007]), np.linspace(-0.001, 0.001, 257))
    line_geom = sim.RCAGeometry(x_el=np.array([-0.001, 0.001]), y_el=np.array([-0.001, 0.001]), fs=1e6,
                                f_demod=0.1e6)
    rng = np.random.default_rng(42)
    lr = (rng.normal(size=(16, 2, 4, 3)) + 1j * rng.normal(size=(16, 2, 4, 3))).astype(np.complex64)
    lq = (rng.normal(size=lr.shape) + 1j * rng.normal(size=lr.shape)).astype(np.complex64)
    lr[:, :, 0] = 0
    for tag, (r, q, st, g, gm) in {"small": (rc, cr, starts, grid, geom),
                                   "line": (lr, lq, 1e-6, line_grid, line_geom)}.items():
        ar, aq = [], []
        for t in range(r.shape[-1]):
            _, a, _ = sim.delay_rca_channel_data(r[..., t], angles, st, g, gm, "RC", use_cuda=False)
            _, b, _ = sim.delay_rca_channel_data(q[..., t], angles, st, g, gm, "CR", use_cuda=False)
            ar.append(a)
            aq.append(b)
        iq = np.concatenate([np.stack(ar, axis=-1), np.stack(aq, axis=-1)], axis=-2)
        ri, qi = np.arange(4), np.arange(4, 8)
        for k in (2, 3, 4):
            cases[f"{tag}_k{k}_power"] = stsw.st_sw_pd(iq, ri, qi, k=k)
            cases[f"{tag}_k{k}_weights"] = stsw.st_sw_weights(iq, ri, qi, k=k)
        cases[f"{tag}_rc"], cases[f"{tag}_cr"] = r, q
    cases.update(angles=angles, small_starts=starts, line_y=line_grid[2])
    return cases


def scene_cases(sim):
    """Channel IQ of single static point scatterers from the reference ``simulate_point``
    (sim.py:131-189, Gaussian envelope, sigma_t = 0.15 us): the pulse model that the
    scene forward model sums over scatterers."""
    # Inputs are float32-exact: the forward-model kernel reads float32 fields.
    f32 = lambda v: np.asarray(v, dtype=np.float32).astype(np.float64)  # noqa: E731
    el_x, el_y = f32((np.arange(16) - 7.5) * 0.2e-3), f32((np.arange(16) - 7.5) * 0.18e-3)
    geom = sim.RCAGeometry(el_x, el_y, c=1540.0, fs=20e6, f_demod=15e6, fnumber=None)
    angles = f32(np.deg2rad(np.array([-8.0, 0.0, 5.0])))
    points = f32([[0.3e-3, 4.0e-3, -0.2e-3], [-1.1e-3, 4.6e-3, 0.9e-3]])
    cases = dict(el_x=el_x, el_y=el_y, angles=angles, points=points, nsamp=160, t_start=f32(4.4e-6))
    for i, point in enumerate(points):
        for config in ("RC", "CR"):
            cases[f"point{i}_{config}"] = sim.simulate_point(geom, angles, tuple(point), 160, float(cases["t_start"]),
                                                             config)
    return cases


def main(root: str) -> None:
    sim, clutter, ensemble, dmas = _import_reference(root)
    import rcabeam.stsw as stsw

    np.savez_compressed(HERE / "scene.npz", **scene_cases(sim))
    np.savez_compressed(HERE / "stsw.npz", **stsw_cases(sim, stsw))
    np.savez_compressed(HERE / "das.npz", **das_cases(sim))
    np.savez_compressed(HERE / "clutter.npz", **clutter_cases(clutter))
    np.savez_compressed(HERE / "order.npz", **order_cases(ensemble))
    np.savez_compressed(HERE / "dmas.npz", **dmas_cases(sim, dmas))
    for f in sorted(HERE.glob("*.npz")):
        print(f.name, f.stat().st_size)


if __name__ == "__main__":
    import os

    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("RCABEAM_REFERENCE")
    if not root:
        sys.exit("usage: make_golden.py <reference checkout> (or set RCABEAM_REFERENCE)")
    main(root)
