"""Pin the float64 oracle to the reference's own outputs (golden vectors) and known answers."""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from oracle import clutter, das, methods

GOLDEN = Path(__file__).resolve().parent / "golden"


def _grid_scan(x, z, y):
    return np.stack(np.meshgrid(x, z, y, indexing="ij"), -1).reshape(-1, 3)


@pytest.fixture(scope="module")
def g():
    return np.load(GOLDEN / "das.npz")


@pytest.mark.parametrize("tag,fnumber", [("full", None), ("f1", 1.0)])
@pytest.mark.parametrize("config", ["RC", "CR"])
def test_das_matches_reference_small(g, tag, fnumber, config):
    """Per-angle and per-channel sums agree with reference sim._delay_numpy (complex64 storage)."""
    scan = _grid_scan(g["small_x"], g["small_z"], g["small_y"])
    iq = g["small_rc"] if config == "RC" else g["small_cr"]
    el = g["small_xe"] if config == "RC" else g["small_ye"]
    args = (iq, scan, el, g["small_angles"], g["small_starts"], 1540.0, float(g["small_fs"]), float(g["small_fd"]),
            fnumber, config)
    per_angle = das.aperture_das(*args, per_angle=True)
    ref = g[f"small_{tag}_{config}_per_angle"].reshape(per_angle.shape)
    np.testing.assert_allclose(per_angle, ref, rtol=1e-6, atol=1e-6)
    ch, ang, cnt = methods.aperture_terms(*args)
    np.testing.assert_allclose(ch, g[f"small_{tag}_{config}_per_channel"].reshape(ch.shape), rtol=1e-6, atol=1e-6)
    np.testing.assert_allclose(ang, ref, rtol=1e-6, atol=1e-6)
    np.testing.assert_array_equal(cnt, g[f"small_{tag}_{config}_count"].ravel())


@pytest.mark.parametrize("config", ["RC", "CR"])
def test_das_matches_reference_targets(g, config):
    """15 MHz / 20 MS/s simulated targets, fnumber 1: relative L2 at the reference's complex64 floor."""
    scan = _grid_scan(g["target_x"], g["target_z"], g["target_y"])
    iq = g["target_rc"] if config == "RC" else g["target_cr"]
    mine = das.aperture_das(iq, scan, g["target_el"], g["target_angles"], float(g["target_t0"]), 1540.0, 20e6, 15e6,
                            1.0, config, per_angle=True)
    ref = g[f"target_{config}_per_angle"].reshape(mine.shape)
    assert np.linalg.norm(mine - ref) / np.linalg.norm(ref) < 1e-6


def test_closed_receive_window_known_answer(g):
    """Reference tests/test_iq_sampling.py:255-266: [1, 2.5, 3, 0]."""
    zero = np.zeros(1)
    scan = _grid_scan(zero, np.array([0, 1.5, 2, 2.25]), zero)
    raw = np.arange(1, 4, dtype=np.complex64).reshape(3, 1, 1)
    out = das.aperture_das(raw, scan, zero, zero, 0.0, 2.0, 1.0, 0.0, None, "RC").ravel()
    np.testing.assert_array_equal(out, [1, 2.5, 3, 0])
    np.testing.assert_array_equal(out, g["closed_window"])


def test_voxel_order_known_answer():
    order = np.load(GOLDEN / "order.npz")
    for key in order.files:
        shape = tuple(int(s) for s in key.split("_")[1].split("x"))
        np.testing.assert_array_equal(das.opw_voxel_order(shape), order[key])
    np.testing.assert_array_equal(das.opw_voxel_order((4, 3, 8))[:8], [0, 1, 2, 3, 24, 25, 26, 27])


def test_dmas_oracle_matches_reference(g):
    """DMAS-CCF-ACF from per-frame channel/angle sums (reference dmas.py:32-85)."""
    ref = np.load(GOLDEN / "dmas.npz")["dmas_f1_power"].ravel()
    scan = _grid_scan(g["small_x"], g["small_z"], g["small_y"])
    mine = methods.dmas_ccf_acf_power(g["small_rc"], g["small_cr"], scan, g["small_xe"], g["small_ye"],
                                      g["small_angles"], g["small_starts"], 1540.0, float(g["small_fs"]),
                                      float(g["small_fd"]), 1.0)
    np.testing.assert_allclose(mine, ref, rtol=1e-5, atol=1e-5)


def test_clutter_oracle_matches_reference():
    c = np.load(GOLDEN / "clutter.npz")
    for method in ("svd", "gram"):
        values, basis = clutter.temporal_basis(c["spectrum_matrix"].reshape(3, 6, 6), method=method)
        np.testing.assert_allclose(values, c[f"spectrum_{method}_values"], rtol=1e-10)
        np.testing.assert_allclose(values, c["spectrum_values"], rtol=2e-6)
        np.testing.assert_allclose(basis.conj().T @ basis, np.eye(6), atol=2e-14)
        out = clutter.svd_clutter_filter(c["spectrum_matrix"].reshape(3, 6, 6), rank_start=1, rank_stop=4,
                                         method=method)
        np.testing.assert_allclose(out, c[f"spectrum_{method}_filtered"], rtol=1e-9, atol=1e-12)
        tissue = clutter.svd_clutter_filter(c["tissue_iq"], rank_start=3, method=method)
        ref = c[f"tissue_{method}_filtered"]
        assert np.linalg.norm(tissue - ref) / np.linalg.norm(ref) < 1e-6  # reference casts back to complex64


def test_clutter_oracle_policy():
    with pytest.raises(ValueError):
        clutter.temporal_basis(np.zeros((2, 3)), method="svd")
    with pytest.raises(ValueError):
        clutter.rank_interval(4, 3, 2)
    with np.errstate(over="ignore", invalid="ignore"), pytest.raises(np.linalg.LinAlgError, match="rescale"):
        clutter.temporal_basis(np.full((2, 3), 1e200 + 1e200j), method="gram")


def test_power_doppler_oracle():
    x = np.array([[1 + 1j, 2, 0, 1j]])
    np.testing.assert_allclose(das.power_doppler(x), [(2 + 4 + 0 + 1) / 4])


@pytest.mark.parametrize("tag", ["small", "line"])
@pytest.mark.parametrize("k", [2, 3, 4])
def test_st_sw_oracle_matches_reference(tag, k):
    """St-SW weights and power against the reference's st_sw_weights / st_sw_pd (stsw.py:10-107)."""
    s = np.load(GOLDEN / "stsw.npz")
    if tag == "small":
        scan = _grid_scan([0.0, 0.008], [0.001, 0.007, 0.03], [0.0])
        xe, ye, starts = np.array([-0.001, 0.001]), np.array([-0.0008, 0.0007]), s["small_starts"]
    else:
        scan = _grid_scan([0.0], [0.007], s["line_y"])
        xe = ye = np.array([-0.001, 0.001])
        starts = 1e-6
    # The fixtures use RCAGeometry's default aperture, f-number 1 (sim.py:12-37).
    args = (s[f"{tag}_rc"], s[f"{tag}_cr"], scan, xe, ye, s["angles"], starts, 1540.0, 1e6, 0.1e6, 1.0, k)
    weights, _ = methods.st_sw_terms(*args)
    ref_w = s[f"{tag}_k{k}_weights"].ravel()
    peak = weights.max()
    # The reference keeps per-angle IQ in complex64 (sim.py:344-393): agreement to its rounding.
    np.testing.assert_allclose(weights / peak, ref_w, rtol=2e-6, atol=1e-6)
    np.testing.assert_allclose(methods.st_sw_power(*args), s[f"{tag}_k{k}_power"].ravel(), rtol=2e-6, atol=1e-6)


@pytest.mark.parametrize("fnumber", [None, 1.0])
def test_c_das_matches_numpy_restatement(g, fnumber):
    """The C oracle (float64, threaded) equals the NumPy restatement, including on the
    reference's golden target case."""
    from oracle import c_das

    rng = np.random.default_rng(7)
    iq = (rng.normal(size=(80, 9, 3, 6)) + 1j * rng.normal(size=(80, 9, 3, 6))).astype(np.complex64)
    el = np.linspace(-1e-3, 1e-3, 9)
    ang, st = np.array([-0.1, 0.0, 0.08]), np.array([1e-6, 1.4e-6, 2e-6])
    scan = _grid_scan(np.linspace(-1e-3, 1e-3, 5), np.linspace(1e-3, 3e-3, 7), np.linspace(-1e-3, 1e-3, 4))
    for config in ("RC", "CR"):
        want = das.aperture_das(iq, scan, el, ang, st, 1540.0, 20e6, 3e6, fnumber, config)
        got = np.zeros_like(want)
        c_das.aperture_accumulate(got, iq, scan, el, ang, st, 1540.0, 20e6, 3e6, fnumber, config)
        assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()
    scan = _grid_scan(g["target_x"], g["target_z"], g["target_y"])
    for config in ("RC", "CR"):
        iq = g["target_rc"] if config == "RC" else g["target_cr"]
        ref = g[f"target_{config}_per_angle"].reshape(len(scan), -1, iq.shape[-1] if iq.ndim == 4 else 1).sum(1)
        got = np.zeros((len(scan), ref.shape[-1]), dtype=np.complex128)
        c_das.aperture_accumulate(got, iq, scan, g["target_el"], g["target_angles"], float(g["target_t0"]), 1540.0,
                                  20e6, 15e6, 1.0, config)
        assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-6


def test_scene_model_matches_reference_simulate_point():
    """The scene forward model (a sum over scatterers of the reference's Gaussian-pulse
    simulate_point, truncated at 4 sigma_t) reproduces the reference's own channel IQ of
    single static points, and superposes them."""
    from oracle import scene

    s = np.load(GOLDEN / "scene.npz")
    pts, ang = s["points"], s["angles"]
    starts = np.full(len(ang), float(s["t_start"]))
    for config, el in (("RC", s["el_x"]), ("CR", s["el_y"])):
        total = 0
        for i, p in enumerate(pts):
            table = np.zeros((1, 11))
            table[0, :3], table[0, 9] = p, 1.0
            got = scene.simulate(table, el, ang, starts, int(s["nsamp"]), 1, prf=500.0, c=1540.0, fs=20e6, fd=15e6,
                                 sigma_t=0.15e-6, half_width=0.6e-6, config=config)[..., 0]
            ref = s[f"point{i}_{config}"]
            assert np.abs(got - ref).max() <= 2e-6 * np.abs(ref).max()
            total = total + ref
        table = np.zeros((len(pts), 11))
        table[:, :3], table[:, 9] = pts, 1.0
        both = scene.simulate(table, el, ang, starts, int(s["nsamp"]), 1, prf=500.0, c=1540.0, fs=20e6, fd=15e6,
                              sigma_t=0.15e-6, half_width=0.6e-6, config=config)[..., 0]
        assert np.abs(both - total).max() <= 4e-6 * np.abs(total).max()
