"""Seeded scenes through every OPW form, against the float64 oracle.

* The forward-model kernel (``rcabeam_simulate_scene_device``) against its float64
  restatement ``oracle.scene`` (moving, wrapping scatterers; both apertures).
* Config 1 at its exact shapes -- 64 + 64 elements, IQ (256, 64, 5, 16), grid
  32 x 64 x 32, 5 unit targets + 2000 speckle + 20 dB noise -- and a reduced
  tissue / blood / noise flow scene, each through ``FilteredOpw`` in the plain
  form (float32 SIMT DAS, float64 Gram), the chosen form (split-BF16 tensor-core
  DAS, 3xBF16 tensor-core Gram) and the FP16-storage form, against the float64
  oracle chain (C oracle DAS -> complex128 Gram -> eigh -> filtered power).
  Bar: relative L2 <= 1e-4 of the filtered (and unfiltered) power; the FP16 form
  is held to the same bar against the oracle run on its FP16-quantized channels
  (the reference's FP16 test convention, tests/test_opw_fp16.py:30-37).
"""

from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

from oracle import c_das  # noqa: E402
from oracle import clutter as oc  # noqa: E402
from oracle import scene as osc  # noqa: E402
from rcabeam_b200 import pipeline, scenes  # noqa: E402
from rcabeam_b200.sim import RCAGeometry  # noqa: E402
from tests._cases import oracle_inputs, rel_l2  # noqa: E402

FORMS = {"plain": ("float32", "complex128"), "chosen": ("bf16x2", "bf16x3"), "fp16": ("float16", "complex128")}


def _fp16_quantized(x: np.ndarray) -> np.ndarray:
    return (x.real.astype(np.float16).astype(np.float32) + 1j * x.imag.astype(np.float16).astype(np.float32)).astype(
        np.complex64)


def _oracle_chain(rc, cr, scene, rank_start):
    o = oracle_inputs(scene.angles, scene.t_start, scene.grid, scene.geom)
    iq = c_das.opw_iq(rc, cr, o["scan"], o["xe"], o["ye"], o["angles"], o["starts"], o["c"], o["fs"], o["fd"],
                      o["fnumber"])
    _, basis = oc.temporal_basis(iq, method="gram")
    filtered = oc.filtered_power(iq, basis, rank_start)
    unfiltered = np.mean(np.abs(iq) ** 2, axis=-1)
    return filtered, unfiltered


def _run_forms(scene, rank_start):
    rc_h, cr_h = scene.rc.cpu().numpy(), scene.cr.cpu().numpy()
    exact = _oracle_chain(rc_h, cr_h, scene, rank_start)
    quant = _oracle_chain(_fp16_quantized(rc_h), _fp16_quantized(cr_h), scene, rank_start)
    errors = {}
    for name, (storage, precision) in FORMS.items():
        plan = pipeline.FilteredOpw(tuple(scene.rc.shape), scene.angles, scene.t_start, scene.grid, scene.geom,
                                    rank_start=rank_start, precision=precision, iq_storage=storage)
        got = plan.run(scene.rc, scene.cr).cpu().numpy().ravel()
        plan.check()
        unfiltered = plan.pd[:, 0].double().cpu().numpy()
        want_f, want_u = quant if name == "fp16" else exact
        errors[name] = (rel_l2(got, want_f), rel_l2(unfiltered, want_u))
    for name, (ef, eu) in errors.items():
        print(f"{scene.info['scene']}: {name:6s} filtered PD rel L2 {ef:.3e}, unfiltered PD {eu:.3e}")
    return errors


def test_forward_model_matches_float64_restatement():
    """Moving scatterers (one wrapping through a periodic tube) rendered on the GPU equal the float64
    restatement to float32 rounding, for both apertures."""
    rng = np.random.default_rng(3)
    el = (np.arange(12) - 5.5) * 0.2e-3
    geom = RCAGeometry(el, el * 1.1, c=1540.0, fs=20e6, f_demod=15e6, fnumber=None)
    angles = np.deg2rad([-6.0, 0.0, 7.0])
    pos = rng.uniform([-1e-3, 4e-3, -1e-3], [1e-3, 6e-3, 1e-3], (30, 3))
    amp = rng.standard_normal(30) + 1j * rng.standard_normal(30)
    d = rng.normal(size=(30, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    table = scenes.scatterer_table(pos, amplitude=amp, direction=d, speed=rng.uniform(0, 40e-3, 30),
                                   s0=rng.uniform(0, 1e-3, 30), period=np.where(np.arange(30) % 3 == 0, 1.2e-3, 0.0))
    ns, nt, t0 = 200, 10, 4.5e-6
    rc, cr = scenes.render(table, geom, angles, t0, ns, nt, prf=200.0)
    for got, config, elements in ((rc, "RC", geom.x_el), (cr, "CR", geom.y_el)):
        want = osc.simulate(table, elements, angles, np.full(3, t0), ns, nt, prf=200.0, c=1540.0, fs=20e6, fd=15e6,
                            sigma_t=scenes.SIGMA_T, half_width=4 * scenes.SIGMA_T, config=config)
        assert np.abs(want).max() > 1.0  # the scatterers are inside the window
        assert rel_l2(got.cpu().numpy(), want) < 2e-6


def test_config1_scene_every_form_matches_fp64_oracle():
    """Config 1 at its exact shapes: unfiltered PD (the configuration's metric) and the
    filtered PD with the static scene's rank removed (rank_start = 1)."""
    scene = scenes.config1_scene(seed=11)
    assert tuple(scene.rc.shape) == (256, 64, 5, 16)
    errors = _run_forms(scene, rank_start=1)
    for name, (ef, eu) in errors.items():
        assert ef <= 1e-4, f"{name}: filtered PD {ef:.3e}"
        assert eu <= 1e-4, f"{name}: unfiltered PD {eu:.3e}"


def test_config1_scene_split_inside_the_noise_band():
    """rank_start = 3 on the static scene removes the scene's rank and two of the 15 noise
    ranks, whose eigenvalues lie within a few percent of each other: the per-voxel filtered
    power then moves to first order with any rotation of the Gram inside that band.  Forms
    with a float64 Gram stay within 1e-4 of the float64 chain; the 3xBF16 Gram's rounding
    rotates the split by ~1e-4 (printed, bounded at 2e-4), which a float64 Gram on the same
    split-BF16 DAS, or the float64 Rayleigh-Ritz correction (``refine=True``), removes."""
    scene = scenes.config1_scene(seed=11)
    rc_h, cr_h = scene.rc.cpu().numpy(), scene.cr.cpu().numpy()
    want, _ = _oracle_chain(rc_h, cr_h, scene, 3)
    got = {}
    for storage, precision, refine in (("float32", "complex128", False), ("bf16x2", "complex128", False),
                                       ("bf16x2", "bf16x3", False), ("bf16x2", "bf16x3", True)):
        plan = pipeline.FilteredOpw(tuple(scene.rc.shape), scene.angles, scene.t_start, scene.grid, scene.geom,
                                    rank_start=3, precision=precision, iq_storage=storage, refine=refine)
        got[(storage, precision, refine)] = rel_l2(plan.run(scene.rc, scene.cr).cpu().numpy().ravel(), want)
        plan.check()
        print(f"config 1, rank_start 3: DAS {storage:8s} Gram {precision:10s} refine {int(refine)} "
              f"filtered PD rel L2 {got[(storage, precision, refine)]:.3e}")
    assert got[("float32", "complex128", False)] <= 1e-4
    assert got[("bf16x2", "complex128", False)] <= 1e-4
    assert got[("bf16x2", "bf16x3", False)] <= 2e-4
    # The float64 Rayleigh-Ritz step on the 16 leading vectors (all 16 frames here) is exact.
    assert got[("bf16x2", "bf16x3", True)] <= 1e-4


def test_config1_scene_fnumber_one():
    """Config 1 with the reference's default receive f-number 1 (aperture-limited)."""
    scene = scenes.config1_scene(seed=12, fnumber=1.0)
    errors = _run_forms(scene, rank_start=1)
    for name, (ef, eu) in errors.items():
        assert ef <= 1e-4 and eu <= 1e-4, f"{name}: {ef:.3e} {eu:.3e}"


def test_flow_scene_every_form_matches_fp64_oracle():
    """A reduced tissue (0 dB, 1 mm/s) / blood (-40 dB, 10-30 mm/s tube) / noise (-50 dB) scene:
    the clutter filter removes the tissue band, so the filtered power is ~40 dB below the
    channel data -- the case that exposes per-sample rounding of the tensor-core forms."""
    scene = scenes.flow_scene(channels=32, samples=192, angles=5, frames=64, grid_shape=(24, 48, 24),
                              depth=(6e-3, 10e-3), t_start=7e-6, n_tissue=700, n_blood=400, tube_radius=0.5e-3,
                              seed=21)
    errors = _run_forms(scene, rank_start=3)
    for name, (ef, eu) in errors.items():
        assert ef <= 1e-4, f"{name}: filtered PD {ef:.3e}"
        assert eu <= 1e-4, f"{name}: unfiltered PD {eu:.3e}"
