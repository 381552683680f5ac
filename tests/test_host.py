"""Host logic that runs without a GPU: C ABI exports, validation, geometry helpers."""

from __future__ import annotations

import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

import rcabeam_b200 as rb
from rcabeam_b200 import _lib
from rcabeam_b200.sim import RCAGeometry, scan_coords, simulate_point

ROOT = Path(__file__).resolve().parent.parent
GOLDEN = Path(__file__).resolve().parent / "golden"


def declared_functions() -> list[str]:
    text = (ROOT / "include" / "rcabeam.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return re.findall(r"\b(rcabeam_\w+)\s*\(", text)


def test_library_exports_every_declared_symbol(built_library):
    names = declared_functions()
    assert len(names) == len(set(names)) >= 17
    handle = ctypes.CDLL(str(built_library))
    for name in names:
        assert hasattr(handle, name), name
    # The ctypes tables cover every declaration with the right arity.
    assert set(_lib.SIGNATURES) | {"rcabeam_status_string"} == set(names)
    text = re.sub(r"/\*.*?\*/", "", (ROOT / "include" / "rcabeam.h").read_text(), flags=re.S)
    for name, args in _lib.SIGNATURES.items():
        decl = re.search(name + r"\s*\((.*?)\);", text, flags=re.S).group(1)
        assert decl.count(",") + 1 == len(args), name


def test_status_strings(built_library):
    lib = _lib.lib()
    assert lib.rcabeam_status_string(0) == b"success"
    assert lib.rcabeam_status_string(1) == b"cuda error"
    assert lib.rcabeam_status_string(2) == b"invalid argument"


def test_argument_rejection_without_gpu(built_library):
    """Null pointers and bad sizes are rejected before any launch (reference ensemble.cu:664-675)."""
    lib = _lib.lib()
    null = None
    assert lib.rcabeam_pack_ensemble_device(null, null, 1, 1, 1, 1) == 2
    assert lib.rcabeam_ensemble_device(*([null] * 12), 2, 1, 1, 1, 1, 1540.0, 1.0, 0.0, -1.0, 0, 2) == 2
    assert lib.rcabeam_opw_device(null, null, 1, 1, 1) == 2
    bogus = ctypes.c_void_p(16)
    # Valid pointers but ns < 2, method out of range, non-finite or nonpositive c.
    args = [bogus] * 12
    assert lib.rcabeam_ensemble_device(*args, 1, 1, 1, 1, 1, 1540.0, 1.0, 0.0, -1.0, 0, 2) == 2
    assert lib.rcabeam_ensemble_device(*args, 4, 1, 1, 1, 1, 1540.0, 1.0, 0.0, -1.0, 6, 2) == 2
    assert lib.rcabeam_ensemble_device(*args, 4, 1, 1, 1, 1, float("nan"), 1.0, 0.0, -1.0, 0, 2) == 2
    assert lib.rcabeam_ensemble_device(*args, 4, 1, 1, 1, 1, -1.0, 1.0, 0.0, -1.0, 0, 2) == 2
    # FP16 with an odd (2-byte) pointer.
    assert lib.rcabeam_opw_fp16_device(ctypes.c_void_p(18), *([bogus] * 9), 4, 1, 1, 1, 1, 1540.0, 1.0, 0.0,
                                       -1.0) == 2
    # Tensor-core Gram: complex128 input, odd frame count, T > 1024, unaligned rows, unknown precision.
    assert lib.rcabeam_gram_accumulate_device(bogus, 8, 8, 1, bogus, 2, bogus) == 2
    assert lib.rcabeam_gram_accumulate_device(bogus, 8, 7, 0, bogus, 3, bogus) == 2
    assert lib.rcabeam_gram_accumulate_device(bogus, 8, 1026, 0, bogus, 2, bogus) == 2
    assert lib.rcabeam_gram_accumulate_device(ctypes.c_void_p(24), 8, 8, 0, bogus, 3, bogus) == 2
    assert lib.rcabeam_gram_accumulate_device(bogus, 8, 8, 0, bogus, 4, bogus) == 2
    size = ctypes.c_size_t(0)
    assert lib.rcabeam_ensemble_workspace_bytes(1000, 4, 2, ctypes.byref(size)) == 0
    assert 0 < size.value <= 2 * 1000 * 6 * 16


def test_python_validation_messages():
    rc = np.zeros((3, 2, 2, 0), dtype=np.complex64)
    geom = RCAGeometry(x_el=np.zeros(2), y_el=np.zeros(2))
    grid = (np.ones(1), np.ones(1), np.ones(1))
    with pytest.raises(ValueError, match="nonempty"):
        rb.ensemble_pd_from_channels(rc, rc, np.zeros(2), 0, grid, geom)
    with pytest.raises(ValueError, match="complex signal"):
        rb.beamform_ensemble(rc, rc, np.zeros(2), 0, grid, geom, method="dmas")
    data = np.zeros((48, 1, 2, 3), dtype=np.complex64)
    g1 = RCAGeometry(np.zeros(1), np.zeros(1), fs=2e6, f_demod=1e6)
    with pytest.raises(ValueError, match="OPW only"):
        rb.ensemble_pd_from_channels(data, data, np.zeros(2), 1e-6, (np.zeros(1), np.ones(1), np.zeros(1)), g1,
                                     method="xdoppler", iq_storage="float16")
    with pytest.raises(ValueError, match="F-number"):
        rb.ensemble_pd_from_channels(data, data, np.zeros(2), 1e-6, (np.zeros(1), np.ones(1), np.zeros(1)),
                                     RCAGeometry(np.zeros(1), np.zeros(1), fnumber=-1.0))
    # St-SW subsets: 2 <= k <= 4 and at least k angles (reference ensemble.py:80-81).
    for k, angles in ((1, 2), (5, 2), (3, 2)):
        with pytest.raises(ValueError, match="St-SW requires"):
            rb.ensemble_pd_from_channels(data[:, :, :angles], data[:, :, :angles], np.zeros(angles), 1e-6,
                                         (np.zeros(1), np.ones(1), np.zeros(1)), g1, method="st_sw", k=k)


def test_st_sw_argument_rejection_without_gpu(built_library):
    """Method 4 needs weights and workspace, no signal, 2 <= k <= 4 and na >= k (reference ensemble.cu:671-673)."""
    lib = _lib.lib()
    b = ctypes.c_void_p(16)
    head = [b] * 8  # rc, cr, scan, xe, ye, angles, starts, pd
    ok_tail = (4, 1, 2, 3, 1, 1540.0, 1.0, 0.0, -1.0, 4)
    assert lib.rcabeam_ensemble_device(*head, None, None, b, b, *ok_tail, 2) == 2   # no weights
    assert lib.rcabeam_ensemble_device(*head, None, b, None, b, *ok_tail, 2) == 2   # no workspace
    assert lib.rcabeam_ensemble_device(*head, b, b, b, b, *ok_tail, 2) == 2        # signal given
    assert lib.rcabeam_ensemble_device(*head, None, b, b, b, *ok_tail, 1) == 2     # k < 2
    assert lib.rcabeam_ensemble_device(*head, None, b, b, b, *ok_tail, 3) == 2     # na = 2 < k
    assert lib.rcabeam_ensemble_device(*head, None, b, b, b, *ok_tail, 5) == 2     # k > 4
    # The no-allocation entry point has no series workspace and rejects St-SW.
    assert lib.rcabeam_ensemble_static_device(*head, None, 4, 1, 2, 3, 1, 1540.0, 1.0, 0.0, -1.0, 4) == 2


def test_filtered_pipeline_domain_rejected_without_gpu():
    from rcabeam_b200.pipeline import FilteredOpw

    with pytest.raises(ValueError, match="domain"):
        FilteredOpw((8, 2, 1, 4), np.zeros(1), 1e-6, (np.zeros(1), np.ones(1), np.zeros(1)),
                    RCAGeometry(np.zeros(2), np.zeros(2)), domain="image")


def test_voxel_order_matches_reference_golden():
    order = np.load(GOLDEN / "order.npz")
    for key in order.files:
        shape = tuple(int(s) for s in key.split("_")[1].split("x"))
        got = rb.opw_voxel_order(shape)
        np.testing.assert_array_equal(got, order[key])
        np.testing.assert_array_equal(np.sort(got), np.arange(np.prod(shape)))
    with pytest.raises(ValueError):
        rb.opw_voxel_order((0, 2, 4))


def test_scan_coords_layout():
    x, z, y = np.array([0.0, 1.0]), np.array([2.0, 3.0, 4.0]), np.array([5.0, 6.0])
    s = scan_coords((x, z, y))
    assert s.dtype == np.float32 and s.shape == (12, 3)
    np.testing.assert_array_equal(s[:3], [[0, 2, 5], [0, 2, 6], [0, 3, 5]])
    np.testing.assert_array_equal(s[-1], [1, 4, 6])


def test_simulate_point_matches_reference():
    g = np.load(GOLDEN / "das.npz")
    el = g["target_el"]
    geom = RCAGeometry(el, el, c=1540.0, fs=20e6, f_demod=15e6, fnumber=1.0)
    for config in ("RC", "CR"):
        mine = simulate_point(geom, g["target_angles"], (0.3e-3, 5.0e-3, -0.2e-3), 256, float(g["target_t0"]),
                              config)[::2]
        np.testing.assert_allclose(mine, g[f"point_{config.lower()}"], rtol=1e-5, atol=1e-6)


def test_depth_axis():
    axis = rb.depth_axis(4e-3, 12e-3, 15e6)
    assert axis[0] == 4e-3 and axis[-1] == 12e-3
    assert np.all(np.diff(axis) <= 1540 / (2 * 15e6) + 1e-15)
    with pytest.raises(ValueError):
        rb.depth_axis(2.0, 1.0, 1e6)
