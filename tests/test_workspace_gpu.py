"""OpwWorkspace: ownership, borrowed outputs, no warm allocation, context checks (reference test_gpu_workspace.py)."""

from __future__ import annotations

import numpy as np
import pytest
import torch

import rcabeam_b200 as rb
from rcabeam_b200 import _lib
from rcabeam_b200.sim import RCAGeometry
from tests._cases import rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs CUDA")
    yield
    assert _lib.device_error() == 0


@pytest.mark.parametrize("storage", ["float32", "float16"])
@pytest.mark.parametrize("spatial", [False, True])
@pytest.mark.parametrize("frames", [3, 8, 66])
def test_workspace_reuses_buffers(storage, spatial, frames):
    rng = np.random.default_rng(222)
    shape = (48, 3, 4, frames)
    rc = (rng.normal(size=shape) + 1j * rng.normal(size=shape)).astype(np.complex64)
    cr = (rng.normal(size=shape) + 1j * rng.normal(size=shape)).astype(np.complex64)
    el = np.linspace(-0.001, 0.001, 3)
    geom = RCAGeometry(el, el, fs=2e6, f_demod=1e6)
    angles = np.linspace(-0.1, 0.1, 4)
    grid = (np.linspace(-0.001, 0.001, 3), np.array([0.005, 0.007]), np.linspace(-0.001, 0.003, 5))
    expected = rb.beamform_ensemble(rc, cr, angles, 1e-6, grid, geom, iq_storage=storage)
    ws = rb.OpwWorkspace(shape, angles, 1e-6, grid, geom, iq_storage=storage, spatial_order=spatial)
    with pytest.raises(RuntimeError, match="Pack"):
        ws.reconstruct()
    ws.pack(torch.from_numpy(rc).cuda(), torch.from_numpy(cr).cuda())
    actual = ws.reconstruct()
    np.testing.assert_allclose(actual.cpu().numpy(), expected, rtol=1e-4, atol=1e-4)
    np.testing.assert_allclose(ws.power.cpu().numpy(), np.mean(abs(expected) ** 2, axis=-1), rtol=1e-4, atol=1e-4)
    pointer = actual.data_ptr()
    angles[:] = 999  # metadata is a construction-time snapshot
    torch.cuda.synchronize()
    before = torch.cuda.memory_stats()["allocation.all.allocated"]
    again = ws.reconstruct()
    assert torch.cuda.memory_stats()["allocation.all.allocated"] == before  # warmed: no device allocation
    assert again.data_ptr() == pointer
    np.testing.assert_allclose(again.cpu().numpy(), expected, rtol=1e-4, atol=1e-4)
    ws.pack(torch.from_numpy(rc * 2).cuda(), torch.from_numpy(cr * 2).cuda())
    assert ws.reconstruct().data_ptr() == pointer
    assert rel_l2(actual.cpu().numpy(), expected * 2) < 1e-5


def test_workspace_rejects_stale_packs_and_streams():
    shape = (48, 1, 1, 3)
    axis = np.array([0.0])
    geom = RCAGeometry(axis, axis, fs=2e6, f_demod=1e6)
    grid = (axis, np.array([0.005]), axis)
    data = torch.zeros(shape, dtype=torch.complex64, device="cuda")
    ws = rb.OpwWorkspace(shape, axis, 0.0, grid, geom, iq_storage="float16")
    ws.pack(data, data)
    ws.reconstruct()
    data[0, 0, 0, 0] = 70000
    with pytest.raises(ValueError, match="FP16 IQ"):
        ws.pack(data, data)
    with pytest.raises(RuntimeError, match="Pack"):
        ws.reconstruct()
    with pytest.raises(RuntimeError, match="reading power"):
        _ = ws.power
    with pytest.raises(ValueError, match="complex64 CUDA"):
        ws.pack(np.zeros(shape, np.complex64), data)
    with torch.cuda.stream(torch.cuda.Stream()), pytest.raises(ValueError, match="default CUDA stream"):
        ws.reconstruct()
    with pytest.raises(ValueError, match="IQ storage"):
        rb.OpwWorkspace(shape, axis, 0.0, grid, geom, iq_storage="invalid")


def test_workspace_large_lateral_plane():
    """A partial last tile with odd lateral tails (reference test_gpu_workspace.py:154-166)."""
    shape = (32, 2, 2, 8)
    rng = np.random.default_rng(22)
    rc = (rng.normal(size=shape) + 1j * rng.normal(size=shape)).astype(np.complex64)
    el = np.array([-0.001, 0.001])
    angles = np.array([-0.1, 0.1])
    grid = (np.linspace(-0.001, 0.001, 65), np.array([0.005]), np.linspace(-0.001, 0.001, 253))
    geom = RCAGeometry(el, el, fs=2e6, f_demod=1e6)
    ws = rb.OpwWorkspace(shape, angles, 0.0, grid, geom, spatial_order=True)
    ws.pack(torch.from_numpy(rc).cuda(), torch.from_numpy(rc).cuda())
    expected = rb.beamform_ensemble(rc, rc, angles, 0.0, grid, geom)
    np.testing.assert_allclose(ws.reconstruct().cpu().numpy(), expected, rtol=1e-4, atol=1e-4)
