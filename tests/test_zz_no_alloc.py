"""The no-allocation ensemble entry point against the workspace entry point.

``rcabeam_ensemble_static_device`` serves callers that cannot allocate device
memory (acquisition loops whose device memory budget is fixed when the scanner
starts, plugins whose host application owns the device allocator): its scratch
lives in a fixed array inside the library.  This file runs last (collection order) so that, if it fails, a
``-x`` run has already run every other test.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

from rcabeam_b200 import _cuda_impl, _lib
from rcabeam_b200.sim import RCAGeometry, scan_coords
from tests._cases import rel_l2

pytestmark = pytest.mark.gpu

MAX_VOXELS = 1 << 18


@pytest.fixture(autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs CUDA")
    yield
    assert _lib.device_error() == 0


def _case(frames=24, nx=16, nz=32, ny=16):
    rng = np.random.default_rng(5)
    el = (np.arange(16) - 7.5) * 0.2e-3
    geom = RCAGeometry(el, el, c=1540.0, fs=20e6, f_demod=15e6, fnumber=1.0)
    angles = np.deg2rad(np.linspace(-8, 8, 3))
    shape = (160, 16, 3, frames)
    rc = (rng.normal(size=shape) + 1j * rng.normal(size=shape)).astype(np.complex64)
    cr = (rng.normal(size=shape) + 1j * rng.normal(size=shape)).astype(np.complex64)
    grid = (np.linspace(-1.5e-3, 1.5e-3, nx), np.linspace(4e-3, 6e-3, nz), np.linspace(-1.5e-3, 1.5e-3, ny))
    return rc, cr, angles, grid, geom


def _device_inputs(rc, cr, angles, grid, geom):
    ns, nc, na, nt = rc.shape
    f32 = lambda v: torch.from_numpy(np.ascontiguousarray(v, dtype=np.float32)).cuda()  # noqa: E731
    packed = []
    for raw in (rc, cr):
        src = torch.from_numpy(np.ascontiguousarray(raw)).cuda()
        dst = torch.empty(ns * nc * na * nt * 8, dtype=torch.uint8, device="cuda")
        _lib.call("rcabeam_pack_ensemble_device", src.data_ptr(), dst.data_ptr(), ns, nc, na, nt)
        packed.append(dst)
    return packed, f32(scan_coords(grid)), f32(geom.x_el), f32(geom.y_el), f32(angles), f32([4e-6] * na)


def _compare(method, rc, cr, angles, grid, geom):
    """Static entry point vs rcabeam_ensemble_device on the same inputs, two calls in a row."""
    ns, nc, na, nt = rc.shape
    (prc, pcr), scan, xe, ye, an, st = _device_inputs(rc, cr, angles, grid, geom)
    nv = scan.shape[0]
    planes = 2 if method == 5 else 1
    with_signal = method in (0, 1, 5)
    consts = (float(geom.c), float(geom.fs), float(geom.f_demod), float(geom.fnumber))
    ref_pd = torch.empty((nv, 2), device="cuda")
    ref_sig = torch.empty((nv * planes, nt), dtype=torch.complex64, device="cuda") if with_signal else None
    ws = torch.empty(_cuda_impl.workspace_bytes(nv, nc, na), dtype=torch.uint8, device="cuda")
    _lib.call("rcabeam_ensemble_device", prc.data_ptr(), pcr.data_ptr(), scan.data_ptr(), xe.data_ptr(), ye.data_ptr(),
              an.data_ptr(), st.data_ptr(), ref_pd.data_ptr(), ref_sig.data_ptr() if with_signal else None, None, None,
              ws.data_ptr(), ns, nc, na, nt, nv, *consts, method, 2)
    torch.cuda.synchronize()
    expected_pd = ref_pd[:, 0].cpu().numpy()
    expected_sig = ref_sig.cpu().numpy() if with_signal else None
    pd = torch.empty((nv, 2), device="cuda")
    sig = torch.empty((nv * planes, nt), dtype=torch.complex64, device="cuda") if with_signal else None
    for _ in range(2):  # two calls in a row share the library's scratch
        pd.fill_(float("nan"))
        if with_signal:
            sig.fill_(float("nan"))
        torch.cuda.synchronize()
        before = torch.cuda.memory_stats().get("allocation.all.allocated", 0)
        free_before = torch.cuda.mem_get_info()[0]
        _lib.call("rcabeam_ensemble_static_device", prc.data_ptr(), pcr.data_ptr(), scan.data_ptr(), xe.data_ptr(),
                  ye.data_ptr(), an.data_ptr(), st.data_ptr(), pd.data_ptr(), sig.data_ptr() if with_signal else None,
                  ns, nc, na, nt, nv, *consts, method)
        torch.cuda.synchronize()
        # Neither torch's allocator nor the driver gave out memory during the call (the driver
        # figure catches a cudaMalloc inside the library; 2 MiB of slack for driver bookkeeping).
        assert torch.cuda.memory_stats().get("allocation.all.allocated", 0) == before
        assert torch.cuda.mem_get_info()[0] >= free_before - (2 << 20)
        if with_signal:
            assert rel_l2(sig.cpu().numpy(), expected_sig) <= 1e-5
            np.testing.assert_allclose(sig.cpu().numpy(), expected_sig, rtol=0,
                                       atol=2e-5 * np.abs(expected_sig).max())
        if method != 5:
            assert rel_l2(pd[:, 0].cpu().numpy(), expected_pd) <= 1e-5


@pytest.mark.parametrize("method", [0, 1, 2, 3, 5])
def test_static_entry_matches_workspace_entry_twice(method):
    _compare(method, *_case())


@pytest.mark.parametrize("method", [0, 3])
def test_static_entry_at_its_voxel_limit(method):
    """262144 voxels (the documented limit): the traversal-order sort fits the fixed scratch."""
    size = ctypes.c_size_t(0)
    assert _lib.lib().rcabeam_voxel_order_workspace_bytes(MAX_VOXELS, ctypes.byref(size)) == 0
    assert 0 < size.value <= 8 << 20
    rc, cr, angles, grid, geom = _case(frames=8, nx=64, nz=64, ny=64)
    _compare(method, rc[:, :8], cr[:, :8], angles, grid,
             RCAGeometry(geom.x_el[:8], geom.y_el[:8], c=geom.c, fs=geom.fs, f_demod=geom.f_demod, fnumber=1.0))


def test_static_entry_rejects_too_many_voxels():
    lib = _lib.lib()
    bogus = ctypes.c_void_p(256)
    status = lib.rcabeam_ensemble_static_device(*([bogus] * 9), 16, 2, 3, 4, MAX_VOXELS + 1, 1540.0, 20e6, 15e6,
                                                 -1.0, 0)
    assert status == 2  # RCABEAM_ERROR_ARGUMENT: beyond the fixed scratch
    assert lib.rcabeam_ensemble_static_device(*([bogus] * 9), 16, 2, 3, 4, 8, 1540.0, 20e6, 15e6, -1.0, 4) == 2
