"""Device orchestration of the frame-batched path through the C ABI.

Mirrors the reference nanobind module ``rcabeam._cuda_impl``
(src/rcabeam/bindings/python.cpp:495-652): ``ensemble_from_channels``,
``pack_opw_channels`` and ``opw_from_packed`` take the same arguments in the
same order.  Host (NumPy) inputs are uploaded and host outputs downloaded;
CUDA ``torch.Tensor`` inputs/outputs are used in place.  Device memory comes
from torch's caching allocator; all kernels run on the legacy default stream.
"""

from __future__ import annotations

import ctypes
import time

import numpy as np
import torch

from rcabeam_b200 import _lib

_COMPLEX64 = (np.complex64, torch.complex64)
# Device scratch for the St-SW correlation series of one voxel tile.
_STSW_SCRATCH_BYTES = 256 << 20


def _ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None or t.numel() == 0 else t.data_ptr()


def _device() -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError("rcabeam_b200 requires a CUDA device")
    return torch.device("cuda", torch.cuda.current_device())


def _to_device(a, dtype: torch.dtype) -> torch.Tensor:
    if isinstance(a, torch.Tensor):
        if not a.is_cuda:
            return a.to(_device(), dtype=dtype, non_blocking=False).contiguous()
        return a.to(dtype=dtype).contiguous()
    arr = np.ascontiguousarray(a)
    if not arr.flags.writeable:
        arr = arr.copy()
    return torch.from_numpy(arr).to(_device(), dtype=dtype)


def workspace_bytes(nv: int, nc: int, na: int) -> int:
    """Geometry-workspace bytes ``rcabeam_ensemble_device`` uses for ``nv`` voxels.

    The C ABI documents 2 * nv * (nc + na) float4 of caller scratch; this
    implementation forms delays on the fly and needs only the buffers of its
    traversal-order sort, a small fraction of that.
    """
    out = ctypes.c_size_t(0)
    _lib.check(_lib.lib().rcabeam_ensemble_workspace_bytes(nv, nc, na, ctypes.byref(out)), "workspace_bytes")
    return int(out.value)


def _storage(half_storage) -> str:
    """Packed storage name: False/"float32", True/"float16", or "bf16x2"."""
    if half_storage in (False, None, "float32"):
        return "float32"
    if half_storage in (True, "float16"):
        return "float16"
    if half_storage == "bf16x2":
        return "bf16x2"
    raise ValueError(f"unknown IQ storage {half_storage!r}")


def ensemble_from_channels(rc, cr, scan, xe, ye, angles, starts, pd, signal, weights, c, fs, fd, fn, method, k,
                           half_storage) -> float:
    """Upload, pack and reconstruct one ensemble; returns raw-upload wall seconds.

    ``half_storage`` is the reference's FP16 flag; ``"bf16x2"`` selects the
    split-BF16 tensor-core path (OPW only, frames a multiple of 4).
    """
    storage = _storage(half_storage)
    ns, nc, na, nt = rc.shape
    nv = scan.shape[0]
    if tuple(cr.shape) != tuple(rc.shape):
        raise ValueError("RC/CR ensemble shapes must match")
    if ns < 2 or not nc or not na or not nt or not nv or method < 0 or method > 5:
        raise ValueError("invalid ensemble dimensions or method")
    if storage != "float32" and method != 0:
        raise ValueError("FP16 IQ storage is supported only for OPW")
    if storage == "bf16x2" and nt % 4:
        raise ValueError("bf16x2 storage requires a frame count divisible by 4")
    if method == 4 and (weights is None or len(weights) != nv):
        raise ValueError("invalid ensemble output shapes")
    if method == 4 and (k < 2 or k > 4 or na < k):
        raise ValueError("St-SW needs 2<=k<=4 and at least k angles")
    host_in = not isinstance(rc, torch.Tensor) or not rc.is_cuda
    begin = time.perf_counter()
    d_rc = _to_device(rc, torch.complex64)
    d_cr = _to_device(cr, torch.complex64)
    if host_in:
        torch.cuda.synchronize()
    upload = time.perf_counter() - begin if host_in else 0.0
    d_scan = _to_device(scan, torch.float32)
    d_xe, d_ye = _to_device(xe, torch.float32), _to_device(ye, torch.float32)
    d_angles, d_starts = _to_device(angles, torch.float32), _to_device(starts, torch.float32)
    dev = d_rc.device
    host_pd = not isinstance(pd, torch.Tensor) or not pd.is_cuda
    d_pd = torch.empty((nv, 2), dtype=torch.float32, device=dev) if host_pd else pd
    planes = 2 if method == 5 else 1
    want_signal = signal is not None and (signal.shape[0] if hasattr(signal, "shape") else 0) > 0
    host_sig = want_signal and (not isinstance(signal, torch.Tensor) or not signal.is_cuda)
    if want_signal:
        d_sig = torch.empty((nv * planes, nt), dtype=torch.complex64, device=dev) if host_sig else signal
    else:
        d_sig = None
    elem = 8 if storage == "float32" else 4
    packed_rc = torch.empty(ns * nc * na * nt * elem, dtype=torch.uint8, device=dev)
    packed_cr = torch.empty_like(packed_rc)
    geometry = torch.empty(workspace_bytes(nv, nc, na), dtype=torch.uint8, device=dev)
    flag = torch.zeros(1, dtype=torch.int32, device=dev)
    if storage == "float16":
        for src, dst in ((d_rc, packed_rc), (d_cr, packed_cr)):
            _lib.call("rcabeam_pack_ensemble_fp16_device", src.data_ptr(), dst.data_ptr(), flag.data_ptr(),
                      ns, nc, na, nt)
        if int(flag.item()):
            raise ValueError("FP16 IQ requires finite components within +/-65504; rescale inputs explicitly")
        _lib.call("rcabeam_opw_fp16_device", packed_rc.data_ptr(), packed_cr.data_ptr(), d_scan.data_ptr(),
                  d_xe.data_ptr(), d_ye.data_ptr(), d_angles.data_ptr(), d_starts.data_ptr(), d_pd.data_ptr(),
                  _ptr(d_sig), geometry.data_ptr(), ns, nc, na, nt, nv, c, fs, fd, fn)
    elif storage == "bf16x2":
        lo_rc = torch.empty_like(packed_rc)
        lo_cr = torch.empty_like(packed_rc)
        for src, hi, lo in ((d_rc, packed_rc, lo_rc), (d_cr, packed_cr, lo_cr)):
            _lib.call("rcabeam_pack_ensemble_split_device", src.data_ptr(), hi.data_ptr(), lo.data_ptr(),
                      flag.data_ptr(), ns, nc, na, nt)
        if int(flag.item()):
            raise ValueError("bf16x2 IQ storage requires finite channel data")
        _lib.call("rcabeam_opw_tc_device", packed_rc.data_ptr(), lo_rc.data_ptr(), packed_cr.data_ptr(),
                  lo_cr.data_ptr(), d_scan.data_ptr(), d_xe.data_ptr(), d_ye.data_ptr(), d_angles.data_ptr(),
                  d_starts.data_ptr(), d_pd.data_ptr(), _ptr(d_sig), geometry.data_ptr(), ns, nc, na, nt, nv, c, fs,
                  fd, fn, 1)
    elif method == 4:
        # St-SW keeps k^2 correlation series per voxel and frame: voxel tiles
        # bound that scratch (reference python.cpp:553-565 tiles for the same reason).
        for src, dst in ((d_rc, packed_rc), (d_cr, packed_cr)):
            _lib.call("rcabeam_pack_ensemble_device", src.data_ptr(), dst.data_ptr(), ns, nc, na, nt)
        tile = max(1, min(nv, _STSW_SCRATCH_BYTES // (k * k * nt * 8)))
        series = torch.empty(tile * k * k * nt, dtype=torch.complex64, device=dev)
        d_w = torch.empty(nv, dtype=torch.float32, device=dev)
        for v0 in range(0, nv, tile):
            count = min(tile, nv - v0)
            _lib.call("rcabeam_ensemble_device", packed_rc.data_ptr(), packed_cr.data_ptr(),
                      d_scan.data_ptr() + 12 * v0, d_xe.data_ptr(), d_ye.data_ptr(), d_angles.data_ptr(),
                      d_starts.data_ptr(), d_pd.data_ptr() + 8 * v0, None, d_w.data_ptr() + 4 * v0,
                      series.data_ptr(), geometry.data_ptr(), ns, nc, na, nt, count, c, fs, fd, fn, method, k)
        if isinstance(weights, torch.Tensor) and weights.is_cuda:
            weights.copy_(d_w)
        else:
            torch.cuda.synchronize()
            np.copyto(np.asarray(weights).reshape(nv), d_w.cpu().numpy())
    else:
        for src, dst in ((d_rc, packed_rc), (d_cr, packed_cr)):
            _lib.call("rcabeam_pack_ensemble_device", src.data_ptr(), dst.data_ptr(), ns, nc, na, nt)
        _lib.call("rcabeam_ensemble_device", packed_rc.data_ptr(), packed_cr.data_ptr(), d_scan.data_ptr(),
                  d_xe.data_ptr(), d_ye.data_ptr(), d_angles.data_ptr(), d_starts.data_ptr(), d_pd.data_ptr(),
                  _ptr(d_sig), None, None, geometry.data_ptr(), ns, nc, na, nt, nv, c, fs, fd, fn, method, k)
    torch.cuda.synchronize()
    if _lib.device_error():
        raise _lib.RcabeamCudaError("a reconstruction kernel timed out waiting on its staging pipeline")
    if host_pd:
        np.copyto(np.asarray(pd).reshape(nv, 2), d_pd.cpu().numpy())
    if host_sig:
        np.copyto(np.asarray(signal).reshape(nv * planes, nt), d_sig.cpu().numpy())
    return upload


def _require_device(t, device: int, name: str) -> None:
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise ValueError(f"resident buffers must be CUDA arrays ({name})")
    if t.device.index != device:
        raise ValueError(f"resident buffers must belong to the current CUDA device ({name})")


def pack_opw_channels(rc, cr, packed_rc, packed_cr, range_error, half_storage) -> None:
    """Pack resident complex64 RC/CR into owned buffers (python.cpp:583-614)."""
    ns, nc, na, nt = rc.shape
    if ns < 2 or not nc or not na or not nt:
        raise ValueError("invalid channel dimensions")
    if tuple(cr.shape) != tuple(rc.shape):
        raise ValueError("RC/CR shapes must match")
    nbytes = ns * nc * na * nt * (4 if half_storage else 8)
    if packed_rc.numel() != nbytes or packed_cr.numel() != nbytes or range_error.numel() != 1:
        raise ValueError("invalid packed buffer sizes")
    device = torch.cuda.current_device()
    for name, t in (("rc", rc), ("cr", cr), ("packed_rc", packed_rc), ("packed_cr", packed_cr),
                    ("range_error", range_error)):
        _require_device(t, device, name)
    if half_storage:
        range_error.zero_()
        _lib.call("rcabeam_pack_ensemble_fp16_device", rc.data_ptr(), packed_rc.data_ptr(), range_error.data_ptr(),
                  ns, nc, na, nt)
        _lib.call("rcabeam_pack_ensemble_fp16_device", cr.data_ptr(), packed_cr.data_ptr(), range_error.data_ptr(),
                  ns, nc, na, nt)
        if int(range_error.item()):
            raise ValueError("FP16 IQ requires finite components within +/-65504; rescale inputs explicitly")
    else:
        _lib.call("rcabeam_pack_ensemble_device", rc.data_ptr(), packed_rc.data_ptr(), ns, nc, na, nt)
        _lib.call("rcabeam_pack_ensemble_device", cr.data_ptr(), packed_cr.data_ptr(), ns, nc, na, nt)
    torch.cuda.synchronize()


def opw_from_packed(rc, cr, scan, xe, ye, angles, starts, pd, signal, geometry_workspace, ns, nc, na, nt, c, fs, fd,
                    fn, half_storage, *, synchronize: bool = True) -> None:
    """OPW of resident packed channels into resident pd/signal (python.cpp:616-652)."""
    nv = scan.shape[0]
    nbytes = ns * nc * na * nt * (4 if half_storage else 8)
    if (rc.numel() != nbytes or cr.numel() != nbytes or xe.numel() != nc or ye.numel() != nc
            or angles.numel() != na or starts.numel() != na or pd.shape[0] != nv
            or (signal is not None and tuple(signal.shape) != (nv, nt))
            or geometry_workspace.numel() < workspace_bytes(nv, nc, na)):
        raise ValueError("invalid resident buffer shapes")
    fn_name = "rcabeam_opw_fp16_device" if half_storage else "rcabeam_ensemble_device"
    if half_storage:
        _lib.call(fn_name, rc.data_ptr(), cr.data_ptr(), scan.data_ptr(), xe.data_ptr(), ye.data_ptr(),
                  angles.data_ptr(), starts.data_ptr(), pd.data_ptr(), _ptr(signal),
                  geometry_workspace.data_ptr(), ns, nc, na, nt, nv, c, fs, fd, fn)
    else:
        _lib.call(fn_name, rc.data_ptr(), cr.data_ptr(), scan.data_ptr(), xe.data_ptr(), ye.data_ptr(),
                  angles.data_ptr(), starts.data_ptr(), pd.data_ptr(), _ptr(signal), None, None,
                  geometry_workspace.data_ptr(), ns, nc, na, nt, nv, c, fs, fd, fn, 0, 2)
    if synchronize:
        torch.cuda.synchronize()
        if _lib.device_error():
            raise _lib.RcabeamCudaError("a reconstruction kernel timed out waiting on its staging pipeline")
