"""Differentiable OPW power Doppler (the differentiation form of the OPW path).

``opw_power_doppler(rc, cr, delay_offsets, sound_speed, geometry)`` is the
OPW ensemble power Doppler of ``ensemble_pd_from_channels`` (reference
src/rcabeam/ensemble.py:133-218, method "opw") as a ``torch.autograd.Function``
with two extra parameters: a delay offset per receive element of each aperture
(``(2, nc)`` seconds, RC then CR) and the sound speed.  Gradients flow to the
channel IQ of both apertures, the offsets and the sound speed through the
hand-written adjoint kernels of the C ABI (``rcabeam_opw_offsets_*``).

Memory: neither pass keeps the beamformed ensemble.  For complex64 channels
the forward packs both apertures and runs the TMA-staged DAS with the offsets
(power only); for complex128 it accumulates power chunk by chunk over
``frame_chunk`` frames (at most 8) with the float64 kernel.  The backward
recomputes, chunk by chunk, the IQ of the voxels whose upstream gradient is
nonzero, forms dL/dIQ = 2 g IQ / nt and scatters it with the adjoint.  The
backward cost therefore scales with the number of voxels that carry gradient
(a region of interest), not with the grid.

Precision follows the channels: complex64 channels run the float32
interpolation / accumulation of the main path (float64 geometry); complex128
channels run float64 throughout (the finite-difference checker).
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from rcabeam_b200 import _lib
from rcabeam_b200.sim import RCAGeometry, scan_coords

MAX_CHUNK = 8


@dataclass
class DasGeometry:
    """Device-resident geometry of one reconstruction (float32 like the C ABI)."""

    scan: torch.Tensor
    xe: torch.Tensor
    ye: torch.Tensor
    angles: torch.Tensor
    starts: torch.Tensor
    fs: float
    fd: float
    fn: float
    shape: tuple

    @classmethod
    def build(cls, grid, geom: RCAGeometry, angles, t_start, device=None) -> "DasGeometry":
        dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        f32 = lambda v: torch.from_numpy(np.ascontiguousarray(v, np.float32)).to(dev)  # noqa: E731
        na = len(angles)
        return cls(scan=f32(scan_coords(grid)), xe=f32(geom.x_el), ye=f32(geom.y_el), angles=f32(angles),
                   starts=f32(np.broadcast_to(np.asarray(t_start, np.float32), (na,))), fs=float(geom.fs),
                   fd=float(geom.f_demod), fn=-1.0 if geom.fnumber is None else float(geom.fnumber),
                   shape=(len(grid[0]), len(grid[1]), len(grid[2])))

    @property
    def voxels(self) -> int:
        return self.scan.shape[0]


def _check_inputs(rc, cr, offsets, sound_speed, geometry):
    for name, t in (("rc", rc), ("cr", cr)):
        if not isinstance(t, torch.Tensor) or not t.is_cuda or t.dtype not in (torch.complex64, torch.complex128):
            raise ValueError(f"{name} must be a complex64 or complex128 CUDA tensor")
        if t.dim() != 4:
            raise ValueError(f"{name} must be (samples, channels, angles, frames)")
    if rc.shape != cr.shape or rc.dtype != cr.dtype:
        raise ValueError("RC and CR channels must share shape and dtype")
    ns, nc, na, _ = rc.shape
    if ns < 2 or geometry.xe.numel() != nc or geometry.ye.numel() != nc or geometry.angles.numel() != na:
        raise ValueError("geometry must match channel data")
    if offsets.shape != (2, nc) or offsets.dtype != torch.float64:
        raise ValueError("delay offsets must be a (2, channels) float64 tensor")
    if sound_speed.dim() != 0 or sound_speed.dtype != torch.float64:
        raise ValueError("sound speed must be a 0-d float64 tensor")


def _geometry_args(geometry, voxels, nvl, offsets, c, shape, frame0, frames):
    ns, nc, na, nt = shape
    return (geometry.scan.data_ptr(), None if voxels is None else voxels.data_ptr(), nvl, geometry.xe.data_ptr(),
            geometry.ye.data_ptr(), geometry.angles.data_ptr(), geometry.starts.data_ptr(), offsets.data_ptr(), c,
            geometry.fs, geometry.fd, geometry.fn, ns, nc, na, nt, frame0, frames)


def _staged_power(rc, cr, offsets, c, geometry) -> torch.Tensor:
    """Whole-grid power of complex64 channels on the TMA-staged DAS (packs both apertures first)."""
    ns, nc, na, nt = rc.shape
    nv = geometry.voxels
    packed = []
    for src in (rc, cr):
        dst = torch.empty_like(src)
        _lib.call("rcabeam_pack_ensemble_device", src.data_ptr(), dst.data_ptr(), ns, nc, na, nt)
        packed.append(dst)
    size = ctypes.c_size_t(0)
    _lib.check(_lib.lib().rcabeam_ensemble_workspace_bytes(nv, nc, na, ctypes.byref(size)), "workspace_bytes")
    work = torch.empty(int(size.value), dtype=torch.uint8, device=rc.device)
    pd = torch.empty((nv, 2), dtype=torch.float32, device=rc.device)
    _lib.call("rcabeam_opw_offsets_power_device", packed[0].data_ptr(), packed[1].data_ptr(), geometry.scan.data_ptr(),
              geometry.xe.data_ptr(), geometry.ye.data_ptr(), geometry.angles.data_ptr(), geometry.starts.data_ptr(),
              offsets.data_ptr(), c, geometry.fs, geometry.fd, geometry.fn, ns, nc, na, nt, nv, pd.data_ptr(),
              work.data_ptr(), work.numel())
    return pd[:, 0].to(torch.float64)


class OpwPowerDoppler(torch.autograd.Function):
    """PD (nv,) float64 of the offset-extended OPW model; see the module docstring."""

    @staticmethod
    def forward(ctx, rc, cr, delay_offsets, sound_speed, geometry: DasGeometry, frame_chunk: int = MAX_CHUNK):
        _check_inputs(rc, cr, delay_offsets, sound_speed, geometry)
        if not 1 <= frame_chunk <= MAX_CHUNK:
            raise ValueError(f"frame_chunk must be in [1, {MAX_CHUNK}]")
        rc, cr = rc.contiguous(), cr.contiguous()
        offsets = delay_offsets.detach().contiguous()
        c = float(sound_speed.item())
        nt = rc.shape[3]
        is128 = int(rc.dtype == torch.complex128)
        if is128:
            pd = torch.zeros(geometry.voxels, dtype=torch.float64, device=rc.device)
            for f0 in range(0, nt, frame_chunk):
                frames = min(frame_chunk, nt - f0)
                _lib.call("rcabeam_opw_offsets_forward_device", rc.data_ptr(), cr.data_ptr(),
                          *_geometry_args(geometry, None, geometry.voxels, offsets, c, rc.shape, f0, frames), None,
                          pd.data_ptr(), is128)
        else:
            pd = _staged_power(rc, cr, offsets, c, geometry)
        ctx.save_for_backward(rc, cr, offsets)
        ctx.geometry, ctx.c, ctx.chunk = geometry, c, frame_chunk
        return pd

    @staticmethod
    def backward(ctx, grad_pd):
        rc, cr, offsets = ctx.saved_tensors
        geometry, c, chunk = ctx.geometry, ctx.c, ctx.chunk
        ns, nc, na, nt = rc.shape
        is128 = int(rc.dtype == torch.complex128)
        grad_pd = grad_pd.to(torch.float64).contiguous()
        voxels = torch.nonzero(grad_pd).flatten().to(torch.int32)
        grad_rc, grad_cr = torch.zeros_like(rc), torch.zeros_like(cr)
        grad_off = torch.zeros((2, nc), dtype=torch.float64, device=rc.device)
        grad_c = torch.zeros(1, dtype=torch.float64, device=rc.device)
        nvl = voxels.numel()
        if nvl:
            weight = (2.0 / nt) * grad_pd[voxels.long()]
            iq = torch.empty((nvl, chunk), dtype=rc.dtype, device=rc.device)
            for f0 in range(0, nt, chunk):
                frames = min(chunk, nt - f0)
                block = iq[:, :frames] if frames == chunk else torch.empty((nvl, frames), dtype=rc.dtype,
                                                                           device=rc.device)
                args = _geometry_args(geometry, voxels, nvl, offsets, c, rc.shape, f0, frames)
                _lib.call("rcabeam_opw_offsets_forward_device", rc.data_ptr(), cr.data_ptr(), *args,
                          block.data_ptr(), None, is128)
                g = (block * weight[:, None].to(block.real.dtype)).contiguous()
                _lib.call("rcabeam_opw_offsets_adjoint_device", rc.data_ptr(), cr.data_ptr(), *args, g.data_ptr(),
                          grad_rc.data_ptr(), grad_cr.data_ptr(), grad_off.data_ptr(), grad_c.data_ptr(), is128)
        sound = grad_c.reshape(()) if ctx.needs_input_grad[3] else None
        return (grad_rc if ctx.needs_input_grad[0] else None, grad_cr if ctx.needs_input_grad[1] else None,
                grad_off if ctx.needs_input_grad[2] else None, sound, None, None)


def opw_power_doppler(rc, cr, delay_offsets, sound_speed, geometry: DasGeometry, *,
                      frame_chunk: int = MAX_CHUNK) -> torch.Tensor:
    """Differentiable OPW power Doppler, ``(nx, nz, ny)`` float64."""
    pd = OpwPowerDoppler.apply(rc, cr, delay_offsets, sound_speed, geometry, frame_chunk)
    return pd.reshape(geometry.shape)
