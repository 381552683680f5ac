"""ctypes wrapper of the C float64 DAS oracle (``das_c.c``) -- TEST INFRASTRUCTURE ONLY.

Same results as ``oracle.das.opw_iq`` / ``aperture_das`` (float64, to rounding
order), threaded over voxels.  The shared library is built by gcc into
``oracle/_build/`` (git-ignored) on first use or by ``build()``; the product
path never loads it.
"""

from __future__ import annotations

import ctypes
import shutil
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
SOURCE = HERE / "das_c.c"
LIB = HERE / "_build" / "liboracle_das.so"

_handle = None


def build(force: bool = False) -> Path:
    """Compile ``das_c.c`` with OpenMP (IEEE float64, no fast-math)."""
    if not force and LIB.exists() and LIB.stat().st_mtime >= SOURCE.stat().st_mtime:
        return LIB
    gcc = shutil.which("gcc") or shutil.which("cc")
    if gcc is None:
        raise RuntimeError("gcc not found: the C oracle cannot be built")
    LIB.parent.mkdir(parents=True, exist_ok=True)
    tmp = LIB.with_suffix(".tmp.so")
    subprocess.run([gcc, "-O2", "-fopenmp", "-fPIC", "-shared", "-fno-fast-math", "-o", str(tmp), str(SOURCE), "-lm"],
                   check=True)
    tmp.replace(LIB)
    return LIB


def _lib():
    global _handle
    if _handle is None:
        handle = ctypes.CDLL(str(build()))
        p, z, d, i = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_double, ctypes.c_int
        handle.oracle_das_accumulate.argtypes = [p, p, z, p, p, p, p, z, z, z, z, d, d, d, d, i, p]
        handle.oracle_das_accumulate.restype = None
        _handle = handle
    return _handle


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def aperture_accumulate(out: np.ndarray, iq, scan, elements, angles, starts, c, fs, fd, fnumber, config: str,
                        offsets=None) -> None:
    """``out`` (nv, nt) complex128 += the float64 DAS of one aperture, summed over channels and angles."""
    iq = np.ascontiguousarray(iq, dtype=np.complex64)
    if iq.ndim == 3:
        iq = iq[..., None]
    ns, nc, na, nt = iq.shape
    scan = np.ascontiguousarray(np.asarray(scan, dtype=np.float64).reshape(-1, 3))
    if out.dtype != np.complex128 or not out.flags.c_contiguous or out.shape != (len(scan), nt):
        raise ValueError("out must be a C-contiguous complex128 (nv, nt) array")
    el = np.ascontiguousarray(elements, dtype=np.float64)
    ang = np.ascontiguousarray(angles, dtype=np.float64)
    st = np.ascontiguousarray(np.broadcast_to(np.asarray(starts, dtype=np.float64), (na,)))
    off = None if offsets is None else np.ascontiguousarray(offsets, dtype=np.float64)
    fn = -1.0 if fnumber is None else float(fnumber)
    _lib().oracle_das_accumulate(_ptr(iq), _ptr(scan), len(scan), _ptr(el), _ptr(ang), _ptr(st),
                                 None if off is None else _ptr(off), ns, nc, na, nt, float(c), float(fs), float(fd),
                                 fn, 1 if config == "CR" else 0, _ptr(out))


def opw_iq(rc, cr, scan, xe, ye, angles, starts, c, fs, fd, fnumber) -> np.ndarray:
    """Coherent OPW IQ ``(nv, nt)`` complex128: RC + CR, each summed over angles and channels."""
    nt = 1 if np.ndim(rc) == 3 else np.shape(rc)[3]
    out = np.zeros((len(np.reshape(scan, (-1, 3))), nt), dtype=np.complex128)
    aperture_accumulate(out, rc, scan, xe, angles, starts, c, fs, fd, fnumber, "RC")
    aperture_accumulate(out, cr, scan, ye, angles, starts, c, fs, fd, fnumber, "CR")
    return out
