"""ctypes binding of the in-tree C ABI library (``lib/librcabeam.so``).

The argument tables below mirror ``include/rcabeam.h``.  Loading fails loudly
when the library has not been built: there is no CPU fallback.
"""

from __future__ import annotations

import ctypes
from ctypes import c_double, c_float, c_int, c_size_t, c_void_p
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "lib" / "librcabeam.so"

P = c_void_p
Z = c_size_t
F = c_float
I = c_int
D = c_double

# name -> argument types (every function returns rcabeam_status, an int enum).
SIGNATURES: dict[str, list] = {
    "rcabeam_opw_device": [P, P, Z, Z, Z],
    "rcabeam_xdoppler_pd_device": [P, P, Z, Z, Z, Z, Z, Z, Z],
    "rcabeam_rc_fmas_pd_device": [P, P, Z, Z, Z, Z, Z, Z, Z],
    "rcabeam_delay_rca_channels_device": [P, P, P, P, P, P, Z, Z, Z, Z, I, F, F, F, F],
    "rcabeam_delay_rca_channel_data_device": [P, P, P, P, P, P, P, P, Z, Z, Z, Z, I, F, F, F, F],
    "rcabeam_opw_pd_from_channels_device": [P, P, P, P, P, P, P, P, Z, Z, Z, Z, F, F, F, F],
    "rcabeam_xdoppler_pd_from_channels_device": [P, P, P, P, P, P, P, P, Z, Z, Z, Z, F, F, F, F],
    "rcabeam_rc_fmas_pd_from_channels_device": [P, P, P, P, P, P, P, P, Z, Z, Z, Z, F, F, F, F],
    "rcabeam_fast_pd_from_channels_device": [P, P, P, P, P, P, P, P, P, P, Z, Z, Z, Z, F, F, F, F],
    "rcabeam_dmas_ccf_acf_from_channels_device": [P, P, P, P, P, P, P, P, Z, Z, Z, Z, F, F, F, F],
    "rcabeam_pack_ensemble_device": [P, P, Z, Z, Z, Z],
    "rcabeam_ensemble_device": [P, P, P, P, P, P, P, P, P, P, P, P, Z, Z, Z, Z, Z, F, F, F, F, I, I],
    "rcabeam_pack_ensemble_fp16_device": [P, P, P, Z, Z, Z, Z],
    "rcabeam_opw_fp16_device": [P, P, P, P, P, P, P, P, P, P, Z, Z, Z, Z, Z, F, F, F, F],
    "rcabeam_pack_ensemble_split_device": [P, P, P, P, Z, Z, Z, Z],
    "rcabeam_opw_tc_device": [P, P, P, P, P, P, P, P, P, P, P, P, Z, Z, Z, Z, Z, F, F, F, F, I],
    "rcabeam_clutter_scale_device": [P, Z, I, P],
    "rcabeam_gram_accumulate_device": [P, Z, Z, I, P, I, P],
    "rcabeam_gram_finish_device": [P, P, Z, Z],
    "rcabeam_heevd_workspace_bytes": [Z, ctypes.POINTER(c_size_t)],
    "rcabeam_heevd_device": [P, P, Z, P, Z, P],
    "rcabeam_project_device": [P, P, P, Z, Z, I, P, Z, I, P],
    "rcabeam_ritz_matrix_device": [P, Z, Z, P, Z, P],
    "rcabeam_ensemble_static_device": [P, P, P, P, P, P, P, P, P, Z, Z, Z, Z, Z, F, F, F, F, I],
    "rcabeam_ensemble_workspace_bytes": [Z, Z, Z, ctypes.POINTER(c_size_t)],
    "rcabeam_opw_offsets_forward_device": [P, P, P, P, Z, P, P, P, P, P, D, F, F, F, Z, Z, Z, Z, Z, Z, P, P, I],
    "rcabeam_opw_offsets_power_device": [P, P, P, P, P, P, P, P, D, F, F, F, Z, Z, Z, Z, Z, P, P, Z],
    "rcabeam_opw_offsets_adjoint_device": [P, P, P, P, Z, P, P, P, P, P, D, F, F, F, Z, Z, Z, Z, Z, Z, P, P, P, P, P,
                                           I],
    "rcabeam_batch_table_bytes": [Z, P, ctypes.POINTER(c_size_t)],
    "rcabeam_batch_prepare": [Z, P, P, Z],
    "rcabeam_batch_run_device": [Z, P, P, Z, P, I, P],
    "rcabeam_simulate_scene_device": [P, Z, P, P, P, P, Z, Z, Z, Z, I, D, D, D, D, D, D],
    "rcabeam_voxel_order_workspace_bytes": [Z, ctypes.POINTER(c_size_t)],
    "rcabeam_voxel_order_device": [P, Z, P, P, Z],
    "rcabeam_wait_selftest_device": [ctypes.c_ulonglong, I, P],
    "rcabeam_device_error": [ctypes.POINTER(c_int)],
}

STATUS = {0: "success", 1: "cuda error", 2: "invalid argument"}

_lib: ctypes.CDLL | None = None


class RcabeamCudaError(RuntimeError):
    """A CUDA launch or device-side error reported by the C ABI."""


def lib() -> ctypes.CDLL:
    """Load the C ABI library once, declaring every entry point's signature."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(
                f"rcabeam_b200 CUDA library missing at {LIB_PATH}; build it with `python -m rcabeam_b200._build`"
            )
        handle = ctypes.CDLL(str(LIB_PATH))
        for name, args in SIGNATURES.items():
            fn = getattr(handle, name)
            fn.argtypes = args
            fn.restype = c_int
        handle.rcabeam_status_string.argtypes = [c_int]
        handle.rcabeam_status_string.restype = ctypes.c_char_p
        _lib = handle
    return _lib


def check(status: int, what: str) -> None:
    """Raise on a non-success rcabeam_status (ValueError for invalid arguments)."""
    if status == 0:
        return
    text = STATUS.get(status, f"status {status}")
    if status == 2:
        raise ValueError(f"{what}: {text}")
    raise RcabeamCudaError(f"{what}: {text}")


def call(name: str, *args) -> None:
    check(getattr(lib(), name)(*args), name)


def device_error() -> int:
    """Read and clear the device error word of the bounded-wait kernels (synchronizes)."""
    code = ctypes.c_int(0)
    check(lib().rcabeam_device_error(ctypes.byref(code)), "rcabeam_device_error")
    return code.value
