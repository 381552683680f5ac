"""B200-native (sm_100a) implementation of rcabeam's OPW path.

Drop-in entry points of the reference library sdiebolt/rcabeam:

* ``beamform_ensemble``, ``ensemble_pd_from_channels``, ``beamform_apertures``
  (reference ``rcabeam.ensemble``);
* ``OpwWorkspace`` (reference ``rcabeam.gpu``) with torch CUDA tensors;
* ``svd_clutter_filter``, ``temporal_basis``, ``filtered_power``,
  ``apply_temporal_filter`` (reference ``rcabeam.gpu_clutter``) and
  ``power_doppler`` (reference ``rcabeam.power``);
* ``RCAGeometry``, ``simulate_point``, ``depth_axis`` (reference ``rcabeam.sim``).

All reconstruction and filtering runs in the in-tree CUDA library
``lib/librcabeam.so`` through the C ABI declared in ``include/rcabeam.h``.
"""

from rcabeam_b200.ensemble import (
    EnsembleTiming,
    beamform_apertures,
    beamform_ensemble,
    ensemble_pd_from_channels,
    opw_voxel_order,
)
from rcabeam_b200.sim import RCAGeometry, depth_axis, scan_coords, simulate_point


def __getattr__(name):
    # GPU-side modules import torch lazily so that geometry helpers stay light.
    if name == "OpwWorkspace":
        from rcabeam_b200.gpu import OpwWorkspace

        return OpwWorkspace
    if name in ("svd_clutter_filter", "temporal_basis", "filtered_power", "apply_temporal_filter", "power_doppler"):
        from rcabeam_b200 import gpu_clutter

        return getattr(gpu_clutter, name)
    raise AttributeError(name)


__all__ = [
    "EnsembleTiming",
    "OpwWorkspace",
    "RCAGeometry",
    "apply_temporal_filter",
    "beamform_apertures",
    "beamform_ensemble",
    "depth_axis",
    "ensemble_pd_from_channels",
    "filtered_power",
    "opw_voxel_order",
    "power_doppler",
    "scan_coords",
    "simulate_point",
    "svd_clutter_filter",
    "temporal_basis",
]
