"""Failure detection of the staging pipelines without a GPU fault.

Every spin-wait of the library's kernels is bounded: after its limit it records
an error code in the device error word and the kernel returns.  Here a pipeline
wait runs out on purpose -- four warps wait on an mbarrier that nothing arrives
on, with a 50 ms limit -- and the host reads the code through the C ABI
(reference status contract: include/rcabeam.h:9-15, ensemble.cu:664-683,
extended to the device error word).  The context stays usable: a reconstruction
afterwards matches the float64 oracle.
"""

from __future__ import annotations

import time

import numpy as np
import pytest
import torch

from oracle import das
from rcabeam_b200 import _lib
from rcabeam_b200 import ensemble as rb
from tests._cases import oracle_inputs, random_case, rel_l2

pytestmark = pytest.mark.gpu


def test_bounded_wait_gives_up_and_reports():
    assert _lib.device_error() == 0
    gave_up = torch.zeros(1, dtype=torch.int32, device="cuda")
    t0 = time.perf_counter()
    _lib.call("rcabeam_wait_selftest_device", 50_000_000, 2, gave_up.data_ptr())
    code = _lib.device_error()  # synchronizes
    elapsed = time.perf_counter() - t0
    assert code == 2
    assert int(gave_up.item()) == 4  # every waiting warp gave up
    assert 0.04 < elapsed < 1.5
    assert _lib.device_error() == 0  # read-and-clear
    with pytest.raises(ValueError):
        _lib.call("rcabeam_wait_selftest_device", 0, 2, gave_up.data_ptr())
    # The context still runs reconstructions correctly.
    rc, cr, angles, starts, _, geom = random_case(3, 40, 4, 3, 6, None)
    grid = (np.linspace(-5e-4, 5e-4, 4), np.linspace(5e-4, 4e-3, 9), np.linspace(-5e-4, 5e-4, 3))
    got = rb.ensemble_pd_from_channels(rc, cr, angles, starts, grid, geom)
    o = oracle_inputs(angles, starts, grid, geom)
    iq = das.opw_iq(rc, cr, o["scan"], o["xe"], o["ye"], o["angles"], o["starts"], o["c"], o["fs"], o["fd"],
                    o["fnumber"])
    assert rel_l2(got.ravel(), das.power_doppler(iq)) < 1e-5
    assert _lib.device_error() == 0
