"""Channel-domain clutter filtering (reference examples/_support/clutter_pipeline.py:85-91, 121-123).

One temporal basis is estimated over the channel Casorati rows of both
apertures, both apertures are filtered, then OPW power is formed.  Checked
against the float64 oracle (oracle.clutter Gram basis + oracle.das OPW) and,
as a size-independent property, against beamformed-domain filtering of the
unfiltered IQ with the same basis (DAS is linear and frame-wise, so the two
must agree).  Bar: filtered PD relative L2 <= 1e-4 against float64.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from oracle import clutter, das
from rcabeam_b200 import _lib, gpu_clutter
from rcabeam_b200.pipeline import FilteredOpw
from rcabeam_b200.sim import RCAGeometry
from tests._cases import oracle_inputs, rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs CUDA")
    yield
    assert _lib.device_error() == 0


def _scene(seed=11, shape=(96, 12, 3, 24)):
    """Channels with rank-3 slow-time clutter (x100) over white noise, and a small RCA geometry."""
    rng = np.random.default_rng(seed)
    ns, nc, na, nt = shape
    t = np.arange(nt)
    out = []
    for _ in range(2):
        clut = sum((rng.normal(size=(ns, nc, na, 1)) + 1j * rng.normal(size=(ns, nc, na, 1)))
                   * 100 * np.exp(2j * np.pi * f * t) for f in (0.0, 0.01, -0.02))
        noise = rng.normal(size=shape) + 1j * rng.normal(size=shape)
        out.append((clut + noise).astype(np.complex64))
    el = (np.arange(nc) - (nc - 1) / 2) * 0.2e-3
    geom = RCAGeometry(el, el, c=1540.0, fs=20e6, f_demod=5e6, fnumber=None)
    angles = np.deg2rad(np.linspace(-6, 6, na))
    grid = (np.linspace(-1e-3, 1e-3, 6), np.linspace(2.0e-3, 3.5e-3, 8), np.linspace(-1e-3, 1e-3, 5))
    return out[0], out[1], angles, 1e-6, grid, geom


def _oracle(rc, cr, angles, t_start, grid, geom, start, stop):
    nt = rc.shape[-1]
    rows = np.concatenate([rc.reshape(-1, nt), cr.reshape(-1, nt)])
    _, basis = clutter.temporal_basis(rows, method="gram")
    kept = basis[:, start:stop]
    filt = [((a.reshape(-1, nt).astype(np.complex128) @ kept) @ kept.conj().T).reshape(a.shape) for a in (rc, cr)]
    o = oracle_inputs(angles, t_start, grid, geom)
    iq = das.opw_iq(filt[0], filt[1], o["scan"], o["xe"], o["ye"], o["angles"], o["starts"], o["c"], o["fs"],
                    o["fd"], o["fnumber"])
    return das.power_doppler(iq)


@pytest.mark.parametrize("storage,precision", [("float32", "complex128"), ("bf16x2", "bf16x3"),
                                               ("float16", "complex128")])
@pytest.mark.parametrize("ranks", [(3, None), (1, 20), (0, 24)])
def test_channel_domain_matches_oracle(storage, precision, ranks):
    rc, cr, angles, t_start, grid, geom = _scene()
    start, stop = ranks
    nt = rc.shape[-1]
    plan = FilteredOpw(rc.shape, angles, t_start, grid, geom, rank_start=start, rank_stop=stop, precision=precision,
                       iq_storage=storage, domain="channel")
    power = plan.run(torch.from_numpy(rc).cuda(), torch.from_numpy(cr).cuda())
    plan.check()
    expected = _oracle(rc, cr, angles, t_start, grid, geom, start, nt if stop is None else stop)
    # FP16 storage quantizes the filtered channels (11-bit significands).
    tol = 2e-3 if storage == "float16" else 1e-4
    assert rel_l2(power.cpu().numpy().ravel(), expected) <= tol


def test_channel_domain_equals_beamformed_filter_with_same_basis():
    """Filter-then-beamform equals beamform-then-filter for one basis (linearity property)."""
    rc, cr, angles, t_start, grid, geom = _scene(seed=3, shape=(96, 12, 3, 32))
    d_rc, d_cr = torch.from_numpy(rc).cuda(), torch.from_numpy(cr).cuda()
    channel = FilteredOpw(rc.shape, angles, t_start, grid, geom, rank_start=3, domain="channel")
    power_channel = channel.run(d_rc, d_cr).clone()
    _, basis = gpu_clutter.temporal_basis((d_rc, d_cr))
    beamformed = FilteredOpw(rc.shape, angles, t_start, grid, geom, rank_start=3)
    beamformed.run(d_rc, d_cr)
    power_same_basis = gpu_clutter.filtered_power(beamformed.iq, basis, rank_start=3).reshape(power_channel.shape)
    # The beamformed side removes 100x clutter after float32 DAS: ~1e-5 of the residual.
    assert rel_l2(power_channel.cpu().numpy(), power_same_basis.cpu().numpy()) <= 1e-4
