"""Host-side logic without a GPU: the shared input validator and the scene tables."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import scene as osc
from rcabeam_b200 import _inputs
from rcabeam_b200.sim import RCAGeometry


def _geom(nc=4, **kw):
    return RCAGeometry(np.linspace(-1e-3, 1e-3, nc), np.linspace(-1e-3, 1e-3, nc), **kw)


GRID = (np.linspace(-1e-3, 1e-3, 3), np.linspace(1e-3, 2e-3, 4), np.linspace(-1e-3, 1e-3, 2))


def test_acquisition_normalizes_to_the_c_abi_types():
    acq = _inputs.acquisition((16, 4, 2, 8), np.array([0.0, 0.1]), 1e-6, GRID, _geom(fnumber=None))
    assert acq.channel_shape == (16, 4, 2, 8) and acq.grid_shape == (3, 4, 2) and acq.voxels == 24
    assert acq.scan.dtype == np.float32 and acq.scan.shape == (24, 3)
    assert all(v.dtype == np.float32 for v in (acq.x_el, acq.y_el, acq.angles, acq.starts))
    np.testing.assert_array_equal(acq.starts, np.float32([1e-6, 1e-6]))
    assert acq.constants[3] == -1.0  # full aperture
    assert _inputs.acquisition((16, 4, 2, 8), [0.0, 0.1], [1e-6, 2e-6], GRID, _geom()).constants[3] == 1.0


@pytest.mark.parametrize("shape,match", [((1, 4, 2, 8), "nonempty"), ((16, 4, 2, 0), "nonempty"), ((16, 4, 2), "nonempty"),
                                         ((16, 5, 2, 8), "channel/angle"), ((16, 4, 3, 8), "channel/angle")])
def test_acquisition_shape_errors(shape, match):
    with pytest.raises(ValueError, match=match):
        _inputs.acquisition(shape, [0.0, 0.1], 1e-6, GRID, _geom())


def test_acquisition_value_errors():
    ok = ((16, 4, 2, 8), [0.0, 0.1], 1e-6)
    with pytest.raises(ValueError, match="F-number"):
        _inputs.acquisition(*ok, GRID, _geom(fnumber=0.0))
    with pytest.raises(ValueError, match="Sound speed"):
        _inputs.acquisition(*ok, GRID, _geom(c=-1.0))
    with pytest.raises(ValueError, match="Grid"):
        _inputs.acquisition(*ok, (GRID[0], np.array([]), GRID[2]), _geom())
    with pytest.raises(ValueError, match="finite"):
        _inputs.acquisition((16, 4, 2, 8), [0.0, np.nan], 1e-6, GRID, _geom())


def test_method_and_storage_contract():
    assert _inputs.method_code("opw", "bf16x2", wants_signal=False) == 0
    assert _inputs.method_code("apertures", "float32", wants_signal=True) == 5
    with pytest.raises(ValueError, match="Unknown method"):
        _inputs.method_code("apertures", "float32", wants_signal=False)
    with pytest.raises(ValueError, match="OPW only"):
        _inputs.method_code("dmas", "float16", wants_signal=False)
    with pytest.raises(ValueError, match="IQ storage"):
        _inputs.method_code("opw", "int8", wants_signal=False)
    with pytest.raises(ValueError, match="St-SW requires"):
        _inputs.check_subsets("st_sw", 3, 2)
    _inputs.check_subsets("opw", 9, 1)


def test_scene_positions_wrap_along_the_tube():
    # o + d * s with s = s0 + speed t wrapped into [0, period): a tube scatterer re-enters at its start.
    table = np.zeros((2, 11))
    table[:, 3] = 1.0           # direction +x
    table[0, 6:9] = 0.5, 2.0, 1.0   # s0, speed, period (wraps)
    table[1, 6:9] = 0.5, 2.0, 0.0   # no wrap
    pos = osc.positions(table, 0.4)  # s = 1.3
    np.testing.assert_allclose(pos[:, 0], [0.3, 1.3])
