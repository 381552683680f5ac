"""Batching form: the persistent queue kernel against the single-ensemble C API.

A queue of uneven ensembles (grids, frame counts, angle counts and methods
differ) runs through one persistent kernel; every ensemble's power must equal
the single-ensemble path (``rcabeam_ensemble_device``, itself pinned to the
float64 oracle) up to float32 summation order (1e-5 relative L2), from a plain
launch and from CUDA-graph replays, with autotuned frame chunks.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from rcabeam_b200 import _lib, batching
from rcabeam_b200.sim import RCAGeometry
from tests._cases import rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs CUDA")
    yield
    assert _lib.device_error() == 0


SPECS = [  # method, depth points, frames, angles
    ("opw", 24, 16, 5),
    ("xdoppler", 16, 34, 3),
    ("dmas", 12, 8, 3),
    ("opw", 40, 66, 7),
    ("xdoppler", 20, 10, 5),
    ("dmas", 9, 130, 2),
    ("opw", 7, 2, 1),
    ("xdoppler", 6, 71, 2),  # a 7-frame tail chunk for every chunk width
]


def _queue(seed=3):
    rng = np.random.default_rng(seed)
    ns, nc = 160, 16
    el = (np.arange(nc) - (nc - 1) / 2) * 0.2e-3
    geom = RCAGeometry(el, el, c=1540.0, fs=20e6, f_demod=15e6, fnumber=None)
    out = []
    for method, nz, nt, na in SPECS:
        angles = np.deg2rad(np.linspace(-8, 8, na)) if na > 1 else np.zeros(1)
        grid = (np.linspace(-1.2e-3, 1.2e-3, 10) + 1.1e-5, np.linspace(3e-3, 6e-3, nz) + 0.7e-5,
                np.linspace(-1.0e-3, 1.0e-3, 8) + 1.9e-5)
        packed = []
        for _ in range(2):
            raw = (rng.normal(size=(ns, nc, na, nt)) + 1j * rng.normal(size=(ns, nc, na, nt))).astype(np.complex64)
            src = torch.from_numpy(raw).cuda()
            dst = torch.empty_like(src)
            _lib.call("rcabeam_pack_ensemble_device", src.data_ptr(), dst.data_ptr(), ns, nc, na, nt)
            packed.append(dst)
        e = batching.Ensemble(packed[0], packed[1], (ns, nc, na, nt), grid, geom, angles, 3e-6, method)
        e.build(torch.device("cuda"))
        out.append(e)
    return out


def _single(ensembles):
    batching.sequential(ensembles)
    return [e.power().clone() for e in ensembles]


@pytest.mark.parametrize("ctas", [0, 1, 2, 3])
@pytest.mark.parametrize("chunk", [16, 32, 64])
def test_queue_matches_single_ensemble_path(chunk, ctas):
    ens = _queue()
    want = _single(ens)
    for e in ens:
        e.frames_per_chunk = chunk
    q = batching.BatchQueue(ens, ctas_per_sm=ctas)
    q.run()
    torch.cuda.synchronize()
    for e, w in zip(ens, want):
        assert w.abs().max() > 0
        assert rel_l2(e.power().cpu().numpy(), w.cpu().numpy()) <= 1e-5, e.method
    done = q.completion_ms()
    assert np.all(done > 0) and np.all(np.isfinite(done))
    assert len(q.parts) == len({e.method for e in ens})  # one persistent launch per method


def test_graph_replay_and_autotune():
    ens = _queue(seed=5)
    want = _single(ens)
    choice = batching.autotune(ens, sample_tiles=4, repeats=1)
    assert set(choice["ctas_per_sm"]) == set(batching.METHODS)
    assert all(k in (0, 2, 3) for k in choice["ctas_per_sm"].values())
    assert all(e.frames_per_chunk in batching.FRAME_CHUNKS for e in ens)
    q = batching.BatchQueue(ens, ctas_per_sm=choice["ctas_per_sm"])
    q.capture()
    for _ in range(2):
        for e in ens:
            e.tensors["pd"].fill_(7.0)  # the graph clears the outputs itself
        q.run()
        torch.cuda.synchronize()
        for e, w in zip(ens, want):
            assert rel_l2(e.power().cpu().numpy(), w.cpu().numpy()) <= 1e-5, e.method


def test_invalid_queue_entries_are_rejected():
    ens = _queue()[:1]
    ens[0].frames_per_chunk = 48
    with pytest.raises(ValueError):
        batching.BatchQueue(ens)
