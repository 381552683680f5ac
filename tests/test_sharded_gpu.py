"""Voxel-sharded filtered OPW with the CUDA kernels: two ranks on one GPU.

Each rank (a separate process on cuda:0) reconstructs its x slab with
``FilteredOpw(..., group=...)``; the clutter basis is shared through the
gloo all-reduces of ``rcabeam_b200.sharded`` (host-side collectives: no
kernel ever waits for another process).  The gathered power must equal the
single-process pipeline on the whole grid.
"""

from __future__ import annotations

import datetime
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _setup():
    from rcabeam_b200.sim import RCAGeometry

    rng = np.random.default_rng(23)
    el = (np.arange(16) - 7.5) * 0.2e-3
    geom = RCAGeometry(el, el, c=1540.0, fs=20e6, f_demod=15e6, fnumber=None)
    angles = np.deg2rad(np.linspace(-8, 8, 3))
    shape = (160, 16, 3, 24)
    rc = (rng.normal(size=shape) + 1j * rng.normal(size=shape)).astype(np.complex64)
    cr = (rng.normal(size=shape) + 1j * rng.normal(size=shape)).astype(np.complex64)
    grid = (np.linspace(-1.5e-3, 1.5e-3, 9), np.linspace(3e-3, 6e-3, 12), np.linspace(-1e-3, 1e-3, 6))
    return rc, cr, angles, 3e-6, grid, geom


def _run(grid_part, group=None):
    from rcabeam_b200 import pipeline

    rc, cr, angles, t0, _, geom = _setup()
    plan = pipeline.FilteredOpw(rc.shape, angles, t0, grid_part, geom, rank_start=3, group=group)
    out = plan.run(torch.from_numpy(rc).cuda(), torch.from_numpy(cr).cuda())
    plan.check()
    return out.cpu()


def _rank(rank, world, port, out):
    import torch.distributed as dist

    from rcabeam_b200 import sharded

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        grid = _setup()[4]
        local = _run(sharded.shard_grid(grid, rank, world), dist.group.WORLD)
        out.put((rank, sharded.gather_power(local, dist.group.WORLD).numpy()))
    finally:
        dist.destroy_process_group()


def test_two_ranks_match_one_process():
    if not torch.cuda.is_available():
        pytest.skip("needs CUDA")
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    results = dict(out.get(timeout=300) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    want = _run(_setup()[4]).numpy()
    for rank in (0, 1):
        np.testing.assert_allclose(results[rank], want, rtol=1e-8, atol=1e-10 * np.abs(want).max())
