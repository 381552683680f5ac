"""Voxel-sharded clutter filter: the collective steps on CPU ranks (gloo).

Two and three ranks each hold an x slab of one (nx, nz, ny, T) ensemble.
They run the product's reduction code (``rcabeam_b200.sharded``: MAX of the
Casorati scale, SUM of the float64 Gram and of the row count, gather of the
power map) around NumPy stand-ins for the per-rank CUDA kernels, and must
reproduce the single-process float64 oracle.  A rank that never joins makes
the others fail with a timeout instead of hanging.
"""

from __future__ import annotations

import datetime
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist

from oracle import clutter as oc
from rcabeam_b200 import sharded

SHAPE = (7, 5, 4, 12)  # nx, nz, ny, frames


def _ensemble():
    rng = np.random.default_rng(17)
    x = rng.normal(size=SHAPE) + 1j * rng.normal(size=SHAPE)
    # A dominant temporal component (clutter) so the filter has something to remove.
    x += 30 * rng.normal(size=SHAPE[:3])[..., None] * np.exp(0.3j * np.arange(SHAPE[3]))
    return x.astype(np.complex128)


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        full = _ensemble()
        local = full[sharded.x_slab(SHAPE[0], rank, world)]
        rows = local.reshape(-1, SHAPE[3])
        # Stand-ins for rcabeam_clutter_scale_device / rcabeam_gram_accumulate_device.
        scale = torch.tensor([max(np.abs(rows.real).max(), np.abs(rows.imag).max())], dtype=torch.float64)
        sharded.reduce_scale(scale, dist.group.WORLD)
        xs = rows / scale.item()
        upper = torch.from_numpy(np.ascontiguousarray(np.stack([(xs.conj().T @ xs).real, (xs.conj().T @ xs).imag],
                                                               axis=-1)).ravel())
        total = sharded.reduce_gram(upper, rows.shape[0], dist.group.WORLD)
        g = upper.numpy().reshape(SHAPE[3], SHAPE[3], 2)
        gram = (g[..., 0] + 1j * g[..., 1]) / total
        lam, vec = np.linalg.eigh((gram + gram.conj().T) / 2)
        basis = vec[:, ::-1]
        power = torch.from_numpy(oc.filtered_power(rows, basis, 3).reshape(local.shape[:3]))
        gathered = sharded.gather_power(power, dist.group.WORLD)
        out.put((rank, gathered.numpy(), scale.item(), total))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_filter_matches_single_process(world):
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    results = [out.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    full = _ensemble()
    _, basis = oc.temporal_basis(full, method="gram")
    want = oc.filtered_power(full, basis, 3).reshape(SHAPE[:3])
    scale = max(np.abs(full.real).max(), np.abs(full.imag).max())
    for rank, gathered, s, total in results:
        assert total == SHAPE[0] * SHAPE[1] * SHAPE[2]
        assert s == scale
        np.testing.assert_allclose(gathered, want, rtol=1e-10, atol=1e-12 * np.abs(want).max())


def _lonely(port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    try:
        dist.init_process_group("gloo", rank=0, world_size=2, timeout=datetime.timedelta(seconds=3))
        out.put("joined")
    except Exception as exc:  # the peer never joins: rendezvous times out
        out.put(type(exc).__name__)


def test_missing_rank_fails_with_a_timeout():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    p = ctx.Process(target=_lonely, args=(_port(), out))
    p.start()
    result = out.get(timeout=120)
    p.join(timeout=60)
    assert result != "joined"


def test_slabs_partition_the_grid():
    for nx in (1, 7, 128):
        for world in (1, 2, 3, 8):
            slabs = [sharded.x_slab(nx, r, world) for r in range(world)]
            covered = np.concatenate([np.arange(nx)[s] for s in slabs])
            np.testing.assert_array_equal(covered, np.arange(nx))
            sizes = [s.stop - s.start for s in slabs]
            assert max(sizes) - min(sizes) <= 1
    grid = (np.arange(10.0), np.arange(3.0), np.arange(2.0))
    part = sharded.shard_grid(grid, 1, 3)
    np.testing.assert_array_equal(part[0], [4.0, 5.0, 6.0])
    with pytest.raises(ValueError):
        sharded.x_slab(4, 3, 3)
