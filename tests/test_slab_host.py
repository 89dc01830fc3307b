"""Slab decomposition driver (exahype_b200.slab) on CPU: oracle slabs
exchanged through gloo ranks / a local ring reproduce the undivided
periodic grid bit for bit."""
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import _oracle as O
from _slab_cpu import OracleSlab, global_ic, run_rank
from exahype_b200 import slab as SL


def undivided(dim, order, n, steps):
    luh, n3, dx = global_ic(dim, order, n)
    t = 0.0
    for _ in range(steps):
        t += O.lib().orc_aderdg_grid_step(dim, order, 0, n3, dx, luh, 0, 0.9, 0.0, None, 1)
    return luh, t


def free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


@pytest.mark.parametrize('dim,order,n,world', [(3, 2, (3, 2, 4), 2), (2, 3, (5, 6), 3)])
def test_gloo_ranks_match_undivided(tmp_path, dim, order, n, world):
    steps = 3
    mp.spawn(run_rank, args=(world, free_port(), dim, order, n, steps, str(tmp_path)), nprocs=world,
             join=True)
    got = np.concatenate([np.load(tmp_path / ('slab%d.npy' % r)) for r in range(world)])
    ref, t = undivided(dim, order, n, steps)
    assert np.array_equal(got, ref)
    for r in range(world):
        assert np.load(tmp_path / ('time%d.npy' % r))[0] == t


@pytest.mark.parametrize('world', [1, 2, 4])
def test_local_ring_matches_undivided(world):
    dim, order, n, steps = 3, 2, (2, 3, 4), 2
    luh, _, _ = global_ic(dim, order, n)
    slabs = [OracleSlab(dim, order, list(n), r, world, luh) for r in range(world)]
    ring = SL.LocalRing(slabs)
    SL.prime(ring)
    SL.step(ring, None, steps)
    got = np.concatenate([s.luh for s in slabs])
    ref, t = undivided(dim, order, n, steps)
    assert np.array_equal(got, ref)
    assert all(s.time == t for s in slabs)


def test_split_rejects_uneven():
    with pytest.raises(ValueError):
        SL.split_last([4, 4, 5], [1.0, 1.0, 1.0], 2)
