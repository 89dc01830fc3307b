"""Slab decomposition on the GPU: slabs of one grid (several on this GPU,
exchanged by a local ring; or one slab per rank through torch.distributed
with NCCL) reproduce the undivided periodic grid bit for bit."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import exahype_b200 as E
from exahype_b200 import slab as SL

pytestmark = pytest.mark.gpu


def undivided(dim, order, n, steps, precision=E.PREC_FP64, **ic):
    g = E.ADERDGGrid(dim, order, n, precision=precision)
    g.init(**ic)
    init = g.get_state()
    g.step(steps)
    out = g.get_state(), g.status()['time'], init
    g.destroy()
    return out


IC = dict(kind=0, param=5.0, seed=3, noise=1e-3)


@pytest.mark.parametrize('dim,order,n,world,precision', [
    (3, 3, (5, 4, 6), 2, E.PREC_FP64),
    (3, 4, (4, 3, 6), 3, E.PREC_FP64),
    (2, 4, (7, 9), 3, E.PREC_FP64),
    (3, 4, (4, 4, 4), 2, E.PREC_MIXED),
])
def test_local_ring_matches_undivided(dim, order, n, world, precision):
    steps = 4
    ref, t, init = undivided(dim, order, n, steps, precision, **IC)
    slabs = [SL.SlabGrid(dim, order, n, r, world, precision=precision) for r in range(world)]
    for s in slabs:
        s.init(**IC)
    assert np.array_equal(SL.gather_state(slabs), init)
    ring = SL.LocalRing(slabs)
    SL.prime(ring)
    SL.step(ring, None, steps)
    assert np.array_equal(SL.gather_state(slabs), ref)
    for s in slabs:
        assert s.status()['time'] == t
        s.destroy()


def test_halo_grid_refuses_plain_step():
    g = E.ADERDGGrid(3, 2, (2, 2, 2))
    g.set_halo(True)
    with pytest.raises(E.ExaError):
        g.step(1)
    g.destroy()


def _nccl_rank(rank, port, outdir):
    import datetime
    import torch
    import torch.distributed as dist
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group('nccl', rank=rank, world_size=1, timeout=datetime.timedelta(seconds=60),
                            device_id=torch.device('cuda', 0))
    try:
        s = SL.SlabGrid(3, 3, (4, 5, 3), rank, 1)
        s.init(**IC)
        ring = SL.DistRing(dist)
        SL.prime(ring, s)
        SL.step(ring, s, 3)
        np.save(os.path.join(outdir, 'state.npy'), s.get_state())
        s.destroy()
    finally:
        dist.destroy_process_group()


def test_dist_ring_nccl_single_rank(tmp_path):
    with socket.socket() as so:
        so.bind(('127.0.0.1', 0))
        port = so.getsockname()[1]
    mp.spawn(_nccl_rank, args=(port, str(tmp_path)), nprocs=1, join=True)
    ref, _, _ = undivided(3, 3, (4, 5, 3), 3, **IC)
    assert np.array_equal(np.load(tmp_path / 'state.npy'), ref)
