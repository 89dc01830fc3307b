"""Slab decomposition on the GPU: slabs of one grid (several on this GPU,
exchanged by a local ring; or one slab per process through the library's
own NCCL transport, exa_aderdg_grid_slab_step) reproduce the undivided
periodic grid bit for bit.  Every GPU run here has one GPU, so the NCCL
transport is exercised with a one-rank communicator (its face layers are
copied on the stream, its dt minimum is NCCL's one-rank all-reduce); the
multi-rank exchange order is covered by the CPU tests of the same driver
(tests/test_slab_host.py)."""
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest

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


@pytest.mark.parametrize('dt_policy', [0, 2])
def test_nccl_ring_single_rank(dt_policy):
    kw = dict(dt_policy=dt_policy, dt_fixed=2e-3) if dt_policy == 2 else {}
    s = SL.SlabGrid(3, 3, (4, 5, 3), 0, 1, **kw)
    s.init(**IC)
    ring = SL.NcclRing(0, 1, SL.NcclRing.make_id())
    SL.prime(ring, s)
    SL.step(ring, s, 3)
    got, t = s.get_state(), s.status()['time']
    s.destroy()
    ring.destroy()
    g = E.ADERDGGrid(3, 3, (4, 5, 3), **kw)
    g.init(**IC)
    g.step(3)
    assert np.array_equal(got, g.get_state())
    assert t == g.status()['time']
    g.destroy()


_NO_TORCH = textwrap.dedent('''
    import sys
    sys.path.insert(0, sys.argv[1])
    import numpy as np
    import exahype_b200 as E
    from exahype_b200 import slab as SL
    E.lib().exa_set_device(0)
    s = SL.SlabGrid(3, 2, (3, 3, 4), 0, 1)
    s.init(kind=0, param=5.0, seed=3, noise=1e-3)
    ring = SL.NcclRing(0, 1, SL.NcclRing.make_id())
    SL.prime(ring, s)
    SL.step(ring, s, 2)
    st = s.status()
    assert st['time'] > 0 and not st['nan']
    ring.destroy()
    s.destroy()
    assert 'torch' not in sys.modules, 'torch was imported on the slab path'
    print('no torch ok')
''')


def test_nccl_ring_needs_no_torch():
    """The slab transport runs in a process that never imports torch."""
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, '-c', _NO_TORCH, root], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert 'no torch ok' in r.stdout
