"""Parity at the benchmark configuration itself: 3D Euler ADER-DG N=4 on the
81^3 periodic grid (531,441 cells), isentropic vortex with seeded density
noise 1e-3.

The GPU grid is stepped with the library's own kernels; after steps 1, 5
and 20 a seeded sample of 2,000 cells of the GPU state is fed both to the
GPU's batched predictor + volume integral (exa_aderdg_predictor_vi, the
kernel the grid runs) and to the reference's own spaceTimePredictor and
volumeIntegral compiled from source (oracle/_ref; the oracle restatement
when that was not built), with the dt the grid took for the next step.
lduh, lQhbnd and lFhbnd must agree within 1e-12 relative L2 over the
sample (the FP64 bar), and the mixed-precision predictor's outputs on the
same sample are held to the mixed bar, 1e-8.  The grid's dt equals the
reference rule's minimum over all cells, and one whole-grid step is
compared with the reference's kernels driven in the reference's step order.
"""
import numpy as np
import pytest

import _oracle as O
import exahype_b200 as E
from exahype_b200 import DeviceBuffer

pytestmark = pytest.mark.gpu
N, ORDER, V = 81, 4, 5
B = ORDER + 1
NN, NF = B ** 3, B ** 2
K = 2000


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _reference_cells(luh_cells, dx, dt):
    """lduh, lQhbnd, lFhbnd of the reference's (or the oracle's) per-cell
    predictor + volume integral on each sampled cell."""
    R = O.ref_lib(3)
    out = {k: [] for k in ('lduh', 'qbnd', 'fbnd')}
    s = O.sizes(3, ORDER)
    dxa = np.asarray(dx, dtype=np.float64)
    for u in luh_cells:
        u = np.ascontiguousarray(u)
        lduh = np.zeros(s['lduh'])
        if R is not None:
            lqi, lqhi, lfhi = np.zeros(s['lQi']), np.zeros(s['lQhi']), np.zeros(s['lFhi'])
            qb, fb = np.zeros(s['qbnd']), np.zeros(s['fbnd'])
            assert R.ref_stp(ORDER, 0, u, lqi, lqhi, lfhi, qb, fb, dxa, dt) == 0
            R.ref_volume_integral(ORDER, lduh, lfhi, dxa)
        else:
            r = O.stp(3, ORDER, u, dx, dt)
            qb, fb = r['lQhbnd'], r['lFhbnd']
            O.lib().orc_volume_integral(3, ORDER, V, 0, lduh, r['lFhi'], dxa)
        out['lduh'].append(lduh)
        out['qbnd'].append(qb)
        out['fbnd'].append(fb)
    return {k: np.concatenate(v) for k, v in out.items()}


def _gpu_cells(luh_cells, dx, dt, precision):
    Kb = E.BatchedADERDG(3, ORDER, dx, precision=precision)
    n = len(luh_cells)
    s = O.sizes(3, ORDER)
    luh = DeviceBuffer.from_array(np.ascontiguousarray(luh_cells).ravel())
    b = {k: DeviceBuffer(n * s[k]) for k in ('lduh', 'qbnd', 'fbnd')}
    Kb.predictor_vi(n, luh, dt, b['lduh'], b['qbnd'], b['fbnd'])
    got = {k: v.download() for k, v in b.items()}
    for v in list(b.values()) + [luh]:
        v.free()
    return got


def _sample(k):
    return np.random.default_rng(100 + k).choice(N ** 3, size=K, replace=False)


@pytest.fixture(scope='module')
def headline():
    """{k: (sampled cells of the state after k steps, dt of step k+1)} and
    the whole state after step 5."""
    g = E.ADERDGGrid(3, ORDER, (N, N, N))
    g.init(kind=0, param=5.0, seed=1234, noise=1e-3)
    snaps, full, done = {}, None, 0
    for k in (1, 5, 20):
        g.step(k - done)
        done = k
        state = g.get_state()
        dt_next = float(g.step(1, want_dt=True)[0])
        g.set_state(state)  # back to the state after k steps
        snaps[k] = (state.reshape(N ** 3, NN * V)[_sample(k)].copy(), dt_next)
        if k == 5:
            full = (state, dt_next)
    g.destroy()
    return snaps, full


@pytest.mark.parametrize('k', [1, 5, 20])
def test_headline_sample_vs_reference(headline, k):
    u, dt = headline[0][k]
    dx = [1.0 / N] * 3
    ref = _reference_cells(u, dx, dt)
    got = _gpu_cells(u, dx, dt, E.PREC_FP64)
    for key in ('lduh', 'qbnd', 'fbnd'):
        e = rel(got[key], ref[key])
        assert e <= 1e-12, (k, key, e)
    mixed = _gpu_cells(u, dx, dt, E.PREC_MIXED)
    for key in ('lduh', 'qbnd', 'fbnd'):
        e = rel(mixed[key], ref[key])
        assert e <= 1e-8, ('mixed', k, key, e)


def test_headline_dt_is_reference_rule(headline):
    """The dt the grid took after step 5 is the reference's CFL x PNPM[N]
    rule minimised over all 531,441 cells (stableTimeStepSize.cpph:21-61 +
    the global min of TimeStepSizeComputation.cpp:83-109)."""
    state, dt = headline[1]
    n = np.full(3, N, dtype=np.int32)
    ref = O.lib().orc_aderdg_grid_dt(3, ORDER, 0, n, np.full(3, 1.0 / N), state, 0, 0.9)
    assert abs(dt - ref) <= 1e-15 * ref


def test_headline_whole_grid_step_vs_reference(headline):
    """One whole-grid step from the state after step 5, on the GPU grid and
    on the reference's kernels in the reference's step order (all host
    cores): the 81^3 state after it within 1e-12 relative L2."""
    R = O.ref_lib(3)
    if R is None or not hasattr(R, 'ref_grid_step_bc'):
        pytest.skip('reference kernels not built')
    state, dt = headline[1]
    g = E.ADERDGGrid(3, ORDER, (N, N, N))
    g.set_state(state)
    dts = g.step(1, want_dt=True)
    got = g.get_state()
    g.destroy()
    ref = state.copy()
    dt_r = O.ref_grid_step(3, ORDER, (N, N, N), ref, dt_policy=0)
    assert abs(dts[0] - dt_r) <= 1e-15 * dt_r
    assert rel(got, ref) <= 1e-12
