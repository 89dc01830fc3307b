"""Limiting ADER-DG grid on the GPU (exa_aderdg_grid_set_limiter) against
the oracle's restated step (orc_limiting_grid_step), 2D and 3D, periodic
and with outflow / reflecting walls: the same
cell statuses and counts every step (exact), the same state within FP64
rounding (1e-11 relative: the DG candidate and the projections sum in
different orders; 1e-9 for the 3D MUSCL-Hancock case, whose step amplifies
rounding differences), the dt sequence to a tenth of that and the DMP bounds
to 100x that (they include Gauss-Lobatto values, which extrapolate)."""
import numpy as np
import pytest

import _limiting_ic as IC
import _oracle as O
from exahype_b200 import ADERDGGrid

pytestmark = pytest.mark.gpu


def run_pair(order, n, luh, steps, scheme=0, nobs=5, cured=0, graph=False, tol=1e-11, bc=None):
    g = ADERDGGrid(len(n), order, n, length=(1.0,) * len(n))
    g.set_state(luh)
    if bc:
        g.set_boundary(bc)
    g.set_limiter(scheme=scheme, nobs=nobs, steps_till_cured=cured)
    if graph:
        g.use_graph(True)
    o = O.LimitingGrid(order, n, luh, scheme=scheme, nobs=nobs, steps_till_cured=cured, bc=bc)
    seen = 0
    for k in range(steps):
        dts = g.step(1, want_dt=True)
        dt_ref = o.step()
        assert abs(dts[0] - dt_ref) <= 0.1 * tol * dt_ref, k
        st, counts = g.limiter_status()
        assert np.array_equal(st, o.status), k
        assert np.array_equal(counts, o.counts), k
        seen += counts[2]
        u = g.get_state()
        assert np.abs(u - o.luh).max() <= tol * np.abs(o.luh).max(), k
        mn, mx = g.limiter_bounds()
        # the extrema include Gauss-Lobatto values, which extrapolate the
        # nodal values (up to ~2x per axis): 1e-9 relative for the bounds
        scale = max(np.abs(o.bmin).max(), np.abs(o.bmax).max())
        assert np.abs(mn - o.bmin).max() <= 100 * tol * scale and np.abs(mx - o.bmax).max() <= 100 * tol * scale, k
    return seen


@pytest.mark.parametrize('order,n,scheme', [(3, (16, 16), 0), (2, (20, 14), 1), (4, (12, 12), 0)])
def test_limiting_grid_vs_oracle(order, n, scheme):
    seen = run_pair(order, n, IC.explosion(order, n), 8, scheme=scheme)
    assert seen > 0  # the run exercised the FV recomputation


def test_limiting_grid_cure_delay_and_observables():
    order, n = 3, (16, 16)
    run_pair(order, n, IC.explosion(order, n), 6, nobs=1, cured=2)


def test_limiting_graph_replay_matches_eager():
    order, n = 3, (16, 16)
    run_pair(order, n, IC.explosion(order, n), 5, graph=True)


def test_smooth_state_unlimited():
    """With nothing troubled, the limiting grid reproduces the plain grid."""
    order, n = 3, (16, 12)
    luh = IC.smooth(order, n, amp=0.05)
    a = ADERDGGrid(2, order, n, length=(1.0, 1.0))
    b = ADERDGGrid(2, order, n, length=(1.0, 1.0))
    a.set_state(luh)
    b.set_state(luh)
    b.set_limiter()
    da = a.step(6, want_dt=True)
    db = b.step(6, want_dt=True)
    assert np.abs(da - db).max() <= 1e-15 * da.max()
    assert np.abs(a.get_state() - b.get_state()).max() <= 1e-13
    st, counts = b.limiter_status()
    assert counts.tolist() == [0, 0, 0] and not st.any()


@pytest.mark.parametrize('order,n,scheme', [(2, (8, 8, 8), 0), (3, (6, 7, 5), 1), (4, (6, 6, 6), 0)])
def test_limiting_grid_3d_vs_oracle(order, n, scheme):
    # 3D MUSCL-Hancock subcells on this state amplify rounding-level input
    # differences ~1e4-fold per step (test_oracle_limiting.py measures it
    # with the oracle alone): 1e-9 there, 1e-11 otherwise
    seen = run_pair(order, n, IC.explosion3d(order, n), 4, scheme=scheme, tol=1e-9 if scheme == 1 else 1e-11)
    assert seen > 0


@pytest.mark.parametrize('order,n,scheme,bc', [(3, (14, 12), 0, [1, 2]), (2, (16, 12), 1, [2, 1]),
                                                (3, (12, 12), 1, [2, 0])])
def test_limiting_grid_walls_vs_oracle(order, n, scheme, bc):
    """outflow / reflecting walls: explosions that touch the walls, so FV
    patches fill their ghost layers from their own boundary layers"""
    luh = IC.explosion(order, n, center=(0.08, 0.1), radius=0.25)
    seen = run_pair(order, n, luh, 8, scheme=scheme, bc=bc)
    assert seen > 0


@pytest.mark.parametrize('order,n,scheme,bc,center', [(2, (8, 7, 6), 0, [2, 1, 2], (0.1, 0.12, 0.15)),
                                                       (3, (6, 6, 5), 1, [1, 2, 2], (0.85, 0.9, 0.8)),
                                                       (2, (7, 6, 6), 1, [2, 2, 0], (0.2, 0.2, 0.8))])
def test_limiting_grid_3d_walls_vs_oracle(order, n, scheme, bc, center):
    # a milder jump than the periodic cases: with (0.125, 0.1) outside, DG
    # cells at a wall can end a step admissible at their nodes but negative
    # between them, and the next step's subcell FV of that state blows up
    # in the oracle as well
    luh = IC.explosion3d(order, n, center=center, radius=0.3, outer=(0.5, 0.4))
    seen = run_pair(order, n, luh, 4, scheme=scheme, bc=bc, tol=1e-9 if scheme == 1 else 1e-11)
    assert seen > 0


def test_limiting_walls_graph_replay():
    order, n = 3, (12, 10)
    run_pair(order, n, IC.explosion(order, n, center=(0.9, 0.9), radius=0.25), 5, graph=True, bc=[2, 1])


def test_limiter_rejects_bad_parameters():
    g = ADERDGGrid(3, 3, (4, 4, 4))
    for bad in (dict(scheme=2), dict(nobs=0), dict(nobs=6), dict(relaxation=-1.0), dict(steps_till_cured=-1)):
        with pytest.raises(Exception):
            g.set_limiter(**bad)
