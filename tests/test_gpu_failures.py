"""Failure detection, with every failure injected on the host (no device
fault, trap or endless wait):

* a non-finite state (the reference's validateNoNansInADERDGSolver,
  exahype/solvers/ADERDGSolver.cpp:1746): one node of one cell set to NaN
  before a step -> the grid's status reports EXA_ENAN and the NaN flag;
* Picard non-convergence (the warning of spaceTimePredictorNonlinear.cpph:
  308-315): a fixed dt four times the stable one -> cells stop at 2(N+1)
  iterations, the grid reports EXA_ENONCONV with the count, and the kept
  result still equals the oracle's step with the same dt;
* in the ensemble, a NaN planted in one solve's state stops that solve at
  the step that produced it (reported failed) while the others complete
  bitwise as they would without it.
"""
import ctypes as C

import numpy as np
import pytest

import _oracle as O
import exahype_b200 as E
from exahype_b200 import _lib

pytestmark = pytest.mark.gpu


def _raw_status(g):
    return int(E.lib().exa_aderdg_grid_status(g.h, None, None, None, None))


@pytest.mark.parametrize('graph', [False, True])
def test_grid_nan_reported(graph):
    g = E.ADERDGGrid(3, 3, (4, 3, 3))
    g.init(kind=0, param=5.0, seed=5, noise=1e-3)
    if graph:
        g.use_graph(True)
    g.step(2)
    st = g.status()
    assert st['code'] == _lib.EXA_OK and not st['nan']
    u = g.get_state()
    u[(7 * 64 + 10) * 5 + 0] = np.nan  # density of node 10 of cell 7
    g.set_state(u)
    g.step(2)
    st = g.status()
    assert st['nan'] and st['code'] == _lib.EXA_ENAN
    assert _raw_status(g) == _lib.EXA_ENAN
    g.destroy()


@pytest.mark.parametrize('graph', [False, True])
def test_grid_debug_scan_locates_first_nonfinite(graph):
    """Debug scan of each phase's outputs: a clean run records nothing; a
    NaN seeded into one node of cell 7 is first seen in the predictor's lduh
    of that cell (the cell whose Picard loop read it), in the step after it
    was seeded."""
    g = E.ADERDGGrid(3, 3, (4, 3, 3))
    g.init(kind=0, param=5.0, seed=5, noise=1e-3)
    if graph:
        g.use_graph(True)
    g.set_debug(True)
    g.step(2)
    assert g.debug_status() == (0, 0, 0)
    u = g.get_state()
    u[(7 * 64 + 10) * 5 + 0] = np.nan
    g.set_state(u)
    g.step(2)
    where, step, index = g.debug_status()
    assert where == 1 and step == 2
    assert 7 * 64 * 5 <= index < 8 * 64 * 5  # lduh of cell 7
    assert g.status()['nan']
    g.set_debug(False)
    g.destroy()


@pytest.mark.parametrize('dim,n', [(2, (6, 6)), (3, (3, 3, 3))])
def test_grid_picard_nonconvergence_reported(dim, n):
    order = 3
    planar = 1 if dim == 2 else 0
    pde = E.PDE_EULER_PLANAR if dim == 2 else E.PDE_EULER
    u0 = O.grid_ic(dim, order, n, kind=0, param=5.0, seed=3, noise=1e-3)
    nn = np.asarray(n, dtype=np.int32)
    dt_cfl = O.lib().orc_aderdg_grid_dt(dim, order, planar, nn, 1.0 / nn, u0, 0, 0.9)
    dt = 4.0 * dt_cfl
    g = E.ADERDGGrid(dim, order, n, pde=pde, dt_policy=2, dt_fixed=dt)
    g.set_state(u0)
    g.step(1)
    st = g.status()
    ref = u0.copy()
    _, its = O.grid_step(dim, order, n, ref, dt_policy=2, dt_fixed=dt, planar=planar)
    maxit = 2 * (order + 1)
    at_cap = int((its == maxit).sum())
    assert at_cap > 0
    assert 0 < st['nonconverged'] <= at_cap
    assert st['picard_iters'] == int(its.sum())
    assert st['code'] == _lib.EXA_ENONCONV and not st['nan']
    assert _raw_status(g) == _lib.EXA_ENONCONV
    got = g.get_state()
    assert np.isfinite(got).all()
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) <= 1e-10
    g.destroy()


def test_grid_converged_run_reports_ok():
    g = E.ADERDGGrid(2, 3, (6, 6), pde=E.PDE_EULER_PLANAR)
    g.init(kind=0, param=5.0, seed=3, noise=1e-3)
    g.step(3)
    st = g.status()
    assert st['code'] == _lib.EXA_OK and st['nonconverged'] == 0 and not st['nan']
    g.destroy()


MIX = [  # order, n, ic_kind, ic_param, pde, seed
    (2, (9, 9), 1, 0.05, E.PDE_EULER, 1),
    (4, (13, 17), 0, 5.0, E.PDE_EULER, 3),
    (3, (27, 27), 1, 0.2, E.PDE_EULER, 2),
]


def _cfg(order, n, kind, param, pde, seed):
    return E.solve_config(order, n, pde=pde, ic_kind=kind, ic_param=param, seed=seed, noise=1e-3)


@pytest.mark.parametrize('graph', [False, True])
def test_ensemble_nan_solve_fails_alone(graph):
    clean = E.Ensemble(8, 1 << 27)
    bad = E.Ensemble(8, 1 << 27)
    for ens in (clean, bad):
        if graph:
            ens.use_graph(True)
    sc = [clean.add(_cfg(*m), steps=6) for m in MIX]
    sb = [bad.add(_cfg(*m), steps=6) for m in MIX]
    for ens in (clean, bad):
        ens.step(2)
        ens.synchronize()
    # plant a NaN in the middle solve's state on the device
    ptr = bad.device_state_ptr(sb[1]).value
    nan = np.array([np.nan])
    _lib.call('exa_memcpy_h2d', C.c_void_p(ptr + 8 * 123), nan.ctypes.data, 8, None)
    E.device.synchronize()
    for _ in range(5):
        for ens in (clean, bad):
            ens.step(1)
            ens.status()
    sc_st, sb_st = clean.status(), bad.status()
    rc = E.lib().exa_ensemble_status(bad.h, None, None, None, None, None)
    assert rc == _lib.EXA_ENAN
    assert sb_st['nan'][sb[1]] == 1 and sb_st['active'][sb[1]] == 0
    assert int(sb_st['steps'][sb[1]]) == 2  # stopped at the step that produced the NaN
    for i in (0, 2):
        assert sb_st['nan'][sb[i]] == 0
        assert int(sb_st['steps'][sb[i]]) == 6 == int(sc_st['steps'][sc[i]])
        assert np.array_equal(bad.get_state(sb[i]), clean.get_state(sc[i]))
    clean.destroy()
    bad.destroy()
