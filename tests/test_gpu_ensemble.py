"""Ensemble of independent 2D solves in one persistent launch per step."""
import numpy as np
import pytest

import exahype_b200 as E
from exahype_b200.device import diff_norms

pytestmark = pytest.mark.gpu

MIX = [  # order, n, ic_kind, ic_param, pde, seed
    (2, (9, 9), 1, 0.05, E.PDE_EULER, 1),
    (3, (27, 27), 1, 0.2, E.PDE_EULER, 2),
    (4, (13, 17), 0, 5.0, E.PDE_EULER, 3),
    (5, (11, 9), 1, 0.3, E.PDE_EULER_PLANAR, 4),
    (3, (40, 12), 0, 5.0, E.PDE_EULER, 5),
    (2, (81, 81), 1, 0.1, E.PDE_EULER, 6),
]


def cfg(order, n, kind, param, pde, seed, noise=1e-3):
    return E.solve_config(order, n, pde=pde, ic_kind=kind, ic_param=param, seed=seed, noise=noise)


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def test_ensemble_matches_single_grids():
    ens = E.Ensemble(16, 1 << 28)
    slots = [ens.add(cfg(*m)) for m in MIX]
    ens.step(8)
    ens.synchronize()
    st = ens.status()
    for sl, (order, n, kind, param, pde, seed) in zip(slots, MIX):
        g = E.ADERDGGrid(2, order, n, pde=pde)
        g.init(kind=kind, param=param, seed=seed, noise=1e-3)
        g.step(8)
        ref = g.get_state()
        got = ens.get_state(sl)
        assert rel(got, ref) < 1e-13, (order, n, rel(got, ref))
        assert abs(st['time'][sl] - g.status()['time']) <= 1e-13 * g.status()['time']
        assert st['steps'][sl] == 8
        g.destroy()
    ens.destroy()


def test_ensemble_step_budget_and_graph():
    a = E.Ensemble(8, 1 << 26)
    b = E.Ensemble(8, 1 << 26)
    b.use_graph(True)
    budgets = [3, 7, -1]
    for ens in (a, b):
        for m, k in zip(MIX[:3], budgets):
            ens.add(cfg(*m), steps=k)
    for _ in range(5):
        a.step(2)
        b.step(2)
        a.status()
        b.status()  # drops finished solves before the next step
    sa, sb = a.status(), b.status()
    assert list(sa['steps'][:3]) == [3, 7, 10]
    assert list(sa['active'][:3]) == [0, 0, 1]
    for sl in range(3):
        assert np.array_equal(a.get_state(sl), b.get_state(sl))
    a.destroy()
    b.destroy()


def test_result_identical_alone_and_in_mix():
    alone = E.Ensemble(4, 1 << 26)
    mixed = E.Ensemble(16, 1 << 28)
    target = (4, (13, 17), 0, 5.0, E.PDE_EULER, 3)
    s_alone = alone.add(cfg(*target), steps=6)
    for m in MIX[:2]:
        mixed.add(cfg(*m), steps=9)
    s_mix = mixed.add(cfg(*target), steps=6)
    for m in MIX[4:]:
        mixed.add(cfg(*m), steps=4)
    for _ in range(9):
        alone.step(1)
        mixed.step(1)
        alone.status()
        mixed.status()
    assert np.array_equal(alone.get_state(s_alone), mixed.get_state(s_mix))
    alone.destroy()
    mixed.destroy()


def test_admission_by_footprint():
    c = cfg(5, (60, 60), 1, 0.2, E.PDE_EULER, 9)
    fp = E.ensemble.footprint(c)
    ens = E.Ensemble(4, int(fp * 1.5))
    s0 = ens.add(c)
    assert s0 is not None
    assert ens.add(c) is None  # does not fit: EXA_EBUSY
    ens.remove(s0)
    assert ens.add(c) is not None
    ens.destroy()


@pytest.mark.parametrize('seed', [0])
def test_mixed_ensemble_vs_fp64(seed):
    a = E.Ensemble(16, 1 << 28, precision=E.PREC_FP64)
    b = E.Ensemble(16, 1 << 28, precision=E.PREC_MIXED)
    sa = [a.add(cfg(*m)) for m in MIX]
    sb = [b.add(cfg(*m)) for m in MIX]
    for _ in range(10):
        a.step(1)
        b.step(1)
    a.synchronize()
    b.synchronize()
    for x, y in zip(sa, sb):
        e = diff_norms(b.device_state_ptr(y), a.device_state_ptr(x), a.state_size(x))
        assert e['rel_l2'] <= 1e-8, e
    a.destroy()
    b.destroy()


def test_contraction_choice_agrees_and_autotuner_applies_it():
    """Every order's predictor gives the same solves with either contraction
    inside the persistent launch (to rounding), and the autotuner's
    contraction stage and schedule stage produce a applied 4-tuple."""
    from exahype_b200.autotune import tune_ensemble
    mix = MIX[:4]
    a = E.Ensemble(8, 1 << 27)
    b = E.Ensemble(8, 1 << 27)
    sa = [a.add(cfg(*m), steps=5) for m in mix]
    sb = [b.add(cfg(*m), steps=5) for m in mix]
    b.tune_contraction(0x0C)  # orders 2 and 3 line-owner, 4 and 5 node-gather: the opposite of the default
    for ens in (a, b):
        ens.step(5)
        ens.status()
    for x, y in zip(sa, sb):
        assert rel(b.get_state(y), a.get_state(x)) < 1e-12
    a.destroy()
    b.destroy()
    c = E.Ensemble(8, 1 << 27)
    for m in mix:
        c.add(cfg(*m))
    best, table = tune_ensemble(c, steps=1, ctas=(1,), grabs=(1, 2), orders=(0,))
    assert len(best) == 5 and best[3] & ~0x3C == 0 and best[4] in (0, 1)
    assert sum(1 for r in table if r['stage'] == 'contraction') == 1 + len({m[0] for m in mix})
    c.step(2)
    assert not c.status()['nan'].any()
    c.destroy()


@pytest.mark.parametrize('precision', [E.PREC_FP64, E.PREC_MIXED])
def test_per_order_launches_equal_persistent(precision):
    """One launch per order and phase gives the solves of the persistent
    launch bit for bit (the same block functions on the same data), with
    step budgets, graph replay and a solve added mid-run."""
    a = E.Ensemble(16, 1 << 28, precision=precision)
    b = E.Ensemble(16, 1 << 28, precision=precision)
    b.set_launch_mode(1)
    for ens in (a, b):
        ens.use_graph(True)
        for m, k in zip(MIX, [6, 3, -1, 5, 4, 6]):
            ens.add(cfg(*m), steps=k)
    for k in range(6):
        for ens in (a, b):
            ens.step(1)
            ens.status()
        if k == 2:
            for ens in (a, b):
                ens.add(cfg(3, (10, 12), 0, 5.0, E.PDE_EULER, 77), steps=3)
    sa, sb = a.status(), b.status()
    assert np.array_equal(sa['steps'], sb['steps']) and np.array_equal(sa['time'], sb['time'])
    for sl in a.cfgs:
        assert np.array_equal(a.get_state(sl), b.get_state(sl)), sl
    a.destroy()
    b.destroy()


@pytest.mark.parametrize('precision,bar', [(E.PREC_FP64, 1e-12), (E.PREC_MIXED, 1e-8)])
def test_ensemble_vs_reference_kernels(precision, bar):
    """Every solve of a small ensemble (orders 2..5) against the reference's
    own kernels compiled from source stepping the same initial state the
    same number of steps (each with its own CFL dt): relative L2 <= 1e-12
    for FP64 and <= 1e-8 for the mixed-precision form."""
    import _oracle as O
    R = O.ref_lib(2)
    if R is None or not hasattr(R, 'ref_grid_step_bc'):
        pytest.skip('reference kernels not built')
    mix = [(2, (10, 9), 1, 0.2, 11), (3, (9, 12), 1, 0.25, 12), (4, (8, 8), 0, 5.0, 13), (5, (7, 9), 1, 0.15, 14)]
    ens = E.Ensemble(8, 1 << 27, precision=precision)
    slots = [ens.add(cfg(o, n, kind, param, E.PDE_EULER, seed)) for o, n, kind, param, seed in mix]
    init = {sl: ens.get_state(sl) for sl in slots}
    steps = 5
    ens.step(steps)
    ens.synchronize()
    for sl, (order, n, _, _, _) in zip(slots, mix):
        ref = init[sl].copy()
        for _ in range(steps):
            O.ref_grid_step(2, order, n, ref, dt_policy=0)
        got = ens.get_state(sl)
        assert rel(got, ref) <= bar, (order, rel(got, ref))
    ens.destroy()
