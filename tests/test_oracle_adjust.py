"""The oracle's solutionAdjustment restatement against the reference's own
kernel (kernels/aderdg/generic/c/{2d,3d}/solutionAdjustment.cpph compiled
in oracle/_ref), both calling the same built-in adjustPointSolution
forms: node positions, loop order and the t / dt handed to the hook must
agree.  The reference computes its Gauss-Legendre nodes at start-up and this
library derives them in extended precision (equal to within 2e-14,
tests/test_dg_tables.py), so a node coordinate can differ in its last bit:
the hook's values agree to a few units in the last place (2e-15
relative)."""
import numpy as np
import pytest

import _oracle as O

HOOKS = [(1, [0.2]), (2, [5.0]), (3, [0.7, 0.15, 3.0, 0.4, 0.55, 0.6])]


@pytest.mark.parametrize('dim', [2, 3])
@pytest.mark.parametrize('order', [2, 3, 4, 5])
@pytest.mark.parametrize('kind,param', HOOKS)
def test_adjustment_vs_reference(dim, order, kind, param):
    R = O.ref_lib(dim)
    if R is None or not hasattr(R, 'ref_solution_adjustment'):
        pytest.skip('reference kernels not built (make -C oracle ref)')
    rng = np.random.default_rng(10 * dim + order + 100 * kind)
    luh = rng.uniform(0.5, 2.0, (order + 1) ** dim * 5)
    center = rng.uniform(0.2, 0.8, dim)
    dx = rng.uniform(0.05, 0.2, dim)
    p = np.zeros(6)
    p[:len(param)] = param
    t, dt = 0.37, 2.5e-3
    ref, mine = luh.copy(), luh.copy()
    assert R.ref_solution_adjustment(order, ref, center, dx, t, dt, kind, p) == 0
    O.lib().orc_solution_adjustment(dim, order, mine, center, dx, t, dt, kind, 1, p)
    assert np.abs(mine - ref).max() <= 2e-15 * np.abs(ref).max()
    assert not np.array_equal(mine, luh)


def test_adjustment_at_start_only():
    luh = np.ones(4 ** 3 * 5)
    p = np.array([0.2, 0, 0, 0, 0, 0.0])
    a = luh.copy()
    O.lib().orc_solution_adjustment(3, 3, a, np.full(3, 0.5), np.full(3, 0.1), 0.1, 1e-3, 1, 0, p)
    assert np.array_equal(a, luh)  # t != 0: the hook does not fire
    O.lib().orc_solution_adjustment(3, 3, a, np.full(3, 0.5), np.full(3, 0.1), 0.0, 1e-3, 1, 0, p)
    assert not np.array_equal(a, luh)
