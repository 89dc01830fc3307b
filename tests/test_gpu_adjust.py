"""Solution adjustment on the GPU (exa_aderdg_solution_adjustment, the
per-cell drop-in and the grid's per-step hook) against the oracle's
restatement of solutionAdjustment.cpph, which test_oracle_adjust.py pins to
the reference's compiled kernel.  The hooks evaluate sin / exp / pow on the
device and in the host's libm: values agree to 1e-14 relative; the grid
runs with the hook after every update and is compared step by step with the
oracle grid (state 1e-12 relative, dt 1e-13)."""
import numpy as np
import pytest

import _oracle as O
import exahype_b200 as E
from exahype_b200 import DeviceBuffer
from exahype_b200.aderdg import BatchedADERDG

pytestmark = pytest.mark.gpu
HOOKS = [(E.ADJUST_SINE_WAVE, [0.2]), (E.ADJUST_ISENTROPIC_VORTEX, [5.0]),
         (E.ADJUST_HEAT_SOURCE, [0.7, 0.15, 3.0, 0.4, 0.55, 0.6])]


def _p6(param):
    p = np.zeros(6)
    p[:len(param)] = param
    return p


@pytest.mark.parametrize('dim', [2, 3])
@pytest.mark.parametrize('order', [2, 3, 4, 5])
@pytest.mark.parametrize('kind,param', HOOKS)
def test_batched_adjustment_vs_oracle(dim, order, kind, param):
    rng = np.random.default_rng(7 * dim + order + 50 * kind)
    nc, nn = 37, (order + 1) ** dim
    dx = rng.uniform(0.05, 0.2, dim)
    luh = rng.uniform(0.5, 2.0, nc * nn * 5)
    centers = rng.uniform(0.1, 0.9, (nc, dim))
    B = BatchedADERDG(dim, order, dx)
    d_luh, d_c = DeviceBuffer.from_array(luh), DeviceBuffer.from_array(centers.ravel())
    t, dt = 0.41, 3e-3
    B.solution_adjustment(nc, d_luh, d_c, t, dt, E.adjust_hook(kind, param))
    got = d_luh.download().reshape(nc, -1)
    for c in range(nc):
        ref = luh[c * nn * 5:(c + 1) * nn * 5].copy()
        O.lib().orc_solution_adjustment(dim, order, ref, np.ascontiguousarray(centers[c]), dx, t, dt, kind, 1,
                                        _p6(param))
        assert np.abs(got[c] - ref).max() <= 1e-14 * np.abs(ref).max(), c


def test_at_start_hook_and_drop_in():
    dim, order = 3, 3
    nn = 4 ** 3
    luh = np.random.default_rng(3).uniform(0.5, 2.0, nn * 5)
    center, dx = np.array([0.45, 0.5, 0.55]), np.array([0.1, 0.1, 0.1])
    hook = E.adjust_hook(E.ADJUST_SINE_WAVE, [0.2], when=E.ADJUST_AT_START)
    a = luh.copy()
    E.solutionAdjustment(dim, order, a, center, dx, 0.25, 1e-3, hook)
    assert np.array_equal(a, luh)  # t != 0: useAdjustSolution says no
    E.solutionAdjustment(dim, order, a, center, dx, 0.0, 0.0, hook)
    ref = luh.copy()
    O.lib().orc_solution_adjustment(dim, order, ref, center, dx, 0.0, 0.0, 1, 0, _p6([0.2]))
    assert np.abs(a - ref).max() <= 1e-14 * np.abs(ref).max()
    with pytest.raises(E.ExaError):
        E.solutionAdjustment(dim, order, a, center, dx, 0.0, 0.0, E.adjust_hook(9))


@pytest.mark.parametrize('dim,order,n', [(3, 3, (5, 4, 3)), (2, 4, (9, 7))])
def test_grid_with_heat_source_vs_oracle(dim, order, n):
    g = E.ADERDGGrid(dim, order, n)
    g.init(kind=1, param=0.2, seed=3, noise=1e-3)
    u = g.get_state()
    param = [2.0, 0.2, 5.0, 0.5, 0.45, 0.5]
    g.set_adjustment(E.adjust_hook(E.ADJUST_HEAT_SOURCE, param))
    nn = np.asarray(n, dtype=np.int32)
    dxv = 1.0 / nn.astype(np.float64)
    dt = O.lib().orc_aderdg_grid_dt(dim, order, 0, nn, dxv, u, 0, 0.9)
    t = 0.0
    idx = np.stack(np.meshgrid(*[np.arange(k) for k in n], indexing='ij'), -1)
    # cells x fastest: cell c = (z * ny + y) * nx + x
    cells = idx.transpose(list(range(dim))[::-1] + [dim]).reshape(-1, dim)
    centers = (cells + 0.5) * dxv
    per = (order + 1) ** dim * 5
    for s in range(5):
        dt_gpu = g.step(1, want_dt=True)[0]
        assert abs(dt_gpu - dt) <= 1e-13 * dt, s
        O.grid_step(dim, order, n, u, dt_policy=2, dt_fixed=dt)
        for c in range(len(centers)):
            blk = u[c * per:(c + 1) * per]
            O.lib().orc_solution_adjustment(dim, order, blk, np.ascontiguousarray(centers[c]), dxv, t + dt, dt,
                                            3, 1, _p6(param))
            u[c * per:(c + 1) * per] = blk
        t += dt
        dt = O.lib().orc_aderdg_grid_dt(dim, order, 0, nn, dxv, u, 0, 0.9)
        got = g.get_state()
        assert np.linalg.norm(got - u) <= 1e-12 * np.linalg.norm(u), s
    # the source heats: total energy grew
    assert u.reshape(-1, 5)[:, 4].sum() > 0


def test_grid_adjustment_rejects_limiter():
    g = E.ADERDGGrid(2, 3, (8, 8))
    g.set_adjustment(E.adjust_hook(E.ADJUST_HEAT_SOURCE, [1.0, 0.2, 1.0, 0.5, 0.5, 0.0]))
    with pytest.raises(E.ExaError):
        g.set_limiter()
    g.set_adjustment(None)
    g.set_limiter()
