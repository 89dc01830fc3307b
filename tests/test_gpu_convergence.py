"""Order of accuracy of the whole ADER-DG step on the GPU: the 2D density
sine wave rho = 1 + A sin(2 pi (x + y)), u = v = 1, p = 1 is transported
unchanged, rho(x, y, t) = rho0(x - t, y - t), so the nodal error against it
must fall like h^(N+1) when the grid is refined (ADER-DG is of order N+1 in
space and time)."""
import numpy as np
import pytest

import exahype_b200 as E

pytestmark = pytest.mark.gpu
A = 0.1


def nodal_error(order, n, t_end):
    g = E.ADERDGGrid(2, order, (n, n), dt_policy=0)
    g.init(kind=1, param=A, seed=0, noise=0.0)
    while g.status()['time'] < t_end:
        g.step(1)
    t = g.status()['time']
    B = order + 1
    x01 = (np.polynomial.legendre.leggauss(B)[0] + 1.0) / 2.0
    u = g.get_state().reshape(n, n, B, B, 5)  # [cy][cx][iy][ix][var]
    cy, cx, iy, ix = np.meshgrid(np.arange(n), np.arange(n), np.arange(B), np.arange(B), indexing='ij')
    h = 1.0 / n
    x, y = (cx + x01[ix]) * h, (cy + x01[iy]) * h
    exact = 1.0 + A * np.sin(2 * np.pi * ((x - t) + (y - t)))
    g.destroy()
    return np.sqrt(np.mean((u[..., 0] - exact) ** 2))


@pytest.mark.parametrize('order', [2, 3, 4])
def test_sine_wave_convergence_order(order):
    t_end = 0.05
    e1 = nodal_error(order, 8, t_end)
    e2 = nodal_error(order, 16, t_end)
    rate = np.log2(e1 / e2)
    assert rate > order + 0.5, (e1, e2, rate)
