"""Design order of the whole ADER-DG step on the isentropic-vortex test.

Shu's isentropic vortex (strength 5, radius 0.1; density, velocity and
pressure from the published closed form) in the free stream u = v = 1,
centred in the periodic square [0, 2]^2 so that the domain boundary lies 10
radii from the centre (the tail there is ~1e-22: the initial state is
periodic to rounding, so the error has no floor).  At t = 0.25 the exact
solution is the initial state moved by (0.25, 0.25), a whole number of
cells at every resolution used, so the exact nodal values are the initial
cells rolled.  The GPU grid steps with a fixed dt (0.9 of the stable dt on
the initial state, t_end divided into whole steps) so time and space are
refined together; ADER-DG is of order N+1 in both, and the nodal L2 error
must fall faster than h^(N+0.5).  3D: the vortex extruded along z on a grid
two cells deep.  N=4 stops at 32^2: at 64^2 its error (~2e-7 after ~770
steps) reaches the level of the Picard stopping rule (the iteration stops
once the squared update falls below 1e-14, as the reference's does), so the
rate there measures that tolerance, not the discretisation.  The coarsest 2D
errors are also checked against the oracle's grid step on the same state and
dt.
"""
import numpy as np
import pytest

import _oracle as O
import exahype_b200 as E

pytestmark = pytest.mark.gpu
GAMMA = 1.4
L = 2.0
T_END = 0.25
NZ = 2


def vortex_nodes(dim, order, n, eps=5.0, R=0.1):
    """Nodal state [cells][nodes][5] in the library's per-cell layout
    (cells x-fastest, nodes at the ascending Gauss-Legendre points)."""
    B = order + 1
    x01 = (np.polynomial.legendre.leggauss(B)[0] + 1.0) / 2.0
    h = L / n
    if dim == 2:
        cy, cx, iy, ix = np.meshgrid(np.arange(n), np.arange(n), np.arange(B), np.arange(B), indexing='ij')
    else:
        _, cy, cx, _, iy, ix = np.meshgrid(np.arange(NZ), np.arange(n), np.arange(n), np.arange(B),
                                           np.arange(B), np.arange(B), indexing='ij')
    x, y = (cx + x01[ix]) * h, (cy + x01[iy]) * h
    xb, yb = (x - L / 2) / R, (y - L / 2) / R
    e = np.exp(0.5 * (1.0 - xb * xb - yb * yb))
    u = 1.0 - eps / (2 * np.pi) * yb * e
    v = 1.0 + eps / (2 * np.pi) * xb * e
    T = 1.0 - (GAMMA - 1) * eps * eps / (8 * GAMMA * np.pi ** 2) * e * e
    rho = T ** (1.0 / (GAMMA - 1))
    p = rho * T
    q = np.stack([rho, rho * u, rho * v, 0.0 * rho, p / (GAMMA - 1) + 0.5 * rho * (u * u + v * v)], -1)
    return q.ravel()


def setup(dim, order, n):
    h = L / n
    ns = (n, n) if dim == 2 else (n, n, NZ)
    length = (L, L) if dim == 2 else (L, L, NZ * h)
    u0 = vortex_nodes(dim, order, n)
    nn = np.asarray(ns, dtype=np.int32)
    planar = 1 if dim == 2 else 0
    dt_cfl = O.lib().orc_aderdg_grid_dt(dim, order, planar, nn, np.full(dim, h), u0, 0, 0.9)
    nsteps = int(np.ceil(T_END / (0.9 * dt_cfl)))
    return ns, length, u0, nsteps, T_END / nsteps


def exact(dim, order, n, u0):
    B = order + 1
    m = int(round(T_END * n / L))
    if dim == 2:
        return np.roll(u0.reshape(n, n, B * B * 5), (m, m), axis=(0, 1)).ravel()
    return np.roll(u0.reshape(NZ, n, n, B ** 3 * 5), (m, m), axis=(1, 2)).ravel()


def gpu_error(dim, order, n):
    ns, length, u0, nsteps, dt = setup(dim, order, n)
    g = E.ADERDGGrid(dim, order, ns, length=length, pde=E.PDE_EULER_PLANAR if dim == 2 else E.PDE_EULER,
                     dt_policy=2, dt_fixed=dt)
    g.set_state(u0)
    g.step(nsteps)
    u = g.get_state()
    st = g.status()
    g.destroy()
    assert not st['nan'] and abs(st['time'] - T_END) <= 1e-12
    e = u - exact(dim, order, n, u0)
    return float(np.sqrt(np.mean(e ** 2))), u


@pytest.mark.parametrize('dim,order,sizes', [(2, 2, (16, 32, 64)), (2, 3, (16, 32, 64)), (2, 4, (16, 32)),
                                              (3, 3, (16, 32)), (3, 4, (16, 32))])
def test_isentropic_vortex_convergence_order(dim, order, sizes):
    errs = [gpu_error(dim, order, n)[0] for n in sizes]
    rates = [np.log2(a / b) for a, b in zip(errs, errs[1:])]
    assert rates[-1] > order + 0.5, (errs, rates)
    assert all(r > order - 0.5 for r in rates), (errs, rates)


def test_vortex_gpu_equals_oracle_coarse():
    """The 2D N=3 16^2 run equals the oracle's grid step by step to the
    FP64 bar after all its steps."""
    dim, order, n = 2, 3, 16
    ns, length, u0, nsteps, dt = setup(dim, order, n)
    _, got = gpu_error(dim, order, n)
    ref = u0.copy()
    dx = np.full(dim, L / n)
    for _ in range(nsteps):
        O.grid_step(dim, order, ns, ref, dt_policy=2, dt_fixed=dt, planar=1, dx=dx)
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) <= 1e-12
