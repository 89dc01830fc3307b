"""The CPU oracle against the reference's golden vectors."""
import numpy as np
import pytest

import _cases
import _oracle as O


@pytest.fixture(scope='module')
def impl():
    return _cases.OracleImpl()


@pytest.mark.parametrize('case', _cases.CASES_3D, ids=lambda c: c.__name__)
def test_oracle_3d(impl, golden3d, case):
    case(impl, golden3d)


@pytest.mark.parametrize('case', _cases.CASES_2D, ids=lambda c: c.__name__)
def test_oracle_2d(impl, golden2d, case):
    case(impl, golden2d)


def test_oracle_pde_fluxes(golden3d, golden2d):
    """GenericEulerKernelTest3D.cpp:132-160 / 2D: flux of one state"""
    import numpy as np
    import _oracle
    Q = np.array([1.0, 0.1, 0.2, 0.3, 3.5])
    F = np.zeros(15)
    _oracle.lib().orc_euler_flux(3, 0, Q, F)
    for i, k in enumerate('fgh'):
        assert np.allclose(F[5 * i:5 * i + 5], golden3d['testPDEFluxes/' + k], rtol=0, atol=1e-15)
    F2 = np.zeros(10)
    _oracle.lib().orc_euler_flux(2, 1, Q, F2)
    for i, k in enumerate('fg'):
        assert np.allclose(F2[5 * i:5 * i + 5], golden2d['testPDEFluxes/' + k], rtol=0, atol=1e-15)


def test_oracle_outflow_keeps_uniform_state():
    """With outflow boundaries a uniform state stays uniform (the boundary
    flux equals the interior flux), and a reflecting wall keeps the density
    of a state at rest."""
    dim, order, n = 2, 3, (4, 3)
    B = order + 1
    nc = n[0] * n[1]
    q = np.zeros((nc, B * B, 5))
    q[..., 0] = 1.0
    q[..., 1] = 0.3
    q[..., 2] = -0.2
    q[..., 4] = 2.5 + 0.5 * (0.3 ** 2 + 0.2 ** 2)
    u = q.ravel().copy()
    O.grid_step(dim, order, n, u, bc=[1, 1])
    assert np.allclose(u, q.ravel(), rtol=0, atol=1e-12)  # the periodic step shows the same 1e-13 rounding
    q[..., 1:3] = 0.0
    q[..., 4] = 2.5
    u = q.ravel().copy()
    O.grid_step(dim, order, n, u, bc=[2, 2])
    assert np.allclose(u.reshape(nc, B * B, 5)[..., 0], 1.0, rtol=0, atol=1e-12)
