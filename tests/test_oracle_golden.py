"""The CPU oracle against the reference's golden vectors."""
import pytest

import _cases


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
