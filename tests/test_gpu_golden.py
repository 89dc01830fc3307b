"""The CUDA library's per-cell drop-ins against the reference's golden
vectors (same cases and eps as GenericEulerKernelTest{2D,3D})."""
import pytest

import _cases

pytestmark = pytest.mark.gpu


@pytest.fixture(scope='module')
def impl():
    from _gpu import GpuImpl
    return GpuImpl()


@pytest.mark.parametrize('case', _cases.CASES_3D, ids=lambda c: c.__name__)
def test_gpu_golden_3d(impl, golden3d, case):
    case(impl, golden3d)


@pytest.mark.parametrize('case', _cases.CASES_2D, ids=lambda c: c.__name__)
def test_gpu_golden_2d(impl, golden2d, case):
    case(impl, golden2d)


def test_gpu_stp_golden_tight(impl, golden3d):
    """The predictor reaches the golden data as closely as the reference's own
    kernels do (lQi 1.1e-12, fluxes ~1e-15)."""
    errs = _cases.stp_3d(impl, golden3d)
    assert errs['lQi'] < 5e-12 and errs['lFhbnd'] < 1e-13, errs
