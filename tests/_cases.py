"""Known-answer cases of the reference's kernel tests, restated over an
implementation object so the same cases check the CPU oracle and the CUDA
library.  Inputs, tolerances and comparisons follow
ExaHyPE/exahype/tests/kernels/c/GenericEulerKernelTest3D.cpp and
GenericEulerKernelTest2D.cpp (order 3, 5 variables, 1 parameter,
eps = 1e-10, GenericEulerKernelTest.h:28-31,78).

An implementation provides:
  stp(dim, order, npar, planar, luh, dx, dt) -> dict(lQi, lFi, lQhi, lFhi, lQhbnd, lFhbnd)
  vi(dim, order, lFhi, dx) -> lduh          (volume integral incl. source block)
  si(dim, order, lduh, lFhbnd, dx) -> lduh  (surface integral, in place semantics)
  riemann(dim, order, npar, planar, FL, FR, QL, QR, direction) -> (FL, FR)
  update(dim, order, npar, luh, lduh, dt) -> luh
"""
import numpy as np

EPS = 1e-10
N, B, V, P, D = 3, 4, 5, 1, 6


def _strided(a, n_nodes, nvar=V, ndata=D):
    """test data use stride nVar; the kernels see stride nData (1 parameter)"""
    out = np.zeros((n_nodes, ndata))
    out[:, :nvar] = np.asarray(a).reshape(n_nodes, nvar)
    return out.ravel()


def _unstride(a, n_nodes, nvar=V, ndata=D):
    return np.asarray(a).reshape(n_nodes, ndata)[:, :nvar].ravel()


def close(a, b, eps=EPS):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape, (a.shape, b.shape)
    err = np.max(np.abs(a - b)) if a.size else 0.0
    assert err <= eps, 'max |diff| = %g > %g' % (err, eps)
    return err


# ------------------------------------------------------------------- 3D
def stp_3d(impl, g):
    """GenericEulerKernelTest3D.cpp:618-773"""
    luh = _strided(g['testSpaceTimePredictorNonlinear/luh'], B ** 3)
    r = impl.stp(3, N, P, 0, luh, [0.05] * 3, 1.083937460199773e-3)
    errs = {}
    errs['lQi'] = close(_unstride(r['lQi'], B ** 4), g['testSpaceTimePredictorNonlinear/lQi'])
    lfi = np.asarray(r['lFi']).reshape(B, B, B, B, 4, V)[:, :, :, :, :3, :].ravel()
    errs['lFi'] = close(lfi, g['testSpaceTimePredictorNonlinear/lFi'])
    errs['lQhi'] = close(_unstride(r['lQhi'], B ** 3), g['testSpaceTimePredictorNonlinear/lQhi'])
    errs['lFhi'] = close(np.asarray(r['lFhi'])[:3 * B ** 3 * V], g['testSpaceTimePredictorNonlinear/lFhi'])
    errs['lQhbnd'] = close(_unstride(r['lQhbnd'], 6 * B * B), g['testSpaceTimePredictorNonlinear/lQhbnd'])
    errs['lFhbnd'] = close(r['lFhbnd'], g['testSpaceTimePredictorNonlinear/lFhbnd'])
    return errs


def vi_3d(impl, g):
    """GenericEulerKernelTest3D.cpp:186-224"""
    lFhi = np.zeros(1280)
    for i in range(0, 320, 5):
        lFhi[i + 1] = 1.0
        lFhi[320 + i + 2] = 1.0
        lFhi[640 + i + 3] = 1.0
    lduh = impl.vi(3, N, lFhi, [0.05] * 3)
    return close(lduh, g['testVolumeIntegralNonlinear/lduh'])


def si_3d(impl, g):
    """GenericEulerKernelTest3D.cpp:267-310"""
    lF = np.zeros(480)
    for i in range(0, 80, 5):
        lF[i + 1] = 1.0
        lF[80 + i + 1] = 1.0
        lF[160 + i + 2] = 1.0
        lF[240 + i + 2] = 1.0
        lF[320 + i + 3] = 1.0
        lF[400 + i + 3] = 1.0
    lduh = np.arange(320) / 10.0
    out = impl.si(3, N, lduh, lF, [0.1] * 3)
    return close(out, g['testSurfaceIntegralNonlinear/lduh'])


def riemann_3d(impl, g):
    """GenericEulerKernelTest3D.cpp:410-488 (normalNonZero = 1)"""
    FL = np.arange(80, dtype=np.float64) + 1.0
    FR = np.arange(80, dtype=np.float64) - 1.0
    QL = _strided(g['testRiemannSolver/QL'], B * B)
    QR = _strided(g['testRiemannSolver/QR'], B * B)
    FL, FR = impl.riemann(3, N, P, 0, FL, FR, QL, QR, 1)
    return max(close(FL, g['testRiemannSolverNonlinear/FL']),
               close(FR, g['testRiemannSolverNonlinear/FR']))


def update_3d(impl, g):
    """GenericEulerKernelTest3D.cpp:495-532 (only the first B^2 nodes are
    compared, as in the reference)"""
    luh = np.zeros(D * B ** 3)
    luh[0::D] = 1.0
    luh[4::D] = 2.5
    lduh = np.arange(V * B ** 3, dtype=np.float64)
    out = impl.update(3, N, P, luh, lduh, 1.40831757919882352703e-03)
    got = _unstride(out, B ** 3)[:B * B * V]
    return close(got, g['testSolutionUpdate/luh'][:B * B * V])


# ------------------------------------------------------------------- 2D
def stp_2d(impl, g):
    """GenericEulerKernelTest2D.cpp:900-1010 (2.5D planar Euler)"""
    luh = _strided(g['testSpaceTimePredictorNonlinear/luh'], B ** 2)
    r = impl.stp(2, N, P, 1, luh, [0.05] * 2, 1.686854344081342e-3)
    errs = {}
    errs['lQi'] = close(_unstride(r['lQi'], B ** 3), g['testSpaceTimePredictorNonlinear/lQi'])
    lfi = np.asarray(r['lFi']).reshape(B, B, B, 3, V)[:, :, :, :2, :].ravel()
    errs['lFi'] = close(lfi, g['testSpaceTimePredictorNonlinear/lFi'])
    errs['lQhi'] = close(_unstride(r['lQhi'], B ** 2), g['testSpaceTimePredictorNonlinear/lQhi'])
    errs['lFhi'] = close(np.asarray(r['lFhi'])[:2 * B * B * V], g['testSpaceTimePredictorNonlinear/lFhi'])
    errs['lQhbnd'] = close(_unstride(r['lQhbnd'], 4 * B), g['testSpaceTimePredictorNonlinear/lQhbnd'])
    errs['lFhbnd'] = close(r['lFhbnd'], g['testSpaceTimePredictorNonlinear/lFhbnd'])
    return errs


def vi_2d(impl, g):
    """GenericEulerKernelTest2D.cpp:758-820, both sub-tests"""
    dx1 = [3.70370370370370349811e-02] * 2
    e1 = close(impl.vi(2, N, g['testVolumeIntegral/lFhi'], dx1), g['testVolumeIntegralNonlinear/lduh_1'])
    lFhi = np.zeros(240)
    for i in range(0, 80, 5):
        lFhi[i + 1] = 1.0
        lFhi[80 + i + 2] = 1.0
    e2 = close(impl.vi(2, N, lFhi, [0.05] * 2), g['testVolumeIntegralNonlinear/lduh_2'])
    return max(e1, e2)


def si_2d(impl, g):
    """GenericEulerKernelTest2D.cpp:265-343, both sub-tests"""
    lF = np.zeros(80)
    for i in range(0, 20, 5):
        lF[i + 1] = 1.0
        lF[20 + i + 1] = 1.0
        lF[40 + i + 2] = 1.0
        lF[60 + i + 2] = 1.0
    e1 = close(impl.si(2, N, g['testSurfaceIntegral/lduh_in'].copy(), lF, [0.1] * 2),
               g['testSurfaceIntegralNonlinear/lduh_1'])
    e2 = close(impl.si(2, N, g['testSurfaceIntegral/lduh_in'].copy(), g['testSurfaceIntegral/lFhbnd_in'],
                       [0.1] * 2), g['testSurfaceIntegralNonlinear/lduh_2'])
    return max(e1, e2)


def riemann_2d(impl, g):
    """GenericEulerKernelTest2D.cpp:501-700: constant state gives FL == FR;
    recorded inputs in directions 0 and 1."""
    q = np.tile([1.0, 0.0, 0.0, 0.0, 2.5], B)
    FL, FR = impl.riemann(2, N, P, 1, np.zeros(20), np.zeros(20), _strided(q, B), _strided(q, B), 0)
    assert np.array_equal(FL, FR)
    errs = []
    for k, d in (('1', 0), ('2', 1)):
        QL = _strided(g['testRiemannSolverNonlinear/QL_%s_in' % k], B)
        QR = _strided(g['testRiemannSolverNonlinear/QR_%s_in' % k], B)
        FL = g['testRiemannSolverNonlinear/FL_%s_in' % k].copy()
        FR = g['testRiemannSolverNonlinear/FR_%s_in' % k].copy()
        FL, FR = impl.riemann(2, N, P, 1, FL, FR, QL, QR, d)
        errs.append(close(FL, g['testRiemannSolverNonlinear/F_%s_out' % k]))
        errs.append(close(FR, g['testRiemannSolverNonlinear/F_%s_out' % k]))
    return max(errs)


def update_2d(impl, g):
    """GenericEulerKernelTest2D.cpp:154-190"""
    luh = np.zeros(D * B * B)
    luh[0::D] = 1.0
    luh[4::D] = 2.5
    out = impl.update(2, N, P, luh, g['testSolutionUpdate/lduh'], 1.40831757919882352703e-03)
    return close(_unstride(out, B * B), g['testSolutionUpdate/luh'])


CASES_3D = [stp_3d, vi_3d, si_3d, riemann_3d, update_3d]
CASES_2D = [stp_2d, vi_2d, si_2d, riemann_2d, update_2d]


class OracleImpl:
    """The CPU oracle (oracle/liboracle.so)."""

    def __init__(self):
        import _oracle
        self.O = _oracle

    def stp(self, dim, order, npar, planar, luh, dx, dt):
        return self.O.stp(dim, order, luh, dx, dt, npar=npar, planar=planar)

    def vi(self, dim, order, lFhi, dx):
        out = np.zeros((order + 1) ** dim * V)
        self.O.lib().orc_volume_integral(dim, order, V, 1, out, np.ascontiguousarray(lFhi, dtype=np.float64),
                                         np.asarray(dx, dtype=np.float64))
        return out

    def si(self, dim, order, lduh, lF, dx):
        lduh = np.array(lduh, dtype=np.float64)
        self.O.lib().orc_surface_integral(dim, order, V, lduh, np.ascontiguousarray(lF, dtype=np.float64),
                                          np.asarray(dx, dtype=np.float64))
        return lduh

    def riemann(self, dim, order, npar, planar, FL, FR, QL, QR, d):
        FL, FR = np.array(FL, dtype=np.float64), np.array(FR, dtype=np.float64)
        self.O.lib().orc_riemann(dim, order, V, npar, planar, FL, FR, np.ascontiguousarray(QL),
                                 np.ascontiguousarray(QR), d)
        return FL, FR

    def update(self, dim, order, npar, luh, lduh, dt):
        luh = np.array(luh, dtype=np.float64)
        self.O.lib().orc_solution_update(dim, order, V, npar, luh, np.ascontiguousarray(lduh, dtype=np.float64),
                                         dt)
        return luh
