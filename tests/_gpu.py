"""GPU-side implementation object for the shared reference cases: every
call goes through libexahype_b200.so (C ABI)."""
import numpy as np

import exahype_b200 as E

V = 5


class GpuImpl:
    def _solver(self, dim, order, npar=0, planar=0, dx=None):
        return E.ADERDGSolver(dim, order, npar=npar, pde=E.PDE_EULER_PLANAR if planar else E.PDE_EULER,
                              dx=dx if dx is not None else [1.0] * dim)

    def stp(self, dim, order, npar, planar, luh, dx, dt):
        s = self._solver(dim, order, npar, planar, dx)
        B, Dd = order + 1, V + npar
        nn = B ** dim
        lQi = np.zeros(nn * B * Dd)
        lFi = np.zeros(nn * B * (dim + 1) * V)
        lQhi = np.zeros(nn * Dd)
        lFhi = np.zeros(nn * (dim + 1) * V)
        qb = np.zeros(2 * dim * B ** (dim - 1) * Dd)
        fb = np.zeros(2 * dim * B ** (dim - 1) * V)
        s.spaceTimePredictor(qb, fb, [lQi], [lFi], lQhi, lFhi, None, np.asarray(luh, dtype=np.float64),
                             dx, dt)
        return dict(lQi=lQi, lFi=lFi, lQhi=lQhi, lFhi=lFhi, lQhbnd=qb, lFhbnd=fb,
                    iters=s.picard_iterations)

    def vi(self, dim, order, lFhi, dx):
        s = self._solver(dim, order)
        out = np.zeros((order + 1) ** dim * V)
        s.volumeIntegral(out, np.asarray(lFhi, dtype=np.float64), dx)
        return out

    def si(self, dim, order, lduh, lF, dx):
        s = self._solver(dim, order)
        lduh = np.array(lduh, dtype=np.float64)
        s.surfaceIntegral(lduh, np.asarray(lF, dtype=np.float64), dx)
        return lduh

    def riemann(self, dim, order, npar, planar, FL, FR, QL, QR, d):
        s = self._solver(dim, order, npar, planar)
        FL, FR = np.array(FL, dtype=np.float64), np.array(FR, dtype=np.float64)
        s.riemannSolver(FL, FR, np.asarray(QL, dtype=np.float64), np.asarray(QR, dtype=np.float64),
                        None, None, None, 0.0, d)
        return FL, FR

    def update(self, dim, order, npar, luh, lduh, dt):
        s = self._solver(dim, order, npar)
        luh = np.array(luh, dtype=np.float64)
        s.solutionUpdate(luh, np.asarray(lduh, dtype=np.float64), dt)
        return luh
