"""ctypes binding of the CPU oracle (oracle/liboracle.so) and, when it was
built, of the reference's own generic kernels (oracle/_ref/libexa_ref*.so).

Test infrastructure only: the product library never loads these.
"""
import ctypes as C
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, 'oracle')

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags='C_CONTIGUOUS')
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags='C_CONTIGUOUS')


def _ensure_built():
    so = os.path.join(ORACLE_DIR, 'liboracle.so')
    srcs = [os.path.join(ORACLE_DIR, f) for f in ('exa_oracle.c', 'exa_oracle.h')]
    if not os.path.exists(so) or any(os.path.getmtime(s) > os.path.getmtime(so) for s in srcs):
        subprocess.check_call(['make', '-s', '-C', ORACLE_DIR, 'liboracle.so'])
    return so


_lib = None


def lib():
    global _lib
    if _lib is not None:
        return _lib
    L = C.CDLL(_ensure_built())
    d, i = C.c_double, C.c_int
    L.orc_euler_flux.argtypes = [i, i, _dp, _dp]
    L.orc_euler_eigenvalues.argtypes = [i, _dp, i, _dp]
    L.orc_stp_nonlinear.restype = i
    L.orc_stp_nonlinear.argtypes = [i, i, i, i, i, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, d]
    L.orc_volume_integral.argtypes = [i, i, i, i, _dp, _dp, _dp]
    L.orc_surface_integral.argtypes = [i, i, i, _dp, _dp, _dp]
    L.orc_riemann.argtypes = [i, i, i, i, i, _dp, _dp, _dp, _dp, i]
    L.orc_solution_update.argtypes = [i, i, i, i, _dp, _dp, d]
    L.orc_stable_dt.restype = d
    L.orc_stable_dt.argtypes = [i, i, i, i, i, _dp, _dp, d]
    L.orc_aderdg_grid_dt.restype = d
    L.orc_aderdg_grid_dt.argtypes = [i, i, i, _ip, _dp, _dp, i, d]
    L.orc_aderdg_grid_step.restype = d
    L.orc_aderdg_grid_step.argtypes = [i, i, i, _ip, _dp, _dp, i, d, d, C.c_void_p, i]
    L.orc_aderdg_grid_step_bc.restype = d
    L.orc_aderdg_grid_step_bc.argtypes = [i, i, i, _ip, _dp, _dp, i, d, d, C.c_void_p, i, C.c_void_p]
    L.orc_aderdg_grid_ic.argtypes = [i, i, _ip, _dp, _dp, i, d, C.c_ulonglong, d]
    L.orc_rusanov_pde.restype = d
    L.orc_rusanov_pde.argtypes = [i, i, C.c_void_p, C.c_void_p, C.c_void_p, _dp, _dp, _dp, _dp, i]
    L.orc_rusanov.restype = d
    L.orc_rusanov.argtypes = [i, i, i, i, _dp, _dp, _dp, _dp, i]
    L.orc_fv_godunov_2d.restype = d
    L.orc_fv_godunov_2d.argtypes = [i, i, i, i, i, _dp, _dp, _dp, d]
    L.orc_fv_musclhancock_2d.restype = d
    L.orc_fv_musclhancock_2d.argtypes = [i, i, i, i, i, _dp, _dp, _dp, d]
    L.orc_fv_stable_dt_2d.restype = d
    L.orc_fv_stable_dt_2d.argtypes = [i, i, i, i, i, _dp, _dp, d]
    L.orc_fv_periodic_ghosts_2d.argtypes = [i, i, i, _dp]
    L.orc_fv_patch_step_2d.restype = d
    L.orc_fv_patch_step_2d.argtypes = [i, i, i, _dp, _dp, d, C.c_void_p]
    L.orc_aderdg_sample_step.argtypes = [i, i, i, C.c_long, _dp, _dp, d, i]
    L.orc_aderdg_slab_predict.argtypes = [i, i, i, _ip, _dp, _dp, d, _dp, _dp, _dp, _dp, _dp]
    L.orc_aderdg_slab_correct.argtypes = [i, i, i, _ip, _dp, _dp, _dp, _dp, _dp, _dp, _dp, d]
    L.orc_amr_prolongation.argtypes = [i, i, i, _dp, _dp, i, _ip]
    L.orc_amr_restriction.argtypes = [i, i, i, _dp, _dp, i, _ip]
    L.orc_fv_patchgrid_step_2d.restype = d
    L.orc_fv_patchgrid_step_2d.argtypes = [i, i, i, i, i, _dp, _dp]
    L.orc_fv_patchgrid_step_2d_bc.restype = d
    L.orc_fv_patchgrid_step_2d_bc.argtypes = [i, i, i, i, i, _dp, _dp, C.c_void_p]
    L.orc_noise_u01.restype = d
    L.orc_noise_u01.argtypes = [C.c_ulonglong, C.c_ulonglong]
    L.orc_limiter_project_on_fv.argtypes = [i, i, i, i, _dp, _dp]
    L.orc_limiter_project_on_dg.argtypes = [i, i, i, i, _dp, _dp]
    L.orc_limiter_local_min_max.argtypes = [i, i, i, i, _dp, _dp, _dp]
    L.orc_limiter_fv_min_max.argtypes = [i, i, i, i, i, _dp, _dp, _dp]
    L.orc_limiter_dmp.restype = i
    L.orc_limiter_dmp.argtypes = [i, i, i, i, _dp, d, d, _dp, _dp]
    L.orc_fv_godunov_3d.restype = d
    L.orc_fv_godunov_3d.argtypes = [i, i, i, i, _dp, _dp, _dp, d]
    L.orc_fv_musclhancock_3d.restype = d
    L.orc_fv_musclhancock_3d.argtypes = [i, i, i, i, _dp, _dp, _dp, d]
    L.orc_fv_stable_dt_3d.restype = d
    L.orc_fv_stable_dt_3d.argtypes = [i, i, i, i, _dp, _dp, d]
    L.orc_fv_periodic_ghosts_3d.argtypes = [i, i, i, _dp]
    L.orc_limiting_grid_step.restype = d
    L.orc_limiting_grid_step.argtypes = [i, i, _ip, _dp, i, _dp, _ip, _ip, _dp, _dp, i, i, d, d, i, i, d, i, d,
                                         C.c_void_p, C.c_void_p]
    L.orc_limiting_initial_bounds.argtypes = [i, i, _ip, _dp, i, _dp, _dp, C.c_void_p]
    L.orc_fv_boundary_ghosts.argtypes = [i, i, i, _dp, i, i]
    L.orc_solution_adjustment.argtypes = [i, i, _dp, _dp, _dp, d, d, i, i, _dp]
    _lib = L
    return L


# ---------------------------------------------------------------- helpers
def sizes(dim, order, nvar=5, npar=0):
    B = order + 1
    nd = nvar + npar
    n_node = B ** dim
    return dict(B=B, nData=nd, luh=n_node * nd, lduh=n_node * nvar,
                lQi=n_node * B * nd, lFi=n_node * B * (dim + 1) * nvar,
                rhs=n_node * B * nvar, lQhi=n_node * nd,
                lFhi=n_node * (dim + 1) * nvar,
                qbnd=2 * dim * B ** (dim - 1) * nd, fbnd=2 * dim * B ** (dim - 1) * nvar)


def stp(dim, order, luh, dx, dt, nvar=5, npar=0, planar=0):
    s = sizes(dim, order, nvar, npar)
    out = {k: np.zeros(s[k]) for k in ('lQi', 'lFi', 'lQhi', 'lFhi')}
    qb, fb = np.zeros(s['qbnd']), np.zeros(s['fbnd'])
    old, rhs = np.zeros(s['lQi']), np.zeros(s['rhs'])
    it = lib().orc_stp_nonlinear(dim, order, nvar, npar, planar, qb, fb, out['lQi'], old, rhs,
                                 out['lFi'], out['lQhi'], out['lFhi'],
                                 np.ascontiguousarray(luh, dtype=np.float64),
                                 np.asarray(dx, dtype=np.float64), dt)
    out.update(lQhbnd=qb, lFhbnd=fb, iters=it)
    return out


def grid_ic(dim, order, n, kind=0, param=5.0, seed=1234, noise=0.0, dx=None):
    n = np.asarray(n, dtype=np.int32)
    if dx is None:
        dx = 1.0 / n.astype(np.float64)
    B = order + 1
    luh = np.zeros(int(np.prod(n)) * B ** dim * 5)
    lib().orc_aderdg_grid_ic(dim, order, n, np.asarray(dx, dtype=np.float64), luh, kind, param,
                             seed, noise)
    return luh


def grid_step(dim, order, n, luh, dt_policy=0, cfl=0.9, dt_fixed=0.0, planar=0,
              nthreads=0, dx=None, bc=None):
    n = np.asarray(n, dtype=np.int32)
    if dx is None:
        dx = 1.0 / n.astype(np.float64)
    iters = np.zeros(int(np.prod(n)), dtype=np.int32)
    bcs = np.asarray(list(bc) + [0] * (3 - len(bc)), dtype=np.int32) if bc is not None else None
    dt = lib().orc_aderdg_grid_step_bc(dim, order, planar, n, np.asarray(dx, dtype=np.float64), luh,
                                       dt_policy, cfl, dt_fixed, iters.ctypes.data, nthreads,
                                       bcs.ctypes.data if bcs is not None else None)
    return dt, iters


def ref_grid_step(dim, order, n, luh, dt_policy=0, dt_fixed=0.0, nthreads=0, dx=None, bc=None):
    """One step of the reference's own kernels on the uniform grid (periodic,
    or boundary rules per dimension through its boundaryConditions kernel)."""
    R = ref_lib(dim)
    n = np.asarray(n, dtype=np.int32)
    if dx is None:
        dx = 1.0 / n.astype(np.float64)
    bcs = np.asarray(list(bc or []) + [0] * (3 - len(bc or [])), dtype=np.int32)
    return R.ref_grid_step_bc(order, n, np.asarray(dx, dtype=np.float64), luh, dt_policy, dt_fixed,
                              nthreads, bcs)


def lim_sizes(dim, order, nvar=5, ghost=0):
    B, S = order + 1, 2 * order + 1
    return dict(B=B, S=S, luh=B ** dim * nvar, lim=(S + 2 * ghost) ** dim * nvar)


def limiter_project_on_fv(dim, order, luh, nvar=5, ghost=0, lim=None):
    """projectOnFVLimiterSpace of every cell of luh ([cell][B^dim][nvar])."""
    s = lim_sizes(dim, order, nvar, ghost)
    luh = np.ascontiguousarray(luh, dtype=np.float64).reshape(-1, s['luh'])
    out = np.zeros((luh.shape[0], s['lim'])) if lim is None else lim.reshape(-1, s['lim'])
    for c in range(luh.shape[0]):
        row = np.ascontiguousarray(out[c])
        lib().orc_limiter_project_on_fv(dim, order, nvar, ghost, np.ascontiguousarray(luh[c]), row)
        out[c] = row
    return out.ravel()


def limiter_project_on_dg(dim, order, lim, nvar=5, ghost=0):
    s = lim_sizes(dim, order, nvar, ghost)
    lim = np.ascontiguousarray(lim, dtype=np.float64).reshape(-1, s['lim'])
    out = np.zeros((lim.shape[0], s['luh']))
    for c in range(lim.shape[0]):
        row = np.zeros(s['luh'])
        lib().orc_limiter_project_on_dg(dim, order, nvar, ghost, np.ascontiguousarray(lim[c]), row)
        out[c] = row
    return out.ravel()


def limiter_local_min_max(dim, order, luh, nvar=5, nobs=5):
    s = lim_sizes(dim, order, nvar)
    luh = np.ascontiguousarray(luh, dtype=np.float64).reshape(-1, s['luh'])
    mn = np.zeros((luh.shape[0], 2 * dim * nobs))
    mx = np.zeros_like(mn)
    for c in range(luh.shape[0]):
        a, b = np.zeros(2 * dim * nobs), np.zeros(2 * dim * nobs)
        lib().orc_limiter_local_min_max(dim, order, nvar, nobs, np.ascontiguousarray(luh[c]), a, b)
        mn[c], mx[c] = a, b
    return mn.ravel(), mx.ravel()


def limiter_fv_min_max(dim, order, lim, nvar=5, nobs=5, ghost=0):
    s = lim_sizes(dim, order, nvar, ghost)
    lim = np.ascontiguousarray(lim, dtype=np.float64).reshape(-1, s['lim'])
    mn = np.zeros((lim.shape[0], 2 * dim * nobs))
    mx = np.zeros_like(mn)
    for c in range(lim.shape[0]):
        a, b = np.zeros(2 * dim * nobs), np.zeros(2 * dim * nobs)
        lib().orc_limiter_fv_min_max(dim, order, nvar, nobs, ghost, np.ascontiguousarray(lim[c]), a, b)
        mn[c], mx[c] = a, b
    return mn.ravel(), mx.ravel()


def limiter_dmp(dim, order, luh, bmin, bmax, relax, scaling, nvar=5, nobs=5):
    """discreteMaximumPrincipleAndMinAndMaxSearch per cell; returns
    (ok[cell], new bmin, new bmax)."""
    s = lim_sizes(dim, order, nvar)
    luh = np.ascontiguousarray(luh, dtype=np.float64).reshape(-1, s['luh'])
    bmin = np.array(bmin, dtype=np.float64).reshape(luh.shape[0], -1)
    bmax = np.array(bmax, dtype=np.float64).reshape(luh.shape[0], -1)
    ok = np.zeros(luh.shape[0], dtype=np.int32)
    for c in range(luh.shape[0]):
        a, b = np.ascontiguousarray(bmin[c]), np.ascontiguousarray(bmax[c])
        ok[c] = lib().orc_limiter_dmp(dim, order, nvar, nobs, np.ascontiguousarray(luh[c]), relax,
                                      scaling, a, b)
        bmin[c], bmax[c] = a, b
    return ok, bmin.ravel(), bmax.ravel()


class LimitingGrid:
    """Oracle state of the limiting ADER-DG grid (2D or 3D): the restated
    step of orc_limiting_grid_step with the same parameters as
    ADERDGGrid.set_limiter; bc = boundary rule per dimension (0 periodic,
    1 outflow, 2 reflecting wall) as in ADERDGGrid.set_boundary."""

    def __init__(self, order, n, luh, length=None, scheme=0, nobs=5, relaxation=1e-4,
                 difference_scaling=1e-3, steps_till_cured=0, check_admissibility=True, dt_policy=0, cfl=0.9,
                 planar=0, bc=None):
        self.dim = len(n)
        self.bc = np.asarray(list(bc or [0] * self.dim) + [0] * (3 - self.dim), dtype=np.int32)
        length = length or (1.0,) * self.dim
        self.order = order
        self.n = np.asarray(list(n) + [1] * (3 - self.dim), dtype=np.int32)
        self.dx = np.array([length[i] / n[i] for i in range(self.dim)] + [1.0] * (3 - self.dim))
        self.luh = np.array(luh, dtype=np.float64)
        nc = int(np.prod(n))
        nf = 2 * self.dim
        self.status = np.zeros(nc, dtype=np.int32)
        self.cure = np.zeros(nc, dtype=np.int32)
        self.bmin = np.zeros(nc * nf * nobs)
        self.bmax = np.zeros(nc * nf * nobs)
        self.p = (scheme, nobs, relaxation, difference_scaling, steps_till_cured, int(check_admissibility))
        self.dt_policy, self.cfl, self.planar = dt_policy, cfl, planar
        lib().orc_limiting_initial_bounds(self.dim, order, self.n, self.luh, nobs, self.bmin, self.bmax,
                                          self.bc.ctypes.data)
        self.dt = lib().orc_aderdg_grid_dt(self.dim, order, planar, self.n, self.dx, self.luh, dt_policy, cfl)
        self.counts = np.zeros(3, dtype=np.int32)

    def step(self):
        """one step with the current dt; returns the dt taken"""
        dt = self.dt
        s, nobs, rel, sc, cured, adm = self.p
        self.dt = lib().orc_limiting_grid_step(self.dim, self.order, self.n, self.dx, self.planar, self.luh,
                                               self.status, self.cure, self.bmin, self.bmax, s, nobs, rel, sc,
                                               cured, adm, dt, self.dt_policy, self.cfl, self.counts.ctypes.data,
                                               self.bc.ctypes.data)
        return dt


# ---------------------------------------------------------------- reference
_ref = {}


def ref_lib(dim):
    """The reference's own kernels (oracle/_ref), or None if not built."""
    if dim in _ref:
        return _ref[dim]
    so = os.path.join(ORACLE_DIR, '_ref', 'libexa_ref%dd.so' % dim)
    L = None
    if os.path.exists(so):
        L = C.CDLL(so)
        d, i = C.c_double, C.c_int
        if hasattr(L, 'ref_limiter'):
            L.ref_limiter.restype = i
            L.ref_limiter.argtypes = [i, i, i, i, i, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                      d, d]
            L.ref_limiter_tables.restype = i
            L.ref_limiter_tables.argtypes = [i, _dp, _dp, _dp, _dp]
        if hasattr(L, 'ref_amr'):
            L.ref_amr.restype = i
            L.ref_amr.argtypes = [i, i, _dp, _dp, _dp, _dp, i, _ip]
        L.ref_stp.restype = i
        L.ref_stp.argtypes = [i, i, _dp, _dp, _dp, _dp, _dp, _dp, _dp, d]
        L.ref_volume_integral.restype = i
        L.ref_volume_integral.argtypes = [i, _dp, _dp, _dp]
        L.ref_surface_integral.restype = i
        L.ref_surface_integral.argtypes = [i, _dp, _dp, _dp]
        L.ref_riemann.restype = i
        L.ref_riemann.argtypes = [i, i, _dp, _dp, _dp, _dp, i]
        L.ref_solution_update.restype = i
        L.ref_solution_update.argtypes = [i, i, _dp, _dp, d]
        L.ref_stable_dt.restype = d
        L.ref_stable_dt.argtypes = [i, i, _dp, _dp]
        L.ref_grid_step.restype = d
        L.ref_grid_step.argtypes = [i, _ip, _dp, _dp, i, d, i]
        L.ref_sample_step.restype = i
        L.ref_sample_step.argtypes = [i, C.c_long, _dp, _dp, d, i]
        if hasattr(L, 'ref_fv_step'):
            L.ref_fv_step.restype = d
            L.ref_fv_step.argtypes = [i, i, _dp, _dp, d, C.c_void_p]
        if hasattr(L, 'ref_solution_adjustment'):
            L.ref_solution_adjustment.restype = i
            L.ref_solution_adjustment.argtypes = [i, _dp, _dp, _dp, d, d, i, _dp]
        if hasattr(L, 'ref_grid_step_bc'):
            L.ref_grid_step_bc.restype = d
            L.ref_grid_step_bc.argtypes = [i, _ip, _dp, _dp, i, d, i, _ip]
        if hasattr(L, 'ref_rusanov_mock'):
            L.ref_rusanov_mock.restype = d
            L.ref_rusanov_mock.argtypes = [_dp, _dp, _dp, _dp, i]
        if hasattr(L, 'ref_fv_boundary'):
            L.ref_fv_boundary.restype = i
            L.ref_fv_boundary.argtypes = [i, i, _dp, i, i]
    _ref[dim] = L
    return L
