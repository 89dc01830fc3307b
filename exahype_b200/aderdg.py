"""Host-side mirror of the reference's ADER-DG solver interface.

``ADERDGSolver`` carries the methods of the toolkit-generated
``Abstract<Solver>`` (Toolkit/src/eu/exahype/solvers/templates/
AbstractGenericADERDGSolverHeader.template:166-177) with the same names,
argument order and in-place semantics, operating on numpy arrays of one
cell; each call runs the CUDA kernels through the C ABI.

``BatchedADERDG`` exposes the batched device entry points over many cells,
and ``ADERDGGrid`` the uniform periodic grid that replaces the Peano
spacetree on one GPU.
"""
import ctypes as C

import numpy as np

from . import _lib
from ._lib import AderdgDesc, GridConfig, call, lib

_dptr = C.POINTER(C.c_double)


def _p(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags['C_CONTIGUOUS']
    return a.ctypes.data_as(_dptr)


def make_desc(dim, order, dx, npar=0, pde=_lib.PDE_EULER, precision=_lib.PREC_FP64, nvar=5):
    d = AderdgDesc()
    d.dim, d.order, d.nvar, d.npar, d.pde, d.precision = dim, order, nvar, npar, pde, precision
    dx = list(dx) + [1.0] * (3 - len(dx))
    for i in range(3):
        d.dx[i] = float(dx[i])
    return d


class ADERDGSolver:
    """Per-cell drop-ins with the generated solver's signatures."""

    NumberOfVariables = 5

    def __init__(self, dim, order, npar=0, pde=_lib.PDE_EULER, dx=None, precision=_lib.PREC_FP64):
        self.dim, self.order, self.npar, self.pde = dim, order, npar, pde
        self.NumberOfParameters = npar
        self.Order = order
        self.CFL = 0.9
        self.desc = make_desc(dim, order, dx if dx is not None else [1.0] * dim, npar, pde, precision)
        self.picard_iterations = 0

    def _dx(self, dx):
        return np.ascontiguousarray(np.broadcast_to(np.asarray(dx, dtype=np.float64), (self.dim,)))

    def spaceTimePredictor(self, lQhbnd, lFhbnd, tempSpaceTimeUnknowns, tempSpaceTimeFluxUnknowns,
                           tempUnknowns, tempFluxUnknowns, tempStateSizedVectors, luh, dx, dt,
                           pointForceSources=None):
        stu = (_dptr * 1)(_p(tempSpaceTimeUnknowns[0]) if tempSpaceTimeUnknowns else None)
        stf = (_dptr * 1)(_p(tempSpaceTimeFluxUnknowns[0]) if tempSpaceTimeFluxUnknowns else None)
        it = C.c_int()
        call('exa_aderdg_spaceTimePredictor', C.byref(self.desc), _p(lQhbnd), _p(lFhbnd), stu, stf,
             _p(tempUnknowns), _p(tempFluxUnknowns), None, _p(np.ascontiguousarray(luh)),
             _p(self._dx(dx)), float(dt), None, C.byref(it))
        self.picard_iterations = it.value

    def volumeIntegral(self, lduh, lFhi, dx):
        call('exa_aderdg_volumeIntegral', C.byref(self.desc), _p(lduh), _p(np.ascontiguousarray(lFhi)),
             _p(self._dx(dx)))

    def surfaceIntegral(self, lduh, lFhbnd, dx):
        call('exa_aderdg_surfaceIntegral', C.byref(self.desc), _p(lduh), _p(np.ascontiguousarray(lFhbnd)),
             _p(self._dx(dx)))

    def riemannSolver(self, FL, FR, QL, QR, tempFaceUnknownsArray, tempStateSizedVectors,
                      tempStateSizedSquareMatrices, dt, normalNonZeroIndex, isBoundaryFace=False):
        call('exa_aderdg_riemannSolver', C.byref(self.desc), _p(FL), _p(FR), _p(np.ascontiguousarray(QL)),
             _p(np.ascontiguousarray(QR)), None, None, None, float(dt), int(normalNonZeroIndex),
             int(bool(isBoundaryFace)))

    def solutionUpdate(self, luh, lduh, dt):
        call('exa_aderdg_solutionUpdate', C.byref(self.desc), _p(luh), _p(np.ascontiguousarray(lduh)),
             float(dt))

    def stableTimeStepSize(self, luh, tempEigenvalues, dx):
        out = C.c_double()
        call('exa_aderdg_stableTimeStepSize', C.byref(self.desc), _p(np.ascontiguousarray(luh)), None,
             _p(self._dx(dx)), C.byref(out))
        return out.value


class BatchedADERDG:
    """Batched device entry points over `ncells` cells (DeviceBuffer args)."""

    def __init__(self, dim, order, dx, pde=_lib.PDE_EULER, precision=_lib.PREC_FP64, npar=0):
        self.desc = make_desc(dim, order, dx, npar, pde, precision)
        self.dim, self.order = dim, order

    def predictor_vi(self, ncells, luh, dt, lduh, qb, fb, iters=None, stats=None, dt_dev=None,
                     stream=None):
        call('exa_aderdg_predictor_vi', C.byref(self.desc), ncells, luh.ptr, float(dt),
             dt_dev.ptr if dt_dev else None, lduh.ptr, qb.ptr, fb.ptr,
             iters.ptr if iters else None, stats.ptr if stats else None, stream)

    def predictor_full(self, ncells, luh, dt, lqi, lfi, lqhi, lfhi, lduh, qb, fb, iters=None,
                       stream=None):
        call('exa_aderdg_predictor_full', C.byref(self.desc), ncells, luh.ptr, float(dt), lqi.ptr,
             lfi.ptr, lqhi.ptr, lfhi.ptr, lduh.ptr, qb.ptr, fb.ptr, iters.ptr if iters else None,
             stream)

    def volume_integral(self, ncells, lduh, lfhi, stream=None):
        call('exa_aderdg_volume_integral', C.byref(self.desc), ncells, lduh.ptr, lfhi.ptr, stream)

    def surface_integral(self, ncells, lduh, fb, stream=None):
        call('exa_aderdg_surface_integral', C.byref(self.desc), ncells, lduh.ptr, fb.ptr, stream)

    def solution_update(self, ncells, luh, lduh, dt, stream=None):
        call('exa_aderdg_solution_update', C.byref(self.desc), ncells, luh.ptr, lduh.ptr, float(dt),
             stream)

    def riemann_faces(self, nfaces, left, right, direction, qb, fb, stream=None):
        call('exa_aderdg_riemann_faces', C.byref(self.desc), nfaces, left.ptr, right.ptr,
             direction.ptr, qb.ptr, fb.ptr, stream)

    def solution_adjustment(self, ncells, luh, centers, t, dt, hook, stream=None):
        """solutionAdjustment on ncells cells: centers = DeviceBuffer
        [ncells][dim], hook = adjust_hook(...)"""
        call('exa_aderdg_solution_adjustment', C.byref(self.desc), ncells, luh.ptr, centers.ptr, float(t),
             float(dt), C.byref(hook), stream)

    def stable_dt(self, ncells, luh, dt_cell=None, dt_min=None, stream=None):
        call('exa_aderdg_stable_dt', C.byref(self.desc), ncells, luh.ptr,
             dt_cell.ptr if dt_cell else None, dt_min.ptr if dt_min else None, stream)


def adjust_hook(kind, param=(), when=_lib.ADJUST_ALWAYS):
    """exa_adjust_t: kind _lib.ADJUST_SINE_WAVE (param a), ADJUST_ISENTROPIC_VORTEX
    (param eps) or ADJUST_HEAT_SOURCE (param A, width, frequency, centre x, y, z);
    when ADJUST_AT_START (only at t == 0) or ADJUST_ALWAYS."""
    h = _lib.AdjustHook()
    h.kind, h.when = int(kind), int(when)
    for i, v in enumerate(list(param)[:6]):
        h.param[i] = float(v)
    return h


def solutionAdjustment(dim, order, luh, center, dx, t, dt, hook):
    """kernels::aderdg::generic::c::solutionAdjustment for one cell (host
    arrays; luh adjusted in place)."""
    arr = np.ascontiguousarray(luh, dtype=np.float64)
    c = np.ascontiguousarray(center, dtype=np.float64)
    d = np.ascontiguousarray(dx, dtype=np.float64)
    call('exa_aderdg_solutionAdjustment', int(dim), int(order), _p(arr), _p(c), _p(d), float(t), float(dt),
         C.byref(hook))
    if arr is not luh:
        luh[...] = arr.reshape(np.shape(luh))
    return luh


def grid_config(dim, order, n, length=None, pde=_lib.PDE_EULER, precision=_lib.PREC_FP64,
                dt_policy=0, cfl=0.9, dt_fixed=0.0):
    c = GridConfig()
    c.dim, c.order = dim, order
    n = list(n) + [1] * (3 - len(n))
    length = list(length) if length is not None else [1.0] * dim
    length = length + [1.0] * (3 - len(length))
    for i in range(3):
        c.n[i] = int(n[i])
        c.length[i] = float(length[i])
    c.pde, c.precision, c.dt_policy, c.cfl, c.dt_fixed = pde, precision, dt_policy, cfl, dt_fixed
    return c


class ADERDGGrid:
    """Uniform periodic ADER-DG grid resident on the current GPU."""

    def __init__(self, dim, order, n, length=None, pde=_lib.PDE_EULER, precision=_lib.PREC_FP64,
                 dt_policy=0, cfl=0.9, dt_fixed=0.0):
        self.cfg = grid_config(dim, order, n, length, pde, precision, dt_policy, cfl, dt_fixed)
        h = C.c_void_p()
        call('exa_aderdg_grid_create', C.byref(self.cfg), C.byref(h))
        self.h = h
        self.dim, self.order = dim, order
        self.ncells = int(lib().exa_aderdg_grid_ncells(h))
        self.nodes_per_cell = (order + 1) ** dim
        self.state_size = self.ncells * self.nodes_per_cell * 5

    @staticmethod
    def footprint(dim, order, n, **kw):
        c = grid_config(dim, order, n, **kw)
        return int(lib().exa_aderdg_grid_footprint(C.byref(c)))

    def init(self, kind=0, param=5.0, seed=1234, noise=0.0):
        call('exa_aderdg_grid_init', self.h, int(kind), float(param), int(seed), float(noise))

    def set_state(self, luh):
        luh = np.ascontiguousarray(luh, dtype=np.float64)
        assert luh.size == self.state_size
        call('exa_aderdg_grid_set_state', self.h, luh.ctypes.data)

    def get_state(self, out=None):
        if out is None:
            out = np.empty(self.state_size)
        call('exa_aderdg_grid_get_state', self.h, out.ctypes.data)
        return out

    def step(self, nsteps=1, want_dt=False):
        if want_dt:
            dts = np.empty(nsteps)
            call('exa_aderdg_grid_step', self.h, int(nsteps), dts.ctypes.data)
            return dts
        call('exa_aderdg_grid_step', self.h, int(nsteps), None)
        return None

    def use_graph(self, enable=True):
        call('exa_aderdg_grid_use_graph', self.h, int(enable))

    def set_debug(self, enable=True):
        """Scan each phase's outputs for non-finite values every step."""
        call('exa_aderdg_grid_set_debug', self.h, int(enable))

    def debug_status(self):
        """(where, step, index) of the first non-finite value seen by the
        debug scan: where 0 none, 1 lduh, 2 lQhbnd, 3 lFhbnd, 4 luh."""
        w, st, ix = C.c_int(), C.c_uint64(), C.c_uint64()
        call('exa_aderdg_grid_debug_status', self.h, C.byref(w), C.byref(st), C.byref(ix))
        return w.value, st.value, ix.value

    def profile(self, enable=True):
        call('exa_aderdg_grid_profile', self.h, int(enable))

    def phase_times(self):
        a, b, n = C.c_double(), C.c_double(), C.c_uint64()
        call('exa_aderdg_grid_phase_times', self.h, C.byref(a), C.byref(b), C.byref(n))
        return dict(predictor_ms=a.value, corrector_ms=b.value, steps=int(n.value))

    def stream(self):
        s = C.c_void_p()
        call('exa_aderdg_grid_stream', self.h, C.byref(s))
        return s

    def device_state_ptr(self):
        p = C.c_void_p()
        call('exa_aderdg_grid_device_state', self.h, C.byref(p))
        return p

    def set_boundary(self, bc):
        """Boundary rule per dimension: _lib.BC_PERIODIC / BC_OUTFLOW /
        BC_REFLECT (see exa_aderdg_grid_set_boundary)."""
        arr = (C.c_int * 3)(*(list(bc) + [0] * (3 - len(bc))))
        call('exa_aderdg_grid_set_boundary', self.h, arr)

    def set_adjustment(self, hook=None):
        """Solution adjustment after every step's update (hook = adjust_hook(...),
        None to turn it off; see exa_aderdg_grid_set_adjustment)."""
        call('exa_aderdg_grid_set_adjustment', self.h, C.byref(hook) if hook is not None else None)

    # -- a-posteriori subcell limiter (exa_aderdg_grid_set_limiter) --
    def set_limiter(self, scheme=0, nobs=5, relaxation=1e-4, difference_scaling=1e-3, steps_till_cured=0,
                    check_admissibility=True, enable=True):
        """Limiting ADER-DG (2D or 3D, any boundary rules): DMP + admissibility check of every
        step's DG candidate, subcell FV recomputation (scheme 0 Godunov, 1
        MUSCL-Hancock) of troubled cells and their neighbours."""
        if not enable:
            call('exa_aderdg_grid_set_limiter', self.h, None)
            self.nobs = None
            return
        c = _lib.LimiterConfig(int(scheme), int(nobs), float(relaxation), float(difference_scaling),
                               int(steps_till_cured), int(bool(check_admissibility)))
        call('exa_aderdg_grid_set_limiter', self.h, C.addressof(c))
        self.nobs = int(nobs)

    def limiter_status(self):
        """(status per cell: Ok 0 .. Troubled 5, counts [patches, FV cells,
        Troubled cells]) of the last step"""
        st = np.zeros(self.ncells, dtype=np.int32)
        counts = np.zeros(3, dtype=np.int32)
        call('exa_aderdg_grid_limiter_status', self.h, st.ctypes.data, counts.ctypes.data)
        return st, counts

    def limiter_bounds(self):
        """DMP bounds for the next step: (min, max), [cell][2 dim][nobs] each"""
        mn = np.zeros(self.ncells * 2 * self.dim * self.nobs)
        mx = np.zeros_like(mn)
        call('exa_aderdg_grid_limiter_bounds', self.h, mn.ctypes.data, mx.ctypes.data)
        return mn, mx

    # -- slab decomposition (see exahype_b200.slab) --
    def set_halo(self, enable=True):
        call('exa_aderdg_grid_set_halo', self.h, int(enable))

    def halo_buffers(self):
        """(send_lo, send_hi, recv_lo, recv_hi) device pointers and the
        number of doubles in each."""
        p = [C.c_void_p() for _ in range(4)]
        n = C.c_size_t()
        call('exa_aderdg_grid_halo_buffers', self.h, *[C.byref(x) for x in p], C.byref(n))
        return [x.value for x in p], int(n.value)

    def dt_slot_ptr(self):
        p = C.c_void_p()
        call('exa_aderdg_grid_dt_slot', self.h, C.byref(p))
        return p.value

    def phase(self, phase):
        call('exa_aderdg_grid_phase', self.h, int(phase))

    def init_slab(self, rank, nranks, kind=0, param=5.0, seed=1234, noise=0.0):
        call('exa_aderdg_grid_init_slab', self.h, int(kind), float(param), int(seed), float(noise),
             int(rank), int(nranks))

    def status(self):
        t, it, nc, nan = C.c_double(), C.c_uint64(), C.c_uint64(), C.c_int()
        st = lib().exa_aderdg_grid_status(self.h, C.byref(t), C.byref(it), C.byref(nc), C.byref(nan))
        if st not in (_lib.EXA_OK, _lib.EXA_ENAN, _lib.EXA_ENONCONV):
            _lib.check(st, 'exa_aderdg_grid_status')
        return dict(time=t.value, picard_iters=int(it.value), nonconverged=int(nc.value),
                    nan=bool(nan.value), code=int(st))

    def destroy(self):
        if self.h:
            call('exa_aderdg_grid_destroy', self.h)
            self.h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


def amr_prolongation(k, order, count, fine, coarse, level_delta, index, coarse_item=None, nvar=5,
                     stream=None):
    """volume/faceUnknownsProlongation for `count` items (DeviceBuffer
    arguments; index: int32 [count][3]; see exa_aderdg_amr_prolongation)."""
    call('exa_aderdg_amr_prolongation', int(k), int(order), int(nvar), int(count), fine.ptr, coarse.ptr,
         coarse_item.ptr if coarse_item is not None else None, int(level_delta), index.ptr, stream)


def amr_restriction(k, order, count, coarse, fine, level_delta, index, nvar=5, stream=None):
    """volume/faceUnknownsRestriction: coarse[i] += R(fine[i])."""
    call('exa_aderdg_amr_restriction', int(k), int(order), int(nvar), int(count), coarse.ptr, fine.ptr,
         int(level_delta), index.ptr, stream)
