"""ctypes binding of libexahype_b200.so (the C ABI in include/exa_kernels.h).

The shared library is built in-tree (``make -C exahype_b200/csrc``) and
loaded from this package directory.  There is no fallback: if the library
is missing every entry point raises.
"""
import ctypes as C
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, 'libexahype_b200.so')

EXA_OK = 0
EXA_EINVAL = 1
EXA_ENONCONV = 2
EXA_ENAN = 3
EXA_ETIMEDOUT = 4
EXA_ECUDA = 5
EXA_ENOMEM = 6
EXA_EBUSY = 7
EXA_ENOTFOUND = 8

PDE_EULER = 0
PDE_EULER_PLANAR = 1
PREC_FP64 = 0
PREC_MIXED = 1
BC_PERIODIC = 0
BC_OUTFLOW = 1
BC_REFLECT = 2
ADJUST_NONE = 0
ADJUST_SINE_WAVE = 1
ADJUST_ISENTROPIC_VORTEX = 2
ADJUST_HEAT_SOURCE = 3
ADJUST_AT_START = 0
ADJUST_ALWAYS = 1


class ExaError(RuntimeError):
    def __init__(self, status, where, detail=''):
        self.status = status
        super().__init__('%s failed: status %d (%s)%s' % (
            where, status, _status_string(status), (': ' + detail) if detail else ''))


class AderdgDesc(C.Structure):
    _fields_ = [('dim', C.c_int), ('order', C.c_int), ('nvar', C.c_int), ('npar', C.c_int),
                ('pde', C.c_int), ('precision', C.c_int), ('dx', C.c_double * 3)]


class GridConfig(C.Structure):
    _fields_ = [('dim', C.c_int), ('order', C.c_int), ('n', C.c_int * 3),
                ('length', C.c_double * 3), ('pde', C.c_int), ('precision', C.c_int),
                ('dt_policy', C.c_int), ('cfl', C.c_double), ('dt_fixed', C.c_double)]


class LimiterConfig(C.Structure):
    _fields_ = [('scheme', C.c_int), ('nobs', C.c_int), ('relaxation', C.c_double),
                ('difference_scaling', C.c_double), ('steps_till_cured', C.c_int),
                ('check_admissibility', C.c_int)]


class AdjustHook(C.Structure):
    """exa_adjust_t: a built-in adjustPointSolution form"""
    _fields_ = [('kind', C.c_int), ('when', C.c_int), ('param', C.c_double * 6)]


class FVDesc(C.Structure):
    _fields_ = [('dim', C.c_int), ('patch', C.c_int), ('ghost', C.c_int), ('nvar', C.c_int),
                ('npar', C.c_int), ('pde', C.c_int), ('dx', C.c_double * 3)]


_lib = None
_lock = threading.Lock()

vp = C.c_void_p
i32 = C.c_int
i64 = C.c_long
f64 = C.c_double
u64 = C.c_uint64
sz = C.c_size_t
dptr = C.POINTER(C.c_double)
dpp = C.POINTER(C.POINTER(C.c_double))
ipt = C.POINTER(C.c_int)

# name -> (restype, argtypes); the list is the C ABI surface the tests check
SIGNATURES = {
    'exa_status_string': (C.c_char_p, [i32]),
    'exa_last_error_string': (C.c_char_p, []),
    'exa_device_count': (i32, []),
    'exa_set_device': (i32, [i32]),
    'exa_device_alloc': (i32, [sz, C.POINTER(vp)]),
    'exa_device_free': (i32, [vp]),
    'exa_host_alloc_pinned': (i32, [sz, C.POINTER(vp)]),
    'exa_host_free_pinned': (i32, [vp]),
    'exa_memcpy_h2d': (i32, [vp, vp, sz, vp]),
    'exa_memcpy_d2h': (i32, [vp, vp, sz, vp]),
    'exa_memset_device': (i32, [vp, i32, sz, vp]),
    'exa_stream_create': (i32, [C.POINTER(vp)]),
    'exa_stream_destroy': (i32, [vp]),
    'exa_stream_synchronize': (i32, [vp]),
    'exa_device_synchronize': (i32, []),
    'exa_timer_create': (i32, [C.POINTER(vp)]),
    'exa_timer_destroy': (i32, [vp]),
    'exa_timer_start': (i32, [vp, vp]),
    'exa_timer_stop': (i32, [vp, vp]),
    'exa_timer_elapsed_ms': (i32, [vp, C.POINTER(C.c_float)]),
    'exa_launch_count': (u64, []),
    'exa_dropin_workspace_doubles': (i32, [i32, C.POINTER(sz)]),
    'exa_nccl_unique_id': (i32, [vp]),
    'exa_slab_comm_create': (i32, [vp, i32, i32, C.POINTER(vp)]),
    'exa_slab_comm_destroy': (i32, [vp]),
    'exa_aderdg_grid_slab_prime': (i32, [vp, vp, f64]),
    'exa_aderdg_grid_slab_step': (i32, [vp, vp, i32, f64]),
    'exa_tune_set': (i32, [i32, i32]),
    'exa_tune_get': (i32, [i32]),
    'exa_diff_norms': (i32, [vp, vp, sz, C.POINTER(f64), vp]),
    'exa_aderdg_spaceTimePredictor': (i32, [C.POINTER(AderdgDesc), dptr, dptr, dpp, dpp, dptr, dptr,
                                            dptr, dptr, dptr, f64, dptr, ipt]),
    'exa_aderdg_spaceTimePredictor_noalloc': (i32, [C.POINTER(AderdgDesc), dptr, dptr, dpp, dpp, dptr,
                                                    dptr, dptr, dptr, dptr, f64, dptr, ipt]),
    'exa_aderdg_volumeIntegral': (i32, [C.POINTER(AderdgDesc), dptr, dptr, dptr]),
    'exa_aderdg_surfaceIntegral': (i32, [C.POINTER(AderdgDesc), dptr, dptr, dptr]),
    'exa_aderdg_riemannSolver': (i32, [C.POINTER(AderdgDesc), dptr, dptr, dptr, dptr, dptr, dpp, dpp,
                                       f64, i32, i32]),
    'exa_aderdg_solutionUpdate': (i32, [C.POINTER(AderdgDesc), dptr, dptr, f64]),
    'exa_aderdg_stableTimeStepSize': (i32, [C.POINTER(AderdgDesc), dptr, dptr, dptr, dptr]),
    'exa_aderdg_predictor_vi': (i32, [C.POINTER(AderdgDesc), i64, vp, f64, vp, vp, vp, vp, vp, vp, vp]),
    'exa_aderdg_predictor_full': (i32, [C.POINTER(AderdgDesc), i64, vp, f64, vp, vp, vp, vp, vp, vp, vp,
                                        vp, vp]),
    'exa_aderdg_volume_integral': (i32, [C.POINTER(AderdgDesc), i64, vp, vp, vp]),
    'exa_aderdg_surface_integral': (i32, [C.POINTER(AderdgDesc), i64, vp, vp, vp]),
    'exa_aderdg_solution_update': (i32, [C.POINTER(AderdgDesc), i64, vp, vp, f64, vp]),
    'exa_aderdg_riemann_faces': (i32, [C.POINTER(AderdgDesc), i64, vp, vp, vp, vp, vp, vp]),
    'exa_aderdg_stable_dt': (i32, [C.POINTER(AderdgDesc), i64, vp, vp, vp, vp]),
    'exa_aderdg_grid_create': (i32, [C.POINTER(GridConfig), C.POINTER(vp)]),
    'exa_aderdg_grid_destroy': (i32, [vp]),
    'exa_aderdg_grid_footprint': (sz, [C.POINTER(GridConfig)]),
    'exa_aderdg_grid_init': (i32, [vp, i32, f64, u64, f64]),
    'exa_aderdg_grid_set_state': (i32, [vp, vp]),
    'exa_aderdg_grid_get_state': (i32, [vp, vp]),
    'exa_aderdg_grid_step': (i32, [vp, i32, vp]),
    'exa_aderdg_grid_use_graph': (i32, [vp, i32]),
    'exa_aderdg_grid_stream': (i32, [vp, C.POINTER(vp)]),
    'exa_aderdg_grid_set_debug': (i32, [vp, i32]),
    'exa_aderdg_grid_debug_status': (i32, [vp, C.POINTER(i32), C.POINTER(u64), C.POINTER(u64)]),
    'exa_aderdg_grid_profile': (i32, [vp, i32]),
    'exa_aderdg_grid_phase_times': (i32, [vp, C.POINTER(f64), C.POINTER(f64), C.POINTER(u64)]),
    'exa_aderdg_grid_device_state': (i32, [vp, C.POINTER(vp)]),
    'exa_aderdg_grid_status': (i32, [vp, C.POINTER(f64), C.POINTER(u64), C.POINTER(u64), C.POINTER(i32)]),
    'exa_aderdg_grid_ncells': (i64, [vp]),
    'exa_fv_grid_create': (i32, [i32, i32, f64, i32, C.POINTER(vp)]),
    'exa_fv_grid_destroy': (i32, [vp]),
    'exa_fv_grid_state_size': (sz, [vp]),
    'exa_fv_grid_init': (i32, [vp, f64, u64, f64]),
    'exa_fv_grid_set_state': (i32, [vp, vp]),
    'exa_fv_grid_get_state': (i32, [vp, vp]),
    'exa_fv_grid_step': (i32, [vp, i32]),
    'exa_fv_grid_status': (i32, [vp, C.POINTER(f64), C.POINTER(f64)]),
    'exa_fv_grid_stream': (i32, [vp, C.POINTER(vp)]),
    'exa_fv_grid_device_state': (i32, [vp, C.POINTER(vp)]),
    'exa_fv_patchgrid_create': (i32, [i32, i32, i32, i32, f64, i32, C.POINTER(vp)]),
    'exa_fv_patchgrid_destroy': (i32, [vp]),
    'exa_fv_patchgrid_state_size': (sz, [vp]),
    'exa_fv_patchgrid_init': (i32, [vp, f64, u64, f64]),
    'exa_fv_patchgrid_set_state': (i32, [vp, vp]),
    'exa_fv_patchgrid_get_state': (i32, [vp, vp]),
    'exa_fv_patchgrid_step': (i32, [vp, i32]),
    'exa_fv_patchgrid_status': (i32, [vp, C.POINTER(f64), C.POINTER(f64)]),
    'exa_fv_patchgrid_stream': (i32, [vp, C.POINTER(vp)]),
    'exa_aderdg_amr_prolongation': (i32, [i32, i32, i32, i64, vp, vp, vp, i32, vp, vp]),
    'exa_aderdg_amr_restriction': (i32, [i32, i32, i32, i64, vp, vp, i32, vp, vp]),
    'exa_limiter_project_on_fv': (i32, [i32, i32, i32, i32, i64, vp, vp, vp]),
    'exa_limiter_project_on_dg': (i32, [i32, i32, i32, i32, i64, vp, vp, vp]),
    'exa_limiter_local_min_max': (i32, [i32, i32, i32, i32, i64, vp, vp, vp, vp]),
    'exa_limiter_fv_min_max': (i32, [i32, i32, i32, i32, i32, i64, vp, vp, vp, vp]),
    'exa_limiter_dmp': (i32, [i32, i32, i32, i32, i64, vp, f64, f64, vp, vp, vp, vp]),
    'exa_limiter_projectOnFVLimiterSpace': (i32, [i32, dptr, i32, i32, i32, dptr]),
    'exa_limiter_projectOnDGSpace': (i32, [i32, dptr, i32, i32, i32, dptr]),
    'exa_limiter_findCellLocalMinAndMax': (i32, [i32, dptr, i32, i32, i32, dptr, dptr]),
    'exa_limiter_discreteMaximumPrincipleAndMinAndMaxSearch': (i32, [i32, dptr, i32, i32, i32, f64, f64, dptr, dptr,
                                                                     C.POINTER(i32)]),
    'exa_aderdg_grid_set_limiter': (i32, [vp, vp]),
    'exa_aderdg_grid_limiter_status': (i32, [vp, vp, vp]),
    'exa_aderdg_grid_limiter_bounds': (i32, [vp, vp, vp]),
    'exa_aderdg_grid_set_halo': (i32, [vp, i32]),
    'exa_aderdg_grid_set_boundary': (i32, [vp, C.POINTER(i32)]),
    'exa_aderdg_grid_set_adjustment': (i32, [vp, vp]),
    'exa_fv_patchgrid_set_boundary': (i32, [vp, C.POINTER(i32)]),
    'exa_aderdg_solution_adjustment': (i32, [C.POINTER(AderdgDesc), i64, vp, vp, f64, f64, vp, vp]),
    'exa_aderdg_solutionAdjustment': (i32, [i32, i32, dptr, dptr, dptr, f64, f64, vp]),
    'exa_aderdg_grid_halo_buffers': (i32, [vp, C.POINTER(vp), C.POINTER(vp), C.POINTER(vp), C.POINTER(vp),
                                           C.POINTER(sz)]),
    'exa_aderdg_grid_dt_slot': (i32, [vp, C.POINTER(vp)]),
    'exa_aderdg_grid_phase': (i32, [vp, i32]),
    'exa_aderdg_grid_init_slab': (i32, [vp, i32, f64, u64, f64, i32, i32]),
    'exa_ensemble_footprint': (sz, [vp]),
    'exa_ensemble_create': (i32, [i32, i32, sz, C.POINTER(vp)]),
    'exa_ensemble_destroy': (i32, [vp]),
    'exa_ensemble_add': (i32, [vp, vp, C.c_longlong, C.POINTER(i32)]),
    'exa_ensemble_remove': (i32, [vp, i32]),
    'exa_ensemble_step': (i32, [vp, i32]),
    'exa_ensemble_use_graph': (i32, [vp, i32]),
    'exa_ensemble_tune': (i32, [vp, i32, i32, i32]),
    'exa_ensemble_tune_contraction': (i32, [vp, i32]),
    'exa_ensemble_set_launch_mode': (i32, [vp, i32]),
    'exa_ensemble_synchronize': (i32, [vp]),
    'exa_ensemble_stream': (i32, [vp, C.POINTER(vp)]),
    'exa_ensemble_get_state': (i32, [vp, i32, vp]),
    'exa_ensemble_device_state': (i32, [vp, i32, C.POINTER(vp)]),
    'exa_ensemble_checkpoint': (i32, [vp, i32, vp, vp]),
    'exa_ensemble_restore': (i32, [vp, vp, vp, vp, C.POINTER(i32)]),
    'exa_ensemble_status': (i32, [vp, vp, vp, vp, vp, vp]),
    'exa_ensemble_active_cells': (i64, [vp]),
    'exa_ensemble_info': (i32, [vp, C.POINTER(i32), C.POINTER(i32), C.POINTER(sz)]),
    'exa_server_footprint': (sz, [vp]),
    'exa_server_create': (i32, [sz, i32, i32, C.POINTER(vp)]),
    'exa_server_destroy': (i32, [vp]),
    'exa_server_submit': (i32, [vp, vp, C.POINTER(u64)]),
    'exa_server_tick': (i32, [vp, C.POINTER(i32)]),
    'exa_server_completed': (i32, [vp, C.POINTER(u64), i32, C.POINTER(i32)]),
    'exa_server_result_size': (sz, [vp, u64]),
    'exa_server_result': (i32, [vp, u64, vp, C.POINTER(f64), C.POINTER(C.c_longlong)]),
    'exa_server_info': (i32, [vp, C.POINTER(i32), C.POINTER(C.c_long), C.POINTER(sz)]),
    'exa_server_run': (i32, [vp, vp, vp, i32, f64, vp, C.POINTER(u64)]),
    'exa_server_tune': (i32, [vp, i32, i32]),
    'exa_server_set_fv_steps': (i32, [vp, i32]),
    'exa_server_device_state': (i32, [vp, u64, C.POINTER(vp)]),
    'exa_server_evict': (i32, [vp, u64]),
    'exa_server_restore': (i32, [vp, u64]),
    'exa_server_evicted': (i32, [vp, u64, C.POINTER(i32)]),
    'exa_server_set_eviction': (i32, [vp, f64]),
    'exa_server_set_result_mode': (i32, [vp, i32]),
    'exa_server_set_staging': (i32, [vp, sz]),
    'exa_server_loop_times': (i32, [vp, dptr]),
    'exa_fv_godunov_update': (i32, [C.POINTER(FVDesc), i64, vp, vp, f64, vp, vp]),
    'exa_fv_musclhancock_update': (i32, [C.POINTER(FVDesc), i64, vp, vp, f64, vp, vp]),
    'exa_fv_stable_dt': (i32, [C.POINTER(FVDesc), i64, vp, vp, vp]),
    'exa_fv_periodic_ghosts': (i32, [C.POINTER(FVDesc), i64, vp, vp]),
    'exa_fv_rusanov': (i32, [i32, i32, i32, i32, dptr, dptr, dptr, dptr, i32, dptr]),
}


def _status_string(s):
    if _lib is None:
        return str(s)
    return _lib.exa_status_string(s).decode()


def lib():
    """Load the library (once).  Raises if it was not built."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise RuntimeError('libexahype_b200.so not found at %s; build it with '
                               '`make -C exahype_b200/csrc -j` (no CPU fallback exists)' % LIB_PATH)
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status, where):
    if status != EXA_OK:
        detail = lib().exa_last_error_string().decode()
        raise ExaError(status, where, detail)
    return status


def call(name, *args):
    """Call an exa_* function and raise ExaError on a non-zero status."""
    return check(getattr(lib(), name)(*args), name)
