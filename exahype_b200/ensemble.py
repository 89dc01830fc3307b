"""Ensembles of independent 2D ADER-DG solves advanced by one persistent
launch per step (exa_ensemble_* in include/exa_kernels.h)."""
import ctypes as C

import numpy as np

from . import _lib
from ._lib import call, lib


class SolveConfig(C.Structure):
    _fields_ = [('order', C.c_int), ('n', C.c_int * 2), ('length', C.c_double * 2), ('pde', C.c_int),
                ('dt_policy', C.c_int), ('cfl', C.c_double), ('dt_fixed', C.c_double), ('ic_kind', C.c_int),
                ('ic_param', C.c_double), ('seed', C.c_uint64), ('noise', C.c_double)]


def solve_config(order, n, length=(1.0, 1.0), pde=_lib.PDE_EULER, dt_policy=0, cfl=0.9, dt_fixed=0.0,
                 ic_kind=1, ic_param=0.2, seed=0, noise=0.0):
    c = SolveConfig()
    c.order = order
    c.n[0], c.n[1] = int(n[0]), int(n[1])
    c.length[0], c.length[1] = float(length[0]), float(length[1])
    c.pde, c.dt_policy, c.cfl, c.dt_fixed = pde, dt_policy, cfl, dt_fixed
    c.ic_kind, c.ic_param, c.seed, c.noise = ic_kind, ic_param, seed, noise
    return c


def footprint(cfg):
    return int(lib().exa_ensemble_footprint(C.byref(cfg)))


class SolveCheckpoint(C.Structure):
    _fields_ = [('time', C.c_double), ('dt', C.c_double), ('dt_next_bits', C.c_uint64),
                ('steps_done', C.c_uint64), ('steps_left', C.c_int64), ('picard', C.c_uint64),
                ('nonconverged', C.c_uint64), ('active', C.c_int), ('nan_flag', C.c_int)]


class Ensemble:
    def __init__(self, max_solves, arena_bytes, precision=_lib.PREC_FP64):
        h = C.c_void_p()
        call('exa_ensemble_create', int(precision), int(max_solves), int(arena_bytes), C.byref(h))
        self.h = h
        self.max_solves = max_solves
        self.cfgs = {}

    def add(self, cfg, steps=-1):
        """Admits a solve; returns its slot, or None when it does not fit now."""
        slot = C.c_int(-1)
        st = lib().exa_ensemble_add(self.h, C.byref(cfg), int(steps), C.byref(slot))
        if st == _lib.EXA_EBUSY:
            return None
        _lib.check(st, 'exa_ensemble_add')
        self.cfgs[slot.value] = cfg
        return slot.value

    def remove(self, slot):
        call('exa_ensemble_remove', self.h, int(slot))
        self.cfgs.pop(slot, None)

    def step(self, nsteps=1):
        call('exa_ensemble_step', self.h, int(nsteps))

    def use_graph(self, enable=True):
        call('exa_ensemble_use_graph', self.h, int(enable))

    def tune(self, ctas_per_sm=0, grab=1, order_policy=0):
        call('exa_ensemble_tune', self.h, int(ctas_per_sm), int(grab), int(order_policy))

    def tune_contraction(self, lines_mask):
        """Per order N: bit N set = line-owner contraction, clear = node-gather."""
        call('exa_ensemble_tune_contraction', self.h, int(lines_mask))

    def set_launch_mode(self, mode):
        """0: one persistent launch per step; 1: one launch per order and phase."""
        call('exa_ensemble_set_launch_mode', self.h, int(mode))

    def synchronize(self):
        call('exa_ensemble_synchronize', self.h)

    def stream(self):
        s = C.c_void_p()
        call('exa_ensemble_stream', self.h, C.byref(s))
        return s

    def state_size(self, slot):
        c = self.cfgs[slot]
        return c.n[0] * c.n[1] * (c.order + 1) ** 2 * 5

    def get_state(self, slot):
        out = np.empty(self.state_size(slot))
        call('exa_ensemble_get_state', self.h, int(slot), out.ctypes.data)
        return out

    def checkpoint(self, slot):
        """(state, SolveCheckpoint) of a solve: what restore() needs to
        continue it bit for bit."""
        out = np.empty(self.state_size(slot))
        ck = SolveCheckpoint()
        call('exa_ensemble_checkpoint', self.h, int(slot), out.ctypes.data, C.byref(ck))
        return out, ck

    def restore(self, cfg, state, ck):
        """Adds a solve from a checkpoint; returns its slot, or None when it
        does not fit now."""
        state = np.ascontiguousarray(state, dtype=np.float64)
        slot = C.c_int(-1)
        st = lib().exa_ensemble_restore(self.h, C.byref(cfg), state.ctypes.data, C.byref(ck), C.byref(slot))
        if st == _lib.EXA_EBUSY:
            return None
        _lib.check(st, 'exa_ensemble_restore')
        self.cfgs[slot.value] = cfg
        return slot.value

    def device_state_ptr(self, slot):
        p = C.c_void_p()
        call('exa_ensemble_device_state', self.h, int(slot), C.byref(p))
        return p

    def status(self):
        n = self.max_solves
        t = np.zeros(n)
        steps = np.zeros(n, dtype=np.uint64)
        act = np.zeros(n, dtype=np.int32)
        pic = np.zeros(n, dtype=np.uint64)
        nan = np.zeros(n, dtype=np.int32)
        st = lib().exa_ensemble_status(self.h, t.ctypes.data, steps.ctypes.data, act.ctypes.data,
                                       pic.ctypes.data, nan.ctypes.data)
        if st not in (_lib.EXA_OK, _lib.EXA_ENAN):
            _lib.check(st, 'exa_ensemble_status')
        return dict(time=t, steps=steps, active=act, picard=pic, nan=nan)

    def active_cells(self):
        return int(lib().exa_ensemble_active_cells(self.h))

    def info(self):
        g, it, fr = C.c_int(), C.c_int(), C.c_size_t()
        call('exa_ensemble_info', self.h, C.byref(g), C.byref(it), C.byref(fr))
        return dict(grid_ctas=g.value, items=it.value, arena_free=fr.value)

    def destroy(self):
        if self.h:
            call('exa_ensemble_destroy', self.h)
            self.h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass
