"""Host-side mirror of the reference's finite-volume solver kernels
(Abstract<Solver> of AbstractGenericFiniteVolumesSolverHeader.template:52-63)
over batches of 2D patches resident on the GPU."""
import ctypes as C

import numpy as np

from . import _lib
from ._lib import FVDesc, call

GODUNOV = 0
MUSCLHANCOCK = 1


def make_fv_desc(patch, ghost, dx, pde=_lib.PDE_EULER, npar=0):
    d = FVDesc()
    d.dim, d.patch, d.ghost, d.nvar, d.npar, d.pde = 2, patch, ghost, 5, npar, pde
    dx = list(dx) + [1.0] * (3 - len(dx))
    for i in range(3):
        d.dx[i] = float(dx[i])
    return d


class FVPatches:
    """Batched FV entry points on `npatches` patches (DeviceBuffer args)."""

    def __init__(self, patch, ghost, dx, pde=_lib.PDE_EULER, npar=0):
        self.desc = make_fv_desc(patch, ghost, dx, pde, npar)
        self.patch, self.ghost = patch, ghost
        self.cells_per_patch = (patch + 2 * ghost) ** 2

    def godunov_update(self, npatches, luh_new, luh, dt, max_dt=None, stream=None):
        call('exa_fv_godunov_update', C.byref(self.desc), npatches, luh_new.ptr, luh.ptr, float(dt),
             max_dt.ptr if max_dt else None, stream)

    def musclhancock_update(self, npatches, luh_new, luh, dt, max_dt=None, stream=None):
        call('exa_fv_musclhancock_update', C.byref(self.desc), npatches, luh_new.ptr, luh.ptr,
             float(dt), max_dt.ptr if max_dt else None, stream)

    def stable_dt(self, npatches, luh, dt_patch, stream=None):
        call('exa_fv_stable_dt', C.byref(self.desc), npatches, luh.ptr, dt_patch.ptr, stream)

    def periodic_ghosts(self, npatches, luh, stream=None):
        call('exa_fv_periodic_ghosts', C.byref(self.desc), npatches, luh.ptr, stream)


def rusanov(fL, fR, qL, qR, normalNonZero, dim=2, pde=_lib.PDE_EULER):
    """riemannsolvers::c::rusanov drop-in on host arrays; returns s_max."""
    dp = C.POINTER(C.c_double)
    s = C.c_double()
    call('exa_fv_rusanov', dim, 5, 0, pde, fL.ctypes.data_as(dp), fR.ctypes.data_as(dp),
         np.ascontiguousarray(qL).ctypes.data_as(dp), np.ascontiguousarray(qR).ctypes.data_as(dp),
         int(normalNonZero), C.byref(s))
    return s.value
