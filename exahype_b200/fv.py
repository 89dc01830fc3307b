"""Host-side mirror of the reference's finite-volume solver kernels
(Abstract<Solver> of AbstractGenericFiniteVolumesSolverHeader.template:52-63)
over batches of 2D patches resident on the GPU."""
import ctypes as C

import numpy as np

from . import _lib
from ._lib import FVDesc, call

GODUNOV = 0
MUSCLHANCOCK = 1


def make_fv_desc(patch, ghost, dx, pde=_lib.PDE_EULER, npar=0, dim=2):
    d = FVDesc()
    d.dim, d.patch, d.ghost, d.nvar, d.npar, d.pde = dim, patch, ghost, 5, npar, pde
    dx = list(dx) + [1.0] * (3 - len(dx))
    for i in range(3):
        d.dx[i] = float(dx[i])
    return d


class FVPatches:
    """Batched FV entry points on `npatches` patches (DeviceBuffer args)."""

    def __init__(self, patch, ghost, dx, pde=_lib.PDE_EULER, npar=0, dim=2):
        self.desc = make_fv_desc(patch, ghost, dx, pde, npar, dim)
        self.patch, self.ghost, self.dim = patch, ghost, dim
        self.cells_per_patch = (patch + 2 * ghost) ** dim

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


class FVGrid:
    """Device-resident periodic 2D FV domain (one patch, fused steps)."""

    def __init__(self, scheme, patch, length=1.0, pde=_lib.PDE_EULER):
        h = C.c_void_p()
        call('exa_fv_grid_create', int(scheme), int(patch), float(length), int(pde), C.byref(h))
        self.h = h
        self.scheme, self.patch = scheme, patch
        self.ghost = 1 if scheme == GODUNOV else 2
        self.side = patch + 2 * self.ghost
        self.state_size = int(_lib.lib().exa_fv_grid_state_size(h))
        self.ncells = patch * patch

    def init(self, amp=0.2, seed=1, noise=0.0):
        call('exa_fv_grid_init', self.h, float(amp), int(seed), float(noise))

    def set_state(self, q):
        q = np.ascontiguousarray(q, dtype=np.float64)
        assert q.size == self.state_size
        call('exa_fv_grid_set_state', self.h, q.ctypes.data)

    def get_state(self):
        out = np.empty(self.state_size)
        call('exa_fv_grid_get_state', self.h, out.ctypes.data)
        return out

    def interior(self, q=None):
        q = self.get_state() if q is None else q
        g, P = self.ghost, self.patch
        return q.reshape(self.side, self.side, 5)[g:g + P, g:g + P]

    def step(self, nsteps=1):
        call('exa_fv_grid_step', self.h, int(nsteps))

    def status(self):
        t, dt = C.c_double(), C.c_double()
        call('exa_fv_grid_status', self.h, C.byref(t), C.byref(dt))
        return dict(time=t.value, dt_next=dt.value)

    def stream(self):
        s = C.c_void_p()
        call('exa_fv_grid_stream', self.h, C.byref(s))
        return s

    def device_state_ptr(self):
        p = C.c_void_p()
        call('exa_fv_grid_device_state', self.h, C.byref(p))
        return p

    def destroy(self):
        if self.h:
            call('exa_fv_grid_destroy', self.h)
            self.h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


class FVPatchGrid:
    """Device-resident periodic grid of npx x npy FV patches (the reference's
    FV layout: per-cell patches with ghost layers exchanged every step)."""

    def __init__(self, scheme, patch, npx, npy, length=1.0, pde=_lib.PDE_EULER):
        h = C.c_void_p()
        call('exa_fv_patchgrid_create', int(scheme), int(patch), int(npx), int(npy), float(length), int(pde),
             C.byref(h))
        self.h = h
        self.scheme, self.patch, self.npx, self.npy = scheme, patch, npx, npy
        self.ghost = 1 if scheme == GODUNOV else 2
        self.side = patch + 2 * self.ghost
        self.state_size = int(_lib.lib().exa_fv_patchgrid_state_size(h))
        self.ncells = patch * patch * npx * npy

    def init(self, amp=0.2, seed=1, noise=0.0):
        call('exa_fv_patchgrid_init', self.h, float(amp), int(seed), float(noise))

    def set_state(self, q):
        q = np.ascontiguousarray(q, dtype=np.float64)
        assert q.size == self.state_size
        call('exa_fv_patchgrid_set_state', self.h, q.ctypes.data)

    def get_state(self):
        out = np.empty(self.state_size)
        call('exa_fv_patchgrid_get_state', self.h, out.ctypes.data)
        return out

    def interiors(self, q=None):
        """[npy][npx][patch][patch][5] view of the patch interiors."""
        q = self.get_state() if q is None else q
        g, P, S = self.ghost, self.patch, self.side
        return q.reshape(self.npy, self.npx, S, S, 5)[:, :, g:g + P, g:g + P]

    def set_boundary(self, bc):
        """Boundary rule per dimension: _lib.BC_PERIODIC / BC_OUTFLOW /
        BC_REFLECT (see exa_fv_patchgrid_set_boundary)."""
        arr = (C.c_int * 2)(*list(bc)[:2])
        call('exa_fv_patchgrid_set_boundary', self.h, arr)

    def step(self, nsteps=1):
        call('exa_fv_patchgrid_step', self.h, int(nsteps))

    def status(self):
        t, dt = C.c_double(), C.c_double()
        call('exa_fv_patchgrid_status', self.h, C.byref(t), C.byref(dt))
        return dict(time=t.value, last_dt=dt.value)

    def stream(self):
        s = C.c_void_p()
        call('exa_fv_patchgrid_stream', self.h, C.byref(s))
        return s

    def destroy(self):
        if self.h:
            call('exa_fv_patchgrid_destroy', self.h)
            self.h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass
