"""A-posteriori subcell limiter kernels (the reference's
kernels/limiter/generic/c/Limiter.cpp) over the C ABI.

Batched functions take DeviceBuffer arguments holding `ncells` cells back to
back (layouts in include/exa_kernels.h); the camel-case functions are the
per-cell drop-ins with the reference's argument lists on host numpy arrays.
"""
import ctypes as C

import numpy as np

from ._lib import call

_dptr = C.POINTER(C.c_double)


def subcells(order):
    """FV subcells per direction of the limiter patch of an order-N cell
    (Limiter.h getBasisSizeLim: 2 (basisSize - 1) + 1)."""
    return 2 * order + 1


def patch_doubles(dim, order, nvar=5, ghost=0):
    """doubles of one limiter patch with `ghost` ghost layers"""
    return (subcells(order) + 2 * ghost) ** dim * nvar


def project_on_fv(dim, order, ncells, luh, lim, nvar=5, ghost=0, stream=None):
    """projectOnFVLimiterSpace for every cell (interior of lim)."""
    call('exa_limiter_project_on_fv', dim, order, nvar, ghost, int(ncells), luh.ptr, lim.ptr, stream)


def project_on_dg(dim, order, ncells, lim, luh, nvar=5, ghost=0, stream=None):
    """projectOnDGSpace for every cell."""
    call('exa_limiter_project_on_dg', dim, order, nvar, ghost, int(ncells), lim.ptr, luh.ptr, stream)


def local_min_max(dim, order, ncells, luh, obs_min, obs_max, nvar=5, nobs=5, stream=None):
    """findCellLocalMinAndMax, copied to all 2 dim face blocks per cell."""
    call('exa_limiter_local_min_max', dim, order, nvar, nobs, int(ncells), luh.ptr, obs_min.ptr, obs_max.ptr,
         stream)


def fv_min_max(dim, order, ncells, lim, obs_min, obs_max, nvar=5, nobs=5, ghost=0, stream=None):
    """findCellLocalLimiterMinAndMax, copied to all face blocks per cell."""
    call('exa_limiter_fv_min_max', dim, order, nvar, nobs, ghost, int(ncells), lim.ptr, obs_min.ptr,
         obs_max.ptr, stream)


def dmp(dim, order, ncells, luh, obs_min, obs_max, dmp_ok, relaxation, difference_scaling, nvar=5, nobs=5,
        stream=None):
    """discreteMaximumPrincipleAndMinAndMaxSearch per cell; dmp_ok: int32
    DeviceBuffer of ncells verdicts."""
    call('exa_limiter_dmp', dim, order, nvar, nobs, int(ncells), luh.ptr, float(relaxation),
         float(difference_scaling), obs_min.ptr, obs_max.ptr, dmp_ok.ptr, stream)


def _d(a):
    return a.ctypes.data_as(_dptr)


def projectOnFVLimiterSpace(dim, luh, numberOfVariables, basisSize, ghostLayerWidth, lim):
    call('exa_limiter_projectOnFVLimiterSpace', dim, _d(luh), numberOfVariables, basisSize, ghostLayerWidth,
         _d(lim))


def projectOnDGSpace(dim, lim, numberOfVariables, basisSize, ghostLayerWidth, luh):
    call('exa_limiter_projectOnDGSpace', dim, _d(lim), numberOfVariables, basisSize, ghostLayerWidth, _d(luh))


def findCellLocalMinAndMax(dim, luh, numberOfVariables, basisSize, numberOfObservables, mn, mx):
    call('exa_limiter_findCellLocalMinAndMax', dim, _d(luh), numberOfVariables, basisSize, numberOfObservables,
         _d(mn), _d(mx))


def discreteMaximumPrincipleAndMinAndMaxSearch(dim, luh, numberOfVariables, basisSize, numberOfObservables,
                                               relaxationParameter, differenceScaling, bmin, bmax):
    """Returns True if the DMP holds; bmin/bmax are updated in place."""
    ok = C.c_int(0)
    call('exa_limiter_discreteMaximumPrincipleAndMinAndMaxSearch', dim, _d(luh), numberOfVariables, basisSize,
         numberOfObservables, float(relaxationParameter), float(differenceScaling), _d(bmin), _d(bmax),
         C.byref(ok))
    return bool(ok.value)
