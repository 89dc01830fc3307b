"""exahype_b200: B200-native ADER-DG / finite-volume cell-update library.

The compute path is libexahype_b200.so (hand-written sm_100a CUDA behind the
C ABI declared in include/exa_kernels.h); this package is the thin Python
host layer over that ABI.
"""
from ._lib import (ADJUST_ALWAYS, ADJUST_AT_START, ADJUST_HEAT_SOURCE, ADJUST_ISENTROPIC_VORTEX, ADJUST_NONE,
                   ADJUST_SINE_WAVE, BC_OUTFLOW, BC_PERIODIC, BC_REFLECT, EXA_OK, PDE_EULER, PDE_EULER_PLANAR,
                   PREC_FP64, PREC_MIXED, ExaError, lib)
from .aderdg import ADERDGGrid, ADERDGSolver, BatchedADERDG, adjust_hook, make_desc, solutionAdjustment
from .device import DeviceBuffer, PinnedBuffer, Stream, Timer, device_count, launch_count
from .ensemble import Ensemble, solve_config
from .fv import FVGrid, FVPatchGrid, FVPatches
from . import limiter

__all__ = ['ADERDGGrid', 'ADERDGSolver', 'BatchedADERDG', 'DeviceBuffer', 'PinnedBuffer', 'Stream',
           'Timer', 'FVPatches', 'FVGrid', 'FVPatchGrid', 'Ensemble', 'solve_config', 'ExaError', 'lib', 'make_desc', 'device_count', 'launch_count',
           'EXA_OK', 'PDE_EULER', 'PDE_EULER_PLANAR', 'PREC_FP64', 'PREC_MIXED', 'BC_PERIODIC', 'BC_OUTFLOW',
           'BC_REFLECT', 'limiter', 'adjust_hook', 'solutionAdjustment', 'ADJUST_NONE', 'ADJUST_SINE_WAVE',
           'ADJUST_ISENTROPIC_VORTEX', 'ADJUST_HEAT_SOURCE', 'ADJUST_AT_START', 'ADJUST_ALWAYS']
