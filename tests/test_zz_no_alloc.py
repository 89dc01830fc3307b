"""The allocation-free predictor entry point, called through the C ABI,
returns what the ordinary drop-in returns, on two calls in a row.

It exists for callers that must not trigger a device allocation (many host
threads calling per-cell kernels at once, where cudaMalloc/cudaFree would
lock and synchronise the device, or a device whose memory a pool allocator
already owns); it stages the cell through a fixed device array instead of a
workspace the library allocates.  This file is collected last on purpose."""
import ctypes as C
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest

import _cases
import exahype_b200 as E
from exahype_b200 import _lib

pytestmark = pytest.mark.gpu
TOL = 1e-12
_dp = C.POINTER(C.c_double)


def _run(fn, desc, luh, dx, dt, dim, order, npar):
    B, D, V = order + 1, 5 + npar, 5
    nn = B ** dim
    out = dict(lQi=np.zeros(nn * B * D), lFi=np.zeros(nn * B * (dim + 1) * V), lQhi=np.zeros(nn * D),
               lFhi=np.zeros(nn * (dim + 1) * V), qb=np.zeros(2 * dim * B ** (dim - 1) * D),
               fb=np.zeros(2 * dim * B ** (dim - 1) * V))
    stu = (_dp * 1)(out['lQi'].ctypes.data_as(_dp))
    stf = (_dp * 1)(out['lFi'].ctypes.data_as(_dp))
    it = C.c_int(-1)
    luh = np.ascontiguousarray(luh, dtype=np.float64)
    dxa = np.asarray(dx, dtype=np.float64)
    st = getattr(E.lib(), fn)(C.byref(desc), out['qb'].ctypes.data_as(_dp), out['fb'].ctypes.data_as(_dp),
                              stu, stf, out['lQhi'].ctypes.data_as(_dp), out['lFhi'].ctypes.data_as(_dp),
                              None, luh.ctypes.data_as(_dp), dxa.ctypes.data_as(_dp), float(dt), None,
                              C.byref(it))
    _lib.check(st, fn)
    out['iters'] = it.value
    return out


def _rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def _cases_inputs(golden3d):
    rng = np.random.default_rng(42)
    luh3 = _cases._strided(golden3d['testSpaceTimePredictorNonlinear/luh'], 4 ** 3)
    q = np.zeros((36, 5))
    q[:, 0] = 1.0 + 0.1 * rng.random(36)
    q[:, 1:3] = 0.2 * rng.standard_normal((36, 2))
    q[:, 4] = 2.5 + 0.1 * rng.random(36)
    return [(3, 3, 1, E.PDE_EULER, luh3, [0.05] * 3, 1.083937460199773e-3),
            (2, 5, 0, E.PDE_EULER_PLANAR, q.ravel(), [0.02, 0.03], 4e-4)]


def test_noalloc_matches_dropin_twice(golden3d):
    for dim, order, npar, pde, luh, dx, dt in _cases_inputs(golden3d):
        desc = E.make_desc(dim, order, dx, npar=npar, pde=pde)
        first = _run('exa_aderdg_spaceTimePredictor_noalloc', desc, luh, dx, dt, dim, order, npar)
        second = _run('exa_aderdg_spaceTimePredictor_noalloc', desc, luh, dx, dt, dim, order, npar)
        ref = _run('exa_aderdg_spaceTimePredictor', desc, luh, dx, dt, dim, order, npar)
        for got in (first, second):
            assert got['iters'] == ref['iters'] > 0
            for k in ('lQi', 'lFi', 'lQhi', 'lFhi', 'qb', 'fb'):
                assert _rel(got[k], ref[k]) <= TOL, (dim, order, k, _rel(got[k], ref[k]))


def test_noalloc_reproduces_golden(golden3d):
    """Same reference known-answer case the drop-in is held to."""
    class Impl(_cases.OracleImpl):
        def __init__(self):
            pass

        def stp(self, dim, order, npar, planar, luh, dx, dt):
            desc = E.make_desc(dim, order, dx, npar=npar,
                               pde=E.PDE_EULER_PLANAR if planar else E.PDE_EULER)
            r = _run('exa_aderdg_spaceTimePredictor_noalloc', desc, luh, dx, dt, dim, order, npar)
            return dict(lQi=r['lQi'], lFi=r['lFi'], lQhi=r['lQhi'], lFhi=r['lFhi'], lQhbnd=r['qb'],
                        lFhbnd=r['fb'])
    _cases.stp_3d(Impl(), golden3d)


def _status(fn, desc, luh, dx, dt, dim, order, npar):
    try:
        _run(fn, desc, luh, dx, dt, dim, order, npar)
    except _lib.ExaError as e:
        return e.status
    return _lib.EXA_OK


def test_noalloc_rejects_what_the_dropin_rejects():
    """Same descriptor checks as the drop-in: an unknown pde, planar Euler in
    3D, nPar = 1 at an order other than 3, a bad order or a non-positive dx
    all return EXA_EINVAL from both entry points."""
    luh = np.ones(4 ** 3 * 6)
    bad = []
    d = E.make_desc(3, 3, [0.1] * 3)
    d.pde = 7
    bad.append((d, 3, 3, 0))
    bad.append((E.make_desc(3, 3, [0.1] * 3, pde=E.PDE_EULER_PLANAR), 3, 3, 0))
    bad.append((E.make_desc(3, 4, [0.1] * 3, npar=1), 3, 4, 1))
    d = E.make_desc(3, 3, [0.1] * 3)
    d.order = 6
    bad.append((d, 3, 6, 0))
    for desc, dim, order, npar in bad:
        B = order + 1
        u = np.ones(B ** dim * (5 + npar))
        for fn in ('exa_aderdg_spaceTimePredictor', 'exa_aderdg_spaceTimePredictor_noalloc'):
            assert _status(fn, desc, u, [0.1] * 3, 1e-4, dim, order, npar) == _lib.EXA_EINVAL, (fn, order)
    desc = E.make_desc(3, 3, [0.1, -0.1, 0.1])
    for fn in ('exa_aderdg_spaceTimePredictor', 'exa_aderdg_spaceTimePredictor_noalloc'):
        assert _status(fn, desc, luh[:4 ** 3 * 5], [0.1, -0.1, 0.1], 1e-4, 3, 3, 0) == _lib.EXA_EINVAL


_FRESH = textwrap.dedent('''
    import ctypes as C, sys
    import numpy as np
    sys.path.insert(0, sys.argv[1])
    import exahype_b200 as E
    from exahype_b200 import _lib
    L = E.lib()
    _lib.check(L.exa_set_device(0), 'set device')
    cap = C.c_size_t(123)
    dp = C.POINTER(C.c_double)
    def call(fn, order):
        B = order + 1
        nn = B ** 3
        desc = E.make_desc(3, order, [0.1] * 3)
        luh = np.zeros(nn * 5)
        luh[0::5] = 1.0
        luh[4::5] = 2.5
        o = [np.zeros(n) for n in (6 * B * B * 5, 6 * B * B * 5, nn * 5, nn * 4 * 5)]
        dx = np.full(3, 0.1)
        _lib.check(getattr(L, fn)(C.byref(desc), *[a.ctypes.data_as(dp) for a in o[:2]], None, None,
                                  *[a.ctypes.data_as(dp) for a in o[2:]], None, luh.ctypes.data_as(dp),
                                  dx.ctypes.data_as(dp), 1e-4, None, None), fn)
    for order in (2, 5, 3):
        call('exa_aderdg_spaceTimePredictor_noalloc', order)
        _lib.check(L.exa_dropin_workspace_doubles(0, C.byref(cap)), 'query')
        assert cap.value == 0, cap.value
    call('exa_aderdg_spaceTimePredictor', 3)
    _lib.check(L.exa_dropin_workspace_doubles(0, C.byref(cap)), 'query')
    assert cap.value > 0, cap.value
    print('fresh ok', cap.value)
''')


def test_noalloc_allocates_nothing_in_a_fresh_process():
    """In a process that never called the drop-in, calls of the allocation-
    free entry point (orders 2, 5, 3) leave the drop-in workspace
    unallocated; the drop-in's first call then allocates it (the query
    sees an allocation when there is one)."""
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, '-c', _FRESH, root], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert 'fresh ok' in r.stdout
