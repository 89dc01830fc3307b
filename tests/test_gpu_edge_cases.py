"""Edge cases of the batched device entry points: empty batches (zero cells,
faces, patches or items) succeed and write nothing; negative counts, NULL
pointers, descriptors outside the supported set and batches above a
documented maximum are rejected with EXA_EINVAL before any device work.  The
reference's generic kernels take one cell per call and have no empty-batch
form; its solvers simply make no call for an empty cell list, which is what
a zero count must amount to here."""
import ctypes as C

import numpy as np
import pytest

from exahype_b200 import DeviceBuffer, _lib, limiter
from exahype_b200.aderdg import BatchedADERDG, amr_prolongation, amr_restriction, make_desc
from exahype_b200.fv import FVPatches

pytestmark = pytest.mark.gpu
SENT = -777.0


def sentinel(n, dtype=np.float64):
    return DeviceBuffer.from_array(np.full(n, SENT if dtype == np.float64 else -7, dtype=dtype))


def untouched(*bufs):
    for b in bufs:
        a = b.download()
        assert (a == (SENT if b.dtype == np.float64 else -7)).all()


def einval(fn, *args):
    with pytest.raises(_lib.ExaError) as e:
        fn(*args)
    assert e.value.status == 1  # EXA_EINVAL


@pytest.mark.parametrize('dim,order', [(2, 3), (3, 4)])
def test_aderdg_empty_batches(dim, order):
    B = BatchedADERDG(dim, order, [0.1] * dim)
    luh, lduh, qb, fb = sentinel(64), sentinel(64), sentinel(64), sentinel(64)
    lqi, lfi, lqhi, lfhi = sentinel(64), sentinel(64), sentinel(64), sentinel(64)
    iters = sentinel(4, np.int32)
    B.predictor_vi(0, luh, 1e-3, lduh, qb, fb, iters=iters)
    B.predictor_full(0, luh, 1e-3, lqi, lfi, lqhi, lfhi, lduh, qb, fb, iters=iters)
    B.volume_integral(0, lduh, lfhi)
    B.surface_integral(0, lduh, fb)
    B.solution_update(0, luh, lduh, 1e-3)
    idx = sentinel(4, np.int32)
    B.riemann_faces(0, idx, idx, idx, qb, fb)
    dt_cell = sentinel(4)
    B.stable_dt(0, luh, dt_cell=dt_cell)
    untouched(luh, lduh, qb, fb, lqi, lfi, lqhi, lfhi, iters, idx, dt_cell)
    # the global minimum of no cells is +inf (the reduction's identity)
    dt_min = sentinel(1)
    B.stable_dt(0, luh, dt_min=dt_min)
    assert dt_min.download()[0] == np.inf


@pytest.mark.parametrize('dim,patch,ghost', [(2, 8, 2), (3, 5, 2)])
def test_fv_empty_batches(dim, patch, ghost):
    P = FVPatches(patch, ghost, [1.0] * dim, dim=dim)
    a, b, dt = sentinel(64), sentinel(64), sentinel(4)
    P.godunov_update(0, a, b, 1e-3, max_dt=dt)
    P.musclhancock_update(0, a, b, 1e-3, max_dt=dt)
    P.stable_dt(0, b, dt)
    P.periodic_ghosts(0, a)
    untouched(a, b, dt)


@pytest.mark.parametrize('dim', [2, 3])
def test_limiter_empty_batches(dim):
    a, b, mn, mx = sentinel(64), sentinel(64), sentinel(64), sentinel(64)
    ok = sentinel(4, np.int32)
    limiter.project_on_fv(dim, 3, 0, a, b, ghost=1)
    limiter.project_on_dg(dim, 3, 0, a, b, ghost=1)
    limiter.local_min_max(dim, 3, 0, a, mn, mx)
    limiter.fv_min_max(dim, 3, 0, a, mn, mx, ghost=1)
    limiter.dmp(dim, 3, 0, a, mn, mx, ok, 1e-4, 1e-3)
    untouched(a, b, mn, mx, ok)


def test_amr_empty_batches():
    fine, coarse = sentinel(64), sentinel(64)
    index = sentinel(4, np.int32)
    for k in (2, 3):
        amr_prolongation(k, 3, 0, fine, coarse, 1, index)
        amr_restriction(k, 3, 0, coarse, fine, 1, index)
    untouched(fine, coarse, index)


def test_negative_counts_rejected():
    B = BatchedADERDG(3, 3, [0.1] * 3)
    buf, ibuf = sentinel(64), sentinel(4, np.int32)
    einval(B.predictor_vi, -1, buf, 1e-3, buf, buf, buf)
    einval(B.volume_integral, -1, buf, buf)
    einval(B.surface_integral, -1, buf, buf)
    einval(B.solution_update, -1, buf, buf, 1e-3)
    einval(B.riemann_faces, -1, ibuf, ibuf, ibuf, buf, buf)
    einval(B.stable_dt, -1, buf)
    P = FVPatches(5, 2, [1.0] * 3, dim=3)
    einval(P.godunov_update, -1, buf, buf, 1e-3)
    einval(P.stable_dt, -1, buf, buf)
    einval(P.periodic_ghosts, -1, buf)
    einval(limiter.project_on_fv, 3, 3, -1, buf, buf)
    einval(amr_prolongation, 3, 3, -1, buf, buf, 1, ibuf)
    untouched(buf, ibuf)


def test_null_pointers_rejected():
    desc = make_desc(3, 3, [0.1] * 3)
    buf = sentinel(64)
    L = _lib.lib()
    st = L.exa_aderdg_predictor_vi(C.byref(desc), 4, None, 1e-3, None, buf.ptr, buf.ptr, buf.ptr, None, None, None)
    assert st == 1
    st = L.exa_aderdg_solution_update(C.byref(desc), 4, buf.ptr, None, 1e-3, None)
    assert st == 1
    st = L.exa_aderdg_riemann_faces(C.byref(desc), 4, None, None, None, buf.ptr, buf.ptr, None)
    assert st == 1
    st = L.exa_aderdg_predictor_vi(None, 4, buf.ptr, 1e-3, None, buf.ptr, buf.ptr, buf.ptr, None, None, None)
    assert st == 1
    untouched(buf)


@pytest.mark.parametrize('field,value', [('dim', 1), ('dim', 4), ('order', 1), ('order', 6), ('nvar', 4),
                                         ('npar', 2), ('pde', 7)])
def test_bad_descriptors_rejected(field, value):
    B = BatchedADERDG(3, 3, [0.1] * 3)
    setattr(B.desc, field, value)
    buf = sentinel(64)
    einval(B.predictor_vi, 1, buf, 1e-3, buf, buf, buf)
    einval(B.solution_update, 1, buf, buf, 1e-3)
    untouched(buf)


def test_non_positive_dx_rejected():
    B = BatchedADERDG(2, 3, [0.1, 0.0])
    buf = sentinel(64)
    einval(B.solution_update, 1, buf, buf, 1e-3)
    untouched(buf)


def test_fv_limits_rejected():
    buf = sentinel(64)
    # MUSCL-Hancock needs two ghost layers, Godunov one
    einval(FVPatches(8, 1, [1.0, 1.0]).musclhancock_update, 1, buf, buf, 1e-3)
    einval(FVPatches(8, 0, [1.0, 1.0]).godunov_update, 1, buf, buf, 1e-3)
    # one CTA stages a whole 3D patch: larger patches are refused
    einval(FVPatches(40, 2, [1.0] * 3, dim=3).musclhancock_update, 1, buf, buf, 1e-3)
    # the patch count is a grid dimension: at most 65535 per call
    einval(FVPatches(4, 1, [1.0, 1.0]).godunov_update, 65536, buf, buf, 1e-3)
    untouched(buf)


def test_limiter_limits_rejected():
    buf = sentinel(64)
    ok = sentinel(4, np.int32)
    einval(limiter.project_on_fv, 3, 7, 1, buf, buf)       # order 1..6
    einval(limiter.project_on_fv, 4, 3, 1, buf, buf)       # dim 2 or 3
    einval(limiter.project_on_fv, 3, 3, 1, buf, buf, 5, 9)  # ghost 0..8
    einval(limiter.local_min_max, 3, 3, 1, buf, buf, buf, 5, 6)  # nobs <= nvar
    einval(limiter.dmp, 3, 3, 1, buf, buf, buf, ok, 1e-4, 1e-3, 5, 0)  # the DMP needs an observable
    untouched(buf, ok)
