"""Limiter kernels on the GPU (exa_limiter_*) against the oracle, which is
pinned to the reference's Limiter.cpp and its known-answer data in
test_oracle_limiter.py.  FP64 throughout: the GPU applies the projections
by sum factorisation, the oracle by the reference's direct sums, so values
agree to rounding (1e-13 relative); extrema and DMP verdicts are compared
exactly where the inputs leave no rounding tie."""
import numpy as np
import pytest

import _oracle as O
from exahype_b200 import DeviceBuffer, limiter

pytestmark = pytest.mark.gpu
V = 5


def rand_cells(dim, order, n, seed, lo=0.5, hi=10.0, nvar=V):
    rng = np.random.default_rng(seed)
    return rng.uniform(lo, hi, size=n * (order + 1) ** dim * nvar)


@pytest.mark.parametrize('dim', [2, 3])
@pytest.mark.parametrize('order', [1, 2, 3, 4, 5, 6])
@pytest.mark.parametrize('ghost', [0, 1, 2])
def test_project_on_fv_vs_oracle(dim, order, ghost):
    ncells = 37
    luh = rand_cells(dim, order, ncells, 11 * dim + order + 100 * ghost)
    s = O.lim_sizes(dim, order, V, ghost)
    fill = np.full(ncells * s['lim'], -123.0)  # ghost entries must stay untouched
    d_luh, d_lim = DeviceBuffer.from_array(luh), DeviceBuffer.from_array(fill)
    limiter.project_on_fv(dim, order, ncells, d_luh, d_lim, ghost=ghost)
    got = d_lim.download()
    ref = O.limiter_project_on_fv(dim, order, luh, ghost=ghost, lim=fill.copy())
    assert np.abs(got - ref).max() <= 1e-13 * np.abs(ref).max()
    if ghost:
        assert (got[ref == -123.0] == -123.0).all()


@pytest.mark.parametrize('dim', [2, 3])
@pytest.mark.parametrize('order', [1, 2, 3, 4, 5, 6])
@pytest.mark.parametrize('ghost', [0, 2])
def test_project_on_dg_vs_oracle(dim, order, ghost):
    ncells = 29
    s = O.lim_sizes(dim, order, V, ghost)
    lim = np.random.default_rng(order + 10 * dim + ghost).uniform(1.0, 10.0, ncells * s['lim'])
    d_lim, d_luh = DeviceBuffer.from_array(lim), DeviceBuffer(ncells * s['luh'])
    limiter.project_on_dg(dim, order, ncells, d_lim, d_luh, ghost=ghost)
    got = d_luh.download()
    ref = O.limiter_project_on_dg(dim, order, lim, ghost=ghost)
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()


@pytest.mark.parametrize('dim', [2, 3])
@pytest.mark.parametrize('order', [2, 3, 4, 5])
def test_round_trip_and_conservation(dim, order):
    """DG -> FV -> DG is the identity; FV -> DG keeps every cell mean."""
    ncells = 64
    luh = rand_cells(dim, order, ncells, 5 + order)
    s = O.lim_sizes(dim, order, V, 1)
    d_luh, d_lim = DeviceBuffer.from_array(luh), DeviceBuffer(ncells * s['lim'])
    d_back = DeviceBuffer(luh.size)
    limiter.project_on_fv(dim, order, ncells, d_luh, d_lim, ghost=1)
    limiter.project_on_dg(dim, order, ncells, d_lim, d_back, ghost=1)
    assert np.abs(d_back.download() - luh).max() <= 1e-12 * np.abs(luh).max()
    # cell means: DG mean = sum w_i w_j (w_k) u, FV mean = average of subcells
    lim = np.random.default_rng(3).uniform(1, 2, ncells * s['lim'])
    d_lim2, d_u = DeviceBuffer.from_array(lim), DeviceBuffer(luh.size)
    limiter.project_on_dg(dim, order, ncells, d_lim2, d_u, ghost=1)
    u = d_u.download().reshape((ncells,) + (order + 1,) * dim + (V,))
    w = np.polynomial.legendre.leggauss(order + 1)[1] / 2  # GL weights on [0, 1]
    S = 2 * order + 1
    L = lim.reshape((ncells,) + (S + 2,) * dim + (V,))
    interior = L[(slice(None),) + (slice(1, S + 1),) * dim]
    fv_mean = interior.reshape(ncells, -1, V).mean(axis=1)
    ww = w
    for _ in range(dim - 1):
        ww = np.multiply.outer(ww, w)
    dg_mean = np.tensordot(u, ww, axes=(tuple(range(1, dim + 1)), tuple(range(dim))))
    assert np.abs(dg_mean - fv_mean).max() <= 1e-13 * np.abs(fv_mean).max()


@pytest.mark.parametrize('dim', [2, 3])
@pytest.mark.parametrize('order', [1, 2, 3, 4, 5, 6])
@pytest.mark.parametrize('nobs', [1, 5])
def test_local_min_max_vs_oracle(dim, order, nobs):
    ncells = 41
    luh = rand_cells(dim, order, ncells, 77 + order + dim, lo=-2.0, hi=3.0)
    nb = ncells * 2 * dim * nobs
    d_luh, d_mn, d_mx = DeviceBuffer.from_array(luh), DeviceBuffer(nb), DeviceBuffer(nb)
    limiter.local_min_max(dim, order, ncells, d_luh, d_mn, d_mx, nobs=nobs)
    rmn, rmx = O.limiter_local_min_max(dim, order, luh, nobs=nobs)
    assert np.abs(d_mn.download() - rmn).max() <= 1e-13 * np.abs(rmn).max()
    assert np.abs(d_mx.download() - rmx).max() <= 1e-13 * np.abs(rmx).max()


@pytest.mark.parametrize('dim', [2, 3])
@pytest.mark.parametrize('order', [2, 4, 6])
@pytest.mark.parametrize('ghost', [0, 1, 2])
def test_fv_min_max_vs_oracle(dim, order, ghost):
    ncells = 19
    s = O.lim_sizes(dim, order, V, ghost)
    lim = np.random.default_rng(order * 3 + ghost).standard_normal(ncells * s['lim'])
    nb = ncells * 2 * dim * 3
    d_lim, d_mn, d_mx = DeviceBuffer.from_array(lim), DeviceBuffer(nb), DeviceBuffer(nb)
    limiter.fv_min_max(dim, order, ncells, d_lim, d_mn, d_mx, nobs=3, ghost=ghost)
    rmn, rmx = O.limiter_fv_min_max(dim, order, lim, nobs=3, ghost=ghost)
    assert np.array_equal(d_mn.download(), rmn)
    assert np.array_equal(d_mx.download(), rmx)


@pytest.mark.parametrize('dim', [2, 3])
@pytest.mark.parametrize('order', [2, 3, 4, 5])
def test_dmp_vs_oracle(dim, order):
    """Verdicts and rewritten face blocks of a batch whose bounds are built so
    that some cells pass, some fail by a clear margin (no rounding ties)."""
    ncells = 200
    luh = rand_cells(dim, order, ncells, 1000 + order + dim, lo=0.5, hi=2.0)
    lmn, lmx = O.limiter_local_min_max(dim, order, luh)
    rng = np.random.default_rng(order)
    widen = rng.choice([0.2, -0.05, 0.0005], size=ncells)
    relax, scal = 1e-3, 1e-3
    nb = 2 * dim * V
    bmin = (lmn.reshape(ncells, nb) - widen[:, None] + rng.uniform(0, 0.01, (ncells, nb))).ravel()
    bmax = (lmx.reshape(ncells, nb) + widen[:, None] - rng.uniform(0, 0.01, (ncells, nb))).ravel()
    ok_ref, mn_ref, mx_ref = O.limiter_dmp(dim, order, luh, bmin, bmax, relax, scal)
    d_luh = DeviceBuffer.from_array(luh)
    d_mn, d_mx = DeviceBuffer.from_array(bmin), DeviceBuffer.from_array(bmax)
    d_ok = DeviceBuffer(ncells, dtype=np.int32)
    limiter.dmp(dim, order, ncells, d_luh, d_mn, d_mx, d_ok, relax, scal)
    assert np.array_equal(d_ok.download(), ok_ref)
    assert 0 < ok_ref.sum() < ncells
    assert np.abs(d_mn.download() - mn_ref).max() <= 1e-13 * np.abs(mn_ref).max()
    assert np.abs(d_mx.download() - mx_ref).max() <= 1e-13 * np.abs(mx_ref).max()


@pytest.mark.parametrize('dim', [2, 3])
def test_drop_ins_on_golden_data(dim):
    """The per-cell drop-ins with the reference's argument lists reproduce
    the reference's known-answer data (limiter_testdata.cpp, order 3)."""
    z = np.load(O.ROOT + '/tests/golden/limiter_%dd.npz' % dim)
    luh_in = z['testFromLuhConversion/luh_in'].copy()
    lim = np.zeros(7 ** dim * V)
    limiter.projectOnFVLimiterSpace(dim, luh_in, V, 4, 0, lim)
    ref = z['testFromLuhConversion/lim_out']
    assert np.abs(lim - ref).max() <= 1e-13 * np.abs(ref).max()
    luh = np.zeros(4 ** dim * V)
    limiter.projectOnDGSpace(dim, z['testToLuhConversion/lim_in'].copy(), V, 4, 0, luh)
    ref = z['testToLuhConversion/luh_out']
    assert np.abs(luh - ref).max() <= 1e-13 * np.abs(ref).max()
    mn, mx = np.zeros(V), np.zeros(V)
    limiter.findCellLocalMinAndMax(dim, luh_in, V, 4, V, mn, mx)
    rmn, rmx = O.limiter_local_min_max(dim, 3, luh_in)
    assert np.abs(mn - rmn[:V]).max() <= 1e-13 * np.abs(rmn).max()
    assert np.abs(mx - rmx[:V]).max() <= 1e-13 * np.abs(rmx).max()
    bmin, bmax = np.tile(rmn[:V] - 1.0, 2 * dim), np.tile(rmx[:V] + 1.0, 2 * dim)
    assert limiter.discreteMaximumPrincipleAndMinAndMaxSearch(dim, luh_in, V, 4, V, 1e-4, 1e-3, bmin, bmax)
    assert np.abs(bmin[:V] - rmn[:V]).max() <= 1e-13 * np.abs(rmn).max()
    bmin, bmax = np.tile(rmn[:V] + 0.5, 2 * dim), np.tile(rmx[:V] + 1.0, 2 * dim)
    assert not limiter.discreteMaximumPrincipleAndMinAndMaxSearch(dim, luh_in, V, 4, V, 1e-4, 1e-3, bmin, bmax)
