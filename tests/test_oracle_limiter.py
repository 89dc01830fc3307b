"""A-posteriori subcell limiter (kernels/limiter/generic/c/Limiter.cpp):
the project's projection tables and the oracle's restatement of the limiter
kernels, pinned against (1) the reference's known-answer data
(exahype/tests/kernels/testdata/limiter_testdata.cpp, extracted to
tests/golden/limiter_{2d,3d}.npz) and (2) the reference's own Limiter.cpp
and LimiterProjectionMatrices.cpp compiled from source (oracle/_ref)."""
import importlib.util
import os

import numpy as np
import pytest

import _oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
V = 5


@pytest.fixture(scope='module')
def gen():
    spec = importlib.util.spec_from_file_location(
        'gen', os.path.join(ROOT, 'exahype_b200', 'csrc', 'gen_dg_tables.py'))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def golden(dim):
    return np.load(os.path.join(ROOT, 'tests', 'golden', 'limiter_%dd.npz' % dim))


def cells(dim, order, n, seed, lo=0.5, hi=10.0):
    rng = np.random.default_rng(seed)
    return rng.uniform(lo, hi, size=n * (order + 1) ** dim * V)


@pytest.mark.parametrize('dim', [2, 3])
def test_golden_dg_to_fv(dim):
    """luh -> subcell means, order 3 (limiter_testdata.cpp lim_out)."""
    z = golden(dim)
    lim = O.limiter_project_on_fv(dim, 3, z['testFromLuhConversion/luh_in'])
    ref = z['testFromLuhConversion/lim_out']
    assert np.abs(lim - ref).max() <= 1e-13 * np.abs(ref).max()


@pytest.mark.parametrize('dim', [2, 3])
def test_golden_fv_to_dg(dim):
    """subcell means -> luh, order 3 (limiter_testdata.cpp luh_out)."""
    z = golden(dim)
    luh = O.limiter_project_on_dg(dim, 3, z['testToLuhConversion/lim_in'])
    ref = z['testToLuhConversion/luh_out']
    assert np.abs(luh - ref).max() <= 1e-13 * np.abs(ref).max()


@pytest.mark.parametrize('dim', [2, 3])
def test_golden_lobatto_values(gen, dim):
    """luh at the Gauss-Lobatto points in the reference's (descending) node
    order with the generated uh2lob table (limiter_testdata.cpp lob_out)."""
    z = golden(dim)
    T = np.array(gen.derive(3)['uh2lob'])
    u = z['testFromLuhConversion/luh_in'].reshape((4,) * dim + (V,))
    if dim == 2:
        lob = np.einsum('yxv,yY,xX->YXv', u, T, T)
    else:
        lob = np.einsum('zyxv,zZ,yY,xX->ZYXv', u, T, T, T)
    ref = z['testFromLuhConversion/lob_out']
    assert np.abs(lob.ravel() - ref).max() <= 1e-13 * np.abs(ref).max()


@pytest.mark.parametrize('order', range(10))
def test_tables_vs_reference_build(gen, order):
    """uh2lim / uh2lob / lim2uh / Lobatto nodes against the reference's
    start-up computation (LimiterProjectionMatrices.cpp:40-140)."""
    R = O.ref_lib(2)
    if R is None or not hasattr(R, 'ref_limiter_tables'):
        pytest.skip('reference kernels not built (make -C oracle ref)')
    B, S = order + 1, 2 * order + 1
    a, b, c, d = np.zeros(B * S), np.zeros(B * B), np.zeros(S * B), np.zeros(B)
    R.ref_limiter_tables(order, a, b, c, d)
    t = gen.derive(order)
    for mine, theirs, tol in (('uh2lim', a, 1e-14), ('uh2lob', b, 1e-13), ('lim2uh', c, 1e-12),
                              ('lob_nodes', d, 1e-15)):
        m = np.array(t[mine]).ravel()
        assert np.abs(m - theirs).max() <= tol * max(1.0, np.abs(theirs).max()), mine


@pytest.mark.parametrize('order', range(10))
def test_projection_identities(gen, order):
    """lim2uh is a left inverse of uh2lim (DG -> FV -> DG is the identity on
    the DG space) and keeps the cell mean: sum_k w_k lim2uh[i][k] = 1/S."""
    t = gen.derive(order)
    U, L = np.array(t['uh2lim']), np.array(t['lim2uh'])
    w = np.array(t['gl_weights'])
    assert np.abs(L.T @ U.T - np.eye(order + 1)).max() < 1e-13
    assert np.abs(L @ w - 1.0 / (2 * order + 1)).max() < 1e-15


def _ref_call(R, what, order, nobs, ghost, inp, out=None, mn=None, mx=None, relax=0.0, scal=0.0):
    p = lambda a: a.ctypes.data if a is not None else None
    return R.ref_limiter(what, order, V, nobs, ghost, p(inp), p(out), p(mn), p(mx), relax, scal)


@pytest.mark.parametrize('dim', [2, 3])
@pytest.mark.parametrize('order', [1, 2, 3, 4, 5])
@pytest.mark.parametrize('ghost', [0, 1, 2])
def test_projections_vs_reference(dim, order, ghost):
    R = O.ref_lib(dim)
    if R is None or not hasattr(R, 'ref_limiter'):
        pytest.skip('reference kernels not built (make -C oracle ref)')
    s = O.lim_sizes(dim, order, V, ghost)
    luh = cells(dim, order, 1, 7 * dim + order + 100 * ghost)
    ref_lim = np.full(s['lim'], 7.5)
    _ref_call(R, 0, order, V, ghost, luh, ref_lim)
    my_lim = O.limiter_project_on_fv(dim, order, luh, ghost=ghost, lim=np.full(s['lim'], 7.5))
    assert np.abs(my_lim - ref_lim).max() <= 1e-13 * np.abs(ref_lim).max()
    lim = np.random.default_rng(order).uniform(1, 10, s['lim'])
    ref_luh = np.zeros(s['luh'])
    _ref_call(R, 1, order, V, ghost, lim, ref_luh)
    my_luh = O.limiter_project_on_dg(dim, order, lim, ghost=ghost)
    assert np.abs(my_luh - ref_luh).max() <= 1e-12 * np.abs(ref_luh).max()


@pytest.mark.parametrize('dim', [2, 3])
@pytest.mark.parametrize('order', [1, 2, 3, 4, 5])
@pytest.mark.parametrize('nobs', [1, 3, 5])
def test_min_max_vs_reference(dim, order, nobs):
    R = O.ref_lib(dim)
    if R is None or not hasattr(R, 'ref_limiter'):
        pytest.skip('reference kernels not built (make -C oracle ref)')
    luh = cells(dim, order, 1, 3 * dim + order + 10 * nobs, lo=-3.0, hi=5.0)
    rmn, rmx = np.zeros(nobs), np.zeros(nobs)
    _ref_call(R, 2, order, nobs, 0, luh, None, rmn, rmx)
    mn, mx = O.limiter_local_min_max(dim, order, luh, nobs=nobs)
    mn, mx = mn.reshape(2 * dim, nobs), mx.reshape(2 * dim, nobs)
    for f in range(2 * dim):  # face 0 result, copied to every face
        assert np.abs(mn[f] - rmn).max() <= 1e-13 * np.abs(rmn).max()
        assert np.abs(mx[f] - rmx).max() <= 1e-13 * np.abs(rmx).max()
    # the extrema over nodes, Lobatto points and subcell means bracket the nodes
    nodes = luh.reshape(-1, V)[:, :nobs]
    assert (mn[0] <= nodes.min(0)).all() and (mx[0] >= nodes.max(0)).all()
    for ghost in (0, 2):
        s = O.lim_sizes(dim, order, V, ghost)
        lim = np.random.default_rng(order + ghost).uniform(-2, 2, s['lim'])
        rmn, rmx = np.zeros(nobs), np.zeros(nobs)
        _ref_call(R, 3, order, nobs, ghost, lim, None, rmn, rmx)
        mn, mx = O.limiter_fv_min_max(dim, order, lim, nobs=nobs, ghost=ghost)
        assert np.array_equal(mn.reshape(2 * dim, nobs)[-1], rmn)
        assert np.array_equal(mx.reshape(2 * dim, nobs)[0], rmx)


@pytest.mark.parametrize('dim', [2, 3])
@pytest.mark.parametrize('order', [2, 3, 4])
def test_dmp_vs_reference(dim, order):
    """discreteMaximumPrincipleAndMinAndMaxSearch: verdict and the rewritten
    face-0 (new local) / face-1 (boundary) blocks, for boundary bounds that
    hold, that fail from below, that fail from above and that pass only by
    the relaxation."""
    R = O.ref_lib(dim)
    if R is None or not hasattr(R, 'ref_limiter'):
        pytest.skip('reference kernels not built (make -C oracle ref)')
    rng = np.random.default_rng(dim * 10 + order)
    luh = cells(dim, order, 1, 99 + order, lo=0.5, hi=2.0)
    lmn, lmx = O.limiter_local_min_max(dim, order, luh)
    lmn, lmx = lmn.reshape(2 * dim, V)[0], lmx.reshape(2 * dim, V)[0]
    verdicts = set()
    for case in range(12):
        widen = [0.3, -0.05, 0.0, 0.01][case % 4]
        bmin = np.tile(lmn - widen, 2 * dim) + rng.uniform(0, 0.02, 2 * dim * V) * (case // 4)
        bmax = np.tile(lmx + widen, 2 * dim) - rng.uniform(0, 0.02, 2 * dim * V) * (case // 4)
        relax, scal = [(1e-4, 1e-3), (0.0, 0.0), (0.05, 0.0)][case % 3]
        rmn, rmx = bmin.copy(), bmax.copy()
        ok_ref = _ref_call(R, 4, order, V, 0, luh, None, rmn, rmx, relax, scal)
        ok, mn, mx = O.limiter_dmp(dim, order, luh, bmin, bmax, relax, scal)
        assert ok[0] == ok_ref, case
        verdicts.add(ok_ref)
        assert np.abs(mn - rmn).max() <= 1e-13 * np.abs(rmn).max()
        assert np.abs(mx - rmx).max() <= 1e-13 * np.abs(rmx).max()
    assert verdicts == {0, 1}
