"""Domain boundaries of the oracle's limiting ADER-DG step
(orc_limiting_grid_step with boundary rules): the subcell ghost filling at a
wall against the reference's own FiniteVolumesSolver::mergeWithBoundaryData
kernels (boundaryLayerExtraction, boundaryConditions,
ghostLayerFillingAtBoundary of finitevolumes/commons/c/commons.cpph, built in
oracle/_ref), and grid-level properties: a wall stops the status spreading
and the bounds merge, and a state mirror-symmetric between two walls stays
so, statuses included."""
import numpy as np
import pytest

import _limiting_ic as IC
import _oracle as O


@pytest.mark.parametrize('dim', [2, 3])
@pytest.mark.parametrize('patch', [3, 5, 7, 9])
@pytest.mark.parametrize('ghost', [1, 2])
@pytest.mark.parametrize('rule', [1, 2])
def test_boundary_ghosts_vs_reference(dim, patch, ghost, rule):
    R = O.ref_lib(dim)
    if R is None or not hasattr(R, 'ref_fv_boundary'):
        pytest.skip('reference kernels not built (make -C oracle ref)')
    S = patch + 2 * ghost
    rng = np.random.default_rng(100 * dim + 10 * patch + ghost + rule)
    for face in range(2 * dim):
        base = rng.uniform(-2.0, 3.0, S ** dim * 5)
        ref, mine = base.copy(), base.copy()
        assert R.ref_fv_boundary(patch, ghost, ref, face, rule) == 0
        O.lib().orc_fv_boundary_ghosts(dim, patch, ghost, mine, face, rule)
        assert np.array_equal(mine, ref), face
        assert not np.array_equal(ref, base)  # the face's ghosts were written


def _two_explosions(order, n):
    """explosions touching the walls x = 0 and x = 1, mirror images"""
    a = IC.explosion(order, n, center=(0.08, 0.5), radius=0.2)
    b = IC.explosion(order, n, center=(0.92, 0.5), radius=0.2)
    return np.where(a.reshape(-1, 5)[:, :1] == 1.0, a.reshape(-1, 5), b.reshape(-1, 5)).ravel()


def _mirror_x(luh, order, n):
    B = order + 1
    q = luh.reshape(n[1], n[0], B, B, 5)[:, ::-1, :, ::-1, :].copy()
    q[..., 1] *= -1
    return q.reshape(-1)


@pytest.mark.parametrize('scheme', [0, 1])
@pytest.mark.parametrize('rule', [1, 2])
def test_walls_keep_mirror_symmetry(scheme, rule):
    order, n = 3, (12, 10)
    luh = _two_explosions(order, n)
    assert np.array_equal(_mirror_x(luh, order, n), luh)
    g = O.LimitingGrid(order, n, luh, scheme=scheme, bc=[rule, 2])
    for k in range(6):
        g.step()
        st = g.status.reshape(n[1], n[0])
        assert g.counts[2] > 0
        assert np.array_equal(st, st[:, ::-1]), k
        assert np.abs(_mirror_x(g.luh, order, n) - g.luh).max() <= 1e-12 * np.abs(g.luh).max(), k
        assert np.isfinite(g.luh).all()


def test_wall_stops_status_spreading_and_bounds_merge():
    order, n = 3, (12, 10)
    luh = IC.explosion(order, n, center=(0.06, 0.5), radius=0.2)
    per = O.LimitingGrid(order, n, luh)
    wall = O.LimitingGrid(order, n, luh, bc=[1, 0])
    per.step()
    wall.step()
    sp, sw = per.status.reshape(n[1], n[0]), wall.status.reshape(n[1], n[0])
    # periodic: the trouble at x = 0 reaches the last column; a wall stops it
    assert sp[:, -1].max() > 0 and sw[:, -1].max() == 0
    # spreading within the domain: no status drops by more than one per face
    assert (sw[:, 1:] >= sw[:, :-1] - 1).all() and (sw[:, :-1] >= sw[:, 1:] - 1).all()
    assert (sw >= np.roll(sw, 1, axis=0) - 1).all() and (sw >= np.roll(sw, -1, axis=0) - 1).all()
    # bounds: face f holds min / max of the cell's own extrema and its
    # neighbour's across f, so the own extrema bound every face; a wall face
    # holds exactly the own extrema
    mn = wall.bmin.reshape(n[1], n[0], 4, 5)
    mx = wall.bmax.reshape(n[1], n[0], 4, 5)
    assert np.array_equal(mn[:, 0, 0], mn[:, 0].max(axis=1))
    assert np.array_equal(mx[:, 0, 0], mx[:, 0].min(axis=1))
    assert np.array_equal(mn[:, -1, 1], mn[:, -1].max(axis=1))
    assert np.array_equal(mx[:, -1, 1], mx[:, -1].min(axis=1))


def test_outflow_and_reflect_differ():
    order, n = 2, (10, 10)
    luh = IC.explosion(order, n, center=(0.1, 0.5), radius=0.2)
    a = O.LimitingGrid(order, n, luh, bc=[1, 1])
    b = O.LimitingGrid(order, n, luh, bc=[2, 2])
    for _ in range(4):
        a.step()
        b.step()
    assert np.abs(a.luh - b.luh).max() > 1e-6


def test_explosion_in_a_box_3d():
    order, n = 2, (8, 8, 8)
    luh = IC.explosion3d(order, n, center=(0.1, 0.5, 0.9), radius=0.25)
    g = O.LimitingGrid(order, n, luh, bc=[2, 1, 2])
    for _ in range(4):
        g.step()
        st = g.status.reshape(n[2], n[1], n[0])
        assert g.counts[2] > 0 and g.counts[2] == (st == 5).sum()
        for ax in (0, 1, 2):
            a, b = np.moveaxis(st, ax, 0)[1:], np.moveaxis(st, ax, 0)[:-1]
            assert (a >= b - 1).all() and (b >= a - 1).all()
    assert np.isfinite(g.luh).all() and g.luh.reshape(-1, 5)[:, 0].min() > 0.0
