"""The oracle's limiting ADER-DG step (orc_limiting_grid_step, a
restatement of LimitingADERDGSolver on a uniform periodic grid) on its own:
it leaves a smooth state to the unlimited DG scheme, and on an explosion it
marks the cells along the discontinuity, spreads their status by face hops
and keeps the state admissible where the unlimited scheme undershoots."""
import numpy as np

import _limiting_ic as IC
import _oracle as O


def pressure(luh):
    q = luh.reshape(-1, 5)
    return 0.4 * (q[:, 4] - 0.5 * (q[:, 1] ** 2 + q[:, 2] ** 2 + q[:, 3] ** 2) / q[:, 0])


def test_smooth_state_is_not_limited():
    order, n = 3, (12, 10)
    luh = IC.smooth(order, n, amp=0.05)
    g = O.LimitingGrid(order, n, luh)
    plain = luh.copy()
    nn = np.asarray(n, dtype=np.int32)
    for _ in range(5):
        dt = g.step()
        O.lib().orc_aderdg_grid_step(2, order, 0, nn, g.dx, plain, 2, 0.9, dt, None, 0)
        assert g.counts.tolist() == [0, 0, 0]
    assert np.array_equal(g.luh, plain)


def test_explosion_limiting():
    order, n = 3, (16, 16)
    g = O.LimitingGrid(order, n, IC.explosion(order, n))
    plain = IC.explosion(order, n)
    nn = np.asarray(n, dtype=np.int32)
    for _ in range(8):
        dt = g.step()
        O.lib().orc_aderdg_grid_step(2, order, 0, nn, g.dx, plain, 2, 0.9, dt, None, 0)
        st = g.status.reshape(n[1], n[0])
        assert g.counts[2] > 0 and g.counts[2] == (st == 5).sum()
        assert g.counts[1] == (st >= 3).sum() and g.counts[0] == (st >= 2).sum()
        # status never drops by more than one across a face (four-hop spreading)
        for ax in (0, 1):
            for sh in (1, -1):
                assert (st >= np.roll(st, sh, axis=ax) - 1).all()
        # troubled cells sit on the discontinuity (circle of radius 0.25)
        cy, cx = np.nonzero(st == 5)
        r = np.hypot((cx + 0.5) / n[0] - 0.5, (cy + 0.5) / n[1] - 0.5)
        assert (np.abs(r - 0.25) < 0.2).all()
    q = g.luh.reshape(-1, 5)
    assert q[:, 0].min() > 0.08 and pressure(g.luh).min() > 0.05
    # the unlimited scheme with the same steps breaks down or undershoots
    pq = plain.reshape(-1, 5)
    assert not np.isfinite(plain).all() or (pq[:, 0].min() < q[:, 0].min()
                                           and pressure(plain).min() < pressure(g.luh).min())


def test_explosion_limiting_3d():
    order, n = 2, (8, 8, 8)
    g = O.LimitingGrid(order, n, IC.explosion3d(order, n))
    for _ in range(4):
        g.step()
        st = g.status.reshape(n[2], n[1], n[0])
        assert g.counts[2] > 0 and g.counts[2] == (st == 5).sum()
        assert g.counts[1] == (st >= 3).sum() and g.counts[0] == (st >= 2).sum()
        for ax in (0, 1, 2):
            for sh in (1, -1):
                assert (st >= np.roll(st, sh, axis=ax) - 1).all()
    q = g.luh.reshape(-1, 5)
    assert np.isfinite(q).all() and q[:, 0].min() > 0.0 and pressure(g.luh).min() > 0.0


def test_3d_muscl_step_amplifies_rounding():
    """The oracle alone: relative perturbations of 1e-15 in the state of a
    3D MUSCL-Hancock limited explosion grow to ~1e-11 in one step (the GPU
    parity test for that case uses 1e-9 for this reason)."""
    order, n = 3, (6, 7, 5)
    o = O.LimitingGrid(order, n, IC.explosion3d(order, n), scheme=1)
    o.step()
    keep = (o.luh.copy(), o.status.copy(), o.cure.copy(), o.bmin.copy(), o.bmax.copy(), o.dt)
    o.step()
    rng = np.random.default_rng(0)
    t = O.LimitingGrid(order, n, keep[0] * (1 + 1e-15 * rng.standard_normal(keep[0].size)), scheme=1)
    t.status[:], t.cure[:], t.bmin[:], t.bmax[:] = keep[1], keep[2], keep[3], keep[4]
    t.dt = keep[5]
    t.step()
    assert np.array_equal(t.status, o.status)
    diff = np.abs(t.luh - o.luh).max() / np.abs(o.luh).max()
    assert 1e-13 < diff < 1e-9
