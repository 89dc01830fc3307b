"""Parity of the CUDA path with the CPU oracle on seeded inputs.

Tolerance: relative L2 <= 1e-12 per array (the north-star bar for the plain
FP64 path), Picard iteration counts identical."""
import numpy as np
import pytest

import _oracle as O
import exahype_b200 as E
from exahype_b200 import DeviceBuffer

pytestmark = pytest.mark.gpu
TOL = 1e-12
V = 5


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def random_cells(rng, ncells, nn, amp=0.3):
    q = np.zeros((ncells, nn, V))
    q[..., 0] = 1.0 + 0.2 * rng.random((ncells, nn))
    q[..., 1:4] = amp * rng.standard_normal((ncells, nn, 3))
    q[..., 4] = 2.5 + 0.3 * rng.random((ncells, nn))
    return q


@pytest.mark.parametrize('dim,order,planar', [(3, 2, 0), (3, 3, 0), (3, 4, 0), (3, 5, 0),
                                              (2, 2, 1), (2, 3, 0), (2, 3, 1), (2, 4, 1), (2, 5, 0)])
def test_predictor_batched_vs_oracle(dim, order, planar):
    rng = np.random.default_rng(100 + 10 * dim + order)
    B = order + 1
    nn = B ** dim
    ncells = 37
    q = random_cells(rng, ncells, nn)
    if planar:
        q[..., 3] = 0.3 * rng.standard_normal((ncells, nn))  # planar pressure ignores it
    dx = [0.05, 0.04, 0.03][:dim]
    dt = 2e-4
    K = E.BatchedADERDG(dim, order, dx, pde=E.PDE_EULER_PLANAR if planar else E.PDE_EULER)
    s = O.sizes(dim, order)
    bufs = {k: DeviceBuffer(ncells * s[k]) for k in ('lQi', 'lFi', 'lQhi', 'lFhi', 'lduh', 'qbnd', 'fbnd')}
    luh = DeviceBuffer.from_array(q.ravel())
    it = DeviceBuffer(ncells, np.int32)
    K.predictor_full(ncells, luh, dt, bufs['lQi'], bufs['lFi'], bufs['lQhi'], bufs['lFhi'], bufs['lduh'],
                     bufs['qbnd'], bufs['fbnd'], iters=it)
    got = {k: b.download().reshape(ncells, -1) for k, b in bufs.items()}
    its = it.download()
    for c in range(ncells):
        r = O.stp(dim, order, q[c].ravel(), dx, dt, planar=planar)
        lduh = np.zeros(s['lduh'])
        O.lib().orc_volume_integral(dim, order, V, 1, lduh, r['lFhi'], np.array(dx))
        assert its[c] == r['iters'], (c, its[c], r['iters'])
        for k, ref in (('lQi', r['lQi']), ('lQhi', r['lQhi']), ('lFhi', r['lFhi']), ('lduh', lduh),
                       ('qbnd', r['lQhbnd']), ('fbnd', r['lFhbnd'])):
            assert rel(got[k][c], ref) < TOL, (k, c, rel(got[k][c], ref))
        # lFi: the last iteration's fluxes
        assert rel(got['lFi'][c], r['lFi']) < TOL


def test_predictor_vi_matches_full():
    """The production (fused) predictor writes the same lduh/faces as the
    reference-temporaries variant (to rounding: for 3D order 4 the production
    path uses the line-owner contraction, which sums in another order), and
    its stats count the iterations."""
    rng = np.random.default_rng(7)
    dim, order, ncells = 3, 4, 150
    B = order + 1
    q = random_cells(rng, ncells, B ** dim)
    dx = [0.02] * 3
    s = O.sizes(dim, order)
    K = E.BatchedADERDG(dim, order, dx)
    luh = DeviceBuffer.from_array(q.ravel())
    a = {k: DeviceBuffer(ncells * s[k]) for k in ('lQi', 'lFi', 'lQhi', 'lFhi', 'lduh', 'qbnd', 'fbnd')}
    b = {k: DeviceBuffer(ncells * s[k]) for k in ('lduh', 'qbnd', 'fbnd')}
    it = DeviceBuffer(ncells, np.int32)
    stats = DeviceBuffer(2, np.uint64)
    stats.zero()
    K.predictor_full(ncells, luh, 1e-4, a['lQi'], a['lFi'], a['lQhi'], a['lFhi'], a['lduh'], a['qbnd'],
                     a['fbnd'])
    K.predictor_vi(ncells, luh, 1e-4, b['lduh'], b['qbnd'], b['fbnd'], iters=it, stats=stats)
    for k in ('lduh', 'qbnd', 'fbnd'):
        assert rel(b[k].download(), a[k].download()) < 1e-13, k
    st = stats.download()
    assert int(st[0]) == int(it.download().astype(np.int64).sum())


def test_cell_local_ops_vs_oracle():
    """Batched surface integral, solution update, stable dt and the face-list
    Riemann solver against the oracle."""
    rng = np.random.default_rng(11)
    for dim, order in ((3, 4), (2, 3), (3, 2)):
        B = order + 1
        nn, nf = B ** dim, B ** (dim - 1)
        ncells = 9
        dx = [0.1, 0.07, 0.05][:dim]
        K = E.BatchedADERDG(dim, order, dx)
        q = random_cells(rng, ncells, nn)
        lduh = rng.standard_normal((ncells, nn * V))
        fb = rng.standard_normal((ncells, 2 * dim * nf * V))
        qb = random_cells(rng, ncells, 2 * dim * nf).reshape(ncells, -1)
        # surface integral
        d_lduh = DeviceBuffer.from_array(lduh)
        d_fb = DeviceBuffer.from_array(fb)
        K.surface_integral(ncells, d_lduh, d_fb)
        got = d_lduh.download().reshape(ncells, -1)
        for c in range(ncells):
            ref = lduh[c].copy()
            O.lib().orc_surface_integral(dim, order, V, ref, fb[c].copy(), np.array(dx))
            assert rel(got[c], ref) < TOL
        # update
        d_luh = DeviceBuffer.from_array(q.ravel())
        d_lduh = DeviceBuffer.from_array(lduh)
        K.solution_update(ncells, d_luh, d_lduh, 3e-3)
        got = d_luh.download().reshape(ncells, -1)
        for c in range(ncells):
            ref = q[c].ravel().copy()
            O.lib().orc_solution_update(dim, order, V, 0, ref, lduh[c].copy(), 3e-3)
            assert rel(got[c], ref) < 1e-15
        # stable dt
        d_luh = DeviceBuffer.from_array(q.ravel())
        dtc = DeviceBuffer(ncells)
        dtm = DeviceBuffer(1)
        K.stable_dt(ncells, d_luh, dtc, dtm)
        dts = dtc.download()
        for c in range(ncells):
            ref = O.lib().orc_stable_dt(dim, order, V, 0, 0, q[c].ravel().copy(), np.array(dx), 0.9)
            assert abs(dts[c] - ref) <= 1e-15 * ref
        assert dtm.download()[0] == dts.min()
        # face list: cell c's +d face against cell (c+1)%n's -d face
        left = np.arange(ncells, dtype=np.int32)
        right = ((left + 1) % ncells).astype(np.int32)
        dirs = (left % dim).astype(np.int32)
        d_qb, d_fb = DeviceBuffer.from_array(qb.ravel()), DeviceBuffer.from_array(fb.ravel())
        K.riemann_faces(ncells, DeviceBuffer.from_array(left), DeviceBuffer.from_array(right),
                        DeviceBuffer.from_array(dirs), d_qb, d_fb)
        got = d_fb.download().reshape(ncells, 2 * dim, nf * V)
        ref_fb = fb.reshape(ncells, 2 * dim, nf * V).copy()
        refq = qb.reshape(ncells, 2 * dim, nf * V)
        for k in range(ncells):  # sequential in face order, as the faces are disjoint
            l, r, d = left[k], right[k], dirs[k]
            FL, FR = ref_fb[l, 2 * d + 1].copy(), ref_fb[r, 2 * d].copy()
            O.lib().orc_riemann(dim, order, V, 0, 0, FL, FR, refq[l, 2 * d + 1].copy(), refq[r, 2 * d].copy(), d)
            ref_fb[l, 2 * d + 1], ref_fb[r, 2 * d] = FL, FR
        assert rel(got, ref_fb) < TOL


def test_grid_ic_matches_oracle():
    for dim, order, n, kind in ((3, 4, (3, 4, 2), 0), (2, 3, (7, 5), 1)):
        g = E.ADERDGGrid(dim, order, n)
        g.init(kind=kind, param=5.0 if kind == 0 else 0.2, seed=99, noise=1e-3)
        ref = O.grid_ic(dim, order, n, kind=kind, param=5.0 if kind == 0 else 0.2, seed=99, noise=1e-3)
        assert rel(g.get_state(), ref) < 1e-14
        g.destroy()


@pytest.mark.parametrize('dim,order,n,kind,planar,policy,steps', [
    (3, 4, (4, 5, 3), 0, 0, 0, 6),
    (3, 3, (3, 3, 4), 0, 0, 1, 4),
    (3, 2, (5, 3, 3), 1, 0, 0, 4),
    (3, 5, (2, 3, 2), 0, 0, 0, 3),
    (2, 3, (27, 27), 1, 0, 1, 100),   # the 27x27 N=3 sine-wave configuration
    (2, 3, (9, 11), 1, 1, 0, 20),
    (2, 2, (12, 7), 0, 0, 0, 10),
    (2, 4, (6, 9), 0, 1, 1, 10),
    (2, 5, (5, 5), 1, 0, 0, 10),
])
@pytest.mark.parametrize('variant', [1, 2, 3])
def test_grid_steps_vs_oracle(dim, order, n, kind, planar, policy, steps, variant):
    """Every step is compared with the oracle stepping the identical input
    state (per-step parity, relative L2 <= 1e-12); a second oracle copy runs
    free for all steps to bound the accumulated drift.  variant (tuning key
    3): FP64 predictor contraction, 1 = node-gather, 2 = line-owner, 3 = the
    progressive line-owner form (3D order 4; line-owner elsewhere)."""
    E._lib.call('exa_tune_set', 3, variant)
    try:
        _grid_steps_vs_oracle(dim, order, n, kind, planar, policy, steps)
    finally:
        E._lib.call('exa_tune_set', 3, 0)


def _grid_steps_vs_oracle(dim, order, n, kind, planar, policy, steps):
    pde = E.PDE_EULER_PLANAR if planar else E.PDE_EULER
    g = E.ADERDGGrid(dim, order, n, pde=pde, dt_policy=policy)
    param = 5.0 if kind == 0 else 0.2
    g.init(kind=kind, param=param, seed=5, noise=1e-3)
    u = g.get_state()
    free = u.copy()
    worst = 0.0
    for s in range(steps):
        dt_gpu = g.step(1, want_dt=True)[0]
        dt_ref, _ = O.grid_step(dim, order, n, u, dt_policy=policy, planar=planar)
        assert abs(dt_gpu - dt_ref) <= 1e-13 * dt_ref, (s, dt_gpu, dt_ref)
        got = g.get_state()
        err = rel(got, u)
        assert err < TOL, (s, err)
        worst = max(worst, err)
        O.grid_step(dim, order, n, free, dt_policy=policy, planar=planar)
        u = got.copy()  # next step: both from the GPU state
    drift = rel(g.get_state(), free)
    assert drift < 1e-10, drift
    st = g.status()
    assert not st['nan'] and st['picard_iters'] > 0
    g.destroy()


def test_grid_graph_replay_is_bitwise_identical():
    a = E.ADERDGGrid(3, 4, (4, 4, 4))
    b = E.ADERDGGrid(3, 4, (4, 4, 4))
    for g in (a, b):
        g.init(kind=0, param=5.0, seed=3, noise=1e-3)
    b.use_graph(True)
    da = a.step(5, want_dt=True)
    db = b.step(5, want_dt=True)
    assert np.array_equal(da, db)
    assert np.array_equal(a.get_state(), b.get_state())
    assert a.status()['time'] == b.status()['time']


@pytest.mark.parametrize('dim,order,n,bc,steps', [
    (2, 3, (9, 7), (1, 1), 8),
    (2, 4, (6, 8), (2, 1), 6),
    (2, 2, (10, 5), (2, 2), 8),
    (3, 4, (4, 3, 5), (1, 2, 1), 4),
    (3, 3, (3, 4, 3), (2, 2, 2), 4),
])
def test_grid_boundary_conditions_vs_oracle(dim, order, n, bc, steps):
    """Outflow / reflecting-wall boundaries (exa_aderdg_grid_set_boundary)
    against the oracle's boundary rules, per step from the identical state."""
    g = E.ADERDGGrid(dim, order, n)
    g.set_boundary(bc)
    g.init(kind=0, param=5.0, seed=8, noise=1e-3)
    u = g.get_state()
    for s in range(steps):
        dt_gpu = g.step(1, want_dt=True)[0]
        dt_ref, _ = O.grid_step(dim, order, n, u, bc=bc)
        assert abs(dt_gpu - dt_ref) <= 1e-13 * dt_ref, (s, dt_gpu, dt_ref)
        got = g.get_state()
        assert rel(got, u) < TOL, (s, rel(got, u))
        u = got.copy()
    g.destroy()


def test_grid_boundary_rejects_bad_rule():
    g = E.ADERDGGrid(2, 3, (4, 4))
    with pytest.raises(E.ExaError):
        g.set_boundary((0, 7))
    g.set_halo(True)
    with pytest.raises(E.ExaError):
        g.set_boundary((1, 1))  # slab halos need a periodic last dimension
    g.destroy()


@pytest.mark.parametrize('dim,pde', [(3, E.PDE_EULER), (2, E.PDE_EULER), (2, E.PDE_EULER_PLANAR)])
def test_progressive_fp64_equals_line_owner_bitwise(dim, pde):
    """The progressive FP64 predictor performs the line-owner kernel's
    operations in the same order: the same grid, stepped with either, is
    identical bit for bit (order 4; 3D one cell per CTA, 2D four cells per
    CTA with a partial last block; also with a dt four times the stable
    one, where cells stop at the iteration cap)."""
    planar = int(pde == E.PDE_EULER_PLANAR)
    n1 = (5, 4, 3) if dim == 3 else (7, 5)
    n2 = (3,) * dim
    out = []
    for variant in (2, 3):
        E._lib.call('exa_tune_set', 3, variant)
        try:
            g = E.ADERDGGrid(dim, 4, n1, pde=pde)
            g.init(kind=0, param=5.0, seed=21, noise=1e-3)
            g.step(4)
            u0 = O.grid_ic(dim, 4, n2, kind=0, param=5.0, seed=22, noise=1e-3)
            nn = np.full(dim, 3, dtype=np.int32)
            dt4 = 4.0 * O.lib().orc_aderdg_grid_dt(dim, 4, planar, nn, np.full(dim, 1.0 / 3), u0, 0, 0.9)
            h = E.ADERDGGrid(dim, 4, n2, pde=pde, dt_policy=2, dt_fixed=dt4)
            h.set_state(u0)
            h.step(1)
            out.append((g.get_state(), h.get_state(), g.status()['picard_iters'], h.status()['nonconverged']))
            g.destroy()
            h.destroy()
        finally:
            E._lib.call('exa_tune_set', 3, 0)
    a, b = out
    assert np.isfinite(a[1]).all()
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    assert a[2] == b[2] and a[3] == b[3]
