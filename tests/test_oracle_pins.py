"""The oracle's restatements that no golden vector covers, pinned to the
reference's own kernels compiled unchanged from source (oracle/_ref):

* the uniform-grid step in the reference's non-fused order (dt ->
  spaceTimePredictor + volumeIntegral -> riemannSolver per face -> surface
  integral + solutionUpdate; exahype/runners/Runner.cpp:1125-1160,
  ADERDGSolver.cpp:2744-2826), 2D and 3D, orders 2-5, several steps;
* the same step with domain-boundary faces through the reference's
  boundaryConditions kernel (c/{2d,3d}/boundaryConditions.cpph) and
  ADERDGSolver::applyBoundaryConditions' Riemann convention
  (ADERDGSolver.cpp:2854-2925);
* stableTimeStepSize (c/{2d,3d}/stableTimeStepSize.cpph:21-61);
* the 2D finite-volume kernels godunov (godunov/c/2d/godunov.cpph:33-120),
  musclhancock (musclhancock/c/2d/musclhancock.cpph:50-240) and the FV
  stableTimeStepSize (commons/c/commons.cpph:26-67), whole patch with ghost
  layers and the admissible dt, patches 4..256;
* the reference's Rusanov unit test (exahype/tests/kernels/finitevolumes/
  riemannsolvers/c/RusanovTest.cpp:71-90): zero flux, unit eigenvalues,
  qL = 0.8, qR = 0.2 -> fL = fR = 0.3.
"""
import ctypes as C

import numpy as np
import pytest

import _oracle as O

V = 5


def _ref(dim):
    R = O.ref_lib(dim)
    if R is None or not hasattr(R, 'ref_grid_step_bc'):
        pytest.skip('reference kernels not built (make -C oracle ref REF=<reference tree>)')
    return R


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def _perturbed(dim, order, n, seed, kind=0, amp=5.0, noise=1e-3):
    return O.grid_ic(dim, order, n, kind=kind, param=amp, seed=seed, noise=noise)


# ------------------------------------------------------------ ADER-DG grid
GRIDS = {2: (5, 4), 3: (3, 2, 2)}


@pytest.mark.parametrize('dim', [2, 3])
@pytest.mark.parametrize('order', [2, 3, 4, 5])
def test_grid_step_vs_reference(dim, order):
    """orc_aderdg_grid_step (the oracle every grid test uses) equals the
    reference's kernels driven in the reference's step order, step by step:
    dt exactly up to the last bits, the state within 1e-13 relative."""
    _ref(dim)
    n = GRIDS[dim]
    u = _perturbed(dim, order, n, seed=100 + order)
    mine, ref = u.copy(), u.copy()
    for step in range(3):
        dt_m, _ = O.grid_step(dim, order, n, mine, dt_policy=0, planar=1 if dim == 2 else 0)
        dt_r = O.ref_grid_step(dim, order, n, ref, dt_policy=0)
        assert abs(dt_m - dt_r) <= 1e-15 * dt_r, (step, dt_m, dt_r)
        e = _rel(mine, ref)
        assert e <= 1e-13, (step, e)


@pytest.mark.parametrize('dim', [2, 3])
def test_grid_step_fixed_dt_sine_vs_reference(dim):
    """The benchmark's 2D sine-wave configuration (fixed dt policy) on
    both: the 27x27 N=3 case for 10 steps in 2D, a 3x3x3 N=4 case in 3D."""
    _ref(dim)
    order = 3 if dim == 2 else 4
    n = (27, 27) if dim == 2 else (3, 3, 3)
    u = O.grid_ic(dim, order, n, kind=1, param=0.2, seed=1)
    mine, ref = u.copy(), u.copy()
    dt = 0.9 / (2 * order + 1) / 2.0 / n[0] * 0.5
    for _ in range(10 if dim == 2 else 3):
        O.grid_step(dim, order, n, mine, dt_policy=2, dt_fixed=dt, planar=1 if dim == 2 else 0)
        O.ref_grid_step(dim, order, n, ref, dt_policy=2, dt_fixed=dt)
    assert _rel(mine, ref) <= 1e-13


@pytest.mark.parametrize('dim', [2, 3])
@pytest.mark.parametrize('bc', [(1, 1, 1), (2, 2, 2), (1, 2, 0), (0, 2, 1)])
@pytest.mark.parametrize('order', [2, 4])
def test_grid_step_boundary_vs_reference(dim, bc, order):
    """orc_aderdg_grid_step_bc's outflow / reflecting-wall faces equal the
    reference's boundaryConditions kernel + applyBoundaryConditions' Riemann
    solve, with the Euler boundaryValues hook of the same rule."""
    _ref(dim)
    n = GRIDS[dim]
    bc = bc[:dim]
    u = _perturbed(dim, order, n, seed=7 + order, kind=0, amp=5.0, noise=1e-2)
    mine, ref = u.copy(), u.copy()
    for step in range(3):
        dt_m, _ = O.grid_step(dim, order, n, mine, dt_policy=0, planar=1 if dim == 2 else 0, bc=bc)
        dt_r = O.ref_grid_step(dim, order, n, ref, dt_policy=0, bc=bc)
        assert abs(dt_m - dt_r) <= 1e-15 * dt_r, (step, dt_m, dt_r)
        assert _rel(mine, ref) <= 1e-13, (step, _rel(mine, ref))
    # the boundary changed the result: the same state stepped periodically differs
    per = u.copy()
    for _ in range(3):
        O.grid_step(dim, order, n, per, dt_policy=0, planar=1 if dim == 2 else 0)
    assert _rel(per, ref) > 1e-6


def test_boundary_rule_mistake_is_caught():
    """A planted mistake in the oracle's wall rule (outflow where the
    reference reflects) is visible at the pin's tolerance."""
    _ref(3)
    n = GRIDS[3]
    u = _perturbed(3, 3, n, seed=3, noise=1e-2)
    mine, ref = u.copy(), u.copy()
    O.grid_step(3, 3, n, mine, dt_policy=0, bc=(1, 1, 1))
    O.ref_grid_step(3, 3, n, ref, dt_policy=0, bc=(2, 2, 2))
    assert _rel(mine, ref) > 1e-8


# -------------------------------------------------------- stable time step
@pytest.mark.parametrize('dim', [2, 3])
@pytest.mark.parametrize('order', [1, 2, 3, 4, 5, 6, 7])
def test_stable_dt_vs_reference(dim, order):
    """orc_stable_dt (CFL 0.9 x PNPM[N] / sum_d max|lambda_d| / dx_d, min
    over nodes) equals the reference's stableTimeStepSize on random cells."""
    R = _ref(dim)
    rng = np.random.default_rng(order * 10 + dim)
    B = order + 1
    nn = B ** dim
    dx = np.array([0.3, 0.2, 0.15][:dim])
    for trial in range(20):
        q = np.zeros((nn, V))
        q[:, 0] = 0.5 + rng.random(nn)
        q[:, 1:1 + dim] = rng.standard_normal((nn, dim))
        q[:, 4] = 2.0 + rng.random(nn) + 0.5 * (q[:, 1:4] ** 2).sum(-1) / q[:, 0]
        q = q.ravel()
        r = R.ref_stable_dt(order, 0, q, dx)
        m = O.lib().orc_stable_dt(dim, order, V, 0, 1 if dim == 2 else 0, q, dx, 0.9)
        assert abs(m - r) <= 1e-15 * r, (trial, m, r)


# ----------------------------------------------------- 2D finite volumes
def _fv_patch(P, g, seed):
    rng = np.random.default_rng(seed)
    S = P + 2 * g
    q = np.zeros((S, S, V))
    q[..., 0] = 1.0 + 0.2 * rng.random((S, S))
    q[..., 1:3] = 0.3 * rng.standard_normal((S, S, 2))
    q[..., 4] = 2.5 + 0.5 * rng.random((S, S)) + 0.5 * (q[..., 1:3] ** 2).sum(-1) / q[..., 0]
    return q.ravel()


@pytest.mark.parametrize('scheme', [0, 1])
@pytest.mark.parametrize('P', [4, 5, 8, 16, 32, 64, 256])
def test_fv2d_vs_reference(scheme, P):
    """orc_fv_godunov_2d / orc_fv_musclhancock_2d / orc_fv_stable_dt_2d (the
    oracle of the EulerFV and serving paths) equal the reference's 2D
    kernels on a perturbed periodic patch: the whole patch after one step,
    ghost layers included (both kernels write the boundary-face
    contributions into the first ghost layer; MUSCL-Hancock leaves the
    ghost cells next to the patch un-evolved), the admissible dt and the
    stable dt.  The 256^2 MUSCL-Hancock case runs the reference on a thread
    with a 1 GiB stack (its work arrays live on the stack)."""
    R = _ref(2)
    g = 1 if scheme == 0 else 2
    dx = np.array([0.3, 0.25])
    u = _fv_patch(P, g, 10 * P + scheme)
    O.lib().orc_fv_periodic_ghosts_2d(P, g, V, u)
    ref = u.copy()
    adm = C.c_double()
    dt = R.ref_fv_step(scheme, P, ref, dx, 0.0, C.byref(adm))
    assert dt > 0, 'patch size not instantiated in the reference harness'
    dt_mine = O.lib().orc_fv_stable_dt_2d(P, g, V, 0, 1, u, dx, 0.9)
    assert abs(dt_mine - dt) <= 1e-15 * dt
    mine = u.copy()
    f = O.lib().orc_fv_godunov_2d if scheme == 0 else O.lib().orc_fv_musclhancock_2d
    adm_mine = f(P, g, V, 0, 1, mine, u.copy(), dx, dt)
    assert abs(adm_mine - adm.value) <= 1e-15 * adm.value
    assert np.abs(mine - ref).max() <= 1e-14 * np.abs(ref).max()


def test_fv2d_muscl_ghost_quirk_is_the_reference_behaviour():
    """The MUSCL-Hancock ghost quirk (cells next to the patch are not
    half-step evolved, musclhancock.cpph:132-185) is what the reference
    computes: the oracle, which reproduces it, matches the reference on the
    whole patch, including the first ghost layer that both kernels write."""
    R = _ref(2)
    P, g = 8, 2
    dx = np.array([0.3, 0.25])
    u = _fv_patch(P, g, 5)
    O.lib().orc_fv_periodic_ghosts_2d(P, g, V, u)
    ref = u.copy()
    adm = C.c_double()
    dt = R.ref_fv_step(1, P, ref, dx, 0.0, C.byref(adm))
    mine = u.copy()
    O.lib().orc_fv_musclhancock_2d(P, g, V, 0, 1, mine, u.copy(), dx, dt)
    S = P + 2 * g
    a, b = mine.reshape(S, S, V), ref.reshape(S, S, V)
    # interior and ghost ring written by the kernels agree bit for bit scale
    assert np.abs(a - b).max() <= 1e-14 * np.abs(b).max()
    # the first ghost layer was written (differs from the periodic copy)
    assert np.abs(b[1, g:g + P] - u.reshape(S, S, V)[1, g:g + P]).max() > 0


# ------------------------------------------------------------- Rusanov KAT
_FLUX = C.CFUNCTYPE(None, C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double))
_EIG = C.CFUNCTYPE(None, C.c_void_p, C.POINTER(C.c_double), C.c_int, C.POINTER(C.c_double))


def test_rusanov_kat_zero_flux_mock():
    """RusanovTest.cpp:71-90 on the oracle's Rusanov (the formula orc_rusanov
    and every FV oracle kernel use) and on the reference's rusanov: the
    ZeroFluxZeroNCP mock (4 variables, 3 parameters, no flux, eigenvalues
    1), qL = 0.8, qR = 0.2 -> fL = fR = 0.3 in every variable, s_max 1."""
    nvar = 4

    @_FLUX
    def flux(ctx, q, F):
        pass

    @_EIG
    def eig(ctx, q, d, lam):
        for i in range(nvar):
            lam[i] = 1.0

    qL = np.full(7, 0.8)
    qR = np.full(7, 0.2)
    for d in range(3):
        fL, fR = np.zeros(nvar), np.zeros(nvar)
        s = O.lib().orc_rusanov_pde(3, nvar, C.cast(flux, C.c_void_p), C.cast(eig, C.c_void_p), None,
                                    fL, fR, qL, qR, d)
        assert s == 1.0
        np.testing.assert_allclose(fL, 0.3, rtol=0, atol=1e-15)
        np.testing.assert_allclose(fR, 0.3, rtol=0, atol=1e-15)
    for dim in (2, 3):
        R = O.ref_lib(dim)
        if R is None or not hasattr(R, 'ref_rusanov_mock'):
            pytest.skip('reference kernels not built')
        fL, fR = np.zeros(nvar), np.zeros(nvar)
        s = R.ref_rusanov_mock(fL, fR, qL, qR, 0)
        assert s == 1.0
        np.testing.assert_allclose(fL, 0.3, rtol=0, atol=1e-15)
        np.testing.assert_allclose(fR, 0.3, rtol=0, atol=1e-15)


def test_rusanov_euler_vs_reference_fv_step_faces():
    """orc_rusanov with the Euler callbacks is the function the FV pins
    above exercise; a direct check against the golden-free formula on
    random states (2D planar and 3D) keeps the refactored callback path
    honest: fL = fR, s_max = max |u_n| + c over both sides."""
    rng = np.random.default_rng(3)
    for dim, planar in ((2, 1), (3, 0)):
        for _ in range(50):
            q = []
            for _s in range(2):
                rho = 0.5 + rng.random()
                u = rng.standard_normal(3) * (np.array([1, 1, 0]) if planar else 1)
                p = 0.5 + rng.random()
                ke = 0.5 * rho * (u[:2] ** 2).sum() if planar else 0.5 * rho * (u ** 2).sum()
                q.append(np.array([rho, *(rho * u), p / 0.4 + ke]))
            fL, fR = np.zeros(V), np.zeros(V)
            d = int(rng.integers(dim))
            s = O.lib().orc_rusanov(dim, V, 0, planar, fL, fR, q[0], q[1], d)
            cs = [np.sqrt(1.4 * 0.4 * (qq[4] - (0.5 * (qq[1] ** 2 + qq[2] ** 2) if planar else
                                                 0.5 * (qq[1:4] ** 2).sum()) / qq[0]) / qq[0]) for qq in q]
            smax = max(abs(qq[d + 1] / qq[0]) + c for qq, c in zip(q, cs))
            assert abs(s - smax) <= 1e-14 * smax
            np.testing.assert_array_equal(fL, fR)
