"""3D finite volumes of the oracle (orc_fv_godunov_3d, orc_fv_musclhancock_3d,
orc_fv_stable_dt_3d) against the reference's own 3D godunov / musclhancock /
commons kernels compiled from source (oracle/_ref), on perturbed periodic
patches: the whole patch array after one step, ghost layers included (both
write the boundary-face contributions into the first ghost layer), the
admissible dt and the stable dt."""
import ctypes as C

import numpy as np
import pytest

import _oracle as O

V = 5


def patch_state(P, g, seed):
    rng = np.random.default_rng(seed)
    S = P + 2 * g
    q = np.zeros((S, S, S, V))
    q[..., 0] = 1.0 + 0.2 * rng.random((S, S, S))
    q[..., 1:4] = 0.3 * rng.standard_normal((S, S, S, 3))
    q[..., 4] = 2.5 + 0.5 * rng.random((S, S, S)) + 0.5 * (q[..., 1:4] ** 2).sum(-1) / q[..., 0]
    return q.ravel()


@pytest.mark.parametrize('scheme', [0, 1])
@pytest.mark.parametrize('P', [4, 5, 7, 9])
def test_fv3d_oracle_vs_reference(scheme, P):
    R = O.ref_lib(3)
    if R is None or not hasattr(R, 'ref_fv_step'):
        pytest.skip('reference kernels not built (make -C oracle ref)')
    g = 1 if scheme == 0 else 2
    dx = np.array([0.3, 0.25, 0.2])
    u = patch_state(P, g, 10 * P + scheme)
    O.lib().orc_fv_periodic_ghosts_3d(P, g, V, u)
    ref = u.copy()
    adm = C.c_double()
    dt = R.ref_fv_step(scheme, P, ref, dx, 0.0, C.byref(adm))
    dt_mine = O.lib().orc_fv_stable_dt_3d(P, g, V, 0, u, dx, 0.9)
    assert abs(dt_mine - dt) <= 1e-15 * dt
    mine = u.copy()
    f = O.lib().orc_fv_godunov_3d if scheme == 0 else O.lib().orc_fv_musclhancock_3d
    adm_mine = f(P, g, V, 0, mine, u.copy(), dx, dt)
    assert abs(adm_mine - adm.value) <= 1e-15 * adm.value
    assert np.abs(mine - ref).max() <= 1e-14 * np.abs(ref).max()
