"""3D finite volumes on the GPU (exa_fv_*_update / exa_fv_stable_dt /
exa_fv_periodic_ghosts with dim = 3) against the oracle, which
tests/test_oracle_fv3d.py pins to the reference's compiled 3D kernels: the
whole luh_new of every patch (first ghost layer included), the admissible
dt per patch and the stable dt per patch, FP64 within 1e-13."""
import numpy as np
import pytest

import _oracle as O
from exahype_b200 import DeviceBuffer
from exahype_b200.fv import FVPatches

pytestmark = pytest.mark.gpu
V = 5


def patches(P, g, n, seed, D=V):
    rng = np.random.default_rng(seed)
    S = P + 2 * g
    q = np.zeros((n, S, S, S, D))
    q[..., 0] = 1.0 + 0.3 * rng.random((n, S, S, S))
    q[..., 1:4] = 0.4 * rng.standard_normal((n, S, S, S, 3))
    q[..., 4] = 2.5 + 0.5 * rng.random((n, S, S, S)) + 0.5 * (q[..., 1:4] ** 2).sum(-1) / q[..., 0]
    if D > V:
        q[..., V:] = rng.random((n, S, S, S, D - V))
    return q.reshape(n, -1)


@pytest.mark.parametrize('scheme', [0, 1])
@pytest.mark.parametrize('P', [4, 7, 9])
def test_fv3d_update_vs_oracle(scheme, P):
    g = 1 if scheme == 0 else 2
    n = 6
    dx = [0.3, 0.25, 0.2]
    u = patches(P, g, n, 100 * P + scheme)
    for i in range(n):
        row = np.ascontiguousarray(u[i])
        O.lib().orc_fv_periodic_ghosts_3d(P, g, V, row)
        u[i] = row
    dt = 0.8 * min(O.lib().orc_fv_stable_dt_3d(P, g, V, 0, np.ascontiguousarray(u[i]), np.array(dx), 0.9)
                   for i in range(n))
    fv = FVPatches(P, g, dx, dim=3)
    d_old, d_new = DeviceBuffer.from_array(u), DeviceBuffer.from_array(u)
    d_adm = DeviceBuffer(n)
    (fv.godunov_update if scheme == 0 else fv.musclhancock_update)(n, d_new, d_old, dt, max_dt=d_adm)
    got, adm = d_new.download().reshape(n, -1), d_adm.download()
    f = O.lib().orc_fv_godunov_3d if scheme == 0 else O.lib().orc_fv_musclhancock_3d
    for i in range(n):
        ref = np.ascontiguousarray(u[i]).copy()
        a = f(P, g, V, 0, ref, np.ascontiguousarray(u[i]), np.array(dx), dt)
        assert np.abs(got[i] - ref).max() <= 1e-13 * np.abs(ref).max(), i
        assert abs(adm[i] - a) <= 1e-14 * a, i


def test_fv3d_stable_dt_and_ghosts():
    P, g, n = 5, 2, 4
    dx = [0.2, 0.2, 0.3]
    u = patches(P, g, n, 7)
    fv = FVPatches(P, g, dx, dim=3)
    d = DeviceBuffer.from_array(u)
    fv.periodic_ghosts(n, d)
    got = d.download().reshape(n, -1)
    dt_p = DeviceBuffer(n)
    fv.stable_dt(n, d, dt_p)
    dts = dt_p.download()
    for i in range(n):
        ref = np.ascontiguousarray(u[i]).copy()
        O.lib().orc_fv_periodic_ghosts_3d(P, g, V, ref)
        assert np.array_equal(got[i], ref)
        r = O.lib().orc_fv_stable_dt_3d(P, g, V, 0, ref, np.array(dx), 0.9)
        assert abs(dts[i] - r) <= 1e-15 * r


def test_fv3d_with_parameters_and_in_place():
    """nPar > 0 strides the data; the parameters stay untouched.  In place
    (luh_new is luh) gives the same interior as separate buffers."""
    P, g, n, D = 4, 1, 3, 6
    dx = [0.1, 0.1, 0.1]
    u = patches(P, g, n, 9, D=D)
    fv = FVPatches(P, g, dx, npar=1, dim=3)
    d_old, d_new = DeviceBuffer.from_array(u), DeviceBuffer.from_array(u)
    fv.godunov_update(n, d_new, d_old, 1e-4)
    got = d_new.download().reshape(n, -1, D)
    assert np.array_equal(got[..., V:], u.reshape(n, -1, D)[..., V:])
    ref = np.zeros_like(got)
    for i in range(n):
        r = np.ascontiguousarray(u[i]).copy()
        O.lib().orc_fv_godunov_3d(P, g, V, 1, r, np.ascontiguousarray(u[i]), np.array(dx), 1e-4)
        ref[i] = r.reshape(-1, D)
    assert np.abs(got - ref).max() <= 1e-13 * np.abs(ref).max()
    d_same = DeviceBuffer.from_array(u)
    fv.godunov_update(n, d_same, d_same, 1e-4)
    assert np.array_equal(d_same.download().reshape(n, -1, D), got)
