"""Mixed-precision predictor against the FP64 path: relative L2 error of the
state after every step <= 1e-8 (the accuracy bar stated for the
mixed-precision form), same Picard behaviour, no NaN."""
import numpy as np
import pytest

import exahype_b200 as E
from exahype_b200.device import diff_norms

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize('dim,order,n,kind,steps', [
    (3, 4, (6, 5, 4), 0, 30),
    (3, 3, (4, 4, 4), 0, 20),
    (3, 2, (5, 5, 5), 1, 20),
    (3, 5, (3, 3, 3), 0, 10),
    (2, 3, (27, 27), 1, 50),
    (2, 4, (16, 12), 0, 30),
    (2, 5, (9, 9), 0, 20),
    (2, 2, (20, 20), 1, 30),
])
@pytest.mark.parametrize('variant', [1, 2, 3, 4])
def test_mixed_vs_fp64_per_step(dim, order, n, kind, steps, variant):
    # variant (tuning key 2): 1 = node-gather contraction, 2 = line-owner,
    # 3 = tensor-core line derivatives, 4 = progressive line-owner (both 3D
    # order 4; line-owner elsewhere)
    E._lib.call('exa_tune_set', 2, variant)
    try:
        _mixed_vs_fp64(dim, order, n, kind, steps)
    finally:
        E._lib.call('exa_tune_set', 2, 0)


def _mixed_vs_fp64(dim, order, n, kind, steps):
    a = E.ADERDGGrid(dim, order, n, precision=E.PREC_FP64)
    b = E.ADERDGGrid(dim, order, n, precision=E.PREC_MIXED)
    param = 5.0 if kind == 0 else 0.2
    for g in (a, b):
        g.init(kind=kind, param=param, seed=17, noise=1e-3)
    worst = 0.0
    for s in range(steps):
        da = a.step(1, want_dt=True)[0]
        db = b.step(1, want_dt=True)[0]
        assert abs(da - db) <= 1e-8 * da
        e = diff_norms(b.device_state_ptr(), a.device_state_ptr(), a.state_size)
        worst = max(worst, e['rel_l2'])
        assert e['rel_l2'] <= 1e-8, (s, e)
    sa, sb = a.status(), b.status()
    assert not sb['nan']
    # the deviation form converges like the FP64 path (iteration counts agree
    # up to cells sitting at the threshold)
    assert abs(sa['picard_iters'] - sb['picard_iters']) <= 0.01 * sa['picard_iters']
    a.destroy()
    b.destroy()


@pytest.mark.parametrize('dim,order,n,pde', [(3, 4, (5, 4, 3), E.PDE_EULER), (2, 5, (7, 5), E.PDE_EULER),
                                             (2, 5, (7, 5), E.PDE_EULER_PLANAR)])
def test_progressive_mixed_equals_line_owner_bitwise(dim, order, n, pde):
    """The progressive mixed predictor (tuning key 2 = 4) performs the
    line-owner kernel's FP32 operations in the same order: the same grid
    stepped with either is identical bit for bit (3D order 4, one cell per
    CTA; 2D order 5, two cells per CTA with a partial last block), Picard
    counts included."""
    out = []
    for variant in (2, 4):
        E._lib.call('exa_tune_set', 2, variant)
        try:
            g = E.ADERDGGrid(dim, order, n, pde=pde, precision=E.PREC_MIXED)
            g.init(kind=0, param=5.0, seed=23, noise=1e-3)
            g.step(5)
            out.append((g.get_state(), g.status()['picard_iters']))
            g.destroy()
        finally:
            E._lib.call('exa_tune_set', 2, 0)
    assert np.array_equal(out[0][0], out[1][0]) and out[0][1] == out[1][1]


def test_diff_norms_utility():
    from exahype_b200 import DeviceBuffer
    rng = np.random.default_rng(0)
    x = rng.standard_normal(100003)
    y = x + 1e-6 * rng.standard_normal(x.size)
    dx, dy = DeviceBuffer.from_array(x), DeviceBuffer.from_array(y)
    e = diff_norms(dy.ptr, dx.ptr, x.size)
    assert abs(e['rel_l2'] - np.linalg.norm(y - x) / np.linalg.norm(x)) < 1e-12
    assert abs(e['rel_linf'] - np.abs(y - x).max() / np.abs(x).max()) < 1e-15
