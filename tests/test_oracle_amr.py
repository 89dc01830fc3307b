"""AMR transfer operators of the oracle (3:1 refinement, fine-grid
projector of DGMatrices.cpp) against the reference's own amrRoutines
compiled from source (oracle/_ref), and the projection identity: restricting
the prolongations of a coarse DG polynomial to all children gives it back."""
import itertools

import numpy as np
import pytest

import _oracle as O

V = 5


def prolong(k, order, coarse, delta, index):
    fine = np.zeros_like(coarse)
    O.lib().orc_amr_prolongation(k, order, V, fine, coarse, delta, np.asarray(index + [0] * (3 - len(index)), np.int32))
    return fine


def restrict(k, order, coarse, fine, delta, index):
    O.lib().orc_amr_restriction(k, order, V, coarse, fine, delta, np.asarray(index + [0] * (3 - len(index)), np.int32))


@pytest.mark.parametrize('dim', [2, 3])
@pytest.mark.parametrize('order', [2, 3, 4, 5])
@pytest.mark.parametrize('delta', [1, 2])
def test_amr_oracle_vs_reference(dim, order, delta):
    R = O.ref_lib(dim)
    if R is None or not hasattr(R, 'ref_amr'):
        pytest.skip('reference kernels not built (make -C oracle ref)')
    rng = np.random.default_rng(10 * dim + order + 100 * delta)
    B = order + 1
    for what, k in ((0, dim), (1, dim), (2, dim - 1), (3, dim - 1)):
        n = B ** k * V
        idx = [int(x) for x in rng.integers(0, 3 ** delta, size=k)]
        iq, i_f = rng.standard_normal(n), rng.standard_normal(n)
        ref_q, ref_f = rng.standard_normal(n), rng.standard_normal(n)  # restriction accumulates into these
        my_q, my_f = ref_q.copy(), ref_f.copy()
        if what in (0, 2):
            ref_q[:] = 0.0
            ref_f[:] = 0.0
        R.ref_amr(what, order, ref_q, ref_f, iq, i_f, delta, np.asarray(idx + [0] * (3 - k), np.int32))
        if what in (0, 2):
            my_q = prolong(k, order, iq, delta, idx)
            my_f = prolong(k, order, i_f, delta, idx)
        else:
            restrict(k, order, my_q, iq, delta, idx)
            restrict(k, order, my_f, i_f, delta, idx)
        scale = max(1.0, np.abs(ref_q).max())
        assert np.abs(my_q - ref_q).max() < 1e-13 * scale, (what, np.abs(my_q - ref_q).max())
        if what >= 2:
            assert np.abs(my_f - ref_f).max() < 1e-13 * max(1.0, np.abs(ref_f).max())


@pytest.mark.parametrize('k,order', [(2, 3), (3, 4), (1, 5)])
def test_restriction_of_prolongations_is_identity(k, order):
    rng = np.random.default_rng(k + order)
    B = order + 1
    coarse = rng.standard_normal(B ** k * V)
    back = np.zeros_like(coarse)
    for idx in itertools.product(range(3), repeat=k):
        restrict(k, order, back, prolong(k, order, coarse, 1, list(idx)), 1, list(idx))
    assert np.abs(back - coarse).max() < 1e-11  # projector tables carry 13 significant digits
