"""AMR transfer operators on the GPU against the oracle (which is pinned to
the reference's compiled amrRoutines in test_oracle_amr.py)."""
import itertools

import numpy as np
import pytest

import _oracle as O
from exahype_b200 import DeviceBuffer
from exahype_b200.aderdg import amr_prolongation, amr_restriction

pytestmark = pytest.mark.gpu
V = 5


@pytest.mark.parametrize('k,order,delta', [(3, 4, 1), (3, 3, 2), (2, 5, 1), (2, 2, 3), (1, 4, 2), (3, 2, 1)])
def test_amr_gpu_vs_oracle(k, order, delta):
    rng = np.random.default_rng(7 * k + order + delta)
    B = order + 1
    n = B ** k * V
    count = 23
    coarse = rng.standard_normal((count, n))
    idx = np.zeros((count, 3), np.int32)
    idx[:, :k] = rng.integers(0, 3 ** delta, size=(count, k))
    d_c, d_i = DeviceBuffer.from_array(coarse), DeviceBuffer.from_array(idx)
    d_f = DeviceBuffer(count * n)
    amr_prolongation(k, order, count, d_f, d_c, delta, d_i)
    got = d_f.download().reshape(count, n)
    for i in range(count):
        ref = np.zeros(n)
        O.lib().orc_amr_prolongation(k, order, V, ref, coarse[i].copy(), delta, idx[i])
        assert np.abs(got[i] - ref).max() < 1e-13 * max(1.0, np.abs(ref).max()), i
    # restriction accumulates into the coarse arrays
    fine = rng.standard_normal((count, n))
    base = rng.standard_normal((count, n))
    d_b, d_f2 = DeviceBuffer.from_array(base), DeviceBuffer.from_array(fine)
    amr_restriction(k, order, count, d_b, d_f2, delta, d_i)
    got = d_b.download().reshape(count, n)
    for i in range(count):
        ref = base[i].copy()
        O.lib().orc_amr_restriction(k, order, V, ref, fine[i].copy(), delta, idx[i])
        assert np.abs(got[i] - ref).max() < 1e-13 * max(1.0, np.abs(ref).max()), i


def test_amr_gpu_children_of_one_parent():
    """A parent prolonged into its 3^k children through coarse_item and the
    children restricted back reproduce the parent."""
    k, order = 3, 4
    B = order + 1
    n = B ** k * V
    rng = np.random.default_rng(1)
    parent = rng.standard_normal(n)
    kids = list(itertools.product(range(3), repeat=k))
    idx = np.zeros((len(kids), 3), np.int32)
    for c, t in enumerate(kids):
        idx[c, :k] = t[::-1]  # (x, y, z)
    d_p = DeviceBuffer.from_array(parent)
    d_i = DeviceBuffer.from_array(idx)
    d_map = DeviceBuffer.from_array(np.zeros(len(kids), np.int64))
    d_f = DeviceBuffer(len(kids) * n)
    amr_prolongation(k, order, len(kids), d_f, d_p, 1, d_i, coarse_item=d_map)
    fine = d_f.download().reshape(len(kids), n)
    back = np.zeros(n)
    for c in range(len(kids)):  # deterministic order on the host side
        part = DeviceBuffer.from_array(np.zeros(n))
        amr_restriction(k, order, 1, part, DeviceBuffer.from_array(fine[c]), 1,
                        DeviceBuffer.from_array(idx[c:c + 1]))
        back += part.download()
    assert np.abs(back - parent).max() < 1e-11
