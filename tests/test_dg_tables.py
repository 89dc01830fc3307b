"""The project's own derivation of the DG operator tables (gen_dg_tables.py)
against the reference's hard-coded tables (DGMatrices.cpp, Gauss-
LegendreQuadrature.cpp; extracted to tests/golden/dg_tables_ref.npz)."""
import importlib.util
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope='module')
def tables():
    spec = importlib.util.spec_from_file_location(
        'gen', os.path.join(ROOT, 'exahype_b200', 'csrc', 'gen_dg_tables.py'))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m.all_tables()


@pytest.fixture(scope='module')
def ref():
    return np.load(os.path.join(ROOT, 'tests', 'golden', 'dg_tables_ref.npz'))


@pytest.mark.parametrize('order', range(10))
def test_tables_match_reference(tables, ref, order):
    t = tables[order]
    # 13-significant-digit tables: identical except for entries whose exact
    # value is 0 (reference prints ~1e-16 noise) or sits on a rounding tie
    for mine, theirs in (('kxi', 'Kxi'), ('ik1', 'iK1'), ('dudx', 'dudx')):
        a, b = np.array(t[mine]), ref['%s/%d' % (theirs, order)]
        scale = max(1.0, np.abs(b).max())
        assert np.abs(a - b).max() <= 2e-13 * scale, mine
        exact = np.mean(a == b)
        assert exact > 0.85, (mine, exact)
    # fine-grid projector of 3:1 refinement (DGMatrices.cpp fineGridProjector1d)
    a, b = np.array(t['fgp']), ref['fgp/%d' % order]
    assert np.abs(a - b).max() <= 2e-14 * max(1.0, np.abs(b).max()), 'fgp'
    assert np.mean(a == b) > 0.95, 'fgp'
    for mine, theirs in (('f0', 'F0'), ('flcoeff', 'FLCoeff'), ('frcoeff', 'FRCoeff'),
                         ('gl_weights', 'weights'), ('gl_nodes', 'nodes'),
                         ('lob_nodes', 'lob_nodes')):
        a, b = np.array(t[mine]), ref['%s/%d' % (theirs, order)]
        assert np.abs(a - b).max() <= 2e-14 * max(1.0, np.abs(b).max()), mine


def test_generated_header_is_current(tables):
    """dg_tables.h must be the output of the generator (hex literals)."""
    text = open(os.path.join(ROOT, 'exahype_b200', 'csrc', 'dg_tables.h')).read()
    for n in (2, 3, 4, 5):
        for v in tables[n]['kxi'][1]:
            assert float(v).hex() in text


def test_operators_are_exact_on_polynomials(tables):
    """Kxi/w differentiates degree-N polynomials exactly at the nodes;
    the GL rule integrates degree 2N+1 exactly."""
    for n in (2, 3, 4, 5):
        t = tables[n]
        x = np.array(t['gl_nodes'])
        w = np.array(t['gl_weights'])
        kxi = np.array(t['kxi'])
        D = (kxi / w[None, :]).T  # D[l][p] = Kxi[p][l]/w_l = phi_p'(x_l)
        for deg in range(n + 1):
            f = x ** deg
            df = deg * x ** (deg - 1) if deg > 0 else 0 * x
            assert np.allclose(D @ f, df, atol=1e-11)
        assert abs(np.sum(w * x ** (2 * n + 1)) - 1.0 / (2 * n + 2)) < 1e-14
