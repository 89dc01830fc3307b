#!/usr/bin/env python3
"""Extract the reference's known-answer data into small numpy fixtures.

Run in a checkout that has the reference sources: the path of the reference
tree is the first argument (or the ``EXA_REFERENCE`` environment variable).  It writes, next to this script:

* ``generic_euler_2d.npz`` / ``generic_euler_3d.npz`` -- every array of
  ``ExaHyPE/exahype/tests/kernels/testdata/generic_euler_testdata.cpp``
  (2D block ``:21-1346``, 3D block ``:1348-...``), keyed
  ``<namespace>/<array>``.  These are the golden vectors the reference's
  ``GenericEulerKernelTest{2D,3D}.cpp`` checks its generic kernels against
  (order 3, 5 variables, 1 material parameter, eps 1e-10).
* ``dg_tables_ref.npz`` -- the reference's hard-coded Gauss-Legendre rule
  (``ExaHyPE/kernels/GaussLegendreQuadrature.cpp:33-164``), Gauss-Lobatto
  nodes (``ExaHyPE/kernels/GaussLobattoQuadrature.cpp:47-160``) and DG
  operator tables (``ExaHyPE/kernels/DGMatrices.cpp:82-3116``), keyed
  ``<table>/<order>`` as dense arrays, used to pin this project's own
  derivation of the tables.
* ``limiter_2d.npz`` / ``limiter_3d.npz`` -- the limiter projection
  known-answer arrays of
  ``ExaHyPE/exahype/tests/kernels/testdata/limiter_testdata.cpp``.

The fixtures are data only; nothing under ``tests/`` reads the reference
tree at test time.
"""
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _parse_arrays(text):
    """Yield (namespace, name, values) for every `const double x[n] = {...}`."""
    ns_stack = []
    pos = 0
    token = re.compile(r'namespace\s+(\w+)\s*\{|\}\s*//\s*(?:namespace|namesapce)?\s*(\w*)|'
                       r'const\s+double\s+(\w+)\s*\[(\d+)\]\s*=?\s*\{([^}]*)\}', re.S)
    for m in token.finditer(text):
        if m.group(1):
            ns_stack.append(m.group(1))
        elif m.group(3):
            body = re.sub(r'//[^\n]*|/\*.*?\*/', ' ', m.group(5), flags=re.S)
            vals = [float(v) for v in re.split(r'[,\s]+', body.strip()) if v]
            n = int(m.group(4))
            assert len(vals) in (n, 0), (m.group(3), len(vals), n)  # `= {}`: no data
            yield ns_stack[-1], m.group(3), np.array(vals)
        else:
            if ns_stack:
                ns_stack.pop()


def extract_generic_euler(ref):
    path = os.path.join(ref, 'ExaHyPE/exahype/tests/kernels/testdata/generic_euler_testdata.cpp')
    text = open(path).read()
    i2 = text.index('#ifdef Dim2')
    i3 = text.index('#ifdef Dim3')
    out = {}
    for tag, block in (('2d', text[i2:i3]), ('3d', text[i3:])):
        arrays = {}
        for ns, name, vals in _parse_arrays(block):
            arrays['%s/%s' % (ns, name)] = vals
        out[tag] = arrays
        np.savez_compressed(os.path.join(HERE, 'generic_euler_%s.npz' % tag), **arrays)
    return out


def extract_dg_tables(ref):
    src = open(os.path.join(ref, 'ExaHyPE/kernels/DGMatrices.cpp')).read()
    gsrc = open(os.path.join(ref, 'ExaHyPE/kernels/GaussLegendreQuadrature.cpp')).read()
    out = {}
    for n in range(10):
        b = n + 1
        for name in ('Kxi', 'iK1', 'dudx'):
            out['%s/%d' % (name, n)] = np.full((b, b), np.nan)
        for name in ('F0', 'FLCoeff', 'FRCoeff'):
            out['%s/%d' % (name, n)] = np.full(b, np.nan)
        out['fgp/%d' % n] = np.full((3, b, b), np.nan)
        out['weights/%d' % n] = np.full(b, np.nan)
        out['nodes/%d' % n] = np.full(b, np.nan)
    for m in re.finditer(r'\b(Kxi|iK1|dudx)\[(\d)\]\[(\d)\]\[(\d)\]\s*=\s*([-+0-9.eE]+);', src):
        out['%s/%s' % (m.group(1), m.group(2))][int(m.group(3)), int(m.group(4))] = float(m.group(5))
    for m in re.finditer(r'\b(F0|FLCoeff|FRCoeff)\[(\d)\]\[(\d)\]\s*=\s*([-+0-9.eE]+);', src):
        out['%s/%s' % (m.group(1), m.group(2))][int(m.group(3))] = float(m.group(4))
    for m in re.finditer(r'fineGridProjector1d\[(\d)\]\[(\d)\]\[(\d)\]\[(\d)\]\s*=\s*([-+0-9.eE]+);', src):
        out['fgp/%s' % m.group(1)][int(m.group(2)), int(m.group(3)), int(m.group(4))] = float(m.group(5))
    for m in re.finditer(r'gaussLegendre(Weights|Nodes)\[(\d)\]\[(\d)\]\s*=\s*([-+0-9.eE]+);', gsrc):
        key = ('weights' if m.group(1) == 'Weights' else 'nodes') + '/' + m.group(2)
        out[key][int(m.group(3))] = float(m.group(4))
    lsrc = open(os.path.join(ref, 'ExaHyPE/kernels/GaussLobattoQuadrature.cpp')).read()
    for n in range(10):
        out['lob_nodes/%d' % n] = np.full(n + 1, np.nan)
    for m in re.finditer(r'gaussLobattoNodes\s*\[(\d)\]\[(\d)\]\s*=\s*([-+0-9.eE]+);', lsrc):
        out['lob_nodes/%s' % m.group(1)][int(m.group(2))] = float(m.group(3))
    for k, v in out.items():
        assert not np.isnan(v).any(), k
    np.savez_compressed(os.path.join(HERE, 'dg_tables_ref.npz'), **out)
    return out


def extract_limiter(ref):
    """Known-answer data of the limiter projections,
    ExaHyPE/exahype/tests/kernels/testdata/limiter_testdata.cpp (order 3,
    5 variables; 2D block from `#ifdef Dim2`, 3D block from `#ifdef Dim3`):
    testFromLuhConversion::{luh_in, lob_out, lim_out} and
    testToLuhConversion::{lim_in, luh_out}.  (The reference's
    LimiterKernelTest.cpp keeps the checks that would use them commented
    out.)"""
    path = os.path.join(ref, 'ExaHyPE/exahype/tests/kernels/testdata/limiter_testdata.cpp')
    text = open(path).read()
    i2 = text.index('#ifdef Dim2')
    i3 = text.index('#ifdef Dim3')
    out = {}
    for tag, block in (('2d', text[i2:i3]), ('3d', text[i3:])):
        arrays = {}
        for ns, name, vals in _parse_arrays(block):
            if vals.size:
                arrays['%s/%s' % (ns, name)] = vals
        out[tag] = arrays
        np.savez_compressed(os.path.join(HERE, 'limiter_%s.npz' % tag), **arrays)
    return out


if __name__ == '__main__':
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get('EXA_REFERENCE')
    if not ref:
        sys.exit('usage: make_golden.py <reference tree>  (or set EXA_REFERENCE)')
    ge = extract_generic_euler(ref)
    tabs = extract_dg_tables(ref)
    lim = extract_limiter(ref)
    print('limiter 2d arrays:', sorted(lim['2d']), ' 3d arrays:', sorted(lim['3d']))
    print('generic_euler 2d arrays:', len(ge['2d']), ' 3d arrays:', len(ge['3d']),
          ' dg tables:', len(tabs))
