#!/usr/bin/env python3
"""Derive the nodal ADER-DG operator tables on Gauss-Legendre nodes and write
them as a C header (``dg_tables.h``) shared by the CUDA kernels and the CPU
oracle.

The tables are the ones the reference kernels index (reference
``ExaHyPE/kernels/DGMatrices.h:47-126``, ``GaussLegendreQuadrature.h``):

* ``gl_nodes[N][i]``, ``gl_weights[N][i]`` -- Gauss-Legendre rule with N+1
  points mapped to the unit interval [0, 1].
* ``kxi[N][k][l]``   -- stiffness matrix  w_l * phi_k'(x_l).
* ``dudx[N][l][k]``  -- nodal derivative  phi_k'(x_l).
* ``ik1[N][k][l]``   -- inverse of the time "stiffness" K1 = F1 - Kxi, with
  F1[k][l] = phi_k(1) phi_l(1).
* ``f0[N][k]``       -- phi_k(0) (time flux at t=0).
* ``flcoeff``/``frcoeff`` -- phi_k(0) and phi_k(1) (face extrapolation).

Everything is computed from the mathematics in 60-digit arithmetic (mpmath)
and then rounded to double.  The reference ships its stiffness-type tables
(Kxi, iK1, dudx) printed with 13 significant digits
(``DGMatrices.cpp:401-476`` for order 4) and its kernels compute with those
rounded values.  To keep the results of this library within 1e-12 of the
reference we round the same three tables to 13 significant digits; all other
tables are kept at full double precision.  ``tests/test_dg_tables.py`` pins
every entry against the reference's values.

Usage: ``python gen_dg_tables.py [out.h]`` (default: ``dg_tables.h`` beside
this script).
"""
import os
import sys

import mpmath as mp

MAX_ORDER = 9
mp.mp.dps = 60


def gauss_legendre_unit(n):
    """n-point Gauss-Legendre nodes/weights on [0,1], ascending nodes."""
    xs, ws = [], []
    for i in range(n):
        x = mp.cos(mp.pi * (i + mp.mpf(3) / 4) / (n + mp.mpf(1) / 2))
        for _ in range(200):
            p0, p1 = mp.mpf(1), x
            for k in range(2, n + 1):
                p0, p1 = p1, ((2 * k - 1) * x * p1 - (k - 1) * p0) / k
            if n == 1:
                p0, p1 = mp.mpf(1), x
            dp = n * (x * p1 - p0) / (x * x - 1)
            step = p1 / dp
            x -= step
            if abs(step) < mp.mpf(10) ** -55:
                break
        xs.append((1 - x) / 2)
        ws.append(1 / ((1 - x * x) * dp * dp))  # 2/(...) on [-1,1], halved
    return xs, ws


def lagrange(xs, k, x):
    r = mp.mpf(1)
    for j, xj in enumerate(xs):
        if j != k:
            r *= (x - xj) / (xs[k] - xj)
    return r


def dlagrange(xs, k, x):
    s = mp.mpf(0)
    for m in range(len(xs)):
        if m == k:
            continue
        r = 1 / (xs[k] - xs[m])
        for j in range(len(xs)):
            if j != k and j != m:
                r *= (x - xs[j]) / (xs[k] - xs[j])
        s += r
    return s


def gauss_lobatto_unit(n):
    """n-point Gauss-Lobatto nodes on [0,1] in the reference's order,
    descending from 1 to 0 (GaussLobattoQuadrature.cpp:47-160); the
    1-point rule is the midpoint, as there."""
    if n == 1:
        return [mp.mpf(1) / 2]
    # interior nodes: roots of P'_{n-1} on [-1,1], by Newton from the
    # Chebyshev-Gauss-Lobatto guesses
    m = n - 1
    xs = []
    for i in range(1, m):
        x = -mp.cos(mp.pi * i / m)
        for _ in range(200):
            p0, p1 = mp.mpf(1), x
            for k in range(2, m + 1):
                p0, p1 = p1, ((2 * k - 1) * x * p1 - (k - 1) * p0) / k
            # P'_m and P''_m from the Legendre ODE
            dp = m * (x * p1 - p0) / (x * x - 1)
            d2p = (2 * x * dp - m * (m + 1) * p1) / (1 - x * x)
            step = dp / d2p
            x -= step
            if abs(step) < mp.mpf(10) ** -55:
                break
        xs.append(x)
    pts = [mp.mpf(-1)] + xs + [mp.mpf(1)]
    return sorted([(1 + x) / 2 for x in pts], reverse=True)


def round13(v):
    """Round to 13 significant digits (the precision of the reference's
    stiffness tables), then to the nearest double."""
    return float('%.12e' % float(v)) if v != 0 else 0.0


def derive(order):
    b = order + 1
    xs, ws = gauss_legendre_unit(b)
    kxi = [[ws[l] * dlagrange(xs, k, xs[l]) for l in range(b)] for k in range(b)]
    dudx = [[dlagrange(xs, k, xs[l]) for k in range(b)] for l in range(b)]
    k1 = mp.matrix(b, b)
    for k in range(b):
        for l in range(b):
            k1[k, l] = lagrange(xs, k, 1) * lagrange(xs, l, 1) - kxi[k][l]
    ik1 = k1 ** -1
    out = {
        'gl_nodes': [float(x) for x in xs],
        'gl_weights': [float(w) for w in ws],
        'kxi': [[round13(kxi[k][l]) for l in range(b)] for k in range(b)],
        'dudx': [[round13(dudx[l][k]) for k in range(b)] for l in range(b)],
        'ik1': [[round13(ik1[k, l]) for l in range(b)] for k in range(b)],
        'f0': [float(lagrange(xs, k, 0)) for k in range(b)],
        # fine-grid projector (3:1 refinement): fgp[s][n][m] = coarse basis
        # polynomial n at node m of subinterval s, phi_n((s + x_m) / 3)
        'fgp': [[[round13(lagrange(xs, n, (sub + xs[m]) / 3)) for m in range(b)] for n in range(b)]
                for sub in range(3)],
        'flcoeff': [float(lagrange(xs, k, 0)) for k in range(b)],
        'frcoeff': [float(lagrange(xs, k, 1)) for k in range(b)],
        'lob_nodes': [float(x) for x in gauss_lobatto_unit(b)],
    }
    out.update(derive_limiter(xs, ws))
    return out


def derive_limiter(xs, ws):
    """Projections between the nodal DG basis of one cell and its FV
    subcell patch of S = 2N+1 subcells per direction (the reference builds
    them at start-up, LimiterProjectionMatrices.cpp:40-140):

    * uh2lim[k][i] -- mean of phi_k over subcell i, [i/S, (i+1)/S] (the
      reference integrates with the B-point Gauss-Legendre rule, exact for
      degree N);
    * uh2lob[k][i] -- phi_k at Gauss-Lobatto node i (descending order);
    * lim2uh[i][k] -- the conservative least-squares inverse: for subcell
      means L, u = sum_i L_i lim2uh[i][:] minimises
      sum_i (sum_k uh2lim[k][i] u_k - L_i)^2 subject to
      sum_k w_k u_k = sum_i L_i / S (the cell mean is kept).  Solved from
      the bordered normal equations [[2 U U^T, -w], [w^T, 0]].
    All three are kept at full double precision (the reference computes
    them in double at run time)."""
    b = len(xs)
    s = 2 * (b - 1) + 1
    dxi = mp.mpf(1) / s
    uh2lim = [[mp.fsum(ws[j] * lagrange(xs, k, i * dxi + dxi * xs[j]) for j in range(b))
               for i in range(s)] for k in range(b)]
    lob = gauss_lobatto_unit(b)
    uh2lob = [[lagrange(xs, k, lob[i]) for i in range(b)] for k in range(b)]
    a = mp.matrix(b + 1, b + 1)
    for i in range(b):
        for j in range(b):
            a[i, j] = 2 * mp.fsum(uh2lim[i][k] * uh2lim[j][k] for k in range(s))
        a[i, b] = -ws[i]
        a[b, i] = ws[i]
    ia = a ** -1
    lim2uh = [[None] * b for _ in range(s)]
    for i in range(s):
        rhs = [2 * uh2lim[j][i] for j in range(b)] + [dxi]
        for k in range(b):
            lim2uh[i][k] = mp.fsum(ia[k, m] * rhs[m] for m in range(b + 1))
    return {
        'uh2lim': [[float(v) for v in row] for row in uh2lim],
        'uh2lob': [[float(v) for v in row] for row in uh2lob],
        'lim2uh': [[float(v) for v in row] for row in lim2uh],
    }


def all_tables():
    return {n: derive(n) for n in range(MAX_ORDER + 1)}


def _fmt(v):
    return float(v).hex()


def write_header(path):
    tabs = all_tables()
    D = MAX_ORDER + 1
    out = []
    out.append('/* Generated by gen_dg_tables.py -- do not edit.\n'
               ' * Nodal ADER-DG operators on Gauss-Legendre nodes of [0,1] for\n'
               ' * orders 0..%d (see the generator for definitions).  Values are\n'
               ' * C99 hexadecimal double literals; unused entries are zero. */\n' % MAX_ORDER)
    out.append('#ifndef EXA_DG_TABLES_H\n#define EXA_DG_TABLES_H\n')
    out.append('#define EXA_DG_MAX_ORDER %d\n' % MAX_ORDER)
    out.append('#ifndef EXA_TABLE_QUAL\n#define EXA_TABLE_QUAL static const\n#endif\n')
    for name in ('gl_nodes', 'gl_weights', 'f0', 'flcoeff', 'frcoeff'):
        out.append('EXA_TABLE_QUAL double exa_%s[%d][%d] = {\n' % (name, D, D))
        for n in range(D):
            row = tabs[n][name] + [0.0] * (D - len(tabs[n][name]))
            out.append('  {' + ', '.join(_fmt(v) for v in row) + '},\n')
        out.append('};\n')
    for name in ('kxi', 'dudx', 'ik1'):
        out.append('EXA_TABLE_QUAL double exa_%s[%d][%d][%d] = {\n' % (name, D, D, D))
        for n in range(D):
            out.append('  {\n')
            m = tabs[n][name]
            for k in range(D):
                row = (m[k] if k < len(m) else []) + [0.0] * (D - (len(m[k]) if k < len(m) else 0))
                out.append('    {' + ', '.join(_fmt(v) for v in row) + '},\n')
            out.append('  },\n')
        out.append('};\n')
    out.append('EXA_TABLE_QUAL double exa_fgp[%d][3][%d][%d] = {\n' % (D, D, D))
    for n in range(D):
        out.append('  {\n')
        for sub in range(3):
            out.append('    {\n')
            m = tabs[n]['fgp'][sub]
            for k in range(D):
                row = (m[k] if k < len(m) else []) + [0.0] * (D - (len(m[k]) if k < len(m) else 0))
                out.append('      {' + ', '.join(_fmt(v) for v in row) + '},\n')
            out.append('    },\n')
        out.append('  },\n')
    out.append('};\n')
    # limiter projections (subcell count S = 2N+1 <= 19)
    S = 2 * MAX_ORDER + 1
    out.append('#define EXA_LIM_MAX_SUBCELLS %d\n' % S)
    out.append('EXA_TABLE_QUAL double exa_lob_nodes[%d][%d] = {\n' % (D, D))
    for n in range(D):
        row = tabs[n]['lob_nodes'] + [0.0] * (D - len(tabs[n]['lob_nodes']))
        out.append('  {' + ', '.join(_fmt(v) for v in row) + '},\n')
    out.append('};\n')
    for name, rows, cols in (('uh2lim', D, S), ('uh2lob', D, D), ('lim2uh', S, D)):
        out.append('EXA_TABLE_QUAL double exa_%s[%d][%d][%d] = {\n' % (name, D, rows, cols))
        for n in range(D):
            out.append('  {\n')
            m = tabs[n][name]
            for k in range(rows):
                row = list(m[k]) if k < len(m) else []
                row = row + [0.0] * (cols - len(row))
                out.append('    {' + ', '.join(_fmt(v) for v in row) + '},\n')
            out.append('  },\n')
        out.append('};\n')
    # CFL safety factors for ADER-DG of order N (reference
    # kernels/aderdg/generic/c/3d/stableTimeStepSize.cpph:33-34)
    out.append('EXA_TABLE_QUAL double exa_pnpm[10] = {1.0, 0.33, 0.17, 0.1, 0.069, '
               '0.045, 0.038, 0.03, 0.02, 0.015};\n')
    out.append('#endif\n')
    with open(path, 'w') as f:
        f.write(''.join(out))


if __name__ == '__main__':
    here = os.path.dirname(os.path.abspath(__file__))
    write_header(sys.argv[1] if len(sys.argv) > 1 else os.path.join(here, 'dg_tables.h'))
