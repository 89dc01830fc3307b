"""The C++ adaptor header (include/exahype_b200.hpp) compiles against the C
ABI, links with libexahype_b200.so, and on a GPU reproduces the reference's
3D predictor golden vectors."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

import _cases

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, 'exahype_b200')


def build(tmp):
    exe = os.path.join(tmp, 'adaptor_stp')
    subprocess.check_call(['g++', '-std=c++14', '-O1', '-Wall', '-Werror',
                           '-I', os.path.join(ROOT, 'include'),
                           os.path.join(ROOT, 'tests', 'cpp', 'adaptor_stp.cpp'),
                           '-L', LIBDIR, '-lexahype_b200', '-Wl,-rpath,' + LIBDIR, '-o', exe])
    return exe


def test_adaptor_compiles_and_links():
    with tempfile.TemporaryDirectory() as tmp:
        assert os.path.exists(build(tmp))


@pytest.mark.gpu
def test_adaptor_stp_golden(golden3d):
    B, D, V = 4, 6, 5
    luh = _cases._strided(golden3d['testSpaceTimePredictorNonlinear/luh'], B ** 3)
    with tempfile.TemporaryDirectory() as tmp:
        exe = build(tmp)
        inp, out = os.path.join(tmp, 'luh.bin'), os.path.join(tmp, 'out.bin')
        luh.tofile(inp)
        subprocess.check_call([exe, inp, out])
        r = np.fromfile(out)
    n_qb, n_fb, n_qhi = 6 * B * B * D, 6 * B * B * V, B ** 3 * D
    qb, fb, qhi = r[:n_qb], r[n_qb:n_qb + n_fb], r[n_qb + n_fb:n_qb + n_fb + n_qhi]
    fhi = r[n_qb + n_fb + n_qhi:]
    _cases.close(_cases._unstride(qb, 6 * B * B), golden3d['testSpaceTimePredictorNonlinear/lQhbnd'])
    _cases.close(fb, golden3d['testSpaceTimePredictorNonlinear/lFhbnd'])
    _cases.close(_cases._unstride(qhi, B ** 3), golden3d['testSpaceTimePredictorNonlinear/lQhi'])
    _cases.close(fhi[:3 * B ** 3 * V], golden3d['testSpaceTimePredictorNonlinear/lFhi'])
