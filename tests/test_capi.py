"""The C-ABI library loads and exports every symbol include/*.h declares;
argument validation needs no GPU."""
import ctypes as C
import os
import re

import exahype_b200 as E
from exahype_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    inc = os.path.join(ROOT, 'include')
    for fn in os.listdir(inc):
        if not fn.endswith('.h'):
            continue
        text = open(os.path.join(inc, fn)).read()
        text = re.sub(r'/\*.*?\*/', ' ', text, flags=re.S)
        for m in re.finditer(r'\b(exa_\w+)\s*\(', text):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    L = E.lib()
    names = declared_symbols()
    assert len(names) > 40
    missing = [n for n in sorted(names) if not hasattr(L, n)]
    assert not missing, missing


def test_bindings_cover_the_header():
    assert declared_symbols() == set(_lib.SIGNATURES), \
        declared_symbols().symmetric_difference(set(_lib.SIGNATURES))


def test_validation_without_gpu():
    L = E.lib()
    cfg = E.aderdg.grid_config(4, 4, (2, 2, 2))
    h = C.c_void_p()
    assert L.exa_aderdg_grid_create(C.byref(cfg), C.byref(h)) == _lib.EXA_EINVAL
    cfg = E.aderdg.grid_config(3, 9, (2, 2, 2))
    assert L.exa_aderdg_grid_create(C.byref(cfg), C.byref(h)) == _lib.EXA_EINVAL
    cfg = E.aderdg.grid_config(3, 4, (2, 2, 2), dt_policy=2, dt_fixed=0.0)
    assert L.exa_aderdg_grid_create(C.byref(cfg), C.byref(h)) == _lib.EXA_EINVAL
    assert L.exa_aderdg_grid_create(None, C.byref(h)) == _lib.EXA_EINVAL
    assert b'order' in L.exa_last_error_string() or len(L.exa_last_error_string()) > 0
    for s in range(9):
        assert len(L.exa_status_string(s)) > 0
    assert L.exa_aderdg_grid_ncells(None) == 0
    assert L.exa_aderdg_grid_destroy(None) == _lib.EXA_OK


def test_footprint_of_the_3d_workload():
    fp = E.ADERDGGrid.footprint(3, 4, (81, 81, 81))
    n = 81 ** 3
    assert fp >= n * (2 * 125 * 5 + 2 * 6 * 25 * 5) * 8
    assert fp < 16e9
