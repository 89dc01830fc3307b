"""Host-side logic of the serving loop (no GPU): the seeded request mix."""
import numpy as np

from exahype_b200 import serving as S


def test_request_mix_is_seeded_and_in_range():
    a = S.request_mix(400, seed=7)
    b = S.request_mix(400, seed=7)
    assert [(k, bytes(r)) for k, r in a] == [(k, bytes(r)) for k, r in b]
    kinds = [k for k, _ in a]
    assert 0.15 < kinds.count('dg') / len(kinds) < 0.35
    for k, r in a:
        assert 20 <= r.steps <= 200
        if k == 'dg':
            assert 2 <= r.dg.order <= 5 and 9 <= r.dg.n[0] <= 243 and r.dg.n[0] == r.dg.n[1]
            assert 0.05 <= r.dg.ic_param <= 0.3
        else:
            assert 64 <= r.fv_patch <= 1024 and r.fv_scheme == 1


def test_footprints_are_positive_and_scale():
    small = S.footprint(S.dg_request(3, 20, 10))
    big = S.footprint(S.dg_request(3, 40, 10))
    assert 3.5 * small < big < 4.5 * small
    assert S.footprint(S.fv_request(128, 10)) > S.footprint(S.fv_request(64, 10))
