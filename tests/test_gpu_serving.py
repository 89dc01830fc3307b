"""Serving engine: admission by footprint, continuous batching, results
identical alone and in a mix, FV requests against the oracle."""
import numpy as np
import pytest

import _oracle as O
import exahype_b200 as E
from exahype_b200 import serving as S

pytestmark = pytest.mark.gpu


def run_to_completion(server, reqs, submit_at=None):
    """Submits reqs[i] at tick submit_at[i] (0 by default), ticks until all
    finish; returns {i: state}."""
    submit_at = submit_at or [0] * len(reqs)
    ids, out, tick = {}, {}, 0
    while len(out) < len(reqs):
        for i, r in enumerate(reqs):
            if i not in ids.values() and submit_at[i] <= tick:
                rid = server.submit(r)
                if rid is not None:
                    ids[rid] = i
        server.tick()
        tick += 1
        for rid in server.completed():
            out[ids[rid]] = server.result(rid)
        assert tick < 10000
    return out


def test_results_identical_alone_and_in_mix():
    x_dg = S.dg_request(4, 15, 12, ic_param=0.25, seed=3, noise=1e-3)
    x_fv = S.fv_request(48, 9, scheme=1, ic_param=0.2, seed=4, noise=1e-3)
    alone = {}
    for name, r in (('dg', x_dg), ('fv', x_fv)):
        srv = S.Server(1 << 28)
        alone[name] = run_to_completion(srv, [r])[0]
        srv.destroy()
    others = [S.dg_request(2, 30, 20, seed=5), S.fv_request(100, 5, scheme=0, seed=6),
              S.dg_request(5, 9, 7, seed=7), S.fv_request(64, 15, scheme=1, seed=8),
              S.dg_request(3, 40, 3, seed=9)]
    reqs = others[:2] + [x_dg] + others[2:4] + [x_fv] + others[4:]
    srv = S.Server(1 << 29)
    got = run_to_completion(srv, reqs, submit_at=[0, 1, 2, 2, 4, 3, 5])
    srv.destroy()
    for name, i in (('dg', 2), ('fv', 5)):
        a, b = alone[name], got[i]
        assert np.array_equal(a[0], b[0]), name
        assert a[1] == b[1] and a[2] == b[2]


def test_dg_request_matches_grid():
    r = S.dg_request(3, 21, 10, ic_param=0.2, seed=11, noise=1e-3)
    srv = S.Server(1 << 28)
    state, t, steps = run_to_completion(srv, [r])[0]
    srv.destroy()
    g = E.ADERDGGrid(2, 3, (21, 21))
    g.init(kind=1, param=0.2, seed=11, noise=1e-3)
    g.step(10)
    ref = g.get_state()
    assert steps == 10
    assert np.linalg.norm(state - ref) / np.linalg.norm(ref) < 1e-13
    assert abs(t - g.status()['time']) <= 1e-13 * t
    g.destroy()


def fv_ic(P, g, amp, length=1.0):
    Sz = P + 2 * g
    h = length / P
    j, k = np.mgrid[0:Sz, 0:Sz]
    x, y = (k - g + 0.5) * h, (j - g + 0.5) * h
    rho = 1.0 + amp * np.sin(2 * np.pi * (x + y))
    q = np.zeros((Sz, Sz, 5))
    q[..., 0] = rho
    q[..., 1] = rho
    q[..., 2] = rho
    q[..., 4] = 1.0 / 0.4 + rho
    return q.ravel()


@pytest.mark.parametrize('scheme', [0, 1])
def test_fv_request_matches_oracle(scheme):
    P, steps, amp = 40, 12, 0.2
    g = 1 if scheme == 0 else 2
    srv = S.Server(1 << 26)
    state, t, n = run_to_completion(srv, [S.fv_request(P, steps, scheme=scheme, ic_param=amp, noise=0.0)])[0]
    srv.destroy()
    ref = fv_ic(P, g, amp)
    tr = 0.0
    for _ in range(steps):
        tr += O.lib().orc_fv_patch_step_2d(scheme, P, 0, ref, np.array([1.0, 1.0]), 0.0, None)
    # compare the interior (ghosts are refreshed at the start of each step)
    Sz = P + 2 * g
    a = state.reshape(Sz, Sz, 5)[g:g + P, g:g + P]
    b = ref.reshape(Sz, Sz, 5)[g:g + P, g:g + P]
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-12
    assert abs(t - tr) <= 1e-12 * tr and n == steps


def test_admission_waits_for_memory():
    big = S.dg_request(5, 60, 4, seed=1)
    fp = S.footprint(big)
    srv = S.Server(int(fp * 1.6))
    a = srv.submit(big)
    assert a is not None
    assert srv.submit(S.dg_request(5, 60, 4, seed=2)) is None  # EXA_EBUSY: does not fit
    for _ in range(4):
        srv.tick()
    assert srv.completed() == [a]
    srv.result(a)
    assert srv.submit(S.dg_request(5, 60, 4, seed=2)) is not None
    srv.destroy()


def test_poisson_stream_small():
    reqs = [S.dg_request(2 + (i % 4), 9 + 3 * i, 20 + i, seed=i) if i % 3 else S.fv_request(64 + 8 * i, 20, seed=i)
            for i in range(12)]
    srv = S.Server(1 << 29)
    res = S.run_poisson(srv, [('x', r) for r in reqs], rate=200.0, seed=0)
    srv.destroy()
    assert len(res['done']) == 12
    assert (res['latency'] > 0).all()
    assert res['cell_updates'] > 0


def test_failed_request_reported_and_others_unchanged():
    """A NaN planted in one live ADER-DG request's state (between ticks, on
    the host side of the call) makes that request finish as failed
    (EXA_ENAN, stopped at the step that produced it) while the other
    requests in the mix complete bit for bit as they do without it."""
    import ctypes as C
    from exahype_b200 import _lib
    mix = [S.dg_request(3, 15, 8, seed=31), S.dg_request(4, 12, 8, seed=32), S.fv_request(80, 8, seed=33),
           S.dg_request(2, 20, 8, seed=34)]
    clean = run_to_completion(S.Server(1 << 28), mix)
    srv = S.Server(1 << 28)
    ids = [srv.submit(r) for r in mix]
    for _ in range(2):
        srv.tick()
    ptr = srv.device_state_ptr(ids[1])
    nan = np.array([np.nan])
    _lib.call('exa_memcpy_h2d', C.c_void_p(ptr + 8 * 77), nan.ctypes.data, 8, None)
    E.device.synchronize()
    got, status = {}, {}
    for _ in range(20):
        srv.tick()
        for rid in srv.completed():
            i = ids.index(rid)
            out, t, steps, st = srv.result(rid, with_status=True)
            got[i] = (out, t, steps)
            status[i] = st
        if len(got) == len(mix):
            break
    srv.destroy()
    assert status[1] == _lib.EXA_ENAN and got[1][2] == 2
    for i in (0, 2, 3):
        assert status[i] == _lib.EXA_OK
        assert np.array_equal(got[i][0], clean[i][0]) and got[i][2] == clean[i][2] == 8


def test_fv_batch_equals_single_patches():
    """FV requests of several sizes and both schemes stepped together in the
    batched serving launch equal each patch stepped alone by the
    single-patch kernels (FVGrid), bit for bit, with requests joining and
    leaving mid-stream."""
    sizes, steps = [64, 100, 37, 256, 90], [6, 9, 4, 7, 5]
    reqs = [S.fv_request(P, k, scheme=1 if i % 2 == 0 else 0, seed=40 + i, noise=1e-3)
            for i, (P, k) in enumerate(zip(sizes, steps))]
    srv = S.Server(1 << 28)
    got = run_to_completion(srv, reqs, submit_at=[0, 1, 0, 3, 2])
    srv.destroy()
    for i, (r, P, k) in enumerate(zip(reqs, sizes, steps)):
        g = E.FVGrid(r.fv_scheme, P)
        g.init(amp=0.2, seed=40 + i, noise=1e-3)
        g.step(k)
        ref, t = g.get_state(), g.status()['time']
        g.destroy()
        assert np.array_equal(got[i][0], ref) and got[i][1] == t and got[i][2] == k, i


def test_evict_restore_continues_bitwise():
    """Evicted requests (state and time-step scalars to host memory, device
    memory back to the arena) restored a few ticks later finish with the
    result of an uninterrupted run, bit for bit, while the other requests
    keep stepping meanwhile; ADER-DG (orders 2 and 4) and both FV schemes."""
    reqs = [S.dg_request(4, 15, 12, ic_param=0.25, seed=3, noise=1e-3),
            S.fv_request(48, 11, scheme=1, ic_param=0.2, seed=4, noise=1e-3),
            S.dg_request(2, 20, 9, seed=5),
            S.fv_request(40, 10, scheme=0, seed=6, noise=1e-3)]
    srv = S.Server(1 << 29)
    ref = run_to_completion(srv, reqs)
    srv.destroy()

    srv = S.Server(1 << 29)
    ids = [srv.submit(r) for r in reqs]
    free0 = None
    out, tick = {}, 0
    while len(out) < len(reqs):
        if tick == 3:
            free0 = srv.info()['arena_free']
            for rid in ids[:2] + ids[3:]:
                srv.evict(rid)
                assert srv.evicted(rid)
            assert srv.info()['arena_free'] > free0
        if tick == 6:
            for rid in ids[:2] + ids[3:]:
                assert srv.restore(rid)
                assert not srv.evicted(rid)
        srv.tick()
        tick += 1
        for rid in srv.completed():
            out[ids.index(rid)] = srv.result(rid)
        assert tick < 1000
    srv.destroy()
    for i in range(len(reqs)):
        assert np.array_equal(ref[i][0], out[i][0]), i
        assert ref[i][1] == out[i][1] and ref[i][2] == out[i][2], i


def test_preemption_admits_a_waiting_request():
    """exa_server_run with eviction after 0.05 s: a small request that does
    not fit beside a long-running large one is admitted by evicting the
    large one, which is restored when memory frees and still ends with its
    uninterrupted result."""
    big = S.dg_request(5, 60, 3000, seed=21)  # runs for about a second
    small = S.fv_request(64, 5, scheme=1, seed=22)
    budget = S.footprint(big) + S.footprint(small) // 2
    assert S.footprint(small) <= budget and S.footprint(big) <= budget
    srv = S.Server(1 << 30)
    alone = run_to_completion(srv, [big])[0]
    srv.destroy()

    srv = S.Server(budget)
    srv.set_eviction(0.05)
    res = S.run_poisson(srv, [('dg', big), ('fv', small)], rate=20.0, seed=1, collect=True, time_limit=120.0)
    srv.destroy()
    assert sorted(res['done']) == [0, 1]
    assert res['evictions'][0] >= 1 and res['evictions'][1] == 0
    # the small request finished before the large one
    assert res['done'][1][0] < res['done'][0][0]
    st, t, steps, state = res['done'][0]
    assert np.array_equal(state, alone[0]) and t == alone[1] and steps == alone[2]


def test_fv_steps_per_tick_same_results():
    """FV requests advancing two or three steps per tick
    (exa_server_set_fv_steps) end with the results of one step per tick,
    bit for bit, including budgets that run out in the middle of a tick."""
    reqs = [S.fv_request(48, 10, scheme=1, seed=31, noise=1e-3), S.dg_request(3, 12, 6, seed=32),
            S.fv_request(33, 7, scheme=0, seed=33, noise=1e-3), S.fv_request(64, 8, scheme=1, seed=34)]
    out = []
    for k in (1, 3, 2):
        srv = S.Server(1 << 29)
        srv.set_fv_steps(k)
        out.append(run_to_completion(srv, reqs, submit_at=[0, 0, 1, 2]))
        srv.destroy()
    for j in (1, 2):
        for i in range(len(reqs)):
            assert np.array_equal(out[0][i][0], out[j][i][0]), (j, i)
            assert out[0][i][1] == out[j][i][1] and out[0][i][2] == out[j][i][2], (j, i)


def test_overlapped_result_hand_out_same_results():
    """exa_server_run hands out results while the next tick runs (result
    mode 1, pinned staging on its own stream) with the same states, times
    and step counts as the synchronous hand-out (mode 0)."""
    reqs = S.request_mix(24, seed=41)
    for _, r in reqs:  # keep the stream small
        if r.kind == S.REQ_ADERDG:
            r.dg.n[0] = r.dg.n[1] = min(r.dg.n[0], 40)
        else:
            r.fv_patch = min(r.fv_patch, 200)
        r.steps = min(r.steps, 30)
    got = []
    # mode 1 twice: the default ring, and a 1 MiB ring that the larger
    # results outgrow and the others wrap around, waiting for older copies
    for mode, staging in ((0, None), (1, None), (1, 1 << 20)):
        srv = S.Server(1 << 30)
        srv.set_result_mode(mode)
        if staging:
            srv.set_staging(staging)
        res = S.run_poisson(srv, reqs, rate=400.0, seed=5, collect=True, time_limit=120.0)
        times = srv.loop_times()
        srv.destroy()
        assert len(res['done']) == len(reqs) and not res['failed']
        assert all(v >= 0.0 for v in times.values()) and times['wait_s'] > 0.0
        got.append(res['done'])
    for j in (1, 2):
        for i in range(len(reqs)):
            a, b = got[0][i], got[j][i]
            assert a[1] == b[1] and a[2] == b[2], (j, i)
            assert np.array_equal(a[3], b[3]), (j, i)
