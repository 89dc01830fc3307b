"""Serving over the C++ engine (exa_server_* in include/exa_kernels.h): a
seeded Poisson stream of solve requests handed to the engine's own request
loop (exa_server_run: admission queue for requests that do not fit yet,
continuous batching -- every tick advances all admitted requests, ADER-DG
ones by one step and FV ones by up to set_fv_steps steps -- and
time-to-solution records, all in C++); this module builds the
requests and the arrival times and summarises the records."""
import ctypes as C

import numpy as np

from . import _lib
from ._lib import call, lib
from .ensemble import SolveConfig, solve_config

REQ_ADERDG = 0
REQ_FV = 1


class RequestRecord(C.Structure):
    _fields_ = [('arrival_s', C.c_double), ('admitted_s', C.c_double), ('completed_s', C.c_double),
                ('sim_time', C.c_double), ('steps_done', C.c_longlong), ('status', C.c_int),
                ('evictions', C.c_int)]


class Request(C.Structure):
    _fields_ = [('kind', C.c_int), ('dg', SolveConfig), ('fv_scheme', C.c_int), ('fv_patch', C.c_int),
                ('fv_length', C.c_double), ('steps', C.c_longlong)]


def dg_request(order, n, steps, ic_param=0.2, seed=0, noise=0.0, pde=_lib.PDE_EULER):
    r = Request()
    r.kind = REQ_ADERDG
    r.dg = solve_config(order, (n, n), pde=pde, ic_kind=1, ic_param=ic_param, seed=seed, noise=noise)
    r.steps = steps
    return r


def fv_request(patch, steps, scheme=1, ic_param=0.2, seed=0, noise=0.0, length=1.0, pde=_lib.PDE_EULER):
    r = Request()
    r.kind = REQ_FV
    r.dg = solve_config(2, (1, 1), pde=pde, ic_param=ic_param, seed=seed, noise=noise)
    r.fv_scheme, r.fv_patch, r.fv_length, r.steps = scheme, patch, length, steps
    return r


def footprint(req):
    return int(lib().exa_server_footprint(C.byref(req)))


class Server:
    def __init__(self, hbm_budget, max_requests=512, precision=_lib.PREC_FP64):
        h = C.c_void_p()
        call('exa_server_create', int(hbm_budget), int(max_requests), int(precision), C.byref(h))
        self.h = h

    def submit(self, req):
        """Returns the request id, or None if it does not fit right now."""
        rid = C.c_uint64()
        st = lib().exa_server_submit(self.h, C.byref(req), C.byref(rid))
        if st == _lib.EXA_EBUSY:
            return None
        _lib.check(st, 'exa_server_submit')
        return rid.value

    def tick(self):
        n = C.c_int()
        st = lib().exa_server_tick(self.h, C.byref(n))
        if st not in (_lib.EXA_OK, _lib.EXA_ENAN):
            _lib.check(st, 'exa_server_tick')
        return n.value

    def completed(self, cap=4096):
        ids = (C.c_uint64 * cap)()
        n = C.c_int()
        call('exa_server_completed', self.h, ids, cap, C.byref(n))
        return [ids[i] for i in range(n.value)]

    def result(self, rid, with_status=False):
        """(final state, simulated time, steps done) of a finished request;
        with_status also returns the status: EXA_ENAN for a solve that
        produced a non-finite state (without with_status that raises)."""
        size = int(lib().exa_server_result_size(self.h, C.c_uint64(rid)))
        out = np.empty(size)
        t, steps = C.c_double(), C.c_longlong()
        st = lib().exa_server_result(self.h, C.c_uint64(rid), out.ctypes.data, C.byref(t), C.byref(steps))
        if st != _lib.EXA_OK and not (with_status and st == _lib.EXA_ENAN):
            _lib.check(st, 'exa_server_result')
        if with_status:
            return out, t.value, steps.value, st
        return out, t.value, steps.value

    def evict(self, rid):
        """Moves a running request's state to host memory and frees its
        device memory (exa_server_evict)."""
        call('exa_server_evict', self.h, C.c_uint64(rid))

    def restore(self, rid):
        """Re-admits an evicted request; False when it does not fit now."""
        st = lib().exa_server_restore(self.h, C.c_uint64(rid))
        if st == _lib.EXA_EBUSY:
            return False
        _lib.check(st, 'exa_server_restore')
        return True

    def evicted(self, rid):
        v = C.c_int()
        call('exa_server_evicted', self.h, C.c_uint64(rid), C.byref(v))
        return bool(v.value)

    def set_eviction(self, wait_s):
        """Preemption in run_poisson / exa_server_run after wait_s seconds of
        waiting (0: off)."""
        call('exa_server_set_eviction', self.h, float(wait_s))

    def tune(self, launch_mode=0, use_graph=True):
        """ADER-DG launch form of a tick (0 persistent, 1 per order) and graph replay."""
        call('exa_server_tune', self.h, int(launch_mode), int(bool(use_graph)))

    def set_fv_steps(self, steps):
        """FV steps per tick (exa_server_set_fv_steps)."""
        call('exa_server_set_fv_steps', self.h, int(steps))

    def set_result_mode(self, mode):
        """exa_server_run's result hand-out (exa_server_set_result_mode):
        1 overlapped with the next tick (the default), 0 synchronous."""
        call('exa_server_set_result_mode', self.h, int(mode))

    def set_staging(self, nbytes):
        """Capacity of the pinned staging ring of the overlapped hand-out
        (exa_server_set_staging; default 256 MiB)."""
        call('exa_server_set_staging', self.h, int(nbytes))

    def loop_times(self):
        """Host seconds of the last exa_server_run: launching ticks, waiting
        for them, handing out results, admission and eviction."""
        out = (C.c_double * 4)()
        call('exa_server_loop_times', self.h, out)
        return dict(zip(('launch_s', 'wait_s', 'results_s', 'admission_s'), list(out)))

    def device_state_ptr(self, rid):
        p = C.c_void_p()
        call('exa_server_device_state', self.h, C.c_uint64(rid), C.byref(p))
        return p.value

    def info(self):
        live, cells, free = C.c_int(), C.c_long(), C.c_size_t()
        call('exa_server_info', self.h, C.byref(live), C.byref(cells), C.byref(free))
        return dict(live=live.value, active_dg_cells=cells.value, arena_free=free.value)

    def destroy(self):
        if self.h:
            call('exa_server_destroy', self.h)
            self.h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


def request_mix(n, seed, dg_fraction=0.25):
    """Seeded request mix: ADER-DG (order ~U{2..5}, side log-uniform in
    [9, 243], steps ~U{20..200}) and FV MUSCL-Hancock (side log-uniform in
    [64, 1024], steps ~U{20..200})."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        steps = int(rng.integers(20, 201))
        if rng.random() < dg_fraction:
            side = int(round(np.exp(rng.uniform(np.log(9), np.log(243)))))
            out.append(('dg', dg_request(int(rng.integers(2, 6)), side, steps, ic_param=float(rng.uniform(0.05, 0.3)),
                                         seed=10_000 + i)))
        else:
            side = int(round(np.exp(rng.uniform(np.log(64), np.log(1024)))))
            out.append(('fv', fv_request(side, steps, scheme=1, ic_param=float(rng.uniform(0.05, 0.3)),
                                         seed=20_000 + i)))
    return out


def result_size(req):
    if req.kind == REQ_ADERDG:
        B = req.dg.order + 1
        return req.dg.n[0] * req.dg.n[1] * B * B * 5
    g = 1 if req.fv_scheme == 0 else 2
    return (req.fv_patch + 2 * g) ** 2 * 5


def run_poisson(server, requests, rate, seed, collect=False, time_limit=None):
    """Runs `requests` ((name, Request) pairs) arriving at seeded Poisson
    times (rate per second) through the engine's C++ request loop; returns
    per-request time-to-solution (completion - arrival), throughput and the
    records."""
    rng = np.random.default_rng(seed)
    n = len(requests)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=n))
    reqs = (Request * n)(*[r for _, r in requests])
    rec = (RequestRecord * n)()
    for i in range(n):
        rec[i].arrival_s = float(arrivals[i])
    outs = ptrs = None
    if collect:
        outs = [np.empty(result_size(r)) for _, r in requests]
        ptrs = (C.POINTER(C.c_double) * n)(*[o.ctypes.data_as(C.POINTER(C.c_double)) for o in outs])
    ticks = C.c_uint64()
    _lib.check(lib().exa_server_run(server.h, reqs, rec, n, float(time_limit or 0.0), ptrs, C.byref(ticks)),
               'exa_server_run')
    done, cell_updates, failed = {}, 0, []
    for i in range(n):
        if rec[i].completed_s < 0:
            continue
        r = requests[i][1]
        cells = r.dg.n[0] * r.dg.n[1] if r.kind == REQ_ADERDG else r.fv_patch * r.fv_patch
        cell_updates += cells * rec[i].steps_done
        done[i] = (rec[i].completed_s, rec[i].sim_time, rec[i].steps_done, outs[i] if collect else None)
        if rec[i].status != _lib.EXA_OK:
            failed.append(i)
    wall = max([rec[i].completed_s for i in done] + [0.0])
    lat = np.array([done[i][0] - arrivals[i] for i in sorted(done)])
    return dict(latency=lat, done=done, arrivals=arrivals, wall=wall, ticks=int(ticks.value),
                cell_updates=cell_updates, failed=failed,
                admitted=np.array([rec[i].admitted_s for i in range(n)]),
                evictions=np.array([rec[i].evictions for i in range(n)]))
