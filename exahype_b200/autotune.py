"""Project autotuner: picks launch/schedule knobs by timing the actual
workload with CUDA events (the measure-then-pick idea of the reference's
shared-memory oracles, Peano/sharedmemoryoracles/, applied to GPU knobs).

tune_ensemble: persistent CTAs per SM x work items per grab x work order
for an Ensemble; tune_predictor: register budget of the predictor kernels
(exa_tune_set keys) for a grid.  Results can be cached in a JSON file keyed
by the workload signature."""
import itertools
import json
import os

from ._lib import call
from .device import Timer


def _time_ensemble(ens, steps):
    t = Timer()
    s = ens.stream()
    ens.step(1)  # warm-up (and work-item rebuild)
    t.start(s)
    ens.step(steps)
    t.stop(s)
    return t.elapsed_ms() / steps


def tune_ensemble(ens, steps=3, ctas=(1, 2), grabs=(1, 4), orders=(0, 1), cache=None, key=None):
    """Times every (ctas_per_sm, grab, order_policy) combination on `ens`
    (which advances while being measured), applies the fastest and returns
    (best, table)."""
    if cache and key and os.path.exists(cache):
        with open(cache) as f:
            got = json.load(f).get(key)
        if got:
            ens.tune(*got['best'])
            return tuple(got['best']), got['table']
    table = []
    for c, g, o in itertools.product(ctas, grabs, orders):
        ens.tune(c, g, o)
        ms = _time_ensemble(ens, steps)
        table.append({'ctas_per_sm': c, 'grab': g, 'order_policy': o, 'ms_per_step': ms})
    best = min(table, key=lambda r: r['ms_per_step'])
    b = (best['ctas_per_sm'], best['grab'], best['order_policy'])
    ens.tune(*b)
    if cache and key:
        data = {}
        if os.path.exists(cache):
            with open(cache) as f:
                data = json.load(f)
        data[key] = {'best': list(b), 'table': table}
        with open(cache, 'w') as f:
            json.dump(data, f, indent=1)
    return b, table


def tune_predictor(grid, steps=3, keys=((0, (0, 1)),)):
    """For each (tuning key, candidate values): time `steps` grid steps per
    value, keep the fastest (exa_tune_set)."""
    chosen = {}
    for key, values in keys:
        best = None
        for v in values:
            call('exa_tune_set', key, v)
            t = Timer()
            s = grid.stream()
            grid.step(1)
            t.start(s)
            grid.step(steps)
            t.stop(s)
            ms = t.elapsed_ms()
            if best is None or ms < best[1]:
                best = (v, ms)
        call('exa_tune_set', key, best[0])
        chosen[key] = best
    return chosen
