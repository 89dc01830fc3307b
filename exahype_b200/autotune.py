"""Project autotuner: picks launch/schedule knobs by timing the actual
workload with CUDA events (the measure-then-pick idea of the reference's
shared-memory oracles, Peano/sharedmemoryoracles/, applied to GPU knobs).

tune_ensemble: the contraction per order, then persistent CTAs per SM x
work items per grab (cells per CTA) x work order, for an Ensemble;
tune_contraction: the contraction per order alone, in the current launch form;
tune_predictor: register budget of the predictor kernels
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


def tune_contraction(ens, steps=3, mask=0x30):
    """Coordinate descent over the contraction of each order present
    (line-owner or node-gather; exa_ensemble_tune_contraction) in the
    ensemble's current launch form and schedule, from `mask` (default: the
    library's, orders 4 and 5 line-owner), flipping one order at a time and
    keeping the faster.  Applies the result and returns (mask, table)."""
    table = []
    present = sorted({c.order for c in ens.cfgs.values()})
    if not present:
        return mask, table
    ens.tune_contraction(mask)
    base = _time_ensemble(ens, steps)
    table.append({'stage': 'contraction', 'lines_mask': mask, 'ms_per_step': base})
    for n in present:
        trial = mask ^ (1 << n)
        ens.tune_contraction(trial)
        ms = _time_ensemble(ens, steps)
        table.append({'stage': 'contraction', 'lines_mask': trial, 'ms_per_step': ms})
        if ms < base:
            mask, base = trial, ms
    ens.tune_contraction(mask)
    return mask, table


def tune_ensemble(ens, steps=3, ctas=(1, 2), grabs=(1, 2, 4, 8), orders=(0, 1), contraction=True, modes=(0, 1),
                  cache=None, key=None):
    """Picks the ensemble's knobs by timing `ens` itself (which advances
    while being measured):

    1. the contraction of each order present (line-owner or node-gather;
       exa_ensemble_tune_contraction): coordinate descent from the default,
       flipping one order at a time and keeping the faster;
    2. the persistent schedule: CTAs per SM x work items per atomic grab
       (the cells-per-CTA schedule: a grab takes that many consecutive
       blocks of cells) x work order (costly orders first / solve order),
       every combination timed.

    3. the launch form (among `modes`): the best persistent schedule against
       one launch per order and phase (exa_ensemble_set_launch_mode).

    Applies the fastest and returns (best, table), best =
    (ctas_per_sm, grab, order_policy, lines_mask, launch_mode)."""
    if cache and key and os.path.exists(cache):
        with open(cache) as f:
            got = json.load(f).get(key)
        if got:
            c, g, o, m, lm = got['best']
            ens.tune_contraction(m)
            ens.tune(c, g, o)
            ens.set_launch_mode(lm)
            return tuple(got['best']), got['table']
    table = []
    mask = 0x30  # orders 4 and 5 line-owner: the library's default
    if contraction and ens.cfgs:
        ens.tune(ctas[0], grabs[0], orders[0])
        mask, table = tune_contraction(ens, steps, mask)
    for c, g, o in itertools.product(ctas, grabs, orders):
        ens.tune(c, g, o)
        ms = _time_ensemble(ens, steps)
        table.append({'stage': 'schedule', 'ctas_per_sm': c, 'grab': g, 'order_policy': o, 'ms_per_step': ms})
    best = min((r for r in table if r['stage'] == 'schedule'), key=lambda r: r['ms_per_step'])
    ens.tune(best['ctas_per_sm'], best['grab'], best['order_policy'])
    mode = 0
    if 1 in modes:
        ens.set_launch_mode(1)
        ms = _time_ensemble(ens, steps)
        table.append({'stage': 'launch_mode', 'launch_mode': 1, 'ms_per_step': ms})
        mode = 1 if (ms < best['ms_per_step'] or 0 not in modes) else 0
    ens.set_launch_mode(mode)
    b = (best['ctas_per_sm'], best['grab'], best['order_policy'], mask, mode)
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
