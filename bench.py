#!/usr/bin/env python3
"""Benchmark of the ADER-DG cell-update path.

Workload (one GPU): 3D compressible Euler, ADER-DG order N=4 (125 nodes per
cell), 81^3 uniform periodic cells on the unit cube, FP64 plain path,
isentropic vortex + seeded uniform density noise of amplitude 1e-3.  A
"step" is one full time step of the whole grid (dt reduction, space-time
predictor + volume integral, Riemann solves, surface integral, update).
Metric: cell-updates/s (one cell advanced one step = 1).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--precision fp64|mixed] [--n 81] [--order 4]

N>1 cuts one periodic 81 x 81 x 81N grid into z-slabs, one per GPU (81^3
cells per GPU, weak scaling): each step exchanges the two boundary face
layers with the neighbouring slabs and reduces the dt minimum over all
ranks; launched one process per GPU by torch.distributed.run; the timing is
the max over ranks.

--impl reference times the reference's own generic CPU kernels (compiled
from its sources into oracle/_ref) on all host cores, each step one whole
step of the grid in the reference's step order.  The default run's CPU
baseline is one such step from the GPU's state after its timed steps, and
the GPU's FP64 and mixed-precision steps from that state are compared with
it over the whole grid (parity_81, mixed.accuracy_vs_oracle).
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# Euler functor operation counts (exahype_b200/csrc/exa_device.cuh):
C_FLUX = 31   # euler_flux, 3 directions
C_EIG = 16    # euler_max_eig, one direction


def flops_per_cell_update(dim, order, kbar, V=5):
    """Algorithmic FLOP per cell-update (k = mean Picard iterations):
    P_iter = d B^(d+1) V B 2 + B^(d+2) V 2 + B^(d+1) (c_F + 5V)
    P_post = B^(d+1) V (d+2) 2 + 2d B^(d-1) V B 4 + d B^d V B 2 + d B^d V 6
             + d B^(d-1) V 8 + B^d V 2 + B^d d (c_lambda + 3)
    Returns (total, predictor share)."""
    B, d = order + 1, dim
    p_iter = d * B ** (d + 1) * V * B * 2 + B ** (d + 2) * V * 2 + B ** (d + 1) * (C_FLUX + 5 * V)
    avg = B ** (d + 1) * V * (d + 2) * 2
    extrap = 2 * d * B ** (d - 1) * V * B * 4
    vi = d * B ** d * V * B * 2
    post_corr = d * B ** d * V * 6 + d * B ** (d - 1) * V * 8 + B ** d * V * 2 + B ** d * d * (C_EIG + 3)
    pred = kbar * p_iter + avg + extrap + vi
    return pred + post_corr, pred


def first_iteration_reuse(dim, order, V=5):
    """FLOP per cell the kernels do not execute: the first Picard iterate is
    luh in every time slice, so iteration 0 evaluates the flux and the
    spatial derivatives of one slice and reuses them for the other B-1
    (identical values; the algorithmic count above keeps them)."""
    B, d = order + 1, dim
    per_slice = d * B ** d * V * B * 2 + B ** d * (C_FLUX + 5 * V)
    return (B - 1) * per_slice


def bytes_per_cell_update(dim, order, V=5):
    """Algorithmic HBM bytes per cell-update: luh read+write, face Q/F
    write + read (2 B^d V 8 + 2 (2d B^(d-1) V 8 2))."""
    B, d = order + 1, dim
    return 2 * B ** d * V * 8 + 2 * (2 * d * B ** (d - 1) * V * 8 * 2)


def predictor_bytes_per_cell(dim, order, V=5):
    """luh read, lduh write, lQhbnd + lFhbnd write."""
    B, d = order + 1, dim
    return 8 * (B ** d * V * 2 + 2 * 2 * d * B ** (d - 1) * V)


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""
    Q = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
         'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
         'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ['nvidia-smi', '-i', str(self.index), '--query-gpu=' + self.Q, '--format=csv,noheader,nounits',
                 '-lms', '200'], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, mx, reasons = [], [], set()
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        for ln in self.lines:
            f = [x.strip() for x in ln.split(',')]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() in ('active', '1'):
                    reasons.add(nm)
        if not sm:
            return None
        return {'sm_mhz': float(np.median(sm)), 'sm_max_mhz': float(max(mx)), 'reasons': sorted(reasons),
                'samples': len(sm)}


def fp64_fma_peak():
    """FP64 FMA TFLOP/s of this GPU from the benchmark's own probe library
    (exahype_b200/libexa_fp64_probe.so, built beside the product library but
    not part of it): the FP64 roofline denominator."""
    import ctypes as C
    so = os.path.join(ROOT, 'exahype_b200', 'libexa_fp64_probe.so')
    P = C.CDLL(so)
    P.exa_probe_fp64_fma_tflops.restype = C.c_int
    P.exa_probe_fp64_fma_tflops.argtypes = [C.POINTER(C.c_double)]
    v = C.c_double()
    rc = P.exa_probe_fp64_fma_tflops(C.byref(v))
    if rc != 0:
        raise RuntimeError('FP64 peak probe failed: cudaError %d' % rc)
    return v.value


def measured_peaks():
    p = os.path.join(ROOT, 'MEASURED_PEAKS.json')
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f), 'measured'
    return {'hbm_gbs': 6650.0, 'bf16_tflops': 1590.0}, 'fallback'


def fp64_predictor_kernel(order):
    """The FP64 predictor kernel the library launches for 3D Euler at this
    order by default (tuning key 3 unset)."""
    if order == 4:
        return 'k_predictor_prog'
    return 'k_predictor_lines' if order >= 4 else 'k_predictor'


def mixed_predictor_kernel(order, variant=0):
    """The mixed-precision predictor kernel for 3D Euler at this order and
    tuning key 2 value."""
    if order == 4 and variant in (0, 4):
        return 'k_predictor_mixed_prog'
    if order == 4 and variant == 3:
        return 'k_predictor_mixed_tc'
    if variant == 1 or (variant == 0 and order < 4):
        return 'k_predictor_mixed'
    return 'k_predictor_mixed_lines'


def ncu_traffic_per_cell(kernel, order):
    """DRAM bytes per cell of the FP64 predictor from the committed ncu summary."""
    p = os.path.join(ROOT, 'profiles', '%s_3d_N%d.md' % (kernel, order))
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith('traffic_bytes_per_cell:'):
            try:
                return float(line.split(':', 1)[1].split()[0])
            except ValueError:
                return None
    return None


# ------------------------------------------------------------ CPU baseline
def reference_step_check(ctx, state):
    """CPU baseline and parity at the benchmark configuration in one pass:
    one whole-grid step of the reference's own kernels (oracle/_ref, all host
    cores; the C oracle when that was not built) from the GPU's state after
    the timed steps is timed, and the GPU's FP64 and mixed-precision steps
    from the same state are compared with it (relative L2 / Linf over the
    whole grid, and the dt)."""
    sys.path.insert(0, os.path.join(ROOT, 'tests'))
    import _oracle as O
    E, args = ctx['E'], ctx['args']
    n, order = args.n, args.order
    cores = os.cpu_count() or 1
    R = O.ref_lib(3)
    kind = 'reference' if R is not None else 'port'
    nn = np.array([n, n, n], dtype=np.int32)
    dx = np.full(3, 1.0 / n)
    def ref_step(u):
        if R is not None:
            return R.ref_grid_step(order, nn, dx, u, 0, 0.0, cores)
        return O.lib().orc_aderdg_grid_step(3, order, 0, nn, dx, u, 0, 0.9, 0.0, None, cores)
    ref = np.ascontiguousarray(state).copy()
    dt_ref = ref_step(ref)  # the step the GPU is compared with (also the warm-up)
    warm = ref.copy()
    t0 = time.perf_counter()
    ref_step(warm)
    t = time.perf_counter() - t0
    del warm
    cpu = {'value': n ** 3 / t, 'unit': 'cell-updates/s', 'cores': cores, 'kind': kind,
           'sample': 'one whole %d^3 grid step (dt + predictor + volume integral + Riemann + surface integral + '
                     'update), the second from the GPU state after the timed steps (the first, untimed, is the '
                     'step the GPU steps are compared with)' % n}
    parity = {'reference': kind, 'from': 'GPU state after warm-up + timed steps, one step on each side'}
    nrm2, nrmi = float(np.linalg.norm(ref)), float(np.abs(ref).max())
    for name, prec in (('fp64', E.PREC_FP64), ('mixed', E.PREC_MIXED)):
        g = E.ADERDGGrid(3, order, (n, n, n), precision=prec)
        g.set_state(state)
        dt = float(g.step(1, want_dt=True)[0])
        got = g.get_state()
        g.destroy()
        d = got - ref
        parity[name] = {'rel_l2': float(np.linalg.norm(d)) / nrm2, 'rel_linf': float(np.abs(d).max()) / nrmi,
                        'dt': dt, 'dt_reference': float(dt_ref), 'dt_rel_diff': abs(dt - dt_ref) / dt_ref,
                        'cells': n ** 3}
        del got, d
    parity['fp64']['bar'] = 1e-12
    parity['mixed']['bar'] = 1e-8
    return cpu, parity


# ---------------------------------------------------------------- reference
def run_reference(args, rank, world):
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, 'tests'))
    import _oracle as O
    n, order = args.n, args.order
    cores = os.cpu_count() or 1
    R = O.ref_lib(3)
    kind = 'reference' if R is not None else 'port'
    dx = np.full(3, 1.0 / n)

    # one step = one whole step of a periodic grid in the reference's order
    # (stableTimeStepSize + global min, predictor + volume integral, Riemann
    # per face, surface integral + update), all host cores, on the n x n
    # cross-section of the benchmark with the benchmark's cell size and as
    # many z-planes (<= n) as fit ~150 s for the whole --warmup + --steps
    # run (the whole n^3 grid takes ~8 s per step on 16 cores); calibrated
    # on a 4-plane slab first
    def grid(nz):
        return O.grid_ic(3, order, (n, n, nz), kind=0, param=5.0, seed=args.seed, noise=1e-3,
                         dx=dx)

    def run(u, nz):
        nn = np.array([n, n, nz], dtype=np.int32)
        if R is not None:
            R.ref_grid_step(order, nn, dx, u, 0, 0.0, cores)
        else:
            O.lib().orc_aderdg_grid_step(3, order, 0, nn, dx, u, 0, 0.9, 0.0, None, cores)
    u = grid(4)
    run(u, 4)
    t0 = time.perf_counter()
    run(u, 4)
    rate = 4 * n * n / max(time.perf_counter() - t0, 1e-6)
    budget = 150.0 / max(1, args.warmup + args.steps)
    nz = int(max(4, min(n, budget * rate / (n * n))))
    u = grid(nz)
    ncells = n * n * nz
    for _ in range(args.warmup):
        run(u, nz)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        run(u, nz)
    t = time.perf_counter() - t0
    value = ncells * args.steps / t
    sample = ('whole periodic %dx%dx%d grid (the benchmark\'s %d^2 cross-section and cell size, %d of its %d '
              'z-planes), every step: dt + predictor + volume integral + Riemann + surface integral + update'
              % (n, n, nz, n, nz, n))
    line = {
        'impl': 'reference', 'metric': METRIC, 'value': value, 'unit': 'cell-updates/s', 'n_gpus': world,
        'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': 1e3 * t / args.steps,
        'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64',
        'data': 'synthetic', 'config': config_dict(args, world),
        'cpu_baseline': {'value': value, 'unit': 'cell-updates/s', 'cores': cores, 'kind': kind,
                         'sample': sample},
        'e2e': {'value': value, 'unit': 'cell-updates/s', 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0},
    }
    print(json.dumps(line), flush=True)


METRIC = '3D Euler ADER-DG N=4 cell-updates/s'


def config_dict(args, world):
    if world == 1:
        wl = '3D Euler ADER-DG N=%d, %d^3 periodic cells, isentropic vortex + 1e-3 density noise' % (
            args.order, args.n)
    else:
        wl = ('3D Euler ADER-DG N=%d, one periodic %dx%dx%d grid cut into %d z-slabs of %d^3 cells, '
              'isentropic vortex + 1e-3 density noise' % (args.order, args.n, args.n, args.n * world, world,
                                                          args.n))
    return {'workload': wl,
            'order': args.order, 'cells': args.n ** 3 * world, 'cells_per_gpu': args.n ** 3,
            'nodes_per_cell': (args.order + 1) ** 3,
            'precision': args.precision, 'dt_policy': 'CFL*PNPM[N], CFL=0.9',
            'l2_flush': 'inputs larger than L2 (state + faces %.1f GB per GPU)' %
                        (args.n ** 3 * (2 * 125 * 5 + 2 * 6 * 25 * 5) * 8 / 1e9 if args.order == 4 else 0),
            'parallelism': 'slab-z%d (NCCL face-layer exchange + dt min)' % world if world > 1 else 'single'}


# ---------------------------------------------------------------- ours
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=20)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='ours', choices=['ours', 'reference'])
    ap.add_argument('--precision', default='fp64', choices=['fp64', 'mixed'])
    ap.add_argument('--n', type=int, default=81)
    ap.add_argument('--order', type=int, default=4)
    ap.add_argument('--seed', type=int, default=2024)
    ap.add_argument('--no-cpu-baseline', action='store_true')
    ap.add_argument('--no-e2e', action='store_true')
    ap.add_argument('--no-mixed', action='store_true')
    ap.add_argument('--no-extras', action='store_true', help='grid workload: skip the ensemble and serving summaries')
    ap.add_argument('--rates', default='', help='serving: comma-separated offered rates (req/s)')
    ap.add_argument('--serving-seconds', type=float, default=20.0, help='serving: seconds of arrivals per rate')
    ap.add_argument('--serving-mode', type=int, default=1, help='serving: ADER-DG launch form (0 persistent, 1 per order: the default)')
    ap.add_argument('--serving-no-graph', action='store_true', help='serving: direct launches instead of graph replay')
    ap.add_argument('--serving-result-mode', type=int, default=1,
                    help='serving: result hand-out (1 overlapped with the next tick: the default, 0 synchronous)')
    ap.add_argument('--serving-fv-steps', type=int, default=3,
                    help='serving: FV steps per tick (exa_server_set_fv_steps)')
    ap.add_argument('--mixed-variant', type=int, default=0,
                    help='contraction of the mixed predictor (tuning key 2): 0 default, 1 node-gather, '
                         '2 line-owner FP32, 3 tensor cores, 4 progressive line-owner (3 and 4: 3D N=4)')
    ap.add_argument('--workload', default='grid3d',
                    choices=['grid3d', 'ensemble', 'serving', 'fv', 'amr', 'limiter'],
                    help='grid3d: the 81^3 N=4 grid (default); ensemble: 512 independent 2D solves; '
                         'serving: Poisson stream of solve requests; fv: one periodic 2D FV patch')
    ap.add_argument('--fv-patch', type=int, default=8192)
    ap.add_argument('--requests', type=int, default=400)
    ap.add_argument('--rate', type=float, default=200.0)
    ap.add_argument('--dg-fraction', type=float, default=0.25)
    ap.add_argument('--nsolves', type=int, default=512)
    ap.add_argument('--ens-orders', default='2,3,4,5', help='ensemble: orders drawn from (comma-separated)')
    ap.add_argument('--ens-sides', default='9,81', help='ensemble: grid sides drawn uniformly from lo,hi')
    ap.add_argument('--limiter-cells', type=int, default=131072)
    ap.add_argument('--tune', action='append', default=[],
                    help='key=value tuning knob passed to exa_tune_set (see include/exa_kernels.h)')
    args = ap.parse_args()
    args.warmup = max(args.warmup, 0)

    rank = int(os.environ.get('RANK', '0'))
    world = int(os.environ.get('WORLD_SIZE', '1'))
    local = int(os.environ.get('LOCAL_RANK', '0'))
    dist = None
    cpu_group = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        # host-side rendezvous, barriers and maxima over gloo; for the grid
        # workload the face layers and the dt minimum move over the
        # library's own NCCL communicator (exahype_b200.slab.NcclRing)
        dist.init_process_group('gloo', timeout=datetime.timedelta(seconds=300))
        cpu_group = dist.group.WORLD

    if args.impl == 'ours':
        import exahype_b200 as E
        E.lib().exa_set_device(local)
        for kv in args.tune:
            k, v = kv.split('=')
            E._lib.call('exa_tune_set', int(k), int(v))
    if args.workload == 'ensemble':
        run_ensemble(args, rank, world, dist)
        return
    if args.workload == 'serving':
        run_serving(args, rank, world, dist)
        return
    if args.workload == 'fv':
        run_fv(args, rank, world, dist)
        return
    if args.workload == 'amr':
        run_amr(args, rank, world, dist)
        return
    if args.workload == 'limiter':
        run_limiter(args, rank, world, dist)
        return
    if args.impl == 'reference':
        run_reference(args, rank, world)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return

    import exahype_b200 as E
    E.lib().exa_set_device(local)
    import ctypes as C
    fp64_peak = C.c_double(fp64_fma_peak())
    peaks, peak_src = measured_peaks()

    def barrier():
        if dist:
            dist.barrier(group=cpu_group)

    def max_over_ranks(x):
        if not dist:
            return x
        import torch
        t = torch.tensor([x], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX, group=cpu_group)
        return float(t.item())

    if args.mixed_variant:
        E._lib.call('exa_tune_set', 2, args.mixed_variant)
    ctx = dict(E=E, args=args, rank=rank, world=world, local=local, barrier=barrier, dist=dist,
               max_over_ranks=max_over_ranks, fp64_peak=fp64_peak.value)
    primary = 'mixed' if args.precision == 'mixed' else 'fp64'
    res = measure(ctx, primary, with_e2e=not args.no_e2e)
    other = None
    if args.precision == 'fp64' and not args.no_mixed:
        other = measure(ctx, 'mixed', with_e2e=False)
        other['accuracy'] = mixed_accuracy(ctx, steps=min(50, args.warmup + args.steps))

    cpu = parity = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu, parity = reference_step_check(ctx, res['state'])
        if other is not None and parity is not None:
            other['accuracy_vs_oracle'] = parity.pop('mixed')

    if rank == 0:
        ncells = res['ncells']
        line = {
            'metric': METRIC, 'value': res['value'], 'unit': 'cell-updates/s', 'n_gpus': world,
            'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': res['ms_per_step'],
            'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None,
            'dtype': 'f64' if primary == 'fp64' else 'f64+f32', 'data': 'synthetic',
            'config': config_dict(args, world),
            'roofline': res['roofline'],
            'roofline_hbm': {
                'achieved': bytes_per_cell_update(3, args.order) * ncells / (res['ms_per_step'] * 1e-3) / 1e9,
                'peak': peaks.get('hbm_gbs'), 'unit': 'GB/s', 'peak_source': peak_src,
                'bytes_per_cell_update': bytes_per_cell_update(3, args.order)},
            'flop_per_cell_update': res['flop_per_cell_update'],
            'cpu_baseline': cpu,
            'parity_81': parity,
            'e2e': res.get('e2e'),
            'gpu_launches': res['launches'],
            'clocks': res['clocks'],
        }
        if other is not None:
            line['mixed'] = {
                'value': other['value'], 'unit': 'cell-updates/s', 'ms_per_step': other['ms_per_step'],
                'speedup_vs_fp64': other['value'] / res['value'], 'roofline': other['roofline'],
                'accuracy_vs_fp64': other['accuracy'], 'accuracy_vs_oracle': other.get('accuracy_vs_oracle'),
                'gpu_launches': other['launches'],
                'clocks': other['clocks'],
                'form': 'Picard deviations dq = q - luh and dF = F(q) - F(luh) in FP32 (FP32 accumulate); '
                        'luh, F(luh) and its derivative, the update, Riemann fluxes, faces and dt in FP64'}
        if world == 1 and not args.no_extras:
            line['ensemble'] = ensemble_summary(args, rank)
            line['serving'] = serving_summary(args)
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier(group=cpu_group)
        dist.destroy_process_group()


class GridRun:
    """The timed grid of this rank.  One GPU: the whole n^3 periodic grid
    (CUDA-graph replay of its steps).  N GPUs: slab `rank` of one periodic
    n x n x (n N) grid (n^3 cells per GPU, weak scaling), its boundary face
    layers and the dt minimum exchanged over NCCL every step."""

    def __init__(self, ctx, prec):
        E, args = ctx['E'], ctx['args']
        n, order, world = args.n, args.order, ctx['world']
        ic = dict(kind=0, param=5.0, seed=args.seed, noise=1e-3)
        self.slab = None
        if world == 1:
            self.g = E.ADERDGGrid(3, order, (n, n, n), precision=prec)
            self.g.init(**ic)
        else:
            from exahype_b200 import slab as SL
            self.SL = SL
            self.slab = SL.SlabGrid(3, order, (n, n, n * world), ctx['rank'], world,
                                    length=(1.0, 1.0, float(world)), precision=prec)
            self.slab.init(**ic)
            self.g = self.slab.grid
            d = ctx['dist']
            uid = [SL.NcclRing.make_id() if ctx['rank'] == 0 else None]
            d.broadcast_object_list(uid, src=0)
            self.ring = SL.NcclRing(ctx['rank'], world, uid[0], timeout_s=60.0)
            self.primed = False
        self.ncells = self.g.ncells
        self.state_size = self.g.state_size

    def step(self, k, per_step_read=False):
        """k steps; per_step_read: each step returns its dt (one GPU) or the
        grid's scalar status (slabs) to the host."""
        if self.slab is None:
            if per_step_read:
                for _ in range(k):
                    self.g.step(1, want_dt=True)
            else:
                self.g.step(k)
            return
        if not self.primed:
            self.SL.prime(self.ring, self.slab)
            self.primed = True
        for _ in range(k if per_step_read else 1):
            self.SL.step(self.ring, self.slab, 1 if per_step_read else k)
            if per_step_read:
                self.g.status()

    def set_state_ptr(self, ptr):
        self.E_call('exa_aderdg_grid_set_state', ptr)
        if self.slab is not None:
            self.primed = False

    def get_state_ptr(self, ptr):
        self.E_call('exa_aderdg_grid_get_state', ptr)

    def E_call(self, name, ptr):
        from exahype_b200 import _lib
        _lib.call(name, self.g.h, ptr)

    def per_step_d2h_bytes(self):
        return 8 if self.slab is None else 56

    def destroy(self):
        if self.slab is not None:
            self.slab.destroy()
            self.ring.destroy()
        else:
            self.g.destroy()


def measure(ctx, precision, with_e2e):
    """Time K steps of the grid on this rank (W untimed warm-up steps
    first); returns the rank-0 view of the numbers."""
    E, args = ctx['E'], ctx['args']
    from exahype_b200 import Timer
    n, order = args.n, args.order
    prec = E.PREC_MIXED if precision == 'mixed' else E.PREC_FP64
    run = GridRun(ctx, prec)
    grid = run.g
    stream = grid.stream()
    initial = grid.get_state() if with_e2e else None
    run.step(args.warmup)
    st0 = grid.status()
    grid.profile(True)
    E.device.synchronize()
    ctx['barrier']()
    clocks = ClockSampler(ctx['local'])
    clocks.start()
    timer = Timer()
    l0 = E.launch_count()
    timer.start(stream)
    run.step(args.steps)
    timer.stop(stream)
    ms = timer.elapsed_ms()
    E.device.synchronize()
    launches = E.launch_count() - l0
    ctx['barrier']()
    clk = clocks.stop()
    st1 = grid.status()
    phases = grid.phase_times()
    ms_max = ctx['max_over_ranks'](ms)
    ncells = run.ncells
    value = ctx['world'] * ncells * args.steps / (ms_max * 1e-3)
    kbar = (st1['picard_iters'] - st0['picard_iters']) / (ncells * args.steps)
    total_flop, pred_flop = flops_per_cell_update(3, order, kbar)
    pred_ms = phases['predictor_ms'] / max(1, phases['steps'])
    achieved = pred_flop * ncells / (pred_ms * 1e-3) / 1e12
    kernel = fp64_predictor_kernel(order)
    traffic_pc = ncu_traffic_per_cell(kernel, order) if precision == 'fp64' else None
    out = dict(value=value, ms_per_step=ms_max / args.steps, ncells=ncells, launches=launches, clocks=clk,
               flop_per_cell_update=total_flop)
    if precision == 'fp64':
        out['roofline'] = {
            'kernel': kernel, 'bound': 'fp64', 'achieved': achieved, 'peak': ctx['fp64_peak'],
            'unit': 'TFLOP/s', 'frac': achieved / ctx['fp64_peak'],
            'peak_source': 'DFMA probe measured in this run (MEASURED_PEAKS.json has no FP64 figure)',
            'flop_per_cell': pred_flop, 'picard_mean_iterations': kbar,
            'flop_per_cell_executed': pred_flop - first_iteration_reuse(3, order),
            'achieved_executed': (pred_flop - first_iteration_reuse(3, order)) * ncells / (pred_ms * 1e-3) / 1e12,
            'traffic': (traffic_pc * ncells if traffic_pc else None), 'ms_per_launch': pred_ms,
            'share_of_step': phases['predictor_ms'] / max(1e-9, phases['predictor_ms'] + phases['corrector_ms'])}
    else:
        out['roofline'] = {
            'kernel': mixed_predictor_kernel(order, args.mixed_variant), 'bound': 'fp64+fp32',
            'achieved_equiv_fp64_flop': achieved,
            'unit': 'TFLOP/s', 'flop_per_cell': pred_flop, 'picard_mean_iterations': kbar,
            'ms_per_launch': pred_ms, 'frac_of_fp64_peak': achieved / ctx['fp64_peak'],
            'share_of_step': phases['predictor_ms'] / max(1e-9, phases['predictor_ms'] + phases['corrector_ms'])}
    if with_e2e:
        from exahype_b200 import PinnedBuffer
        pin = PinnedBuffer(grid.state_size)
        pin.array[:] = initial
        grid.profile(False)
        ctx['barrier']()
        t2 = Timer()
        t2.start(stream)
        run.set_state_ptr(pin.array.ctypes.data)
        run.step(args.steps, per_step_read=True)
        run.get_state_ptr(pin.array.ctypes.data)
        t2.stop(stream)
        ms_e2e = ctx['max_over_ranks'](t2.elapsed_ms())
        ctx['barrier']()
        sb = grid.state_size * 8
        out['e2e'] = {'value': ctx['world'] * ncells * args.steps / (ms_e2e * 1e-3), 'unit': 'cell-updates/s',
                      'h2d_bytes_per_step': sb / args.steps,
                      'd2h_bytes_per_step': run.per_step_d2h_bytes() + sb / args.steps,
                      'note': 'one solve per timed region: state upload from pinned host memory, K steps each '
                              'returning its dt to the host, final state download'}
        pin.free()
    if ctx['rank'] == 0 and precision == 'fp64' and ctx['world'] == 1:
        out['state'] = grid.get_state()
        out['dt'] = grid.step(1, want_dt=True)[0]
    run.destroy()
    return out


def mixed_accuracy(ctx, steps):
    """Relative L2 / Linf of the mixed-precision state against the FP64 path
    after every step, both started from the identical state."""
    E, args = ctx['E'], ctx['args']
    from exahype_b200.device import diff_norms
    n, order = args.n, args.order
    a = E.ADERDGGrid(3, order, (n, n, n), precision=E.PREC_FP64)
    b = E.ADERDGGrid(3, order, (n, n, n), precision=E.PREC_MIXED)
    for g in (a, b):
        g.init(kind=0, param=5.0, seed=args.seed + ctx['rank'], noise=1e-3)
    l2, linf = [], []
    for _ in range(steps):
        a.step(1, want_dt=True)  # synchronises the grid's stream
        b.step(1, want_dt=True)
        e = diff_norms(b.device_state_ptr(), a.device_state_ptr(), a.state_size)
        l2.append(e['rel_l2'])
        linf.append(e['rel_linf'])
    a.destroy()
    b.destroy()
    return {'steps': steps, 'rel_l2_per_step': l2, 'rel_linf_per_step': linf, 'max_rel_l2': max(l2),
            'max_rel_linf': max(linf), 'target_rel_l2': 1e-8}


def ensemble_summary(args, rank):
    """The ensemble workload (512 seeded 2D solves) in brief, for the
    default run's line."""
    import argparse as _ap
    a = _ap.Namespace(**vars(args))
    a.steps, a.warmup = 10, 3
    out = ensemble_measure(a, rank, None)
    keep = ('value', 'ms_per_step', 'cells', 'launches_per_step', 'tuned', 'form', 'per_order_launches')
    res = {k: {kk: out[k][kk] for kk in keep if kk in out[k]} for k in ('fp64', 'mixed')}
    res['mixed']['max_rel_l2_vs_fp64_first16'] = out['mixed'].get('max_rel_l2_vs_fp64_first16')
    res['mixed_speedup'] = out['mixed']['value'] / out['fp64']['value']
    res['workload'] = '%d independent 2D Euler solves, sides 9..81, N 2..5, one persistent launch per step' % a.nsolves
    res['unit'] = 'cell-updates/s'
    return res


def serving_summary(args):
    """One steady-state serving stream at the stated 200 req/s (60 s of
    arrivals) for the default run's line."""
    from exahype_b200 import serving as S
    srv = S.Server(64 << 30, max_requests=4096)
    srv.set_fv_steps(args.serving_fv_steps)
    srv.set_result_mode(args.serving_result_mode)
    S.run_poisson(srv, [('dg', S.dg_request(o, 9, 3)) for o in (2, 3, 4, 5)] + [('fv', S.fv_request(64, 3))],
                  rate=1e4, seed=1)
    r = serving_stream(S, srv, 200.0, 60.0, args.seed + 500, args.dg_fraction)
    srv.destroy()
    r['workload'] = ('Poisson stream, 25 % ADER-DG 2D (N 2..5, 9^2..243^2) and 75 % FV MUSCL-Hancock '
                     '(64^2..1024^2), 20..200 steps each, C++ request loop')
    return r


# ---------------------------------------------------------------- ensemble
def ensemble_mix(nsolves, seed, orders=(2, 3, 4, 5), sides=(9, 81)):
    """Seeded ensemble: grid side ~U{9..81}, order ~U{2..5}, sine-wave
    density amplitude ~U(0.05, 0.3) (the default mix; other orders and
    sides for per-order measurements)."""
    rng = np.random.default_rng(seed)
    return [(int(orders[rng.integers(0, len(orders))]), int(rng.integers(sides[0], sides[1] + 1)),
             float(rng.uniform(0.05, 0.3)), int(1000 + i)) for i in range(nsolves)]


def run_ensemble(args, rank, world, dist):
    """All solves advanced by one persistent launch per step (CUDA-graph
    replayed), schedule picked by the autotuner; FP64 and mixed precision."""
    import exahype_b200 as E
    E.lib().exa_set_device(int(os.environ.get('LOCAL_RANK', '0')))
    out = ensemble_measure(args, rank, dist)
    if rank == 0:
        line = {'metric': '2D Euler ADER-DG ensemble cell-updates/s (512 solves, N in 2..5, 9^2..81^2 cells)',
                'value': out['fp64']['value'] * world, 'unit': 'cell-updates/s', 'n_gpus': world,
                'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': out['fp64']['ms_per_step'],
                'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64',
                'data': 'synthetic', 'config': {'workload': 'ensemble of %d 2D solves, one persistent launch per '
                                                            'step in a CUDA graph' % args.nsolves,
                                                'cells': out['fp64']['cells']},
                'fp64': out['fp64'], 'mixed': out['mixed'],
                'mixed_speedup': out['mixed']['value'] / out['fp64']['value']}
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def ensemble_measure(args, rank, dist):
    """FP64 and mixed-precision runs of the seeded ensemble (autotuned
    schedule, graph-replayed steps); returns their figures."""
    import exahype_b200 as E
    from exahype_b200 import Timer
    from exahype_b200.autotune import tune_contraction, tune_ensemble
    mix = ensemble_mix(args.nsolves, args.seed + rank, tuple(int(x) for x in args.ens_orders.split(',')),
                       tuple(int(x) for x in args.ens_sides.split(',')))
    out = {}
    for prec_name, prec in (('fp64', E.PREC_FP64), ('mixed', E.PREC_MIXED)):
        cfgs = [E.solve_config(o, (n, n), ic_kind=1, ic_param=amp, seed=sd, noise=0.0) for o, n, amp, sd in mix]
        arena = int(sum(E.ensemble.footprint(c) for c in cfgs) * 1.05) + (1 << 24)
        ens = E.Ensemble(len(cfgs), arena, precision=prec)
        for c in cfgs:
            assert ens.add(c) is not None
        # the specified form first: one persistent launch per step, its
        # contraction per order and schedule autotuned
        best, table = tune_ensemble(ens, steps=3, modes=(0,))
        ens.use_graph(True)

        def timed():
            ens.step(args.warmup)
            ens.synchronize()
            st0 = ens.status()
            if dist:
                dist.barrier()
            t = Timer()
            s = ens.stream()
            l0 = E.launch_count()
            t.start(s)
            ens.step(args.steps)
            t.stop(s)
            ms = t.elapsed_ms()
            launches = E.launch_count() - l0
            st1 = ens.status()
            steps_done = (st1['steps'] - st0['steps']).astype(np.int64)
            updates = sum(int(steps_done[sl]) * c.n[0] * c.n[1] for sl, c in ens.cfgs.items())
            return updates / (ms * 1e-3), ms / args.steps, launches / args.steps
        value, ms_step, lps = timed()
        cells = ens.active_cells()
        # the same step as one launch per order and phase (replayed as one
        # graph), its contraction per order tuned again in that form (each
        # order's kernel has its own occupancy there)
        ens.set_launch_mode(1)
        mask1, _ = tune_contraction(ens, steps=3, mask=best[3])
        v1, ms1, lps1 = timed()
        ens.set_launch_mode(0)
        ens.tune_contraction(best[3])
        out[prec_name] = {'value': value, 'ms_per_step': ms_step, 'cells': cells, 'launches_per_step': lps,
                          'form': 'one persistent cooperative launch per step, CUDA-graph replay',
                          'tuned': {'ctas_per_sm': best[0], 'grab': best[1], 'order_policy': best[2],
                                    'line_owner_orders': [n for n in range(2, 6) if (best[3] >> n) & 1]},
                          'tuning_table': table,
                          'per_order_launches': {'value': v1, 'ms_per_step': ms1, 'graph_launches_per_step': lps1,
                                                 'speedup_vs_persistent': v1 / value,
                                                 'line_owner_orders': [n for n in range(2, 6) if (mask1 >> n) & 1],
                                                 'form': 'one launch per order and phase + commit, one graph'}}
        if prec_name == 'fp64':
            ref_states = {sl: ens.get_state(sl) for sl in list(ens.cfgs)[:16]}
        else:
            errs = [float(np.linalg.norm(ens.get_state(sl) - r) / np.linalg.norm(r)) for sl, r in ref_states.items()]
            out['mixed']['max_rel_l2_vs_fp64_first16'] = max(errs)
        ens.destroy()
    return out


# ---------------------------------------------------------------- FV
# Algorithmic FP64 work per FV cell-update (C_FLUX = 31 per flux vector,
# C_EIG = 16 per max-eigenvalue, as for ADER-DG):
#   Godunov: 2 Rusanov faces (2 eig + 2 flux + 20) + update (40) + next dt (2 eig + 4)
#   MUSCL-Hancock: + minmod slopes / extrapolation (70) + half-step (4 flux + 60)

def fv_flop_per_cell(scheme):
    faces = 2 * (2 * 16 + 2 * 31 + 20)
    base = faces + 40 + (2 * 16 + 4)
    return base if scheme == 0 else base + 70 + 4 * 31 + 60


def run_fv(args, rank, world, dist):
    """One periodic 2D FV patch per GPU (replicas over GPUs), MUSCL-Hancock
    (headline) and Godunov, fused device-resident steps."""
    import exahype_b200 as E
    from exahype_b200 import PinnedBuffer, Timer
    local = int(os.environ.get('LOCAL_RANK', '0'))
    E.lib().exa_set_device(local)
    import ctypes as C
    fp64_peak = C.c_double(fp64_fma_peak())
    peaks, peak_src = measured_peaks()
    P = args.fv_patch
    out = {}
    for scheme, name in ((1, 'musclhancock'), (0, 'godunov')):
        g = E.FVGrid(scheme, P)
        g.init(amp=0.2, seed=args.seed + rank, noise=1e-3)
        q0 = g.get_state() if scheme == 1 else None
        g.step(args.warmup)
        stream = g.stream()
        E.device.synchronize()
        if dist:
            dist.barrier()
        clocks = ClockSampler(local)
        clocks.start()
        t = Timer()
        l0 = E.launch_count()
        t.start(stream)
        g.step(args.steps)
        t.stop(stream)
        ms = t.elapsed_ms()
        launches = E.launch_count() - l0
        clk = clocks.stop()
        if dist:
            import torch
            x = torch.tensor([ms], dtype=torch.float64)
            dist.all_reduce(x, op=dist.ReduceOp.MAX)
            ms = float(x.item())
        cells = P * P
        ups = world * cells * args.steps / (ms * 1e-3)
        per = ms / args.steps
        bytes_alg = 80.0 * cells  # state read + write per cell-update
        flop = fv_flop_per_cell(scheme) * cells
        hbm = bytes_alg / (per * 1e-3) / 1e9
        tf = flop / (per * 1e-3) / 1e12
        # the bound follows the arithmetic intensity: FLOP per algorithmic
        # byte against the ridge of the measured FP64 and HBM peaks
        intensity = fv_flop_per_cell(scheme) / 80.0
        ridge = fp64_peak.value * 1e12 / (peaks['hbm_gbs'] * 1e9) if peaks.get('hbm_gbs') else None
        fp64_bound = ridge is not None and intensity > ridge
        r = {'value': ups, 'ms_per_step': per, 'gpu_launches': launches, 'clocks': clk,
             'roofline': {'kernel': 'k_fv_muscl_periodic' if scheme else
                          ('k_fv_godunov<fused>' if '5=1' in args.tune else 'k_fv_godunov_sweep'),
                          'bound': 'fp64' if fp64_bound else 'hbm',
                          'achieved': tf if fp64_bound else hbm,
                          'peak': fp64_peak.value if fp64_bound else peaks.get('hbm_gbs'),
                          'unit': 'TFLOP/s' if fp64_bound else 'GB/s',
                          'frac': (tf / fp64_peak.value) if fp64_bound else
                                  (hbm / peaks['hbm_gbs'] if peaks.get('hbm_gbs') else None),
                          'intensity_flop_per_byte': intensity, 'ridge_flop_per_byte': ridge,
                          'hbm_achieved_gbs': hbm, 'hbm_peak_gbs': peaks.get('hbm_gbs'),
                          'hbm_frac': hbm / peaks['hbm_gbs'] if peaks.get('hbm_gbs') else None,
                          'fp64_achieved_tflops': tf, 'fp64_peak_tflops': fp64_peak.value,
                          'fp64_frac': tf / fp64_peak.value, 'flop_per_cell_update': fv_flop_per_cell(scheme),
                          'bytes_per_cell_update': 80, 'peak_source': peak_src + ' (HBM); DFMA probe (FP64)',
                          'note': 'step time includes the one-thread commit launch'}}
        if scheme == 1:
            pin = PinnedBuffer(g.state_size)
            pin.array[:] = q0
            if dist:
                dist.barrier()
            t2 = Timer()
            t2.start(stream)
            E._lib.call('exa_fv_grid_set_state', g.h, pin.array.ctypes.data)
            for _ in range(args.steps):
                g.step(1)
                g.status()
            E._lib.call('exa_fv_grid_get_state', g.h, pin.array.ctypes.data)
            t2.stop(stream)
            ms2 = t2.elapsed_ms()
            sb = g.state_size * 8
            r['e2e'] = {'value': world * cells * args.steps / (ms2 * 1e-3), 'unit': 'cell-updates/s',
                        'h2d_bytes_per_step': sb / args.steps, 'd2h_bytes_per_step': 16 + sb / args.steps,
                        'note': 'state upload from pinned host memory, K steps each returning time and dt '
                                'to the host, final state download'}
            pin.free()
        out[name] = r
        g.destroy()
    # the reference's FV layout: a grid of 10x10-subcell patches exchanging
    # ghost layers every step (EulerFV demonstrator patch size)
    for scheme, name in ((1, 'musclhancock_patches10'), (0, 'godunov_patches10')):
        npx = max(1, P // 10)
        g = E.FVPatchGrid(scheme, 10, npx, npx)
        g.init(amp=0.2, seed=args.seed + rank, noise=1e-3)
        g.step(args.warmup)
        stream = g.stream()
        E.device.synchronize()
        if dist:
            dist.barrier()
        t = Timer()
        l0 = E.launch_count()
        t.start(stream)
        g.step(args.steps)
        t.stop(stream)
        ms = t.elapsed_ms()
        launches = E.launch_count() - l0
        cells = g.ncells
        out[name] = {'value': world * cells * args.steps / (ms * 1e-3), 'ms_per_step': ms / args.steps,
                     'cells': cells, 'patches': npx * npx, 'gpu_launches': launches,
                     'hbm_gbs_algorithmic': 80.0 * cells / (ms / args.steps * 1e-3) / 1e9}
        g.destroy()
    if rank == 0:
        m = out['musclhancock']
        line = {'metric': '2D Euler FV MUSCL-Hancock cell-updates/s', 'value': m['value'],
                'unit': 'cell-updates/s', 'n_gpus': world, 'steps': args.steps, 'warmup': args.warmup,
                'ms_per_step': m['ms_per_step'], 'higher_is_better': True, 'scaling': 'weak',
                'vs_baseline': None, 'dtype': 'f64', 'data': 'synthetic',
                'config': {'workload': 'one periodic %d^2 FV patch per GPU, density sine + 1e-3 noise' % P,
                           'l2_flush': 'inputs larger than L2 (%.1f GB per state copy)' % ((P + 4) ** 2 * 40 / 1e9),
                           'parallelism': 'replicas%d' % world if world > 1 else 'single'},
                'roofline': m['roofline'], 'e2e': m.get('e2e'), 'gpu_launches': m['gpu_launches'],
                'clocks': m['clocks'], 'godunov': out['godunov'],
                'patch_grid_10': {'musclhancock': out['musclhancock_patches10'],
                                  'godunov': out['godunov_patches10']}}
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


# ---------------------------------------------------------------- AMR
def run_amr(args, rank, world, dist):
    """AMR transfer operators on 3D N=4 cells: every coarse cell prolonged
    into one descendant and every fine cell restricted into its own parent
    slot (one level), items resident on the GPU."""
    import exahype_b200 as E
    from exahype_b200 import DeviceBuffer, Timer
    from exahype_b200.aderdg import amr_prolongation, amr_restriction
    E.lib().exa_set_device(int(os.environ.get('LOCAL_RANK', '0')))
    peaks, peak_src = measured_peaks()
    k, order, count = 3, args.order, 200000
    n = (order + 1) ** k * 5
    rng = np.random.default_rng(args.seed)
    coarse = DeviceBuffer.from_array(rng.standard_normal(count * n))
    fine = DeviceBuffer(count * n)
    idx = np.zeros((count, 3), np.int32)
    idx[:, :k] = rng.integers(0, 3, size=(count, k))
    d_i = DeviceBuffer.from_array(idx)
    out = {}
    for name, fn in (('prolongation', lambda: amr_prolongation(k, order, count, fine, coarse, 1, d_i)),
                     ('restriction', lambda: amr_restriction(k, order, count, coarse, fine, 1, d_i))):
        for _ in range(args.warmup):
            fn()
        E.device.synchronize()
        t = Timer()
        t.start(None)
        for _ in range(args.steps):
            fn()
        t.stop(None)
        ms = t.elapsed_ms() / args.steps
        moved = count * n * 8 * (2 if name == 'prolongation' else 3)  # read in (+ read out) + write out
        out[name] = {'ms_per_call': ms, 'items_per_s': world * count / (ms * 1e-3),
                     'hbm_gbs': moved / (ms * 1e-3) / 1e9,
                     'hbm_frac': moved / (ms * 1e-3) / 1e9 / peaks['hbm_gbs'] if peaks.get('hbm_gbs') else None}
    if rank == 0:
        line = {'metric': 'AMR volume transfers (3D N=%d, one level) items/s' % order,
                'value': out['prolongation']['items_per_s'], 'unit': 'items/s', 'n_gpus': world,
                'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': out['prolongation']['ms_per_call'],
                'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64',
                'data': 'synthetic', 'config': {'workload': '%d cells of 3D N=%d, random child index' % (count, order)},
                'roofline': {'bound': 'hbm', 'peak_source': peak_src}, **out}
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def explosion_state(order, n, radius=0.25):
    """nodal Euler state of a periodic unit square, cells x fastest: density
    1 / pressure 1 inside the circle of `radius` around the centre, 0.125 /
    0.1 outside, at rest"""
    xi = (np.polynomial.legendre.leggauss(order + 1)[0] + 1) / 2
    X = (np.arange(n)[None, :, None, None] + xi[None, None, None, :]) / n
    Y = (np.arange(n)[:, None, None, None] + xi[None, None, :, None]) / n
    X, Y = np.broadcast_arrays(X, Y)
    inside = (X - 0.5) ** 2 + (Y - 0.5) ** 2 < radius ** 2
    q = np.zeros(X.shape + (5,))
    q[..., 0] = np.where(inside, 1.0, 0.125)
    q[..., 4] = np.where(inside, 1.0, 0.1) / 0.4
    return q.reshape(-1)


def explosion_state_3d(order, n, radius=0.25):
    """3D counterpart of explosion_state (sphere in the periodic unit cube)"""
    xi = (np.polynomial.legendre.leggauss(order + 1)[0] + 1) / 2
    c = np.arange(n)
    X = (c[None, None, :, None, None, None] + xi[None, None, None, None, None, :]) / n
    Y = (c[None, :, None, None, None, None] + xi[None, None, None, None, :, None]) / n
    Z = (c[:, None, None, None, None, None] + xi[None, None, None, :, None, None]) / n
    X, Y, Z = np.broadcast_arrays(X, Y, Z)
    inside = (X - 0.5) ** 2 + (Y - 0.5) ** 2 + (Z - 0.5) ** 2 < radius ** 2
    q = np.zeros(X.shape + (5,))
    q[..., 0] = np.where(inside, 1.0, 0.125)
    q[..., 4] = np.where(inside, 1.0, 0.1) / 0.4
    return q.reshape(-1)


def limiting_grid_measure(E, Timer, args, order=3, n=729, steps=20, dim=2):
    """ms per step of the limiting grid and of the same grid unlimited"""
    res = {'workload': '%d^%d cells %dD N=%d, %s explosion, Godunov subcells'
                       % (n, dim, dim, order, 'cylindrical' if dim == 2 else 'spherical'),
           'steps': steps}
    state = explosion_state(order, n) if dim == 2 else explosion_state_3d(order, n)
    for name in ('unlimited', 'limited'):
        g = E.ADERDGGrid(dim, order, (n,) * dim, length=(1.0,) * dim)
        g.set_state(state)
        if name == 'limited':
            g.set_limiter()
        g.use_graph(True)
        g.step(max(args.warmup, 3))
        stream = g.stream()
        t = Timer()
        l0 = E.launch_count()
        t.start(stream)
        g.step(steps)
        t.stop(stream)
        ms = t.elapsed_ms() / steps
        E.device.synchronize()
        res[name] = {'ms_per_step': ms, 'cell_updates_per_s': n ** dim / (ms * 1e-3),
                     'gpu_launches_per_step': (E.launch_count() - l0) / steps}
        if name == 'limited':
            _, counts = g.limiter_status()
            res[name].update({'cells_with_patch': int(counts[0]), 'fv_cells': int(counts[1]),
                              'troubled_cells': int(counts[2])})
        del g
    res['limiting_overhead'] = res['limited']['ms_per_step'] / res['unlimited']['ms_per_step'] - 1
    return res


def fv3d_measure(E, Timer, args, patch=9, npatches=32768):
    """3D Godunov / MUSCL-Hancock on batches of 9^3 patches (the subcell
    patches of N=4 cells), inputs larger than L2"""
    from exahype_b200 import DeviceBuffer
    from exahype_b200.fv import FVPatches
    res = {'workload': '%d patches of %d^3 cells' % (npatches, patch)}
    rng = np.random.default_rng(args.seed)
    for name, scheme, g in (('godunov', 0, 1), ('musclhancock', 1, 2)):
        S = patch + 2 * g
        u = np.zeros((npatches, S ** 3, 5))
        u[..., 0] = 1.0 + 0.1 * rng.random((npatches, S ** 3))
        u[..., 4] = 2.5
        d_old, d_new = DeviceBuffer.from_array(u.reshape(-1)), DeviceBuffer.from_array(u.reshape(-1))
        fv = FVPatches(patch, g, [1.0, 1.0, 1.0], dim=3)
        f = fv.godunov_update if scheme == 0 else fv.musclhancock_update
        for _ in range(3):
            f(npatches, d_new, d_old, 1e-4)
        E.device.synchronize()
        t = Timer()
        t.start(None)
        for _ in range(args.steps):
            f(npatches, d_new, d_old, 1e-4)
        t.stop(None)
        ms = t.elapsed_ms() / args.steps
        cells = npatches * patch ** 3
        res[name] = {'ms_per_call': ms, 'cell_updates_per_s': cells / (ms * 1e-3),
                     'hbm_gbs_at_80B': cells * 80 / (ms * 1e-3) / 1e9}
        del d_old, d_new
    return res


def run_limiter(args, rank, world, dist):
    """Limiter kernels on 3D N=4 cells resident on the GPU: DG -> FV subcell
    projection into patches with one ghost layer, FV -> DG projection back,
    and the DMP check with its min/max search (5 observables); inputs larger
    than L2."""
    import ctypes as C
    import exahype_b200 as E
    from exahype_b200 import DeviceBuffer, Timer, limiter
    E.lib().exa_set_device(int(os.environ.get('LOCAL_RANK', '0')))
    peaks, peak_src = measured_peaks()
    dim, order, count, ghost, V = 3, args.order, args.limiter_cells, 1, 5
    B, S = order + 1, 2 * order + 1
    n_luh, n_lim = B ** dim * V, (S + 2 * ghost) ** dim * V
    rng = np.random.default_rng(args.seed)
    luh_h = rng.uniform(0.5, 2.0, count * n_luh)
    luh = DeviceBuffer.from_array(luh_h)
    lim = DeviceBuffer(count * n_lim)
    lim.zero()
    back = DeviceBuffer(count * n_luh)
    nb = 2 * dim * V
    bmin = DeviceBuffer.from_array(np.full(count * nb, 0.4))
    bmax = DeviceBuffer.from_array(np.full(count * nb, 2.2))
    ok = DeviceBuffer(count, dtype=np.int32)
    lu_b, li_b = n_luh * 8, S ** dim * V * 8
    kernels = (
        ('project_on_fv', lambda: limiter.project_on_fv(dim, order, count, luh, lim, ghost=ghost), lu_b + li_b),
        ('project_on_dg', lambda: limiter.project_on_dg(dim, order, count, lim, back, ghost=ghost), lu_b + li_b),
        ('dmp', lambda: limiter.dmp(dim, order, count, luh, bmin, bmax, ok, 1e-4, 1e-3),
         lu_b + 2 * nb * 8 + 2 * 2 * V * 8 + 4),
    )
    out = {}
    for name, fn, bytes_per_cell in kernels:
        for _ in range(max(args.warmup, 3)):
            fn()
        E.device.synchronize()
        t = Timer()
        t.start(None)
        for _ in range(args.steps):
            fn()
        t.stop(None)
        ms = t.elapsed_ms() / args.steps
        gbs = count * bytes_per_cell / (ms * 1e-3) / 1e9
        out[name] = {'ms_per_call': ms, 'cells_per_s': world * count / (ms * 1e-3),
                     'bytes_per_cell': bytes_per_cell, 'hbm_gbs': gbs,
                     'hbm_frac': gbs / peaks['hbm_gbs'] if peaks.get('hbm_gbs') else None}
    # limiting ADER-DG grid: 2D N=3 cylindrical explosion (discontinuous
    # density and pressure), with and without the limiter, graph-replayed
    lg = limiting_grid_measure(E, Timer, args)
    lg3 = limiting_grid_measure(E, Timer, args, order=4, n=48, steps=10, dim=3)
    fv3 = fv3d_measure(E, Timer, args)
    # CPU baseline: the reference's own Limiter.cpp (oracle/_ref) on a sample
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        so = os.path.join(ROOT, 'oracle', '_ref', 'libexa_ref3d.so')
        if os.path.exists(so):
            R = C.CDLL(so)
            R.ref_limiter.restype = C.c_int
            R.ref_limiter.argtypes = [C.c_int] * 5 + [C.c_void_p] * 4 + [C.c_double] * 2
            sample = 256
            src = np.ascontiguousarray(luh_h[:sample * n_luh])
            dst = np.zeros(n_lim)
            t0 = time.perf_counter()
            for c in range(sample):
                R.ref_limiter(0, order, V, V, ghost, src[c * n_luh:].ctypes.data, dst.ctypes.data, None, None,
                              0.0, 0.0)
            dt = time.perf_counter() - t0
            cpu = {'value': sample / dt, 'unit': 'cells/s', 'cores': 1, 'kind': 'reference',
                   'sample': 'projectOnFVLimiterSpace of %d cells, one thread' % sample}
    if rank == 0:
        line = {'metric': 'limiter DG->FV subcell projection (3D N=%d) cells/s' % order,
                'value': out['project_on_fv']['cells_per_s'], 'unit': 'cells/s', 'n_gpus': world,
                'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': out['project_on_fv']['ms_per_call'],
                'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64',
                'data': 'synthetic',
                'config': {'workload': '%d cells of 3D N=%d, patches of %d^3 subcells + %d ghost layer'
                           % (count, order, S, ghost), 'l2': 'inputs larger than L2'},
                'roofline': {'bound': 'hbm', 'achieved': out['project_on_fv']['hbm_gbs'],
                             'peak': peaks.get('hbm_gbs'), 'unit': 'GB/s',
                             'frac': out['project_on_fv']['hbm_frac'], 'peak_source': peak_src},
                'cpu_baseline': cpu, 'kernels': out, 'limiting_grid': lg, 'limiting_grid_3d': lg3, 'fv3d': fv3}
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


# ---------------------------------------------------------------- serving
def serving_stream(S, srv, rate, seconds, seed, dg_fraction):
    """One Poisson stream of `rate` req/s over `seconds` of arrivals through
    the engine's C++ loop; steady-state figures from the second half of the
    arrivals."""
    n = max(8, int(round(rate * seconds)))
    reqs = S.request_mix(n, seed=seed, dg_fraction=dg_fraction)
    res = S.run_poisson(srv, reqs, rate=rate, seed=seed + 17, time_limit=seconds * 2.0 + 30.0)
    loop = srv.loop_times()
    arr = res['arrivals']
    T = float(arr[-1])
    comp = {i: res['done'][i][0] for i in res['done']}
    lat = {i: comp[i] - arr[i] for i in comp}
    second = [i for i in range(n) if arr[i] >= 0.5 * T]
    steady = [lat[i] for i in second if i in lat]
    q3 = [lat[i] for i in range(n) if 0.5 * T <= arr[i] < 0.75 * T and i in lat]
    q4 = [lat[i] for i in range(n) if arr[i] >= 0.75 * T and i in lat]
    last = max(comp.values()) if comp else 0.0
    # steady-state throughput: completions per second inside the second half
    # of the arrival window (the first half fills the engine); the rate over
    # the whole run, drain included, is reported beside it
    achieved = sum(1 for c in comp.values() if 0.5 * T <= c < T) / (0.5 * T) if T > 0 else 0.0
    overall = len(comp) / max(T, last) if T > 0 else 0.0
    growth = (float(np.median(q4)) / float(np.median(q3))) if q3 and q4 else None
    kinds = [reqs[i][0] for i in range(n)]
    out = {'offered_rate_per_s': rate, 'requests': n, 'arrival_window_s': T, 'completed': len(comp),
           'failed': len(res['failed']), 'achieved_rate_per_s': achieved, 'completion_rate_overall_per_s': overall,
           'p50_s': float(np.percentile(steady, 50)) if steady else None,
           'p99_s': float(np.percentile(steady, 99)) if steady else None,
           'p50_dg_s': float(np.percentile([lat[i] for i in second if i in lat and kinds[i] == 'dg'], 50))
           if any(kinds[i] == 'dg' and i in lat for i in second) else None,
           'p50_fv_s': float(np.percentile([lat[i] for i in second if i in lat and kinds[i] == 'fv'], 50))
           if any(kinds[i] == 'fv' and i in lat for i in second) else None,
           'latency_growth_last_quarter': growth, 'ticks': res['ticks'], 'wall_s': res['wall'],
           'aggregate_cell_updates_per_s': res['cell_updates'] / res['wall'] if res['wall'] > 0 else 0.0}
    out['drain_after_last_arrival_s'] = last - T
    # host seconds of the loop: launching ticks, waiting for them, handing
    # out results (overlapped with the next tick), admission
    out['loop_s'] = {k: round(v, 3) for k, v in loop.items()}
    # sustained: everything completed, at >= 95 % of the offered rate in
    # the steady half, within a short drain after the last arrival, and the
    # latency of the last quarter of the arrivals did not grow against the
    # third
    out['sustained'] = bool(len(comp) == n and last - T <= max(5.0, 0.1 * T) and growth is not None
                            and growth < 1.5 and achieved >= 0.95 * rate)
    return out


def run_serving(args, rank, world, dist):
    """Seeded Poisson streams of solve requests (ADER-DG 2D N=2..5, sides
    9..243 log-uniform, 20-200 steps; FV MUSCL-Hancock patches 64..1024
    log-uniform, 20-200 steps), continuous batching on one GPU through the
    engine's C++ request loop; one stream per offered rate, each
    --serving-seconds of arrivals, steady-state latency from the second half
    of the arrivals."""
    import exahype_b200 as E
    from exahype_b200 import serving as S
    E.lib().exa_set_device(int(os.environ.get('LOCAL_RANK', '0')))
    budget = 64 << 30
    srv = S.Server(budget, max_requests=4096)
    srv.tune(args.serving_mode, not args.serving_no_graph)
    srv.set_fv_steps(args.serving_fv_steps)
    srv.set_result_mode(args.serving_result_mode)
    # warm-up: a few small requests through every code path
    S.run_poisson(srv, [('dg', S.dg_request(o, 9, 3)) for o in (2, 3, 4, 5)] + [('fv', S.fv_request(64, 3))],
                  rate=1e4, seed=1)
    if dist:
        dist.barrier()
    rates = [float(r) for r in args.rates.split(',')] if args.rates else [args.rate]
    runs = [serving_stream(S, srv, r, args.serving_seconds, args.seed + rank + 100 * k, args.dg_fraction)
            for k, r in enumerate(rates)]
    srv.destroy()
    head = runs[-1] if len(runs) == 1 else max(runs, key=lambda x: (x['sustained'], x['offered_rate_per_s']))
    if rank == 0:
        line = {'metric': 'serving p99 time-to-solution (Poisson req/s, ADER-DG + FV MUSCL-Hancock mix)',
                'value': head['p99_s'], 'unit': 's', 'higher_is_better': False,
                'n_gpus': world, 'steps': None, 'warmup': 5, 'dtype': 'f64', 'data': 'synthetic',
                'scaling': 'weak', 'vs_baseline': None, 'headline_rate': head['offered_rate_per_s'],
                'runs': runs,
                'config': {'workload': 'serving', 'dg_fraction': args.dg_fraction,
                           'seconds_of_arrivals': args.serving_seconds,
                           'dg': 'order U{2..5}, side log-U[9,243], steps U{20..200}',
                           'fv': 'MUSCL-Hancock, side log-U[64,1024], steps U{20..200}',
                           'loop': 'exa_server_run (C++), FV patches batched per tick',
                           'fv_steps_per_tick': args.serving_fv_steps,
                           'result_hand_out': 'overlapped' if args.serving_result_mode else 'synchronous',
                           'dg_launch': ('per order' if args.serving_mode else 'persistent') +
                                        (', direct' if args.serving_no_graph else ', graph'),
                           'hbm_budget_gb': budget / 2 ** 30}}
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == '__main__':
    main()
