"""Slab decomposition of one periodic ADER-DG grid over several GPUs.

The reference runs a distributed grid through Peano's MPI layer: for every
face on a rank boundary, ADERDGSolver::sendDataToNeighbour
(exahype/solvers/ADERDGSolver.cpp:3379) ships that face's extrapolated
predictor lQhbnd and flux lFhbnd, and the receiving rank's
mergeWithNeighbourData (:3451) solves the Riemann problem with the received
data (:3521); the global time step is a min-reduction over ranks
(exahype/mappings/TimeStepSizeComputation.cpp:83-109).

Here the grid is cut into equal slabs along its last dimension (z in 3D, y
in 2D), one slab per process/GPU.  A slab is an ADERDGGrid of the slab's
size with halos on; one step is

    predict (+ pack the two boundary face layers)      on the grid's stream
    exchange  send_hi(r) -> recv_lo(r+1), send_lo(r) -> recv_hi(r-1)
    correct   (faces across the slab ends read recv_lo / recv_hi)
    all-reduce MIN of the next-dt slot
    commit

The exchange is two face layers per step (a 81x81 layer of N=4 faces is
13 MB) and the reduction is 8 bytes, against a ~60 ms step: NCCL send/recv
on the grid's stream is enough; nothing here waits on the host.

Transports:

* `NcclRing` -- the GPU transport: exchange and reduction run inside the
  library (exa_aderdg_grid_slab_step, C++ over NCCL on the grid's stream);
  Python only passes the communicator's id between processes at start-up.
* `DistRing` (torch.distributed, gloo) and `LocalRing` (all slabs in one
  process) drive the same phases from Python for the CPU tests of this
  driver with oracle slabs (any object with `phase`, `halo_tensors`,
  `dt_slot_tensor`, `stream_ctx`, `fixed_dt`).
"""
import ctypes as C

import numpy as np

from . import _lib
from .aderdg import ADERDGGrid

PHASE_PREDICT = 0
PHASE_CORRECT = 1
PHASE_COMMIT = 2
PHASE_PRIME_LOCAL = 3
PHASE_PRIME_COMMIT = 4


class _DeviceArray:
    """Zero-copy view of library-owned device memory for torch.as_tensor."""

    def __init__(self, ptr, count, typestr):
        self.__cuda_array_interface__ = {
            'shape': (int(count),), 'typestr': typestr, 'data': (int(ptr), False),
            'version': 3, 'strides': None}


def split_last(n, length, nranks):
    """Slab sizes: the last dimension's cells divided evenly over nranks."""
    n = list(n)
    length = list(length)
    if n[-1] % nranks:
        raise ValueError('last dimension (%d cells) does not divide over %d slabs' % (n[-1], nranks))
    n[-1] //= nranks
    length[-1] = length[-1] / nranks
    return n, length


class SlabGrid:
    """Slab `rank` of `nranks` of a periodic ADER-DG grid of `n` cells over
    `length` (whole-domain sizes), on the current GPU."""

    def __init__(self, dim, order, n, rank, nranks, length=None, pde=_lib.PDE_EULER,
                 precision=_lib.PREC_FP64, dt_policy=0, cfl=0.9, dt_fixed=0.0):
        length = list(length) if length is not None else [1.0] * dim
        n_loc, len_loc = split_last(n, length, nranks)
        self.rank, self.nranks = rank, nranks
        self.grid = ADERDGGrid(dim, order, n_loc, len_loc, pde=pde, precision=precision,
                               dt_policy=dt_policy, cfl=cfl, dt_fixed=dt_fixed)
        self.grid.set_halo(True)
        self.fixed_dt = dt_policy == 2
        self.ncells = self.grid.ncells
        self._views = None

    def init(self, kind=0, param=5.0, seed=1234, noise=0.0):
        self.grid.init_slab(self.rank, self.nranks, kind=kind, param=param, seed=seed, noise=noise)

    def phase(self, p):
        self.grid.phase(p)

    def _torch_views(self):
        if self._views is None:
            import torch
            ptrs, count = self.grid.halo_buffers()
            halos = [torch.as_tensor(_DeviceArray(p, count, '<f8'), device='cuda') for p in ptrs]
            slot = torch.as_tensor(_DeviceArray(self.grid.dt_slot_ptr(), 1, '<i8'), device='cuda')
            self._views = (halos, slot)
        return self._views

    def halo_tensors(self):
        return self._torch_views()[0]

    def dt_slot_tensor(self):
        return self._torch_views()[1]

    def stream_ctx(self):
        import torch
        return torch.cuda.stream(torch.cuda.ExternalStream(self.grid.stream().value))

    def synchronize(self):
        _lib.call('exa_stream_synchronize', self.grid.stream())

    def get_state(self):
        return self.grid.get_state()

    def status(self):
        return self.grid.status()

    def destroy(self):
        self._views = None
        self.grid.destroy()


class DistRing:
    """Slab exchange and dt reduction through torch.distributed: rank r
    holds slab r of world_size.  Works with NCCL (slabs on GPUs; the ops
    are ordered on each slab's stream) and gloo (CPU slabs)."""

    def __init__(self, dist, group=None):
        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)

    def exchange(self, slab):
        s_lo, s_hi, r_lo, r_hi = slab.halo_tensors()
        with slab.stream_ctx():
            if self.world == 1:
                r_lo.copy_(s_hi)
                r_hi.copy_(s_lo)
                return
            d = self.dist
            up, down = (self.rank + 1) % self.world, (self.rank - 1) % self.world
            # per peer, messages match in issue order (NCCL) or by tag (gloo):
            # the upward message is the receiver's recv_lo, the downward one
            # its recv_hi
            ops = [d.P2POp(d.isend, s_hi, up, self.group, 1),
                   d.P2POp(d.isend, s_lo, down, self.group, 2),
                   d.P2POp(d.irecv, r_lo, down, self.group, 1),
                   d.P2POp(d.irecv, r_hi, up, self.group, 2)]
            for w in d.batch_isend_irecv(ops):
                w.wait()

    def reduce_dt(self, slab):
        with slab.stream_ctx():
            self.dist.all_reduce(slab.dt_slot_tensor(), op=self.dist.ReduceOp.MIN, group=self.group)

    def slabs(self, slab):
        return [slab]


class LocalRing:
    """All slabs of a ring in this process (several slabs on one GPU, or
    CPU slabs): exchange and reduction are plain copies between steps."""

    def __init__(self, slabs):
        self.all = list(slabs)

    def _sync(self):
        for s in self.all:
            if hasattr(s, 'synchronize'):
                s.synchronize()

    def exchange(self, _slab=None):
        self._sync()
        w = len(self.all)
        for r, s in enumerate(self.all):
            s_lo, s_hi, _, _ = s.halo_tensors()
            self.all[(r + 1) % w].halo_tensors()[2].copy_(s_hi)
            self.all[(r - 1) % w].halo_tensors()[3].copy_(s_lo)
        self._sync_copies()

    def _sync_copies(self):
        t = self.all[0].halo_tensors()[0]
        if t.is_cuda:
            import torch
            torch.cuda.synchronize(t.device)

    def reduce_dt(self, _slab=None):
        self._sync()
        slots = [s.dt_slot_tensor() for s in self.all]
        m = min(int(x.item()) for x in slots)
        for x in slots:
            x.fill_(m)
        self._sync_copies()

    def slabs(self, _slab=None):
        return self.all


class NcclRing:
    """Slab transport inside the library (C++ over NCCL): one communicator
    per process, rank `rank` of `nranks`; `uid` is the 128-byte id made by
    rank 0 with NcclRing.make_id() and handed to every rank (e.g. over a
    host-side process group).  prime / step run whole steps through
    exa_aderdg_grid_slab_prime / _step, which wait with a deadline and abort
    the communicator if a peer stops answering (EXA_ETIMEDOUT)."""

    native = True

    def __init__(self, rank, nranks, uid, timeout_s=60.0):
        h = C.c_void_p()
        buf = C.create_string_buffer(bytes(uid), 128)
        _lib.call('exa_slab_comm_create', buf, int(nranks), int(rank), C.byref(h))
        self.h = h
        self.rank, self.world = rank, nranks
        self.timeout_s = float(timeout_s)

    @staticmethod
    def make_id():
        buf = C.create_string_buffer(128)
        _lib.call('exa_nccl_unique_id', buf)
        return buf.raw

    def prime(self, slab):
        _lib.call('exa_aderdg_grid_slab_prime', slab.grid.h, self.h, self.timeout_s)

    def step(self, slab, nsteps):
        _lib.call('exa_aderdg_grid_slab_step', slab.grid.h, self.h, int(nsteps), self.timeout_s)

    def slabs(self, slab):
        return [slab]

    def destroy(self):
        if self.h:
            _lib.call('exa_slab_comm_destroy', self.h)
            self.h = None


def _each(ring, slab, fn):
    for s in ring.slabs(slab):
        fn(s)


def prime(ring, slab=None):
    """Initial dt: local minimum per slab, MIN over slabs, commit."""
    if getattr(ring, 'native', False):
        ring.prime(slab)
        return
    first = ring.slabs(slab)[0]
    if first.fixed_dt:
        _each(ring, slab, lambda s: s.phase(PHASE_PRIME_COMMIT))
        return
    _each(ring, slab, lambda s: s.phase(PHASE_PRIME_LOCAL))
    ring.reduce_dt(slab)
    _each(ring, slab, lambda s: s.phase(PHASE_PRIME_COMMIT))


def step(ring, slab=None, nsteps=1):
    """Advance every slab of the ring by nsteps time steps."""
    if getattr(ring, 'native', False):
        ring.step(slab, nsteps)
        return
    fixed = ring.slabs(slab)[0].fixed_dt
    for _ in range(nsteps):
        _each(ring, slab, lambda s: s.phase(PHASE_PREDICT))
        ring.exchange(slab)
        _each(ring, slab, lambda s: s.phase(PHASE_CORRECT))
        if not fixed:
            ring.reduce_dt(slab)
        _each(ring, slab, lambda s: s.phase(PHASE_COMMIT))


def gather_state(slabs):
    """Whole-domain state (cells in the undivided grid's order) from the
    slabs of a LocalRing: the last dimension is the slowest cell index, so
    slab states concatenate."""
    return np.concatenate([s.get_state() for s in slabs])
