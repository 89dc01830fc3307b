"""CPU slab with the slab interface of exahype_b200.slab (phase,
halo_tensors, dt_slot_tensor, stream_ctx, fixed_dt), computed by the oracle:
lets the slab driver (exchange order, neighbour ranks, dt reduction) run as
gloo ranks without a GPU.  Test infrastructure only."""
import contextlib
import struct

import numpy as np
import torch

import _oracle as O
from exahype_b200 import slab as SL


def _bits(x):
    return struct.unpack('<q', struct.pack('<d', x))[0]


def _double(b):
    return struct.unpack('<d', struct.pack('<q', int(b)))[0]


class OracleSlab:
    def __init__(self, dim, order, n_global, rank, nranks, luh_global, dt_policy=0, cfl=0.9):
        n_loc, _ = SL.split_last(n_global, [1.0] * dim, nranks)
        self.dim, self.order, self.dt_policy, self.cfl = dim, order, dt_policy, cfl
        self.fixed_dt = False
        self.n = np.array(n_loc + [1] * (3 - dim), dtype=np.int32)
        self.dx = np.array([1.0 / n_global[i] if i < dim else 1.0 for i in range(3)])
        self.ncells = int(np.prod(n_loc))
        B = order + 1
        nn, nfv = B ** dim, B ** (dim - 1) * 5
        self.luh = np.ascontiguousarray(luh_global[rank * self.ncells * nn * 5:(rank + 1) * self.ncells * nn * 5])
        self.lduh = np.zeros(self.ncells * nn * 5)
        self.qb = np.zeros(self.ncells * 2 * dim * nfv)
        self.fb = np.zeros_like(self.qb)
        count = self.ncells // n_loc[-1] * 2 * nfv
        self.halo = [torch.zeros(count, dtype=torch.float64) for _ in range(4)]
        self.slot = torch.zeros(1, dtype=torch.int64)
        self.dt = 0.0
        self.time = 0.0

    def halo_tensors(self):
        return self.halo

    def dt_slot_tensor(self):
        return self.slot

    def stream_ctx(self):
        return contextlib.nullcontext()

    def phase(self, p):
        L = O.lib()
        h = [t.numpy() for t in self.halo]
        if p == SL.PHASE_PRIME_LOCAL:
            self.slot[0] = _bits(L.orc_aderdg_grid_dt(self.dim, self.order, 0, self.n, self.dx, self.luh,
                                                      self.dt_policy, self.cfl))
        elif p == SL.PHASE_PRIME_COMMIT:
            self.dt = _double(self.slot[0])
        elif p == SL.PHASE_PREDICT:
            L.orc_aderdg_slab_predict(self.dim, self.order, 0, self.n, self.dx, self.luh, self.dt, self.lduh,
                                      self.qb, self.fb, h[0], h[1])
        elif p == SL.PHASE_CORRECT:
            L.orc_aderdg_slab_correct(self.dim, self.order, 0, self.n, self.dx, self.luh, self.lduh, self.qb,
                                      self.fb, h[2], h[3], self.dt)
            self.slot[0] = _bits(L.orc_aderdg_grid_dt(self.dim, self.order, 0, self.n, self.dx, self.luh,
                                                      self.dt_policy, self.cfl))
        elif p == SL.PHASE_COMMIT:
            self.time += self.dt
            self.dt = _double(self.slot[0])


def global_ic(dim, order, n, kind=0, param=5.0, seed=7, noise=1e-3):
    B = order + 1
    nc = int(np.prod(n))
    luh = np.zeros(nc * B ** dim * 5)
    n3 = np.array(list(n) + [1] * (3 - dim), dtype=np.int32)
    dx = np.array([1.0 / n[i] if i < dim else 1.0 for i in range(3)])
    O.lib().orc_aderdg_grid_ic(dim, order, n3, dx, luh, kind, param, seed, noise)
    return luh, n3, dx


def run_rank(rank, world, port, dim, order, n, steps, outdir):
    """gloo rank of the CPU slab driver test: slab `rank` of the grid
    advanced `steps` steps through exahype_b200.slab with a DistRing."""
    import os
    import datetime
    import torch.distributed as dist
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        luh, _, _ = global_ic(dim, order, n)
        s = OracleSlab(dim, order, list(n), rank, world, luh)
        ring = SL.DistRing(dist)
        SL.prime(ring, s)
        SL.step(ring, s, steps)
        np.save(os.path.join(outdir, 'slab%d.npy' % rank), s.luh)
        np.save(os.path.join(outdir, 'time%d.npy' % rank), np.array([s.time]))
    finally:
        dist.destroy_process_group()
