"""One grid decomposed in x over the ranks of a torch.distributed process group.

The reference's active model runs one domain in one process; its legacy model
(qjrmsCode/) decomposes x and y over MPI ranks, trading hs-wide halos with Irecv/Isend
(qjrmsCode/Exchange.cpp:106-176) and reducing dt with MPI_Allreduce(MIN)
(qjrmsCode/Initializer.cpp:263). Here each rank owns one x slab of the grid (its own
awfl_create_slab context and state on its GPU) and, before every x split, trades hs+1
columns with the slabs on either side over the process group (NCCL on GPUs: point-to-point
sends into the receiver's own buffer, no peer-memory reads); the y and z splits need
nothing from other ranks. The extra column lets each slab reconstruct its neighbour's edge
cell itself, so the interior cells advance bit for bit as in the undivided grid. The CFL
time step is the minimum over the slabs (one all-reduce).

`neighbours` and `exchange_columns` hold the exchange logic; they run with NCCL (CUDA
tensors) or gloo (host tensors) alike.
"""
from __future__ import annotations

from . import capi


def neighbours(slab, nslabs, periodic):
    """(slab below, slab above) of `slab`; None at a wall of the grid (and for a single
    periodic slab, which wraps onto itself without an exchange)."""
    if nslabs == 1:
        return None, None
    lo = slab - 1 if slab > 0 else (nslabs - 1 if periodic else None)
    hi = slab + 1 if slab < nslabs - 1 else (0 if periodic else None)
    return lo, hi


def exchange_columns(send, recv, slab, nslabs, periodic, group=None):
    """Trade halo columns with the neighbouring slabs: send[1] (this slab's last columns)
    goes to the slab above and arrives there as its recv[0]; send[0] (its first columns)
    goes to the slab below as its recv[1]. send and recv are [2, n] tensors on the
    process group's device. Every rank posts its operations as one batch
    (batch_isend_irecv) in the same order (upward send, receive from below, downward
    send, receive from above), so that two slabs that are each other's neighbour on both
    sides (a periodic pair) match their messages in order on any backend; tags 0 (upward)
    and 1 (downward) separate them where the backend honours tags."""
    import torch.distributed as dist
    lo, hi = neighbours(slab, nslabs, periodic)
    if lo is None and hi is None:
        return
    ranks = dist.get_process_group_ranks(group) if group is not None else list(range(nslabs))
    ops = []
    if hi is not None:
        ops.append(dist.P2POp(dist.isend, send[1], ranks[hi], group=group, tag=0))
    if lo is not None:
        ops.append(dist.P2POp(dist.irecv, recv[0], ranks[lo], group=group, tag=0))
    if lo is not None:
        ops.append(dist.P2POp(dist.isend, send[0], ranks[lo], group=group, tag=1))
    if hi is not None:
        ops.append(dist.P2POp(dist.irecv, recv[1], ranks[hi], group=group, tag=1))
    # one batch (one NCCL group): no rank's send waits for a receive that its peer has
    # queued behind a send of its own
    for r in dist.batch_isend_irecv(ops):
        r.wait()


def route_columns(sends, periodic):
    """The same exchange between slabs held in one process (a list of [2, n] send
    tensors, one per slab, in slab order): the receive buffers, zero where an end is a
    wall."""
    import torch
    n = len(sends)
    recvs = [torch.zeros_like(s) for s in sends]
    for s in range(n):
        lo, hi = neighbours(s, n, periodic)
        if lo is not None:
            recvs[s][0].copy_(sends[lo][1])
        if hi is not None:
            recvs[s][1].copy_(sends[hi][0])
    return recvs


class SlabDomain:
    """This rank's slab of an nx x ny x nz grid decomposed in x over the ranks of a
    torch.distributed process group (backend "nccl", one GPU per rank). step() advances
    the rank's state one time step; cfl() is the grid's time step."""

    def __init__(self, nx, ny, nz, group=None, device=None, xlen=20000.0, ylen=20000.0, zlen=10000.0,
                 bc=("periodic", "periodic", "wall"), ord_=5, precision=capi.FP64, **kw):
        import torch
        import torch.distributed as dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.nslabs = dist.get_world_size(group)
        self.device = torch.cuda.current_device() if device is None else device
        self.ctx = capi.Context.slab(nx, ny, nz, self.nslabs, self.rank, xlen=xlen, ylen=ylen, zlen=zlen, bc=bc,
                                     ord_=ord_, precision=precision, device=self.device, **kw)
        self.periodic = (capi.BC[bc[0]] if isinstance(bc[0], str) else int(bc[0])) == capi.BC_PERIODIC
        dtype = torch.float64 if precision == capi.FP64 else torch.float32
        half = self.ctx.halo_elems // 2
        self.send = torch.empty((2, half), dtype=dtype, device="cuda:%d" % self.device)
        self.recv = torch.zeros_like(self.send)
        self.dimswitch = 1

    def new_state(self):
        return self.ctx.new_state()

    def cfl(self, state, cfl=0.8):
        import torch
        import torch.distributed as dist
        t = torch.tensor([self.ctx.cfl(state, cfl)], dtype=torch.float64, device="cuda:%d" % self.device)
        dist.all_reduce(t, op=dist.ReduceOp.MIN, group=self.group)
        return t.item()

    def split(self, state, dt, d):
        """One split on torch's current stream (the stream the process group's NCCL
        operations are ordered with; enter another one with torch.cuda.stream(...))."""
        if d != 0 or self.nslabs == 1:
            self.ctx.split(state, dt, d)
            return
        self.ctx.slab_pack(state, self.send)
        exchange_columns(self.send, self.recv, self.rank, self.nslabs, self.periodic, self.group)
        self.ctx.split_slab(state, self.recv, dt)

    def step(self, state, dt):
        """Temporal_ader::timeStep on this slab: three splits in the dimSwitch order, the x
        split after the column exchange."""
        ds = self.dimswitch
        for spl in range(3):
            self.split(state, dt, spl if ds else 2 - spl)
        self.dimswitch = 1 - ds
